"""The C-ABI library loads without a GPU and exports every entry point that include/adock_b200.h declares."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    hdr = (ROOT / "include" / "adock_b200.h").read_text()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(adock_\w+)\s*\(", hdr)))


def test_header_declares_entry_points():
    names = _declared()
    for n in ("adock_version", "adock_last_error", "adock_grid_vina", "adock_grid_fit", "adock_eg", "adock_mc",
              "adock_stage_a", "adock_neighbours", "adock_prepare", "adock_rescore64"):
        assert n in names


def test_library_exports_declared_symbols():
    from adock_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("libadock_b200.so not built")
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for n in _declared():
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTS) <= set(_declared())


def test_version_and_argument_errors_without_gpu():
    """Argument checks run on the host before any CUDA call: a bad size is rejected with a message."""
    from adock_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("libadock_b200.so not built")
    lib = _lib.load()
    assert lib.adock_version() == 1
    with pytest.raises(RuntimeError, match="n_lt"):
        _lib.call("adock_grid_vina", None, None, 0, 1, 1, 1, 1, 18, 1, 0, 0.0, 0.0, 0.0, 0.375, 4, 4, 4, 1, 0, 1, None)
    with pytest.raises(RuntimeError, match="KM"):
        lig = _lib.Ligands()
        lig.L, lig.AM, lig.KM, lig.P = 1, 64, 40, 1
        sf = _lib.SF()
        sf.n_types = 18
        w = _lib.Work()
        _lib.call("adock_prepare", lig, sf, w, None)
