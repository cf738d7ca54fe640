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


def test_pipeline_entry_points_reject_bad_arguments_without_gpu():
    """The device-pipeline entry points check sizes and limits on the host and refuse with a message: start
    selection beyond 16,384 (conformer, rotation) totals, clustering beyond 4,096 poses or 32 representatives,
    conformer counts out of range, and grid cell lists too coarse for the cutoff."""
    from adock_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("libadock_b200.so not built")
    p = ctypes.c_void_p(8)      # never dereferenced: every call below fails its argument check first
    with pytest.raises(RuntimeError, match="16384"):
        _lib.call("adock_select_starts", 1, 64, 512, 8, 4, p, p, p, p, p, p, None, 10, p, None, None)
    w = _lib.Work()
    w.info = 8
    with pytest.raises(RuntimeError, match="4096"):
        _lib.call("adock_cluster", w, 1, 5000, p, p, 64, 2.0, 9, p, p, None)
    with pytest.raises(RuntimeError, match="n_out"):
        _lib.call("adock_cluster", w, 1, 16, p, p, 64, 2.0, 40, p, p, None)
    lig = _lib.Ligands()
    lig.L, lig.AM, lig.KM, lig.P = 1, 64, 8, 1
    sf = _lib.SF()
    sf.n_types = 18
    with pytest.raises(RuntimeError, match="NT"):
        _lib.call("adock_conformers", lig, _lib.Work(), sf, 0, 1, 0, p, p, p, None)
    with pytest.raises(RuntimeError, match="C must"):
        _lib.call("adock_conformers", lig, _lib.Work(), sf, 8, 9, 0, p, p, p, None)
    dims = (ctypes.c_int * 3)(4, 4, 4)
    org = (ctypes.c_float * 3)(0, 0, 0)
    prm = (ctypes.c_float * 15)(8.0, 0, 0.5, 3, 2, 0, 0.5, 1.5, -0.7, 0, -0.035, -0.005, 0.84, -0.035, -0.587)
    lt = (ctypes.c_int * 1)(0)
    tab = (ctypes.c_int * 18)()
    rad = (ctypes.c_float * 18)(*([1.9] * 18))
    with pytest.raises(RuntimeError, match="cell size"):
        _lib.call("adock_grid_vina_cells", p, p, 10, p, ctypes.addressof(dims), ctypes.addressof(org), 1.0,
                  ctypes.addressof(rad), ctypes.addressof(tab), ctypes.addressof(tab), ctypes.addressof(tab), 18,
                  ctypes.addressof(lt), 1, 0.0, 0.0, 0.0, 0.375, 8, 8, 8, ctypes.addressof(prm), 0, p, None)


def test_proposal_entry_points_reject_bad_arguments_without_gpu():
    """The proposal kernels' host checks: only 1 or 3 translation components, at most 512 targets per chain, and
    no ligand-best hint without its key scratch."""
    from adock_b200 import _lib
    if not _lib.LIB_PATH.exists():
        pytest.skip("libadock_b200.so not built")
    p = ctypes.c_void_p(8)      # never dereferenced: every call below fails its argument check first
    with pytest.raises(RuntimeError, match="n_comp"):
        _lib.call("adock_mlp_nll", p, p, 4, 2, p, p, None)
    lig = _lib.Ligands()
    w = _lib.Work()
    w.info = 8
    with pytest.raises(RuntimeError, match="n_comp"):
        _lib.call("adock_prop_sample", lig, w, p, p, 4, p, p, 27, 32, 2, 1, 0, p, None)
    with pytest.raises(RuntimeError, match="512"):
        _lib.call("adock_prop_sample", lig, w, p, p, 4, p, p, 27, 600, 1, 1, 0, p, None)
    with pytest.raises(RuntimeError, match="null"):
        _lib.call("adock_prop_hint", 4, 8, p, p, 27, p, None, p, None)
