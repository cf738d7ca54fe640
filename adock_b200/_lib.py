"""ctypes binding of ``libadock_b200.so`` (declarations in ``include/adock_b200.h``).

The library is built in-tree (``adock_b200/csrc/build.py``). There is no fallback: if it is missing or fails
to load, every entry point raises."""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libadock_b200.so"

ADOCK_GRID_F32, ADOCK_GRID_F16, ADOCK_GRID_BF16 = 0, 1, 2

P = ctypes.c_void_p
I = ctypes.c_int
F = ctypes.c_float


class SF(ctypes.Structure):
    _fields_ = [("prm", F * 15), ("n_types", I), ("radius", F * 64), ("hyd", I * 64), ("don", I * 64),
                ("acc", I * 64)]


class Ligands(ctypes.Structure):
    _fields_ = [("ref", P), ("typ", P), ("tm", P), ("ax", P), ("axp", P), ("axu", P), ("pr", P), ("na", P),
                ("nt", P), ("np", P), ("rg", P), ("gslot", P), ("rec_idx", P), ("L", I), ("AM", I), ("KM", I),
                ("P", I)]


class Grids(ctypes.Structure):
    _fields_ = [("flat", P), ("offs", P), ("dims", P), ("origin", P), ("lo", P), ("hi", P), ("R", I),
                ("dtype", I), ("spacing", F), ("penalty", F), ("nmaps", P)]


class Receptors(ctypes.Structure):
    _fields_ = [("xyz", P), ("typ", P), ("n", P), ("RN", I)]


class Work(ctypes.Structure):
    _fields_ = [("atoms", P), ("masks", P), ("tors", P), ("pairs", P), ("info", P), ("rg", P)]


class McArgs(ctypes.Structure):
    _fields_ = [("chain_lig", P), ("chain_id", P), ("n_chains", I), ("nbr", P), ("nbr_n", P), ("nb_max", I),
                ("cur", P), ("cur_e", P), ("best", P), ("best_e", P), ("init_opt", I), ("mc_steps", I),
                ("bfgs_iters", I), ("temp", F), ("amp_pos", F), ("amp_rot", F), ("seed", ctypes.c_ulonglong),
                ("step_offset", I), ("exact", I), ("order", P), ("queue", P), ("evals", P), ("variant", I),
                ("prop", P), ("prop_k", I), ("prop_stats", P), ("log_x", P), ("log_y", P), ("log_n", P),
                ("log_cap", I), ("prop_frac", F), ("lig_active", P),
                ("prop_tries", I), ("hint", P)]


SP = ctypes.POINTER
_SIGS = {
    "adock_version": ([], I),
    "adock_last_error": ([], ctypes.c_char_p),
    "adock_grid_vina": ([P, P, I, P, P, P, P, I, P, I, F, F, F, F, I, I, I, P, I, P, P], I),
    "adock_grid_fit": ([P, P, I, P, I, P, I, P, F, F, F, F, I, I, I, P, P, P], I),
    "adock_grid_vina_cells": ([P, P, I, P, P, P, F, P, P, P, P, I, P, I, F, F, F, F, I, I, I, P, I, P, P], I),
    "adock_grid_fit_cells": ([P, P, I, P, P, P, F, P, I, P, I, P, F, F, F, F, I, I, I, P, P, P], I),
    "adock_grid_convert": ([P, P, ctypes.c_longlong, I, P], I),
    "adock_prepare": ([SP(Ligands), SP(SF), SP(Work), P], I),
    "adock_eg": ([SP(Ligands), SP(Work), SP(Grids), SP(SF), SP(Receptors), P, I, P, P, P, I, P], I),
    "adock_mc": ([SP(Ligands), SP(Work), SP(Grids), SP(SF), SP(Receptors), SP(McArgs), P], I),
    "adock_stage_a": ([SP(Ligands), SP(Work), SP(Grids), SP(SF), P, I, P, I, P, P, I, F, P, P, P], I),
    "adock_neighbours": ([SP(Ligands), SP(Work), SP(SF), SP(Receptors), P, I, P, F, P, P, I, P], I),
    "adock_stage_a_boxes": ([SP(Ligands), SP(Work), SP(Grids), SP(SF), P, I, P, I, P, P, I, P, F, P, P, P], I),
    "adock_conformers": ([SP(Ligands), SP(Work), SP(SF), I, I, ctypes.c_ulonglong, P, P, P, P], I),
    "adock_lattice": ([SP(Grids), I, P, P, P, P, F, F, I, P, P, P], I),
    "adock_select_starts": ([I, I, I, I, I, P, P, P, P, P, P, P, I, P, P, P], I),
    "adock_segment_update": ([I, I, I, I, I, F, P, P, P, P, P, P, P], I),
    "adock_cluster": ([SP(Work), I, I, P, P, I, F, I, P, P, P], I),
    "adock_pose_atoms": ([SP(Work), I, P, P, I, P, I, P, P, P], I),
    "adock_rescore64": ([SP(Ligands), SP(Work), SP(Grids), SP(SF), SP(Receptors), P, I, P, P, P, P, P], I),
    "adock_mc_noalloc_scratch_bytes": ([I, I, I, I], ctypes.c_size_t),
    "adock_mc_noalloc": ([SP(Ligands), SP(Grids), SP(SF), SP(Receptors), SP(McArgs), P], I),
    "adock_prop_features": ([SP(Ligands), SP(Work), SP(Grids), SP(SF), P, I, P, P, P, P, P], I),
    "adock_prop_hint": ([I, I, P, P, I, P, P, P, P], I),
    "adock_prop_sample": ([SP(Ligands), SP(Work), P, P, I, P, P, I, I, I, ctypes.c_ulonglong, I, P, P], I),
    "adock_gemm_bf16": ([I, I, I, P, ctypes.c_longlong, ctypes.c_longlong, P, ctypes.c_longlong, ctypes.c_longlong, P,
                         ctypes.c_longlong, F, P, I, P, P, ctypes.c_longlong, P], I),
    "adock_gemm_bf16_mma": ([I, I, I, P, ctypes.c_longlong, ctypes.c_longlong, P, ctypes.c_longlong,
                             ctypes.c_longlong, P, ctypes.c_longlong, F, P, I, P, P, ctypes.c_longlong, P], I),
    "adock_gemm_status": ([], I),
    "adock_mlp_nll": ([P, P, I, I, P, P, P], I),
    "adock_silu_backward": ([P, P, ctypes.c_longlong, P, P], I),
    "adock_bias_grad": ([P, I, I, P, P], I),
    "adock_adam": ([P, P, P, P, P, ctypes.c_longlong, F, F, F, F, I, F, P], I),
    "adock_f32_to_bf16": ([P, P, ctypes.c_longlong, P], I),
}
EXPORTS = tuple(_SIGS)

_lib = None
_lock = threading.Lock()
# kernel launches issued through call() (each launching entry point issues one kernel)
LAUNCHES = [0]
_NO_LAUNCH = {"adock_version", "adock_last_error", "adock_mc_noalloc_scratch_bytes", "adock_gemm_status"}


def load():
    """Load the library (once) and declare the signatures. Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m adock_b200.csrc.build`")
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (args, res) in _SIGS.items():
                f = getattr(lib, name)
                f.argtypes = args
                f.restype = res
            _lib = lib
    return _lib


def call(name, *args):
    """Call an entry point; a non-zero status raises RuntimeError with the library's message."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if name not in _NO_LAUNCH and rc == 0:
        LAUNCHES[0] += 1
    if rc != 0:
        msg = lib.adock_last_error().decode(errors="replace")
        raise RuntimeError(f"{name} failed ({rc}): {msg}")
    return rc


def ptr(t):
    """Device (or host) address of a contiguous torch tensor / numpy array; None -> NULL."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        assert t.flags["C_CONTIGUOUS"]
        return t.ctypes.data
    assert t.is_contiguous(), "tensor must be contiguous"
    return t.data_ptr()


def stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


def make_sf(sfp: dict) -> SF:
    from .params import search_prm
    s = SF()
    prm = search_prm(sfp)
    for i in range(15):
        s.prm[i] = float(prm[i])
    rad = np.asarray(sfp["radius"], np.float32)
    n = len(rad)
    assert n <= 64, "at most 64 scoring types"
    s.n_types = n
    for i in range(n):
        s.radius[i] = float(rad[i])
        s.hyd[i] = int(sfp["hydrophobic"][i])
        s.don[i] = int(sfp["donor"][i])
        s.acc[i] = int(sfp["acceptor"][i])
    return s
