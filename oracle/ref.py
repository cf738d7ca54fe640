"""ctypes binding of the reference's own CPU build (``oracle/_ref/*.so``, made by ``oracle/build_ref.py``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference arms, as the checker / the timed reference. The product never imports it.

The launchers follow the reference's generated host source (``src/adock/cpukernel.py:91-142``):
``launch_<kernel>(n_blocks, <kernel arguments>)`` with the kernel signatures of ``src/adock/mckernel.py:328-458``
and ``launch_build_grid_tiled`` (``cpukernel.py:104-137``). Inputs are the packed numpy arrays of
``pack_host`` (``mckernel.py:547-599``).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
_LIG = [P] * 7 + [P, P, P, P] + [I, P]                 # ref typ tm ax axp axu pr | na nt np rg | P_MAX gslot
_GRID = [P, P, P, P, P, P, P, I, F, F]                  # flat origin lo hi rec_idx offs dims T spacing pen
_SF = [P] * 5
_REC = [P, P, P, I]
_SIGS = {
    "launch_eg_kernel": [ctypes.c_longlong] + _LIG + _GRID + _SF + _REC + [I, P, I, P, P, P],
    "launch_mc_kernel": [ctypes.c_longlong] + _LIG + _GRID + _SF + _REC + [I, P, P, I, P, P, I, P, P, P, P, I, I, I, F,
                                                                            F, F, ctypes.c_uint64, I],
    "launch_stagea_kernel": [ctypes.c_longlong, P, P, P, I, P, I, P, P, I, P, P, P, P, P, P, P, F, F, F, P, P],
    "launch_build_grid_tiled": [P, P, I, P, P, P, P, P, I, F, F, F, F, I, I, I, P, I, P, I],
}
_FIT_SIG = [P, P, I, P, P, I, P, F, F, F, F, I, I, I, P, P]

_LIBS = {}


def available() -> bool:
    return (REF_DIR / "adock_ref_64_8.so").exists()


def threads() -> int:
    n = int(os.environ.get("ADOCK_CPU_THREADS", "0"))
    return n or len(os.sched_getaffinity(0))


def lib(am=64, km=8):
    key = (am, km)
    if key not in _LIBS:
        so = REF_DIR / f"adock_ref_{am}_{km}.so"
        if not so.exists():
            raise FileNotFoundError(f"{so} missing: run `python oracle/build_ref.py` where the reference is present")
        L = ctypes.CDLL(str(so))
        for name, sig in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = sig
            f.restype = None
        L.set_threads.argtypes = [I]
        _LIBS[key] = L
    L = _LIBS[key]
    L.set_threads(threads())
    return L


def fit_lib():
    if "fit" not in _LIBS:
        so = REF_DIR / "adock_ref_gridfit.so"
        L = ctypes.CDLL(str(so))
        L.launch_build_grid_fit.argtypes = _FIT_SIG
        L.launch_build_grid_fit.restype = None
        L.set_threads.argtypes = [I]
        _LIBS["fit"] = L
    L = _LIBS["fit"]
    L.set_threads(threads())
    return L


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], type(a)
    return a.ctypes.data


def _c(a, dt):
    return np.ascontiguousarray(np.asarray(a), dtype=dt)


class RefProblem:
    """Packed problem for the reference CPU kernels.

    lig: [ref, typ, tm, ax, axp, axu, pr, na, nt, np, rg, P, gslot] (pack_host order);
    grid: dict flat, origin [R,3], lo, hi, rec_idx [L], offs [R], dims [R,3], T, spacing, penalty;
    sf: [prm(15), radius, hyd, don, acc]; rec: (xyz [R,RN,3], typ [R,RN], n [R]) or None."""

    def __init__(self, AM, KM, lig, sf, grid, rec=None):
        self.AM, self.KM = AM, KM
        ref, typ, tm, ax, axp, axu, pr, na, nt, npr, rg, Pm, gsl = lig
        self.lig = [_c(ref, np.float32), _c(typ, np.int32), _c(tm, np.uint8), _c(ax, np.int32), _c(axp, np.float32),
                    _c(axu, np.float32), _c(pr, np.int32), _c(na, np.int32), _c(nt, np.int32), _c(npr, np.int32),
                    _c(rg, np.float32), int(Pm), _c(gsl, np.int32)]
        self.sf = [_c(sf[0], np.float32), _c(sf[1], np.float32), _c(sf[2], np.int32), _c(sf[3], np.int32),
                   _c(sf[4], np.int32)]
        g = grid
        self.grid = [_c(g["flat"], np.float32), _c(g["origin"], np.float32), _c(g["lo"], np.float32),
                     _c(g["hi"], np.float32), _c(g["rec_idx"], np.int32), _c(g["offs"], np.int64),
                     _c(g["dims"], np.int64), int(g["T"]), float(g["spacing"]), float(g["penalty"])]
        if rec is not None:
            self.rec = [_c(rec[0], np.float32), _c(rec[1], np.int32), _c(rec[2], np.int32), int(np.asarray(rec[0]).shape[1])]
        else:
            self.rec = [np.zeros(3, np.float32), np.zeros(1, np.int32), np.zeros(1, np.int32), 0]
        self.SD, self.DM = 7 + KM, 6 + KM
        self.L = len(self.lig[7])

    def _args(self, exact):
        lg = [_p(a) if isinstance(a, np.ndarray) else a for a in self.lig]
        gr = [_p(a) if isinstance(a, np.ndarray) else a for a in self.grid]
        sf = [_p(a) for a in self.sf]
        rc = [_p(a) if isinstance(a, np.ndarray) else a for a in self.rec]
        return lg + gr + sf + rc + [int(exact)]

    def energy_grad(self, chain_lig, state, exact=False):
        N = state.shape[0]
        e = np.zeros(N, np.float32)
        g = np.zeros((N, self.DM), np.float32)
        cl = _c(chain_lig, np.int32)
        st = _c(state, np.float32)
        lib(self.AM, self.KM).launch_eg_kernel(N, *self._args(exact), _p(cl), N, _p(st), _p(e), _p(g))
        return e, g

    def run_mc(self, chain_lig, chain_id, cur, cur_e, best, best_e, init_opt, mc_steps, bfgs_iters, temp, amp_pos,
               amp_rot, seed, step_offset, exact=False, nbr=None, nbr_n=None):
        """In place on the float32 numpy arrays cur/cur_e/best/best_e."""
        N = cur.shape[0]
        if N == 0:
            return
        for x in (cur, cur_e, best, best_e):
            assert x.flags["C_CONTIGUOUS"] and x.dtype == np.float32
        cl, ci = _c(chain_lig, np.int32), _c(chain_id, np.int32)
        if nbr is not None:
            nbr, nbr_n = _c(nbr, np.int32), _c(nbr_n, np.int32)
            nb = [_p(nbr), _p(nbr_n), int(nbr.shape[1])]
        else:
            nb = [None, None, 0]
        lib(self.AM, self.KM).launch_mc_kernel(
            N, *self._args(exact), _p(cl), _p(ci), N, *nb, _p(cur), _p(cur_e), _p(best), _p(best_e), int(init_opt),
            int(mc_steps), int(bfgs_iters), float(temp), float(amp_pos), float(amp_rot),
            ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), int(step_offset))

    def stage_a(self, conf_h, quats, trans, ntrans, cap):
        L, C = conf_h.shape[:2]
        Q, NT = quats.shape[0], trans.shape[1]
        be = np.empty(L * C * Q, np.float32)
        bi = np.empty(L * C * Q, np.int32)
        conf, qu, tr, nt = _c(conf_h, np.float32), _c(quats, np.float32), _c(trans, np.float32), _c(ntrans, np.int32)
        flat, org, lo, hi, ri, go, gd = self.grid[:7]
        lib(self.AM, self.KM).launch_stagea_kernel(
            L * C * Q, _p(conf), _p(self.lig[12]), _p(self.lig[7]), C, _p(qu), Q, _p(tr), _p(nt), NT, _p(flat),
            _p(org), _p(lo), _p(hi), _p(ri), _p(go), _p(gd), self.grid[8], self.grid[9], float(cap), _p(be), _p(bi))
        return be.reshape(L, C * Q), bi.reshape(L, C * Q).astype(np.int64)


def build_grid(rec_xyz, rec_types, sfp, origin, spacing, n, lig_types, per_term=False, tile=8):
    """Reference host grid builder (cpukernel.py:210-228) -> numpy [T, nx, ny, nz] ([5, T, ...] if per_term)."""
    from adock_b200.params import grid_prm
    if np.isscalar(n):
        n = (int(n),) * 3
    nx, ny, nz = map(int, n)
    rx = _c(np.asarray(rec_xyz).reshape(-1, 3), np.float32)
    rt = _c(rec_types, np.int32)
    lt = _c(lig_types, np.int32)
    out = np.zeros(((5 if per_term else 1) * len(lt) * nx * ny * nz,), np.float32)
    keep = [_c(sfp["radius"], np.float32), _c(sfp["hydrophobic"], np.int32), _c(sfp["donor"], np.int32),
            _c(sfp["acceptor"], np.int32), grid_prm(sfp)]
    lib().launch_build_grid_tiled(_p(rx), _p(rt), len(rx), _p(keep[0]), _p(keep[1]), _p(keep[2]), _p(keep[3]), _p(lt),
                                  len(lt), float(origin[0]), float(origin[1]), float(origin[2]), float(spacing), nx, ny,
                                  nz, _p(keep[4]), int(per_term), _p(out), int(tile))
    return out.reshape(((5, len(lt)) if per_term else (len(lt),)) + (nx, ny, nz))


def build_grid_fit(rec_xyz, rec_ext, W, rad_rec, rad_lig, prm12, origin, spacing, n):
    """Reference fitted grid kernel text (gridfit.py:13-58) run on the host -> numpy [TL, nx, ny, nz]."""
    if np.isscalar(n):
        n = (int(n),) * 3
    nx, ny, nz = map(int, n)
    rx = _c(np.asarray(rec_xyz).reshape(-1, 3), np.float32)
    re = _c(rec_ext, np.int32)
    W = _c(W, np.float32)
    rr, rl, pr = _c(rad_rec, np.float32), _c(rad_lig, np.float32), _c(prm12, np.float32)
    TL = len(rl)
    out = np.zeros(TL * nx * ny * nz, np.float32)
    fit_lib().launch_build_grid_fit(_p(rx), _p(re), len(rx), _p(rr), _p(rl), TL, _p(W), float(origin[0]),
                                    float(origin[1]), float(origin[2]), float(spacing), nx, ny, nz, _p(pr), _p(out))
    return out.reshape(TL, nx, ny, nz)
