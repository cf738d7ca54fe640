"""ctypes binding of the oracle's C restatement (``oracle/port.c`` -> ``oracle/liboracle_port.so``).

TEST INFRASTRUCTURE ONLY: the checker for tests/, smoke() and bench.py's CPU-baseline leg. The same packed
arrays the product consumes (``pack_host`` layout) go in; results come back as numpy arrays."""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_port.so"
P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float


class Lig(ctypes.Structure):
    _fields_ = [(n, P) for n in ("ref", "typ", "tm", "ax", "axp", "axu", "pr", "na", "nt", "np", "rg", "gslot",
                                 "rec_idx")] + [("L", I), ("AM", I), ("KM", I), ("P", I)]


class Grid(ctypes.Structure):
    _fields_ = [(n, P) for n in ("flat", "offs", "dims", "origin", "lo", "hi")] + [("spacing", F), ("penalty", F)]


class SF(ctypes.Structure):
    _fields_ = [("prm", F * 15)] + [(n, P) for n in ("radius", "hyd", "don", "acc")]


class Rec(ctypes.Structure):
    _fields_ = [("xyz", P), ("typ", P), ("n", P), ("RN", I)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            from . import build_port
            build_port.build()
        L = ctypes.CDLL(str(LIB))
        L.port_set_threads.argtypes = [I]
        L.port_grid_vina.argtypes = [P, P, I, P, P, P, P, P, I, F, F, F, F, I, I, I, P, I, P]
        L.port_grid_fit.argtypes = [P, P, I, P, P, I, P, F, F, F, F, I, I, I, P, P]
        SPL, SPG, SPS, SPR = (ctypes.POINTER(x) for x in (Lig, Grid, SF, Rec))
        L.port_eg.argtypes = [SPL, SPG, SPS, SPR, I, P, I, P, P, P]
        L.port_mc.argtypes = [SPL, SPG, SPS, SPR, I, P, P, I, P, P, I, P, P, P, P, I, I, I, F, F, F, ctypes.c_uint64, I]
        L.port_mc.restype = ctypes.c_longlong
        L.port_stage_a.argtypes = [SPL, SPG, P, I, P, I, P, P, I, F, P, P]
        for f in (L.port_set_threads, L.port_grid_vina, L.port_grid_fit, L.port_eg, L.port_stage_a):
            f.restype = None
        _lib = L
    n = int(os.environ.get("ADOCK_CPU_THREADS", "0")) or len(os.sched_getaffinity(0))
    _lib.port_set_threads(n)
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(np.asarray(a), dtype=dt)


def _p(a):
    return None if a is None else a.ctypes.data


def build_grid(rec_xyz, rec_types, sfp, origin, spacing, n, lig_types, per_term=False):
    from adock_b200.params import grid_prm
    if np.isscalar(n):
        n = (int(n),) * 3
    nx, ny, nz = map(int, n)
    rx, rt, lt = _c(np.asarray(rec_xyz).reshape(-1, 3), np.float32), _c(rec_types, np.int32), _c(lig_types, np.int32)
    k = [_c(sfp["radius"], np.float32), _c(sfp["hydrophobic"], np.int32), _c(sfp["donor"], np.int32),
         _c(sfp["acceptor"], np.int32), grid_prm(sfp)]
    out = np.zeros(((5 if per_term else 1) * len(lt) * nx * ny * nz,), np.float32)
    lib().port_grid_vina(_p(rx), _p(rt), len(rx), _p(k[0]), _p(k[1]), _p(k[2]), _p(k[3]), _p(lt), len(lt),
                         float(origin[0]), float(origin[1]), float(origin[2]), float(spacing), nx, ny, nz, _p(k[4]),
                         int(per_term), _p(out))
    return out.reshape(((5, len(lt)) if per_term else (len(lt),)) + (nx, ny, nz))


def build_grid_fit(rec_xyz, rec_ext, W, rad_rec, rad_lig, prm12, origin, spacing, n):
    if np.isscalar(n):
        n = (int(n),) * 3
    nx, ny, nz = map(int, n)
    rx, re = _c(np.asarray(rec_xyz).reshape(-1, 3), np.float32), _c(rec_ext, np.int32)
    W, rr, rl, pr = _c(W, np.float32), _c(rad_rec, np.float32), _c(rad_lig, np.float32), _c(prm12, np.float32)
    out = np.zeros(len(rl) * nx * ny * nz, np.float32)
    lib().port_grid_fit(_p(rx), _p(re), len(rx), _p(rr), _p(rl), len(rl), _p(W), float(origin[0]), float(origin[1]),
                        float(origin[2]), float(spacing), nx, ny, nz, _p(pr), _p(out))
    return out.reshape(len(rl), nx, ny, nz)


class PortProblem:
    """Packed problem for the C restatement (same arrays as the reference's pack_host)."""

    def __init__(self, AM, KM, lig, sf, grid, rec=None):
        ref, typ, tm, ax, axp, axu, pr, na, nt, npr, rg, Pm, gsl = lig
        self.AM, self.KM, self.P = AM, KM, int(Pm)
        self.keep = [_c(ref, np.float32), _c(typ, np.int32), _c(tm, np.uint8), _c(ax, np.int32), _c(axp, np.float32),
                     _c(axu, np.float32), _c(pr, np.int32), _c(na, np.int32), _c(nt, np.int32), _c(npr, np.int32),
                     _c(rg, np.float32), _c(gsl, np.int32), _c(grid["rec_idx"], np.int32)]
        self.L = len(self.keep[7])
        self.lig = Lig(*[_p(a) for a in self.keep], self.L, AM, KM, self.P)
        self.gkeep = [_c(grid["flat"], np.float32), _c(grid["offs"], np.int64), _c(grid["dims"], np.int64),
                      _c(grid["origin"], np.float32), _c(grid["lo"], np.float32), _c(grid["hi"], np.float32)]
        self.grid = Grid(*[_p(a) for a in self.gkeep], float(grid["spacing"]), float(grid["penalty"]))
        self.skeep = [_c(sf[1], np.float32), _c(sf[2], np.int32), _c(sf[3], np.int32), _c(sf[4], np.int32)]
        s = SF()
        for i, v in enumerate(np.asarray(sf[0], np.float32)):
            s.prm[i] = float(v)
        s.radius, s.hyd, s.don, s.acc = [_p(a) for a in self.skeep]
        self.sf = s
        if rec is not None:
            self.rkeep = [_c(rec[0], np.float32), _c(rec[1], np.int32), _c(rec[2], np.int32)]
            self.rec = Rec(*[_p(a) for a in self.rkeep], int(np.asarray(rec[0]).shape[1]))
        else:
            self.rkeep = []
            self.rec = Rec(None, None, None, 0)
        self.SD, self.DM = 7 + KM, 6 + KM

    @classmethod
    def from_problem(cls, prob):
        from adock_b200.problem import pack_host
        AM, KM, lig, sf = pack_host(prob)
        gs = prob.gs
        grid = dict(flat=gs.flat.float().cpu().numpy(), origin=gs.origin.cpu().numpy(), lo=gs.lo.cpu().numpy(),
                    hi=gs.hi.cpu().numpy(), rec_idx=prob.rec_idx.cpu().numpy(), offs=gs.offs.cpu().numpy(),
                    dims=gs.dims.cpu().numpy(), spacing=gs.spacing, penalty=gs.penalty)
        rec = None
        if prob.rec is not None:
            rx, rt, rm = prob.rec
            rec = (rx.cpu().numpy(), rt.cpu().numpy(), rm.sum(1).cpu().numpy())
        return cls(AM, KM, lig, sf, grid, rec)

    def energy_grad(self, chain_lig, state, exact=False):
        N = state.shape[0]
        e = np.zeros(N, np.float32)
        g = np.zeros((N, self.DM), np.float32)
        cl, st = _c(chain_lig, np.int32), _c(state, np.float32)
        lib().port_eg(self.lig, self.grid, self.sf, self.rec, int(exact), _p(cl), N, _p(st), _p(e), _p(g))
        return e, g

    def run_mc(self, chain_lig, chain_id, cur, cur_e, best, best_e, init_opt, mc_steps, bfgs_iters, temp, amp_pos,
               amp_rot, seed, step_offset, exact=False, nbr=None, nbr_n=None):
        """In place on float32 numpy cur/cur_e/best/best_e; returns the number of energy evaluations."""
        N = cur.shape[0]
        for x in (cur, cur_e, best, best_e):
            assert x.flags["C_CONTIGUOUS"] and x.dtype == np.float32
        cl, ci = _c(chain_lig, np.int32), _c(chain_id, np.int32)
        nb = [None, None, 0]
        if nbr is not None:
            nbr, nbr_n = _c(nbr, np.int32), _c(nbr_n, np.int32)
            nb = [_p(nbr), _p(nbr_n), int(nbr.shape[1])]
        return int(lib().port_mc(self.lig, self.grid, self.sf, self.rec, int(exact), _p(cl), _p(ci), N, *nb, _p(cur),
                                 _p(cur_e), _p(best), _p(best_e), int(init_opt), int(mc_steps), int(bfgs_iters),
                                 float(temp), float(amp_pos), float(amp_rot),
                                 ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), int(step_offset)))

    def stage_a(self, conf_h, quats, trans, ntrans, cap):
        L, C = conf_h.shape[:2]
        Q, NT = quats.shape[0], trans.shape[1]
        be = np.empty(L * C * Q, np.float32)
        bi = np.empty(L * C * Q, np.int32)
        cf, qu, tr, nt = _c(conf_h, np.float32), _c(quats, np.float32), _c(trans, np.float32), _c(ntrans, np.int32)
        lib().port_stage_a(self.lig, self.grid, _p(cf), C, _p(qu), Q, _p(tr), _p(nt), NT, float(cap), _p(be), _p(bi))
        return be.reshape(L, C * Q), bi.reshape(L, C * Q).astype(np.int64)
