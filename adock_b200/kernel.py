"""``B200KernelProblem``: drop-in for the reference ``KernelProblem`` (``src/adock/mckernel.py:602-726``).

Same constructor argument (a Problem), same attributes (``AM, KM, L, SD, DM``) and the same methods
(``pack``, ``unpack``, ``energy_grad``, ``receptor_neighbours``, ``stage_a``, ``run_mc``) with the same array
layouts; the work runs in the sm_100a kernels of ``libadock_b200.so`` through its C-ABI. Errors are raised as
``RuntimeError`` (argument checks of the C-ABI) or ``AssertionError`` (layout checks, as in the reference).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from .problem import pack_host


class B200KernelProblem:
    """Packs a batch (ligand preps + GridSet + pair potential) into device arrays for the search kernels.

    State layout per chain: [t(3), q(4) (w,x,y,z), theta(KM)], theta in LigandBatch torsion order.
    ``grid_dtype``: 'f32', 'f16' or 'bf16' storage of the maps read by the search (FP32 interpolation)."""

    def __init__(self, prob, grid_dtype="f32"):
        self.AM, self.KM, lig, sf = pack_host(prob)
        AM, KM, L = self.AM, self.KM, prob.lb.L
        dev = prob.gs.origin.device
        if dev.type != "cuda":
            raise RuntimeError("B200KernelProblem needs CUDA tensors (there is no CPU path)")
        self.device = dev
        _lib.load()
        T = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
        ref, typ, tm, ax, axp, axu, pr, na, nt, npairs, rg, P, gsl = lig
        self.P = int(P)
        self.t_lig = [T(ref), T(typ), T(tm), T(ax), T(axp), T(axu), T(pr), T(na), T(nt), T(npairs), T(rg), T(gsl),
                      prob.rec_idx.to(device=dev, dtype=torch.int32).contiguous()]
        self.na_host, self.nt_host = na.copy(), nt.copy()
        self.h2d_bytes = int(sum(t.numel() * t.element_size() for t in self.t_lig[:12]))
        lt = _lib.Ligands()
        for name, t in zip(("ref", "typ", "tm", "ax", "axp", "axu", "pr", "na", "nt", "np", "rg", "gslot", "rec_idx"),
                           self.t_lig):
            setattr(lt, name, _lib.ptr(t))
        lt.L, lt.AM, lt.KM, lt.P = L, AM, KM, self.P
        self.c_lig = lt
        # scoring tables
        sfp = dict(prob.pot.p)
        sfp.setdefault("radius", sf[1])
        sfp.setdefault("hydrophobic", sf[2])
        sfp.setdefault("donor", sf[3])
        sfp.setdefault("acceptor", sf[4])
        self.c_sf = _lib.make_sf(sfp)
        # grids
        gs = prob.gs
        self.grid_dtype = grid_dtype
        flat, code = gs.storage(grid_dtype)
        self.t_grid = [flat, gs.offs.to(dev, torch.int64).contiguous(), gs.dims.to(dev, torch.int64).contiguous(),
                       gs.origin.float().contiguous(), gs.lo.float().contiguous(), gs.hi.float().contiguous()]
        sizes = torch.diff(self.t_grid[1], append=torch.tensor([flat.numel()], device=dev))
        self.t_nmaps = (sizes // self.t_grid[2].prod(1)).to(torch.int32).contiguous()
        g = _lib.Grids()
        g.flat, g.offs, g.dims, g.origin, g.lo, g.hi = [_lib.ptr(t) for t in self.t_grid]
        g.R, g.dtype, g.spacing, g.penalty = int(gs.origin.shape[0]), code, float(gs.spacing), float(gs.penalty)
        g.nmaps = _lib.ptr(self.t_nmaps)
        self.c_grids = g
        # receptor atoms for exact mode
        r = _lib.Receptors()
        if prob.rec is not None:
            rx, rt, rm = prob.rec
            self.t_rec = [rx.float().to(dev).contiguous(), rt.to(dev, torch.int32).contiguous(),
                          rm.sum(1).to(dev, torch.int32).contiguous()]
            r.xyz, r.typ, r.n = [_lib.ptr(t) for t in self.t_rec]
            r.RN = int(rx.shape[1])
        else:
            self.t_rec = []
            r.xyz = r.typ = r.n = None
            r.RN = 0
        self.c_rec = r
        # B200 working layout
        self.t_work = [torch.empty(L * AM * 4, dtype=torch.float32, device=dev),
                       torch.empty(L * AM, dtype=torch.int32, device=dev),
                       torch.empty(L * KM * 2 * 4, dtype=torch.float32, device=dev),
                       torch.empty(L * (-(-self.P // 32) * 32) * 2, dtype=torch.int32, device=dev),
                       torch.empty(L * 4, dtype=torch.int32, device=dev),
                       torch.empty(L, dtype=torch.float32, device=dev)]
        w = _lib.Work()
        w.atoms, w.masks, w.tors, w.pairs, w.info, w.rg = [_lib.ptr(t) for t in self.t_work]
        self.c_work = w
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.evals = torch.zeros(2, dtype=torch.int64, device=dev)  # energy evaluations, atom evaluations
        with torch.cuda.device(dev):
            _lib.call("adock_prepare", self.c_lig, self.c_sf, self.c_work, _lib.stream_ptr())
        self.L, self.SD, self.DM = L, 7 + KM, 6 + KM

    # ---- state packing ----
    def pack(self, t, q, theta):
        """t [N,3], q [N,4], theta [N,K<=KM] -> state [N, SD] float32 contiguous."""
        N, K = theta.shape
        s = torch.zeros(N, self.SD, device=t.device, dtype=torch.float32)
        s[:, :3], s[:, 3:7] = t, q
        s[:, 7:7 + min(K, self.KM)] = theta[:, :self.KM]
        return s.contiguous()

    def unpack(self, s, K):
        th = torch.zeros(s.shape[0], K, device=s.device, dtype=s.dtype)
        th[:, :min(K, self.KM)] = s[:, 7:7 + min(K, self.KM)]
        th = torch.remainder(th + math.pi, 2 * math.pi) - math.pi
        return s[:, :3].clone(), s[:, 3:7] / s[:, 3:7].norm(dim=-1, keepdim=True), th

    def _i32(self, x):
        return x.to(device=self.device, dtype=torch.int32).contiguous()

    # ---- kernels ----
    def energy_grad(self, chain_lig, state, exact=False):
        """chain_lig int32 [N], state [N, SD] -> (e [N], g [N, DM])."""
        N = state.shape[0]
        e = torch.zeros(N, device=self.device)
        g = torch.zeros(N, self.DM, device=self.device)
        if exact:
            assert self.c_rec.RN > 0, "exact mode needs receptor atoms (Problem.rec)"
        cl = self._i32(chain_lig)
        st = state.to(self.device, torch.float32).contiguous()
        with torch.cuda.device(self.device):
            _lib.call("adock_eg", self.c_lig, self.c_work, self.c_grids, self.c_sf, self.c_rec, _lib.ptr(cl), N,
                      _lib.ptr(st), _lib.ptr(e), _lib.ptr(g), int(exact), _lib.stream_ptr())
        return e, g

    def chain_order(self, chain_lig):
        """Processing order for the persistent MC kernel: most expensive chains first (cost ~ BFGS iterations x
        (atoms + pairs / 32))."""
        cl = chain_lig.long()
        if not hasattr(self, "_cost"):
            na = torch.as_tensor(self.na_host, device=self.device).float()
            npr = self.t_lig[9].float()
            self._cost = (25 + na) / 3 * (na + npr / 16 + 8)
        return torch.argsort(-self._cost[cl], stable=True).to(torch.int32)

    def tune(self, chain_lig, state):
        """Pick the MC launch variant for this batch with the autotuner (cached per shape and device)."""
        from .autotune import tune_mc
        self.mc_variant = tune_mc(self, self._i32(chain_lig), state.contiguous())
        return self.mc_variant

    def prop_features(self, chain_lig, state, cur_e=None, hint=None):
        """Proposal-network feature rows [N, 320] (BF16) of N states; with the states' energies cur_e [N] and the
        ligand-best rows hint [L, 32] (prop_hint) the ligand-best columns are filled, else they are 0."""
        N = state.shape[0]
        out = torch.empty(N, 320, dtype=torch.bfloat16, device=self.device)
        cl = self._i32(chain_lig)
        st = state.to(self.device, torch.float32).contiguous()
        ce = None if cur_e is None else cur_e.to(self.device, torch.float32).contiguous()
        if hint is not None:
            assert hint.shape == (self.L, 32) and hint.dtype == torch.float32 and hint.is_contiguous()
        with torch.cuda.device(self.device):
            _lib.call("adock_prop_features", self.c_lig, self.c_work, self.c_grids, self.c_sf, _lib.ptr(cl), N,
                      _lib.ptr(st), _lib.ptr(ce), _lib.ptr(hint), _lib.ptr(out), _lib.stream_ptr())
        return out

    def prop_hint(self, chain_lig, best, best_e):
        """Ligand-best rows [L, 32]: per ligand, the best state (t, q, torsions 0..19) of its chain with the lowest
        finite best energy, that energy (column 27) and a valid flag (column 28); zeros for a ligand without one."""
        N = best.shape[0]
        hint = torch.empty(self.L, 32, device=self.device)
        keys = torch.empty(self.L, dtype=torch.int64, device=self.device)
        cl = self._i32(chain_lig)
        b = best.float().contiguous()
        be = best_e.float().contiguous()
        with torch.cuda.device(self.device):
            _lib.call("adock_prop_hint", self.L, N, _lib.ptr(cl), _lib.ptr(b), int(b.shape[1]), _lib.ptr(be),
                      _lib.ptr(keys), _lib.ptr(hint), _lib.stream_ptr())
        return hint

    def prop_sample(self, chain_lig, chain_id, net_out, state, k, seed, segment, n_comp=1):
        """Target states [N, k, 32] (t, q, torsions 0..19) drawn from the network's Gaussian (net_out [N, 64]) over
        moves from the states state [N, SD] the network read."""
        N = net_out.shape[0]
        targets = torch.empty(N, k, 32, device=self.device)
        cl, ci = self._i32(chain_lig), self._i32(chain_id)
        no = net_out.float().contiguous()
        st = state.float().contiguous()
        assert st.shape == (N, self.SD)
        with torch.cuda.device(self.device):
            _lib.call("adock_prop_sample", self.c_lig, self.c_work, _lib.ptr(cl), _lib.ptr(ci), N, _lib.ptr(no),
                      _lib.ptr(st), self.SD, int(k), int(n_comp), int(seed) & 0xFFFFFFFFFFFFFFFF, int(segment),
                      _lib.ptr(targets),
                      _lib.stream_ptr())
        return targets

    def run_mc(self, chain_lig, chain_id, cur, cur_e, best, best_e, init_opt, mc_steps, bfgs_iters, temp,
               amp_pos, amp_rot, seed, step_offset, exact=False, nbr=None, nbr_n=None, order=None, variant=None,
               prop=None, prop_stats=None, log=None, prop_frac=1.0, lig_active=None, prop_tries=1, hint=None):
        """In place on cur/cur_e/best/best_e (float32 contiguous CUDA tensors). exact=True with nbr [N, NB] int32 /
        nbr_n [N]: each chain's exact inter energy loops only over its receptor-atom neighbour list.
        variant: MC launch variant (default: the tuned one, else the library default).
        prop: learned moves [N, k, 32] for steps 0..k-1 of this launch (plain MC fallback after 8 rejections);
        prop_stats: int64 [4] counters; log: (x BF16 [cap, 320], y [cap, 32], n int32 [1]) training-data log;
        prop_frac: fraction of steps that take the learned move (the others take the plain random move);
        lig_active: int32 [L] device flags, chains of ligands with 0 are left unchanged (None: all run);
        prop_tries: candidate targets per learned step (prop then holds steps x prop_tries targets per chain);
        hint: ligand-best rows [L, 32] (prop_hint) for the logged features (None: those columns are 0)."""
        N = cur.shape[0]
        if N == 0:
            return
        for x in (cur, cur_e, best, best_e):
            assert x.is_contiguous() and x.dtype == torch.float32 and x.device.type == "cuda"
        if exact:
            assert self.c_rec.RN > 0, "exact mode needs receptor atoms (Problem.rec)"
        cl, ci = self._i32(chain_lig), self._i32(chain_id)
        if order is None:
            order = self.chain_order(cl)
        a = _lib.McArgs()
        a.chain_lig, a.chain_id, a.n_chains = _lib.ptr(cl), _lib.ptr(ci), N
        keep = [cl, ci, order]
        if nbr is not None:
            nbr, nbr_n = self._i32(nbr), self._i32(nbr_n)
            keep += [nbr, nbr_n]
            a.nbr, a.nbr_n, a.nb_max = _lib.ptr(nbr), _lib.ptr(nbr_n), int(nbr.shape[1])
        else:
            a.nbr = a.nbr_n = None
            a.nb_max = 0
        a.cur, a.cur_e, a.best, a.best_e = _lib.ptr(cur), _lib.ptr(cur_e), _lib.ptr(best), _lib.ptr(best_e)
        a.init_opt, a.mc_steps, a.bfgs_iters = int(init_opt), int(mc_steps), int(bfgs_iters)
        a.temp, a.amp_pos, a.amp_rot = float(temp), float(amp_pos), float(amp_rot)
        a.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        a.step_offset, a.exact = int(step_offset), int(exact)
        a.order, a.queue, a.evals = _lib.ptr(order), _lib.ptr(self.queue), _lib.ptr(self.evals)
        a.variant = int(getattr(self, "mc_variant", 0) if variant is None else variant)
        if prop is not None:
            assert prop.is_contiguous() and prop.shape[0] == N and prop.shape[2] == 32 and prop.dtype == torch.float32
            a.prop, a.prop_k = _lib.ptr(prop), int(prop.shape[1])
            a.prop_frac = float(prop_frac)
            a.prop_tries = int(prop_tries)
            keep.append(prop)
        if prop_stats is not None:
            a.prop_stats = _lib.ptr(prop_stats)
        if log is not None:
            lx, ly, ln = log
            a.log_x, a.log_y, a.log_n, a.log_cap = _lib.ptr(lx), _lib.ptr(ly), _lib.ptr(ln), int(lx.shape[0])
        if lig_active is not None:
            assert lig_active.dtype == torch.int32 and lig_active.is_contiguous() and lig_active.numel() == self.L
            a.lig_active = _lib.ptr(lig_active)
            keep.append(lig_active)
        if hint is not None:
            assert hint.shape == (self.L, 32) and hint.dtype == torch.float32 and hint.is_contiguous()
            a.hint = _lib.ptr(hint)
            keep.append(hint)
        with torch.cuda.device(self.device):
            _lib.call("adock_mc", self.c_lig, self.c_work, self.c_grids, self.c_sf, self.c_rec, a, _lib.stream_ptr())
        self._keep_mc = keep

    def stage_a(self, conf_h, quats, trans, ntrans, cap):
        """conf_h [L, C, AM, 3] heavy-atom conformer coords (ligand frame), quats [Q, 4], trans [L, NT, 3],
        ntrans [L] -> (best_e [L, C*Q], best_i [L, C*Q] index into trans)."""
        L, C = conf_h.shape[:2]
        Q, NT = quats.shape[0], trans.shape[1]
        be = torch.empty(L * C * Q, device=self.device)
        bi = torch.empty(L * C * Q, dtype=torch.int32, device=self.device)
        keep = [conf_h.float().contiguous(), quats.float().contiguous(), trans.float().contiguous(),
                self._i32(ntrans)]
        with torch.cuda.device(self.device):
            _lib.call("adock_stage_a", self.c_lig, self.c_work, self.c_grids, self.c_sf, _lib.ptr(keep[0]), C,
                      _lib.ptr(keep[1]), Q, _lib.ptr(keep[2]), _lib.ptr(keep[3]), NT, float(cap), _lib.ptr(be),
                      _lib.ptr(bi), _lib.stream_ptr())
        return be.view(L, C * Q), bi.view(L, C * Q).long()

    # ---- device pipeline of the search driver (adock_b200.search) ----
    def conformers(self, NT, C, seed):
        """Stage-A conformers: (theta [L, C, KM], heavy-atom coordinates [L, C, AM, 3], intra energies [L, C])."""
        L = self.L
        theta = torch.empty(L, C, self.KM, device=self.device)
        conf = torch.empty(L, C, self.AM, 3, device=self.device)
        e = torch.empty(L, C, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("adock_conformers", self.c_lig, self.c_work, self.c_sf, int(NT), int(C),
                      int(seed) & 0xFFFFFFFFFFFFFFFF, _lib.ptr(theta), _lib.ptr(conf), _lib.ptr(e), _lib.stream_ptr())
        return theta, conf, e

    def lattice(self, B, box, box_rec, box_slot, box_n, step, probe_max, nt_max):
        """Probe-filtered translation lattices of B boxes: (trans [B, nt_max, 3], counts [B] int32)."""
        trans = torch.empty(B, nt_max, 3, device=self.device)
        cnt = torch.empty(B, dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("adock_lattice", self.c_grids, int(B), _lib.ptr(box), _lib.ptr(box_rec), _lib.ptr(box_slot),
                      _lib.ptr(box_n), float(step), float(probe_max), int(nt_max), _lib.ptr(trans), _lib.ptr(cnt),
                      _lib.stream_ptr())
        return trans, cnt

    def stage_a_boxes(self, conf, quats, trans, ntrans, lig_box, cap):
        """Rigid Stage-A scores with per-box lattices: (best_e [L, C*Q], best_i [L, C*Q] int32)."""
        L, C = conf.shape[:2]
        Q = quats.shape[0]
        be = torch.empty(L, C * Q, device=self.device)
        bi = torch.empty(L, C * Q, dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("adock_stage_a_boxes", self.c_lig, self.c_work, self.c_grids, self.c_sf, _lib.ptr(conf), int(C),
                      _lib.ptr(quats), int(Q), _lib.ptr(trans), _lib.ptr(ntrans), int(trans.shape[1]),
                      _lib.ptr(lig_box), float(cap), _lib.ptr(be), _lib.ptr(bi), _lib.stream_ptr())
        return be, bi

    def select_starts(self, best_e, best_i, e_conf, quats, theta, trans, lig_box, M):
        """M start states per ligand (state [L*M, SD], Stage-A energies [L*M])."""
        L, C = e_conf.shape
        Q = quats.shape[0]
        state = torch.zeros(L * M, self.SD, device=self.device)
        e = torch.empty(L * M, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("adock_select_starts", L, int(C), int(Q), self.KM, int(M), _lib.ptr(best_e), _lib.ptr(best_i),
                      _lib.ptr(e_conf), _lib.ptr(quats), _lib.ptr(theta), _lib.ptr(trans), _lib.ptr(lig_box),
                      int(trans.shape[1]), _lib.ptr(state), _lib.ptr(e), _lib.stream_ptr())
        return state, e

    def segment_update(self, L, M, seg, next_sg, es_rounds, es_tol, best_e, seg_lim, glob, stall, active,
                       chain_steps):
        """Per-ligand budget and early-stop flags after an MC segment (in place on glob, stall, active)."""
        with torch.cuda.device(self.device):
            _lib.call("adock_segment_update", int(L), int(M), int(seg), int(next_sg), int(es_rounds), float(es_tol),
                      _lib.ptr(best_e), _lib.ptr(seg_lim), _lib.ptr(glob), _lib.ptr(stall), _lib.ptr(active),
                      _lib.ptr(chain_steps), _lib.stream_ptr())

    def cluster(self, e_total, X, L, P, cut, n_out):
        """Greedy cluster representatives of P poses per ligand: (reps [L, n_out] int32, counts [L] int32)."""
        reps = torch.empty(L, n_out, dtype=torch.int32, device=self.device)
        cnt = torch.empty(L, dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("adock_cluster", self.c_work, int(L), int(P), _lib.ptr(e_total.contiguous()),
                      _lib.ptr(X.contiguous()), int(X.shape[1]), float(cut), int(n_out), _lib.ptr(reps), _lib.ptr(cnt),
                      _lib.stream_ptr())
        return reps, cnt

    def pose_atoms(self, lb, chain_lig, states):
        """All-atom world coordinates [n, A, 3] of states (atom order and padding of the LigandBatch lb)."""
        if not hasattr(self, "_atoms_all") or self._atoms_all[0] is not lb:
            ref = lb.ref.to(self.device, torch.float32).contiguous()
            bits = torch.as_tensor(lb.atom_masks().view(np.int32), device=self.device).contiguous()
            self._atoms_all = (lb, ref, bits)
        _, ref, bits = self._atoms_all
        n = states.shape[0]
        X = torch.empty(n, lb.A, 3, device=self.device)
        cl = self._i32(chain_lig)
        st = states.to(self.device, torch.float32).contiguous()
        with torch.cuda.device(self.device):
            _lib.call("adock_pose_atoms", self.c_work, self.KM, _lib.ptr(ref), _lib.ptr(bits), int(lb.A), _lib.ptr(cl),
                      int(n), _lib.ptr(st), _lib.ptr(X), _lib.stream_ptr())
        return X

    def receptor_neighbours(self, prob, chain_lig, states, K, margin):
        """Per chain: indices of receptor atoms within cutoff + margin of any heavy atom of the chain's pose,
        in receptor order (mckernel.py:662-688). Returns (nbr [N, NB] int32, nbr_n [N] int32)."""
        assert self.c_rec.RN > 0, "neighbour lists need receptor atoms (Problem.rec)"
        cut = float(prob.pot.p["cutoff"]) + margin
        N = states.shape[0]
        cl = self._i32(chain_lig)
        st = states.to(self.device, torch.float32).contiguous()
        cnt = torch.zeros(N, dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.call("adock_neighbours", self.c_lig, self.c_work, self.c_sf, self.c_rec, _lib.ptr(cl), N, _lib.ptr(st),
                      cut, None, _lib.ptr(cnt), 0, _lib.stream_ptr())
            NB = max(1, int(cnt.max()) if N else 1)
            nbr = torch.zeros(N, NB, dtype=torch.int32, device=self.device)
            _lib.call("adock_neighbours", self.c_lig, self.c_work, self.c_sf, self.c_rec, _lib.ptr(cl), N, _lib.ptr(st),
                      cut, _lib.ptr(nbr), _lib.ptr(cnt), NB, _lib.stream_ptr())
        return nbr, cnt

    def rescore64(self, chain_lig, states, exact=True):
        """Float64 re-score on the device: (e_total [N] f64, e_intra [N] f64, X [N, AM, 3] f32 world coordinates).
        exact=True uses pairwise inter energies over all receptor atoms (needs Problem.rec), else the grid."""
        N = states.shape[0]
        cl = self._i32(chain_lig)
        st = states.to(self.device, torch.float32).contiguous()
        et = torch.zeros(N, dtype=torch.float64, device=self.device)
        ei = torch.zeros(N, dtype=torch.float64, device=self.device)
        X = torch.zeros(N, self.AM, 3, device=self.device)
        rec = self.c_rec if exact else _lib.Receptors()
        if exact:
            assert self.c_rec.RN > 0, "exact re-score needs receptor atoms (Problem.rec)"
        with torch.cuda.device(self.device):
            _lib.call("adock_rescore64", self.c_lig, self.c_work, self.c_grids, self.c_sf, rec, _lib.ptr(cl), N,
                      _lib.ptr(st), _lib.ptr(et), _lib.ptr(ei), _lib.ptr(X), _lib.stream_ptr())
        return et, ei, X


# reference name, so callers that select the class by name find it
KernelProblem = B200KernelProblem
