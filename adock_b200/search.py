"""Search entry point of the docking hot path (reference ``src/adock/search.py:322-366, 476-537, 544-671``).

``dock_problem_kernel(prob, boxes_c, boxes_s, cfg, seed, log, stats)`` keeps the reference signature and
returns the same per-ligand dicts ``{coords [n_out, A, 3], affinity, inter, intra, total}``. The stages are the
reference's: Stage A rigid enumeration -> Monte-Carlo + BFGS chains (one persistent launch per segment) ->
BFGS refinement of every chain's best state -> exact polish of the top chains on receptor neighbour lists ->
finalize (float64 re-score on the device, RMSD, greedy clustering at 2 A, affinity with the N_rot factor).

``kernel_factory`` selects the kernel object (default ``B200KernelProblem``); any object with the reference
``KernelProblem`` methods works, which is how the reference's own CPU kernels are timed on the same driver.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from .ligand import internal_coords, pose_coords, random_quat
from .problem import heavy_index

LAST_STATS = {}


def _lattice(center, size, step, device):
    axes = [torch.arange(-float(size[d]) / 2 + 1.0, float(size[d]) / 2 - 1.0 + 1e-6, step, device=device)
            for d in range(3)]
    return torch.stack(torch.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3) + center


@torch.no_grad()
def stage_a_kernel(prob, kp, boxes_c, boxes_s, cfg, gen):
    """Conformers x rotations x probe-filtered translation lattice, per-atom capped nearest-grid energy, top-M
    start poses (search.py:322-366). Returns (t [L,M,3], q [L,M,4], theta [L,M,K], e [L,M])."""
    lb, gs = prob.lb, prob.gs
    dev = lb.ref.device
    L, K = lb.L, lb.K
    C, NT, Q, M = cfg["stageA_conformers"], cfg["stageA_conformer_trials"], cfg["stageA_rotations"], cfg["n_chains"]
    th = (torch.rand((L, NT, K), generator=gen, device=dev) * 2 - 1) * math.pi
    th[:, 0] = 0.0
    th = th * lb.tvalid[:, None, :]
    Xc = internal_coords(lb, th)
    e_intra = prob.intra(Xc)
    ci = torch.topk(-e_intra, min(C, NT), dim=1).indices
    th_c = torch.gather(th, 1, ci[..., None].expand(L, ci.shape[1], K))
    e_c = torch.gather(e_intra, 1, ci)
    Xc = internal_coords(lb, th_c)
    C = Xc.shape[1]
    hidx = heavy_index(lb, kp.AM)
    conf_h = torch.gather(Xc, 2, hidx[:, None, :, None].expand(L, C, kp.AM, 3))
    quats = random_quat((Q,), gen, dev)
    step = cfg["stageA_translation_step"]
    # one lattice per distinct (receptor, box): screening batches share a single box
    Ts, cache = [], {}
    for l in range(L):
        c, s = boxes_c[l], boxes_s[l]
        key = (int(prob.rec_idx[l]), tuple(np.round(np.asarray(c.cpu() if torch.is_tensor(c) else c, float), 6)),
               tuple(np.round(np.asarray(s, float), 6)))
        if key not in cache:
            T = _lattice(torch.as_tensor(c, device=dev, dtype=torch.float32), s, step, dev)
            ep = gs.lookup_nearest(T, torch.zeros(len(T), dtype=torch.long, device=dev),
                                   prob.rec_idx[l].expand(len(T)))
            T = T[ep <= cfg.get("stageA_probe_max", 0.0)]
            cache[key] = T if len(T) else torch.as_tensor(c, device=dev, dtype=torch.float32)[None]
        Ts.append(cache[key])
    nT = torch.tensor([len(T) for T in Ts], device=dev)
    NTm = int(nT.max())
    if len(cache) == 1:
        trans = Ts[0][None].expand(L, NTm, 3).contiguous()
    else:
        trans = torch.zeros(L, NTm, 3, device=dev)
        for l, T in enumerate(Ts):
            trans[l, :len(T)] = T
    best_e, best_i = kp.stage_a(conf_h, quats, trans, nT, cfg.get("stageA_atom_cap", 1e9))
    best_e = best_e.to(dev) + e_c.repeat_interleave(Q, dim=1)
    best_i = best_i.to(dev)
    k = min(M, C * Q)
    top = torch.topk(-best_e, k, dim=1).indices
    if k < M:
        top = top[:, torch.arange(M, device=dev) % k]
    li = torch.arange(L, device=dev)[:, None]
    t0 = trans[li, best_i[li, top]]
    return t0, quats[top % Q], th_c[li, top // Q], best_e[li, top]


@torch.no_grad()
def finalize_kernel(prob, kp, states, chain_lig, L, P, cfg, stats=None):
    """Exact re-score (float64 on the device when the kernel object offers it), heavy-atom RMSD [L,P,P], one
    device->host transfer, greedy clustering, affinity = (inter + intra - intra_top) / (1 + w_rot N_rot)
    (search.py:506-537)."""
    lb = prob.lb
    bt, bq, bth = kp.unpack(states, lb.K)
    X = pose_coords(lb, bt.view(L, P, 3), bq.view(L, P, 4), torch.zeros_like(bt).view(L, P, 3), bth.view(L, P, lb.K))
    if hasattr(kp, "rescore64"):
        et, ei, _ = kp.rescore64(chain_lig, states, exact=prob.rec is not None)
        etot, eintra = et.view(L, P), ei.view(L, P)
    else:
        etot = kp.energy_grad(chain_lig, states, exact=prob.rec is not None)[0].view(L, P).to(X.device)
        eintra = prob.intra(X)
    hv = lb.heavy[:, None, None, :].float()
    D = ((((X[:, :, None] - X[:, None, :]) ** 2).sum(-1) * hv).sum(-1) / hv.sum(-1).clamp(min=1)).sqrt()
    Xc, Ec, Ic, Dc = X.cpu().numpy(), etot.double().cpu().numpy(), eintra.double().cpu().numpy(), D.cpu().numpy()
    if stats is not None:
        stats["d2h_bytes"] = stats.get("d2h_bytes", 0) + Xc.nbytes + Ec.nbytes + Ic.nbytes + Dc.nbytes
    Nt = lb.n_tors_vina.cpu().numpy()
    rw = prob.pot.p["rot_weight"]
    cut, n_out = cfg["cluster_rmsd"], cfg["n_out"]
    results = []
    for l in range(L):
        reps = []
        for i in np.argsort(Ec[l], kind="stable"):
            if all(Dc[l, i, j] >= cut for j in reps):
                reps.append(i)
                if len(reps) == n_out:
                    break
        ri = np.array(reps)
        inter = Ec[l, ri] - Ic[l, ri]
        aff = (inter + Ic[l, ri] - Ic[l, ri[0]]) / (1 + rw * Nt[l])
        results.append({"coords": Xc[l, ri], "affinity": aff, "inter": inter, "intra": Ic[l, ri], "total": Ec[l, ri]})
    return results


def dock_problem_kernel(prob, boxes_c, boxes_s, cfg, seed=0, log=None, stats=None, kernel_factory=None):
    """Engine-v2 search (search.py:544-671): Stage A -> MC + BFGS in segments -> BFGS refinement -> exact polish
    -> finalize. cfg keys as the reference presets (n_chains, mc_steps, mc_segment, bfgs_iters, final_bfgs_iters,
    polish_top, polish_iters, mc_temperature, mc_amp_pos, mc_amp_rot, early_stop_rounds, Stage-A keys)."""
    lb = prob.lb
    dev = lb.ref.device
    if kernel_factory is None:
        from .kernel import B200KernelProblem as kernel_factory
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    L = lb.L
    f = 1
    while (L * cfg["n_chains"] * f * 2 <= cfg.get("min_total_chains", 0)
           and cfg["mc_steps"] // (f * 2) >= cfg.get("min_chain_steps", 32)):
        f *= 2
    if f > 1:
        cfg = dict(cfg, n_chains=cfg["n_chains"] * f, mc_steps=cfg["mc_steps"] // f,
                   mc_segment=max(1, cfg.get("mc_segment", cfg["mc_steps"]) // f))
    M = cfg["n_chains"]
    tick = {}

    def _mark(k):
        if dev.type == "cuda":
            torch.cuda.synchronize(dev)
        tick[k] = time.perf_counter()

    _mark("t0")
    kp = kernel_factory(prob)
    t, q0, th, _ = stage_a_kernel(prob, kp, boxes_c, boxes_s, cfg, gen)
    _mark("stageA")
    N = L * M
    cur = kp.pack(t.reshape(N, 3), q0.reshape(N, 4), th.reshape(N, -1))
    best = cur.clone()
    cur_e = torch.zeros(N, device=dev)
    best_e = torch.full((N,), float("inf"), device=dev)
    chain_lig = torch.arange(L, device=dev, dtype=torch.int32).repeat_interleave(M)
    chain_id = torch.arange(N, device=dev, dtype=torch.int32)
    if cfg.get("autotune", True) and hasattr(kp, "tune") and cfg["mc_steps"] > 0:
        kp.tune(chain_lig, cur)
    seg = max(1, cfg.get("mc_segment", cfg["mc_steps"]))
    n_seg = max(1, math.ceil(cfg["mc_steps"] / seg)) if cfg["mc_steps"] > 0 else 0
    active = torch.ones(L, dtype=torch.bool, device=dev)
    stall = torch.zeros(L, dtype=torch.long, device=dev)
    glob = torch.full((L,), float("inf"), device=dev)
    es_rounds, es_tol = cfg.get("early_stop_rounds", 0), cfg.get("early_stop_tol", 0.01)
    if cfg.get("mc_size_ref", 0) > 0:
        nh = lb.heavy.sum(1).float()
        seg_lim = torch.ceil(n_seg * (50 + nh) / (50 + cfg["mc_size_ref"])).long().clamp(min=1)
        n_seg = int(seg_lim.max()) if n_seg > 0 else 0
    else:
        seg_lim = torch.full((L,), n_seg, dtype=torch.long, device=dev)
    chain_steps = 0
    seed64 = int(seed) * 1_000_003 + 12345
    mc = (cfg["mc_temperature"], cfg["mc_amp_pos"], cfg["mc_amp_rot"], seed64)
    ev = mc_counts0 = None
    if stats is not None and dev.type == "cuda":
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        if hasattr(kp, "evals"):
            mc_counts0 = kp.evals.clone()   # the autotuner's sample launches above also count
    if n_seg == 0:
        kp.run_mc(chain_lig, chain_id, cur, cur_e, best, best_e, True, 0, cfg["bfgs_iters"], *mc, 0)
    for sg in range(n_seg):
        active = active & (seg_lim > sg)
        if bool(active.all()):
            idx = None
        else:
            idx = active.repeat_interleave(M).nonzero().squeeze(1)
            if len(idx) == 0:
                break
        if idx is None:
            kp.run_mc(chain_lig, chain_id, cur, cur_e, best, best_e, sg == 0, seg, cfg["bfgs_iters"], *mc, sg * seg)
            chain_steps += N * seg
        else:
            c_, ce_, b_, be_ = cur[idx].contiguous(), cur_e[idx].contiguous(), best[idx].contiguous(), best_e[idx].contiguous()
            kp.run_mc(chain_lig[idx], chain_id[idx], c_, ce_, b_, be_, sg == 0, seg, cfg["bfgs_iters"], *mc, sg * seg)
            cur[idx], cur_e[idx], best[idx], best_e[idx] = c_, ce_, b_, be_
            chain_steps += len(idx) * seg
        if es_rounds > 0 or log is not None or n_seg > 1:
            gb = best_e.view(L, M).min(1).values
            improved = gb < glob - es_tol
            glob = torch.minimum(glob, gb)
            stall = torch.where(improved, torch.zeros_like(stall), stall + 1)
            if es_rounds > 0:
                active = active & (stall < es_rounds)
            if log is not None:
                log(f"segment {sg}: active {int(active.sum())}/{L}, best E mean {glob.mean().item():.3f}")
    mc_counts = None
    if ev is not None:
        ev[1].record()
        if hasattr(kp, "evals"):
            mc_counts = kp.evals.clone()   # counters of the MC phase alone (no host sync)
    _mark("mc")
    if cfg.get("final_bfgs_iters", 0) > 0:
        fe = torch.zeros(N, device=dev)
        bb = best.clone()
        kp.run_mc(chain_lig, chain_id, best, fe, bb, best_e, True, 0, cfg["final_bfgs_iters"], *mc, 0)
        best = bb
    _mark("refine")
    P = min(cfg.get("polish_top", 0), M)
    if P > 0 and cfg.get("polish_iters", 0) > 0 and prob.rec is not None:
        top = torch.topk(-best_e.view(L, M), P, dim=1).indices
        sel = (top + torch.arange(L, device=dev)[:, None] * M).reshape(-1)
        pc, pb = best[sel].contiguous(), best[sel].clone()
        pe, pbe = torch.zeros(L * P, device=dev), torch.full((L * P,), float("inf"), device=dev)
        nb = (kp.receptor_neighbours(prob, chain_lig[sel], pc, lb.K, cfg.get("polish_nbr_margin", 2.0))
              if cfg.get("polish_nbr_margin", 2.0) > 0 else (None, None))
        kp.run_mc(chain_lig[sel], chain_id[sel], pc, pe, pb, pbe, True, 0, cfg["polish_iters"], *mc, 0, exact=True,
                  nbr=nb[0], nbr_n=nb[1])
        best, M, chain_lig = pb, P, chain_lig[sel]
    _mark("polish")
    res = finalize_kernel(prob, kp, best, chain_lig, L, M, cfg, stats=stats)
    _mark("final")
    if stats is not None and hasattr(kp, "h2d_bytes"):
        stats["h2d_bytes"] = stats.get("h2d_bytes", 0) + kp.h2d_bytes
    if stats is not None:
        ks = list(tick)
        stats.update(widen=f, chain_steps=chain_steps, chain_steps_full=int(seg_lim.sum()) * cfg["n_chains"] * seg,
                     **{f"t_{b}": round(tick[b] - tick[a], 4) for a, b in zip(ks[:-1], ks[1:])})
        if ev is not None:
            stats["mc_ms"] = ev[0].elapsed_time(ev[1])
        if hasattr(kp, "evals"):
            ev_ = kp.evals.tolist()
            stats["evals"], stats["atom_evals"] = int(ev_[0]), int(ev_[1])
        if mc_counts is not None:
            mc_ = (mc_counts - mc_counts0).tolist()
            stats["mc_evals"], stats["mc_atom_evals"] = int(mc_[0]), int(mc_[1])
    return res


def dock_problem(prob, boxes_c, boxes_s, cfg, seed=0, log=None):
    """Search entry point (search.py:399-411): the kernel engine with the stock Vina-family potential."""
    LAST_STATS.clear()
    return dock_problem_kernel(prob, boxes_c, boxes_s, cfg, seed=seed, log=log, stats=LAST_STATS)
