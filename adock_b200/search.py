"""Search entry point of the docking hot path as a device pipeline (reference interface
``src/adock/search.py:544`` ``dock_problem_kernel`` and ``:399`` ``dock_problem``).

``dock_problem_kernel(prob, boxes_c, boxes_s, cfg, seed, log, stats)`` returns, per ligand, the reference's result
dict ``{coords [n, A, 3], affinity, inter, intra, total}`` (n <= n_out cluster representatives, best first) and
follows the reference's stages and preset keys. Every stage is a kernel on the caller's stream; the host only
queues launches and reads the results once at the end:

=============  ==========================================================================================
Stage A        ``adock_conformers`` (NT torsion sets -> C lowest-intra conformers), ``adock_lattice`` (probe-
               filtered translations, one lattice per distinct box), ``adock_stage_a_boxes`` (capped rigid
               scores of conformer x rotation x translation), ``adock_select_starts`` (M start states per ligand)
MC             ``adock_mc`` per segment of ``mc_segment`` steps; ligands whose budget (``mc_size_ref``) or early
               stop (``early_stop_rounds``) ended keep their chains untouched through a per-ligand flag that
               ``adock_segment_update`` maintains on the device (the reference compacts active chains on the host)
refine         ``adock_mc`` with 0 steps and ``final_bfgs_iters`` BFGS iterations on each chain's best state
polish         the ``polish_top`` best chains per ligand, ``adock_neighbours``, ``adock_mc`` in exact mode
finalize       ``adock_rescore64`` (float64 exact energies), ``adock_cluster`` (greedy 2 A representatives),
               ``adock_pose_atoms`` (all-atom coordinates of the representatives), affinity
               (inter + intra - intra_top) / (1 + w_rot N_rot), one device -> host copy
=============  ==========================================================================================

The polish sizes its neighbour lists from a device count, which is the one host wait before the end. The random
streams are the library's own counter-based ones (conformer angles, rotations, MC moves), so a seed gives the same
search on every run, but not the reference's torch-generator draws.
"""
from __future__ import annotations

import math

import numpy as np
import torch

LAST_STATS = {}
_SEED_MIX = 1_000_003


def _widen(cfg, L):
    """More, shorter chains at equal chain-steps while L * n_chains stays under ``min_total_chains``."""
    f = 1
    while (L * cfg["n_chains"] * f * 2 <= cfg.get("min_total_chains", 0)
           and cfg["mc_steps"] // (f * 2) >= cfg.get("min_chain_steps", 32)):
        f *= 2
    if f == 1:
        return cfg, 1
    return dict(cfg, n_chains=cfg["n_chains"] * f, mc_steps=cfg["mc_steps"] // f,
                mc_segment=max(1, cfg.get("mc_segment", cfg["mc_steps"]) // f)), f


def _host(x, dtype=np.float64):
    return np.asarray(x.detach().cpu() if torch.is_tensor(x) else x, dtype)


def _boxes(prob, boxes_c, boxes_s, step):
    """Distinct (receptor, centre, size) boxes of the batch: table [B, 6], receptor [B], lattice points per axis
    [B, 3], and the box of each ligand [L]."""
    L = prob.lb.L
    c = _host(boxes_c).reshape(L, 3)
    s = np.stack([_host(x) for x in boxes_s]).reshape(L, 3) if len(boxes_s) == L else np.tile(_host(boxes_s), (L, 1))
    rec = _host(prob.rec_idx, np.int64).reshape(L)
    key = np.concatenate([rec[:, None].astype(np.float64), np.round(c, 6), np.round(s, 6)], 1)
    uniq, first, lig_box = np.unique(key, axis=0, return_index=True, return_inverse=True)
    table = np.concatenate([c[first], s[first]], 1).astype(np.float32)
    # points per axis of arange(-s/2 + 1, s/2 - 1 + 1e-6, step)
    n = np.array([[len(np.arange(-sd / 2 + 1.0, sd / 2 - 1.0 + 1e-6, step)) for sd in row] for row in s[first]],
                 np.int32)
    return table, rec[first].astype(np.int32), np.maximum(n, 1), lig_box.reshape(L).astype(np.int32)


def _quaternions(Q, seed):
    """Q uniformly distributed unit quaternions (w, x, y, z) from the seed."""
    g = np.random.default_rng(np.random.SeedSequence([int(seed) & 0xFFFFFFFF, 0x51A7E]))
    q = g.standard_normal((Q, 4))
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


@torch.no_grad()
def stage_a_starts(prob, kp, boxes_c, boxes_s, cfg, seed):
    """Stage A on the device: start states [L * M, 7 + KM] (ligand-major) and their Stage-A energies [L * M]."""
    dev = kp.device
    L, M = prob.lb.L, cfg["n_chains"]
    NT = cfg["stageA_conformer_trials"]
    C = min(cfg["stageA_conformers"], NT)
    Q = cfg["stageA_rotations"]
    step = cfg["stageA_translation_step"]
    table, box_rec, box_n, lig_box = _boxes(prob, boxes_c, boxes_s, step)
    slot = prob.gs.slot.cpu().numpy() if torch.is_tensor(prob.gs.slot) else np.asarray(prob.gs.slot)
    box_slot = slot[box_rec, 0].astype(np.int32)          # type 0 (C_H) is the probe, as in the reference
    assert (box_slot >= 0).all(), "the probe type (C_H) has no map"
    nt_max = int(box_n.prod(1).max())
    host = {"table": table, "box_rec": box_rec, "box_slot": box_slot, "box_n": box_n, "lig_box": lig_box,
            "quats": _quaternions(Q, seed)}
    d = {k: torch.as_tensor(v, device=dev) for k, v in host.items()}
    theta, conf, e_conf = kp.conformers(NT, C, seed)
    trans, ntrans = kp.lattice(len(table), d["table"], d["box_rec"], d["box_slot"], d["box_n"], step,
                               cfg.get("stageA_probe_max", 0.0), nt_max)
    best_e, best_i = kp.stage_a_boxes(conf, d["quats"], trans, ntrans, d["lig_box"], cfg.get("stageA_atom_cap", 1e9))
    state, e_start = kp.select_starts(best_e, best_i, e_conf, d["quats"], theta, trans, d["lig_box"], M)
    kp._keep_stage_a = (d, trans, ntrans)
    return state, e_start


@torch.no_grad()
def finalize_device(prob, kp, states, chain_lig, L, P, cfg, stats=None):
    """Float64 exact re-score, greedy clustering and all-atom coordinates of the representatives on the device,
    then one device -> host copy; returns the per-ligand result dicts."""
    lb = prob.lb
    n_out = int(cfg["n_out"])
    et, ei, Xh = kp.rescore64(chain_lig, states, exact=prob.rec is not None)
    reps, n_reps = kp.cluster(et, Xh, L, P, cfg["cluster_rmsd"], n_out)
    dev = kp.device
    pick = (torch.arange(L, device=dev)[:, None] * P + reps.clamp(min=0).long()).reshape(-1)
    X = kp.pose_atoms(lb, chain_lig[pick], states[pick])                       # [L * n_out, A, 3]
    total, intra = et[pick].view(L, n_out), ei[pick].view(L, n_out)
    inter = total - intra
    ntv = lb.n_tors_vina.to(dev, torch.float64)
    affinity = (total - intra[:, :1]) / (1.0 + float(prob.pot.p["rot_weight"]) * ntv[:, None])
    energies = torch.stack([affinity, inter, intra, total], 0)               # [4, L, n_out] float64
    blob = torch.cat([X.reshape(-1).view(torch.uint8), energies.reshape(-1).view(torch.uint8),
                      n_reps.to(torch.int32).view(torch.uint8)]).cpu().numpy()
    nx = X.numel() * 4
    Xc = blob[:nx].view(np.float32).reshape(L, n_out, lb.A, 3)
    E = blob[nx:nx + energies.numel() * 8].view(np.float64).reshape(4, L, n_out)
    k = blob[nx + energies.numel() * 8:].view(np.int32)
    if stats is not None:
        stats["d2h_bytes"] = stats.get("d2h_bytes", 0) + int(blob.nbytes)
    return [{"coords": Xc[l, :k[l]], "affinity": E[0, l, :k[l]], "inter": E[1, l, :k[l]], "intra": E[2, l, :k[l]],
             "total": E[3, l, :k[l]]} for l in range(L)]


def dock_problem_kernel(prob, boxes_c, boxes_s, cfg, seed=0, log=None, stats=None, kernel_factory=None):
    """Stage A -> MC + BFGS in segments -> BFGS refinement -> exact polish -> finalize, all on the device.

    cfg: the reference preset keys (n_chains, mc_steps, mc_segment, mc_size_ref, bfgs_iters, final_bfgs_iters,
    polish_top, polish_iters, polish_nbr_margin, mc_temperature, mc_amp_pos, mc_amp_rot, early_stop_rounds,
    early_stop_tol, min_total_chains, min_chain_steps, stageA_*, cluster_rmsd, n_out); cfg["autotune"] = False
    skips the launch-variant autotuner. kernel_factory(prob) may supply the kernel object (default
    ``B200KernelProblem``), e.g. one built once and reused across calls."""
    lb = prob.lb
    L = lb.L
    cfg, widen = _widen(cfg, L)
    M = cfg["n_chains"]
    if kernel_factory is None:
        from .kernel import B200KernelProblem as kernel_factory
    kp = kernel_factory(prob)
    dev = kp.device
    marks = {}

    def mark(name):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks[name] = ev

    mark("t0")
    # ---- Stage A
    N = L * M
    cur, _ = stage_a_starts(prob, kp, boxes_c, boxes_s, cfg, seed)
    mark("stageA")
    best = cur.clone()
    cur_e = torch.zeros(N, device=dev)
    best_e = torch.full((N,), float("inf"), device=dev)
    chain_lig = torch.arange(L, device=dev, dtype=torch.int32).repeat_interleave(M)
    chain_id = torch.arange(N, device=dev, dtype=torch.int32)
    mc = (cfg["mc_temperature"], cfg["mc_amp_pos"], cfg["mc_amp_rot"], int(seed) * _SEED_MIX + 12345)
    if cfg.get("autotune", True) and hasattr(kp, "tune") and cfg["mc_steps"] > 0:
        kp.tune(chain_lig, cur)
    # ---- MC in segments with per-ligand budgets and early stop kept on the device
    seg = max(1, cfg.get("mc_segment", cfg["mc_steps"]))
    n_seg = math.ceil(cfg["mc_steps"] / seg) if cfg["mc_steps"] > 0 else 0
    if cfg.get("mc_size_ref", 0) > 0 and n_seg > 0:
        nh = np.array([int(np.asarray(p.heavy, bool).sum()) for p in lb.preps], np.float64)
        seg_lim = np.maximum(np.ceil(n_seg * (50 + nh) / (50 + cfg["mc_size_ref"])), 1).astype(np.int32)
        n_seg = int(seg_lim.max())
    else:
        seg_lim = np.full(L, n_seg, np.int32)
    seg_lim_d = torch.as_tensor(seg_lim, device=dev)
    active = (seg_lim_d > 0).to(torch.int32)
    glob = torch.full((L,), float("inf"), device=dev)
    stall = torch.zeros(L, dtype=torch.int32, device=dev)
    chain_steps = torch.zeros(1, dtype=torch.int64, device=dev)
    es_rounds, es_tol = int(cfg.get("early_stop_rounds", 0)), float(cfg.get("early_stop_tol", 0.01))
    evals0 = kp.evals.clone() if hasattr(kp, "evals") else None   # the autotuner's sample launches also count
    mark("mc0")
    if n_seg == 0:
        kp.run_mc(chain_lig, chain_id, cur, cur_e, best, best_e, True, 0, cfg["bfgs_iters"], *mc, 0)
    for sg in range(n_seg):
        kp.run_mc(chain_lig, chain_id, cur, cur_e, best, best_e, sg == 0, seg, cfg["bfgs_iters"], *mc, sg * seg,
                  lig_active=active if n_seg > 1 else None)
        kp.segment_update(L, M, seg, sg + 1, es_rounds, es_tol, best_e, seg_lim_d, glob, stall, active, chain_steps)
        if log is not None:
            log(f"segment {sg}: active {int(active.sum())}/{L}, best E mean {glob.mean().item():.3f}")
    mark("mc")
    evals_mc = kp.evals.clone() if evals0 is not None else None
    # ---- refinement of every chain's best state
    if cfg.get("final_bfgs_iters", 0) > 0:
        refined_e = torch.zeros(N, device=dev)
        refined = best.clone()
        kp.run_mc(chain_lig, chain_id, best, refined_e, refined, best_e, True, 0, cfg["final_bfgs_iters"], *mc, 0)
        best = refined
    mark("refine")
    # ---- exact polish of the best chains of each ligand on receptor neighbour lists
    P = min(cfg.get("polish_top", 0), M)
    if P > 0 and cfg.get("polish_iters", 0) > 0 and prob.rec is not None:
        top = torch.topk(best_e.view(L, M), P, dim=1, largest=False).indices
        pick = (top + torch.arange(L, device=dev)[:, None] * M).reshape(-1)
        start = best[pick].contiguous()
        polished = start.clone()
        margin = cfg.get("polish_nbr_margin", 2.0)
        nbr, nbr_n = (kp.receptor_neighbours(prob, chain_lig[pick], start, lb.K, margin) if margin > 0
                      else (None, None))
        kp.run_mc(chain_lig[pick], chain_id[pick], start, torch.zeros(L * P, device=dev), polished,
                  torch.full((L * P,), float("inf"), device=dev), True, 0, cfg["polish_iters"], *mc, 0, exact=True,
                  nbr=nbr, nbr_n=nbr_n)
        best, M, chain_lig = polished, P, chain_lig[pick]
    mark("polish")
    res = finalize_device(prob, kp, best, chain_lig, L, M, cfg, stats=stats)   # ends with the one host copy
    mark("final")
    torch.cuda.current_stream().synchronize()
    if stats is not None:
        phases = (("t_stageA", "t0", "stageA"), ("t_tune", "stageA", "mc0"), ("t_mc", "mc0", "mc"),
                  ("t_refine", "mc", "refine"), ("t_polish", "refine", "polish"), ("t_final", "polish", "final"))
        stats.update(widen=widen, chain_steps=int(chain_steps.item()),
                     chain_steps_full=int(seg_lim.sum()) * cfg["n_chains"] * seg,
                     **{k: round(marks[a].elapsed_time(marks[b]) / 1e3, 4) for k, a, b in phases})
        stats["mc_ms"] = marks["mc0"].elapsed_time(marks["mc"])
        if hasattr(kp, "h2d_bytes"):
            stats["h2d_bytes"] = stats.get("h2d_bytes", 0) + kp.h2d_bytes
        if evals0 is not None:
            tot = kp.evals.tolist()
            stats["evals"], stats["atom_evals"] = int(tot[0]), int(tot[1])
            mc_ = (evals_mc - evals0).tolist()
            stats["mc_evals"], stats["mc_atom_evals"] = int(mc_[0]), int(mc_[1])
    return res


def dock_problem(prob, boxes_c, boxes_s, cfg, seed=0, log=None):
    """Search entry point (reference ``search.py:399``): the kernel engine; statistics in ``LAST_STATS``."""
    LAST_STATS.clear()
    return dock_problem_kernel(prob, boxes_c, boxes_s, cfg, seed=seed, log=log, stats=LAST_STATS)
