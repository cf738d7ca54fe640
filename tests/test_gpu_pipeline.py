"""The device pipeline of the search (Stage-A conformers, lattice, start selection, segment bookkeeping,
clustering, all-atom coordinates) against restatements on the host, and the whole finalize and search against
fixtures recorded from the reference itself (tests/golden/finalize.npz, dock.npz).

Bars: integer and index results bit-exact (selected starts, cluster representatives, segment flags, lattice
membership up to points on the probe threshold); coordinates within 1e-4 A of float64; energies rel 1e-4 with a
1e-4 floor (the reference's CPU<->GPU bar, tests/test_cpukernel.py:17-20).
"""
from pathlib import Path

import numpy as np
import pytest
import torch

from helpers import ligands, lig_types, make_problem, oracle_grid, random_states, receptor, rel_close

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
DEV = torch.device("cuda:0")


def _case(kind="mixed", rec_kind="cfg0"):
    from adock_b200 import params
    from adock_b200.grid import build_grid, grid_dims
    from adock_b200.kernel import B200KernelProblem
    sfp = params.sf_params("vina")
    rec = receptor(rec_kind)
    ligs = ligands(kind)
    lt = lig_types(ligs)
    o = rec["center"] - rec["size"] / 2
    G = build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, params.GRID_SPACING, grid_dims(rec["size"], params.GRID_SPACING),
                   lt, device=DEV)
    pg = make_problem(rec, ligs, sfp, G, lt, DEV)
    pc = make_problem(rec, ligs, sfp, G.cpu().numpy(), lt, "cpu")
    return pg, pc, B200KernelProblem(pg), rec


# ---- counter-based stream of the library (SplitMix64 over (seed, chain, step, slot)), restated in Python
M64 = (1 << 64) - 1


def _splitmix(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def _uniform01(seed, chain, step, slot):
    key = ((chain << 32) ^ (step << 8) ^ slot) & M64
    return np.float32((_splitmix(seed ^ _splitmix(key)) >> 40) * (1.0 / 16777216.0))


def test_conformers_match_host_restatement():
    """adock_conformers: the torsion sets of the library's stream (set 0 = input conformer), float64 intra
    energies of every set, the C lowest chosen in ascending order, coordinates of the chosen sets."""
    from adock_b200.problem import pack_host
    from oracle.fp64 import Packed, internal
    pg, pc, kp, _ = _case("mixed")
    NT, C, seed = 64, 8, 1234
    theta, conf, e = kp.conformers(NT, C, seed)
    theta, conf, e = theta.cpu().numpy(), conf.cpu().numpy(), e.cpu().numpy()
    AM, KM, lig, sf = pack_host(pc)
    model = Packed(lig, sf)
    s = _splitmix(seed ^ 0xC0F0A11CE5)
    pi = np.float32(3.14159265)
    for l in range(pc.lb.L):
        na, nt = int(model.na[l]), int(model.nt[l])
        th = np.zeros((NT, KM), np.float32)
        for t in range(1, NT):
            for k in range(nt):
                th[t, k] = (np.float32(2.0) * _uniform01(s, l, t, k) - np.float32(1.0)) * pi
        X = internal(model.ref[l, :na], model.tm[l, :nt, :na], model.axp[l], model.axu[l], nt, th)
        e64 = model.intra(l, X)
        order = np.argsort(e64, kind="stable")
        # each chosen row is one of the generated sets, with its energy, in ascending order
        rows = [int(np.flatnonzero((th == theta[l, r]).all(1))[0]) for r in range(C)]
        assert rel_close(e[l], e64[rows]) < 1e-4
        assert np.all(np.diff(e[l]) >= 0)
        # and the chosen energies are the C lowest (a swap between near-equal energies is allowed)
        assert rel_close(np.sort(e64[rows]), e64[order[:C]], 1e-4) < 1e-4
        np.testing.assert_allclose(conf[l, :, :na], X[rows], atol=1e-4)
        assert np.all(conf[l, :, na:] == 0)


def _lattice_host(gs, center, size, step, probe_max):
    G = gs.flat.float().cpu().numpy()[:int(np.prod(gs.dims[0].tolist()))].reshape(gs.dims[0].tolist())   # slot 0
    axes = [np.arange(-s / 2 + 1.0, s / 2 - 1.0 + 1e-6, step) for s in size]
    P = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3) + center
    f = np.clip(np.rint((P - gs.origin[0].numpy()) / gs.spacing).astype(np.int64), 0, np.array(G.shape) - 1)
    v = G[f[:, 0], f[:, 1], f[:, 2]]
    return P, v


def test_lattice_matches_host_restatement():
    """adock_lattice: the probe-filtered lattice points in lattice order, one lattice per box; the box centre alone
    when nothing passes."""
    pg, pc, kp, rec = _case("mixed")
    c, s = rec["center"], rec["size"]
    boxes = np.array([np.concatenate([c, s]), np.concatenate([c + 1.0, [10.0, 12.0, 9.0]]),
                      np.concatenate([c, s])], np.float32)
    probes = [0.0, 0.0, -1e9]
    for b, pm in enumerate(probes):
        n = np.array([[len(np.arange(-x / 2 + 1.0, x / 2 - 1.0 + 1e-6, 1.5)) for x in boxes[b, 3:]]], np.int32)
        ntm = int(n.prod())
        d = lambda a, dt: torch.as_tensor(np.asarray(a, dt), device=DEV)
        trans, cnt = kp.lattice(1, d(boxes[b:b + 1], np.float32), d([0], np.int32), d([0], np.int32), d(n, np.int32),
                                1.5, pm, ntm)
        P, v = _lattice_host(pc.gs, boxes[b, :3].astype(np.float64), boxes[b, 3:].astype(np.float64), 1.5, pm)
        keep = v <= pm
        got = trans[0, :int(cnt[0])].cpu().numpy()
        if not keep.any():
            assert int(cnt[0]) == 1
            np.testing.assert_allclose(got[0], boxes[b, :3], atol=1e-6)
            continue
        border = np.abs(v) < 1e-5
        assert abs(int(cnt[0]) - int(keep.sum())) <= int(border.sum())
        if not border[keep].any() and int(cnt[0]) == int(keep.sum()):
            np.testing.assert_allclose(got, P[keep], atol=1e-4)


def test_select_starts_is_exact():
    """adock_select_starts: per ligand the M lowest Stage-A totals (ties: lower index; cycled when fewer than M),
    each start assembled from its translation, rotation and conformer."""
    pg, pc, kp, _ = _case("mixed")
    g = np.random.default_rng(3)
    L, C, Q, M, B, NTM = pc.lb.L, 3, 5, 9, 2, 11
    best_e = g.normal(size=(L, C * Q)).astype(np.float32)
    best_e[0, 1] = best_e[0, 3]                                # a tie within conformer 0
    best_i = g.integers(0, NTM, size=(L, C * Q)).astype(np.int32)
    e_conf = g.normal(size=(L, C)).astype(np.float32)
    quats = g.normal(size=(Q, 4)).astype(np.float32)
    theta = g.normal(size=(L, C, kp.KM)).astype(np.float32)
    trans = g.normal(size=(B, NTM, 3)).astype(np.float32)
    lig_box = np.array([1, 0, 1, 0][:L], np.int32)
    d = lambda a: torch.as_tensor(a, device=DEV)
    for M_ in (M, 40):
        state, e = kp.select_starts(d(best_e), d(best_i), d(e_conf), d(quats), d(theta), d(trans), d(lig_box), M_)
        state, e = state.cpu().numpy().reshape(L, M_, -1), e.cpu().numpy().reshape(L, M_)
        for l in range(L):
            tot = best_e[l] + np.repeat(e_conf[l], Q)
            order = np.lexsort((np.arange(C * Q), tot))
            pick = order[np.arange(M_) % min(M_, C * Q)]
            np.testing.assert_array_equal(e[l], tot[pick])
            np.testing.assert_array_equal(state[l, :, :3], trans[lig_box[l], best_i[l, pick]])
            np.testing.assert_array_equal(state[l, :, 3:7], quats[pick % Q])
            np.testing.assert_array_equal(state[l, :, 7:], theta[l, pick // Q])


def test_segment_update_is_exact():
    """adock_segment_update: best over each ligand's chains, the stall counter (improvement > tol resets it), the
    active flag under the segment budget and the early stop, and the chain-step count."""
    pg, pc, kp, _ = _case("mixed")
    L, M, seg = 4, 3, 5
    best_e = torch.tensor([[-1.0, -2, -3], [0, 0, 0], [5, 4, 3], [-9, -9, -9]], device=DEV).reshape(-1)
    glob = torch.tensor([-2.5, -0.001, float("inf"), -9.0], device=DEV)
    stall = torch.tensor([0, 4, 2, 1], dtype=torch.int32, device=DEV)
    active = torch.tensor([1, 1, 1, 0], dtype=torch.int32, device=DEV)
    seg_lim = torch.tensor([9, 9, 3, 9], dtype=torch.int32, device=DEV)
    steps = torch.zeros(1, dtype=torch.int64, device=DEV)
    kp.segment_update(L, M, seg, 3, 5, 0.01, best_e, seg_lim, glob, stall, active, steps)
    np.testing.assert_array_equal(glob.cpu().numpy(), np.array([-3.0, -0.001, 3.0, -9.0], np.float32))
    assert stall.tolist() == [0, 5, 0, 2]
    assert active.tolist() == [1, 0, 0, 0]       # ligand 1 stalled 5 rounds, ligand 2 ran out of budget
    assert int(steps) == 3 * M * seg


def test_cluster_and_pose_atoms():
    """adock_cluster against a host restatement of the greedy clustering on the same energies and coordinates;
    adock_pose_atoms against float64 kinematics of every atom."""
    from adock_b200.problem import pack_host
    from oracle.fp64 import Packed, internal, world
    pg, pc, kp, _ = _case("mixed")
    L, P = pc.lb.L, 24
    cl, st = random_states(pc, P, seed=11, sigma=2.0)
    st[1::3] = st[0::3]                                        # duplicate poses (RMSD 0)
    st[2::3, :3] += 0.5                                        # near-duplicates (RMSD 0.5)
    clg, stg = torch.as_tensor(cl, device=DEV), torch.as_tensor(st, device=DEV)
    et, ei, Xh = kp.rescore64(clg, stg, exact=True)
    reps, nrep = kp.cluster(et, Xh, L, P, 2.0, 9)
    reps, nrep = reps.cpu().numpy(), nrep.cpu().numpy()
    E, X = et.cpu().numpy().reshape(L, P), Xh.cpu().numpy().reshape(L, P, kp.AM, 3)
    for l in range(L):
        na = pc.lb.preps[l].n
        want = []
        for i in np.argsort(E[l], kind="stable"):
            if all(np.sqrt(((X[l, i, :na] - X[l, j, :na]) ** 2).sum(-1).mean()) >= 2.0 for j in want):
                want.append(int(i))
                if len(want) == 9:
                    break
        assert nrep[l] == len(want) and reps[l, :len(want)].tolist() == want
        assert np.all(reps[l, len(want):] == -1)
    Xa = kp.pose_atoms(pg.lb, clg, stg).cpu().numpy()
    model = Packed(*pack_host(pc)[2:])
    lb = pc.lb
    for l in range(L):
        sel = cl == l
        n, nt = lb.preps[l].n, lb.preps[l].n_tors
        Xi = internal(lb.ref[l, :n].numpy(), lb.tmask[l, :nt, :n].numpy(), lb.axis_p[l].numpy(), lb.axis_u[l].numpy(),
                      nt, st[sel, 7:])
        want = world(Xi, st[sel])
        np.testing.assert_allclose(Xa[sel][:, :n], want, atol=1e-4)
        np.testing.assert_allclose(Xa[sel][:, n:], np.broadcast_to(st[sel][:, None, :3], Xa[sel][:, n:].shape), atol=1e-5)
        np.testing.assert_allclose(Xa[sel][:, :n], model.pose_heavy(l, st[sel]), atol=1e-4)


def _golden_problem_gpu():
    from adock_b200 import params, synth
    from adock_b200.grid import make_gridset
    from adock_b200.ligand import LigandBatch
    from adock_b200.problem import PairPotential, Problem, pad_receptors
    g = dict(np.load(GOLD / "grid.npz"))
    rec = synth.receptor_dict(g["rec_xyz"], g["rec_types"], np.full(3, 10.0), np.full(3, 12.0))
    ligs = [synth.ligand(24, 5, 0), synth.ligand(13, 2, 9), synth.ligand(41, 11, 4)]
    sfp = params.sf_params("vina")
    lt = np.unique(np.concatenate([[0]] + [l.types for l in ligs]))
    gs = make_gridset([rec], sfp, 0.375, 10.0, device=DEV, lig_types=[lt])
    return Problem(gs, LigandBatch(ligs, DEV), torch.zeros(3, dtype=torch.long, device=DEV), PairPotential(sfp, DEV),
                   rec=pad_receptors([rec], DEV))


def test_finalize_matches_reference_finalize():
    """finalize_device on the fixed final states of the fixture against the reference's finalize_kernel on the same
    states: identical cluster representatives, energies within 1e-4 (reference float32 vs float64 here),
    coordinates within 1e-4 A."""
    from adock_b200.kernel import B200KernelProblem
    from adock_b200.search import finalize_device
    gold = dict(np.load(GOLD / "finalize.npz"))
    prob = _golden_problem_gpu()
    kp = B200KernelProblem(prob)
    L, P = prob.lb.L, int(gold["P"])
    st = torch.as_tensor(gold["state"], device=DEV)
    cl = torch.as_tensor(gold["chain_lig"], device=DEV)
    et, _, _ = kp.rescore64(cl, st, exact=True)
    assert rel_close(et.cpu().numpy(), gold["e_exact"]) < 1e-4
    res = finalize_device(prob, kp, st, cl, L, P, {"cluster_rmsd": float(gold["cluster_rmsd"]),
                                                   "n_out": int(gold["n_out"])})
    counts = gold["counts"]
    off = np.concatenate([[0], np.cumsum(counts)])
    for l, r in enumerate(res):
        k = counts[l]
        assert len(r["affinity"]) == k
        reps = gold["reps"][off[l]:off[l + 1]]
        np.testing.assert_array_equal(np.argmin(np.abs(et.cpu().numpy().reshape(L, P)[l][None, :] -
                                                       r["total"][:, None]), 1), reps)
        for key in ("affinity", "inter", "intra", "total"):
            assert rel_close(r[key], gold[key][off[l]:off[l + 1]]) < 1e-4, key
        np.testing.assert_allclose(r["coords"], gold["coords"][off[l]:off[l + 1]], atol=1e-4)


def test_search_matches_reference_search_distribution():
    """The whole search (dock_screen -> dock_problem_kernel on the device) against the reference's own
    dock_problem_kernel on the host cores: 3 small ligands, config-0 receptor, 16 chains x 300 steps, seeds 0-7.
    Independent stochastic searches: per ligand the median best affinity over the seeds agrees within
    0.05 kcal/mol, and the lowest found within 0.1."""
    from adock_b200 import params, synth
    from adock_b200.screen import dock_screen
    gold = dict(np.load(GOLD / "dock.npz"))
    rec = synth.config_receptor(0)
    ligs = [synth.ligand(int(n), int(r), int(s)) for n, r, s in gold["ligands"]]
    cfg = params.workload_preset(int(gold["n_chains"]), int(gold["mc_steps"]))
    ours = np.array([[float(np.min(x["affinity"])) for x in
                      dock_screen(rec, {"center": rec["center"], "size": rec["size"]}, ligs, cfg, device=DEV, seed=int(sd))]
                     for sd in gold["seeds"]])
    ref = gold["best_affinity"]
    assert np.all(np.abs(np.median(ours, 0) - np.median(ref, 0)) <= 0.05), (np.median(ours, 0), np.median(ref, 0))
    assert np.all(np.abs(ours.min(0) - ref.min(0)) <= 0.1), (ours.min(0), ref.min(0))
