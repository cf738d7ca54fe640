"""Generate the golden fixtures in tests/golden/ from the reference implementation itself.

Run where a reference checkout is present:  python tests/golden/make_golden.py --reference DIR
(or with ADOCK_REFERENCE=DIR). The reference package is imported unmodified with empty stand-ins for ``cupy`` and
``rdkit`` (its CPU path and the functions used here do not touch them); its host kernels are compiled by its own
``adock.cpukernel`` into a temporary cache directory. The synthetic inputs come from ``adock_b200.synth`` with
fixed seeds, so every fixture records (inputs, reference outputs). Fixtures:

  pack.npz        reference mckernel.pack_host of a 3-ligand synthetic batch
  pair_terms.npz  reference scoring.pair_terms (float64) for 8 type pairs x 10 distances, Vina and Vinardo
  fitted.npz      reference fit.terms Spec/FittedPotential: W table, radii, grid prm, features of 3 known pairs
  grid.npz        reference cpukernel.build_grid_cpu maps (small receptor, ragged 13x15x17, 4 types, per_term too)
  search.npz      reference CpuKernelProblem: energy_grad (grid + exact) of 32 poses, stage_a, one MC step
  batch.npz       reference ligand.LigandBatch padded arrays of the 3-ligand batch
  finalize.npz    reference search.finalize_kernel on fixed final states (12 per ligand, in near-duplicate groups):
                  per-state exact totals, the representatives it picks and its result arrays
  dock.npz        reference search.dock_problem_kernel (device "cpu"): 3 small ligands against the config-0
                  receptor, 16 chains x 300 steps, seeds 0-7: best affinity per (seed, ligand)
"""
import argparse
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def _import_reference(ref):
    import tempfile
    for name in ("cupy", "rdkit", "rdkit.Chem"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["rdkit"].Chem = sys.modules["rdkit.Chem"]
    os.environ.setdefault("ADOCK_CPU_CACHE", tempfile.mkdtemp(prefix="adock_ref_cpu_"))
    sys.path.insert(0, str(Path(ref) / "src"))
    import torch  # noqa: F401
    from adock import config, cpukernel, grid, ligand, mckernel, scoring, search
    from adock.fit import terms
    return dict(config=config, cpukernel=cpukernel, grid=grid, ligand=ligand, mckernel=mckernel, scoring=scoring,
                search=search, terms=terms)


def _ligands():
    from adock_b200 import synth
    return [synth.ligand(24, 5, 0), synth.ligand(13, 2, 9), synth.ligand(41, 11, 4)]


def _receptor():
    from adock_b200 import synth
    xyz, types_ = synth.receptor(400, 20.0, seed=3)
    return synth.receptor_dict(xyz, types_, np.full(3, 10.0), np.full(3, 12.0))


def main(ref):
    import torch
    R = _import_reference(ref)
    cfg = R["config"].load_config()
    sfp = R["config"].sf_params(cfg, "vina")
    ligs = _ligands()
    rec = _receptor()
    out = {}

    # ---------------- pair terms (float64) ----------------
    pt = {}
    for sf in ("vina", "vinardo"):
        pot = R["scoring"].PairPotential(R["config"].sf_params(cfg, sf))
        idx = cfg["_xs_index"]
        pairs = [("C_H", "C_H"), ("C_H", "C_P"), ("N_D", "O_A"), ("O_DA", "O_DA"), ("N_P", "O_A"), ("Cl_H", "C_H"),
                 ("Met_D", "O_A"), ("S_P", "N_DA")]
        rs = np.array([1.0, 2.0, 2.9, 3.3, 3.6, 4.0, 4.5, 5.5, 7.99, 8.01])
        ti = np.array([idx[a] for a, _ in pairs])
        tj = np.array([idx[b] for _, b in pairs])
        r = torch.tensor(np.repeat(rs[None], len(pairs), 0), dtype=torch.float64)
        e = pot.energy(r, torch.as_tensor(ti)[:, None].expand(r.shape), torch.as_tensor(tj)[:, None].expand(r.shape))
        terms = pot.terms(r, torch.as_tensor(ti)[:, None].expand(r.shape), torch.as_tensor(tj)[:, None].expand(r.shape))
        pt[f"{sf}_ti"], pt[f"{sf}_tj"], pt[f"{sf}_r"] = ti, tj, rs
        pt[f"{sf}_energy"], pt[f"{sf}_terms"] = e.numpy(), terms.numpy()
    np.savez_compressed(HERE / "pair_terms.npz", **pt)

    # ---------------- fitted function ----------------
    T = R["terms"]
    spec = T.Spec(cfg, "vina", buried_threshold=177.0, buried_radius=10.0, ion_rmin=2.0)
    w = np.array([-0.04205807783159489, -0.004991743991543715, 0.8156755426614062, -0.037384251945279,
                  -0.5992849056216177, -0.010445834116223103, -0.033401801182270895, 0.04364980965614507,
                  -0.05896339457313388, -0.2891157216623504, 0.5160035204995856, -0.019994960794392377,
                  -0.009641505343954668, -0.025311347297737166, -0.004635982193796613, 0.7775323047062759,
                  -0.023113067408981426, -0.2059719834408973], np.float32)
    lig_list = np.array([0, 1, 2, 3, 4, 8, 9, 10, 18 + 3, 36 + 8])
    pot = T.FittedPotential(spec, w, lig_list)
    X = torch.tensor([[[0.0, 0.0, 0.0]]], dtype=torch.float64)
    feats = []
    for lt, rt, r in ((0, 0 + 18, 4.0), (3 + 18, 8 + 18 * 4, 3.0), (8, 17, 2.1)):
        Rr = torch.tensor([[r, 0.0, 0.0]], dtype=torch.float64)
        feats.append(T.inter_features(X, torch.tensor([lt]), Rr, torch.tensor([rt]), T.Spec(cfg, "vina", buried_threshold=100))[0].numpy())
    np.savez_compressed(HERE / "fitted.npz", W=pot.W.numpy(), lig_list=lig_list, weights=w, rad_lig=pot.radius.numpy(),
                        rec_radius=spec.rec_radius, indicator_sum=spec.indicator().sum((2, 3)),
                        feats=np.array(feats), feat_pairs=np.array([[0, 18, 4.0], [21, 80, 3.0], [8, 17, 2.1]]))

    # ---------------- grids ----------------
    o = rec["center"] - rec["size"] / 2
    lt = np.array([0, 3, 8, 9])
    G = R["cpukernel"].build_grid_cpu(rec["rec_xyz"], rec["rec_types"], sfp, o, 0.375, (13, 15, 17), lt).numpy()
    Gt = R["cpukernel"].build_grid_cpu(rec["rec_xyz"], rec["rec_types"], sfp, o, 0.375, (5, 6, 7), lt, per_term=True).numpy()
    np.savez_compressed(HERE / "grid.npz", rec_xyz=rec["rec_xyz"], rec_types=rec["rec_types"], origin=o, lig_types=lt,
                        grid=G, grid_per_term=Gt)

    # ---------------- packing + search kernels ----------------
    lb = R["ligand"].LigandBatch(ligs, "cpu")
    types_all = np.unique(np.concatenate([[0]] + [l.types for l in ligs]))
    gs = R["grid"].make_gridset([rec], sfp, 0.375, 10.0, device="cpu", lig_types=[types_all])
    prob = R["search"].Problem(gs, lb, torch.zeros(len(ligs), dtype=torch.long), R["scoring"].PairPotential(sfp),
                               rec=R["search"].pad_receptors([rec], "cpu"))
    AM, KM, lig, sf = R["mckernel"].pack_host(prob)
    names = ["ref", "typ", "tm", "ax", "axp", "axu", "pr", "na", "nt", "np", "rg", "P", "gslot"]
    pk = {n: np.asarray(a) for n, a in zip(names, lig)}
    pk.update(AM=AM, KM=KM, prm=sf[0], radius=sf[1], hyd=sf[2], don=sf[3], acc=sf[4], grid_lt=types_all,
              grid_dims=gs.dims.numpy(), grid_slot=gs.slot.numpy(), grid_origin=gs.origin.numpy())
    np.savez_compressed(HERE / "pack.npz", **pk)

    kp = R["cpukernel"].CpuKernelProblem(prob)
    g = torch.Generator().manual_seed(0)
    n = 16
    c = torch.tensor(rec["center"], dtype=torch.float32)
    t = c + torch.randn((len(ligs) * n, 3), generator=g) * 1.0
    q = R["ligand"].random_quat((len(ligs) * n,), g, "cpu")
    th = (torch.rand((len(ligs) * n, lb.K), generator=g) * 2 - 1) * np.pi
    th = th * lb.tvalid.repeat_interleave(n, 0)
    st = kp.pack(t, q, th)
    cl = torch.arange(len(ligs), dtype=torch.int32).repeat_interleave(n)
    e, gr = kp.energy_grad(cl, st)
    ex, gx = kp.energy_grad(cl, st, exact=True)
    # Stage A
    C, Q = 2, 24
    conf = torch.zeros(len(ligs), C, AM, 3)
    for l, p in enumerate(ligs):
        conf[l, :, :p.n] = torch.as_tensor(p.ref) + torch.randn(C, 1, 3, generator=g) * 0.1
    quats = R["ligand"].random_quat((Q,), g, "cpu")
    trans = (c + (torch.rand(len(ligs), 100, 3, generator=g) - 0.5) * 6).contiguous()
    ntr = torch.tensor([100, 60, 9])
    be, bi = kp.stage_a(conf, quats, trans, ntr, 0.3)
    # one MC step from given energies
    ci = torch.arange(len(cl), dtype=torch.int32) * 5 + 1
    cur, best = st.clone(), st.clone()
    cur_e = e.clone()
    best_e = torch.full((len(cl),), float("inf"))
    kp.run_mc(cl, ci, cur, cur_e, best, best_e, False, 1, 1, 1.2, 2.0, 2.0, 4242, 3)
    np.savez_compressed(HERE / "search.npz", state=st.numpy(), chain_lig=cl.numpy(), e=e.numpy(), g=gr.numpy(),
                        e_exact=ex.numpy(), g_exact=gx.numpy(), conf=conf.numpy(), quats=quats.numpy(),
                        trans=trans.numpy(), ntrans=ntr.numpy(), stage_e=be.numpy(), stage_i=bi.numpy(),
                        mc_chain_id=ci.numpy(), mc_cur=cur.numpy(), mc_cur_e=cur_e.numpy(), mc_best_e=best_e.numpy())
    # ---------------- LigandBatch arrays ----------------
    names = ["ref", "types", "amask", "axis", "tmask", "tvalid", "pairs", "pmask", "rg", "n_tors_vina", "axis_p",
             "axis_u"]
    np.savez_compressed(HERE / "batch.npz", **{k: getattr(lb, k).numpy() for k in names})

    # ---------------- finalize on fixed states ----------------
    # per ligand 4 base poses x 3 near-duplicates (0.2 A translation jitter): the greedy 2 A clustering must keep
    # one representative per group
    P, groups = 12, 4
    L = len(ligs)
    tb = c + torch.randn((L, groups, 1, 3), generator=g) * 1.5
    qb = R["ligand"].random_quat((L, groups, 1), g, "cpu")
    thb = (torch.rand((L, groups, 1, lb.K), generator=g) * 2 - 1) * np.pi
    t = (tb + torch.randn((L, groups, 3, 3), generator=g) * 0.2).reshape(L * P, 3)
    q = qb.expand(L, groups, 3, 4).reshape(L * P, 4)
    th = (thb.expand(L, groups, 3, lb.K) * lb.tvalid[:, None, None, :]).reshape(L * P, lb.K)
    fst = kp.pack(t, q, th)
    fcl = torch.arange(L, dtype=torch.int32).repeat_interleave(P)
    fe, _ = kp.energy_grad(fcl, fst, exact=True)
    cfg_f = dict(cfg["search"]["v2_default"])
    res = R["search"].finalize_kernel(prob, kp, fst, fcl, L, P, cfg_f)
    reps, out = [], {}
    for l, r in enumerate(res):
        # the representative states, recovered from their (exactly equal) totals
        el = fe.view(L, P)[l].numpy()
        reps.append([int(np.flatnonzero(el == v)[0]) for v in r["total"]])
    out["counts"] = np.array([len(r["affinity"]) for r in res])
    for k in ("affinity", "inter", "intra", "total"):
        out[k] = np.concatenate([r[k] for r in res])
    out["coords"] = np.concatenate([r["coords"] for r in res])
    np.savez_compressed(HERE / "finalize.npz", state=fst.numpy(), chain_lig=fcl.numpy(), P=P, e_exact=fe.numpy(),
                        reps=np.concatenate(reps), cluster_rmsd=cfg_f["cluster_rmsd"], n_out=cfg_f["n_out"], **out)

    # ---------------- the whole search on the host cores, several seeds ----------------
    # the config-0 receptor (1,500 atoms, 22.5 A box) and three small ligands, where independent searches converge
    from adock_b200 import synth
    rec0 = synth.config_receptor(0)
    ligs0 = [synth.ligand(n, r, sd) for n, r, sd in ((12, 2, 101), (16, 3, 102), (20, 4, 103))]
    L0 = len(ligs0)
    t0 = np.unique(np.concatenate([[0]] + [l.types for l in ligs0]))
    gs0 = R["grid"].make_gridset([rec0], sfp, 0.375, 10.0, device="cpu", lig_types=[t0])
    prob0 = R["search"].Problem(gs0, R["ligand"].LigandBatch(ligs0, "cpu"), torch.zeros(L0, dtype=torch.long),
                                R["scoring"].PairPotential(sfp), rec=R["search"].pad_receptors([rec0], "cpu"))
    cfg_d = dict(cfg["search"]["v2_default"], n_chains=16, mc_steps=300, mc_segment=300, mc_size_ref=0,
                 min_total_chains=0)
    bc = torch.tensor(rec0["center"], dtype=torch.float32)[None].expand(L0, 3)
    bs = [rec0["size"]] * L0
    seeds = list(range(8))
    best = np.zeros((len(seeds), L0))
    for i, sd in enumerate(seeds):
        r = R["search"].dock_problem_kernel(prob0, bc, bs, cfg_d, seed=sd)
        best[i] = [float(np.min(x["affinity"])) for x in r]
    np.savez_compressed(HERE / "dock.npz", seeds=np.array(seeds), best_affinity=best,
                        ligands=np.array([[12, 2, 101], [16, 3, 102], [20, 4, 103]]), n_chains=cfg_d["n_chains"],
                        mc_steps=cfg_d["mc_steps"])
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("ADOCK_REFERENCE"),
                    help="reference checkout (default: $ADOCK_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference DIR or set ADOCK_REFERENCE")
    main(a.reference)
