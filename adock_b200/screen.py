"""The callers of the search: one pocket x many ligands (``dock_screen``, reference ``src/adock/screen.py:39-78``)
and many pockets x one ligand each (``dock_batch``, reference ``src/adock/dock.py:69-125``).

``dock_screen(receptor, box, ligands, ...)`` builds the receptor maps once on the GPU for the union of the
ligands' types (plus C_H, the Stage-A probe type), then docks the ligands in batches against receptor 0 with
``dock_problem_kernel``. ``dock_batch(complexes, ...)`` takes prepared complexes (the reference's ``prepare_complex``
output: receptor atoms, box and ligand prep), builds one map set per receptor with each complex's own ligand types,
and docks every ligand against its own receptor and box in one search (receptor index = complex index). Inputs are
host data; results come back as host numpy arrays. ``dock_screen`` is the public call the end-to-end benchmark
times.
"""
from __future__ import annotations

import numpy as np
import torch

from . import params
from .grid import make_gridset
from .ligand import LigandBatch
from .problem import PairPotential, Problem, pad_receptors
from .search import LAST_STATS, dock_problem, dock_problem_kernel


def _nbytes(ts):
    return int(sum(t.numel() * t.element_size() for t in ts))


def dock_screen(receptor, box, ligands, cfg=None, device="cuda", seed=0, batch=None, sf="vina", grid_dtype="f32",
                stats=None, log=None):
    """receptor: dict rec_xyz [N,3], rec_types [N]; box: dict center, size; ligands: preps (LigandPrep fields).

    cfg: search preset (default v2_default); batch: ligands per search launch (None = all in one batch).
    Returns one result dict per ligand (coords [n_out, A, 3], affinity, inter, intra, total)."""
    cfg = dict(params.V2_DEFAULT if cfg is None else cfg)
    dev = torch.device(device)
    sfp = params.sf_params(sf)
    rec = {"rec_xyz": np.asarray(receptor["rec_xyz"], np.float32), "rec_types": np.asarray(receptor["rec_types"]),
           "center": np.asarray(box["center"], float), "size": np.asarray(box["size"], float)}
    types = np.unique(np.concatenate([np.asarray(p.types)[np.asarray(p.types) >= 0] for p in ligands]))
    gs = make_gridset([rec], sfp, params.GRID_SPACING, params.OUT_OF_BOX_PENALTY, device=dev, lig_types=[types])
    pot = PairPotential(sfp, dev)
    rec_t = pad_receptors([rec], dev)
    h2d = rec["rec_xyz"].nbytes + rec["rec_types"].nbytes + _nbytes(rec_t)
    B = len(ligands) if not batch else int(batch)
    out = [None] * len(ligands)
    st_all = {}
    # shape buckets: ligands with <= 64 heavy atoms and with more run in separate launches (the kernel's atoms per
    # lane follow the largest ligand of a launch), each bucket in batches of B
    nh = np.array([int(np.asarray(p.heavy).sum()) for p in ligands])
    buckets = [np.where(nh <= 64)[0], np.where(nh > 64)[0]]
    chunks = [idx[b0:b0 + B] for idx in buckets for b0 in range(0, len(idx), B)]
    for idx in chunks:
        chunk = [ligands[i] for i in idx]
        lb = LigandBatch(chunk, dev)
        h2d += _nbytes([lb.ref, lb.types, lb.amask, lb.axis, lb.tmask, lb.tvalid, lb.pairs, lb.pmask, lb.rg,
                        lb.n_tors_vina])
        prob = Problem(gs, lb, torch.zeros(len(chunk), dtype=torch.long, device=dev), pot, rec=rec_t)
        bc = torch.tensor(rec["center"], dtype=torch.float32, device=dev)[None].expand(len(chunk), 3)
        st = {}
        res = dock_problem_kernel(prob, bc, [rec["size"]] * len(chunk), cfg, seed=seed, log=log, stats=st)
        for k, v in st.items():
            if isinstance(v, (int, float)):
                st_all[k] = st_all.get(k, 0) + v
        for i, r in zip(idx, res):
            out[i] = r
    if stats is not None:
        stats.update(st_all)
        stats["h2d_bytes"] = stats.get("h2d_bytes", 0) + int(h2d)
    return out


def dock_batch(complexes, cfg=None, sf="vina", seed=0, device="cuda", log=None, timings=None, grid_dtype="f32"):
    """complexes: dicts with rec_xyz [N, 3], rec_types [N], center [3], size [3] and lig (a ligand prep).

    One search over all complexes: maps per receptor for its ligand's own types (plus the probe type), ligand l
    docked against receptor l in box l. Returns one result dict per complex (coords trimmed to the ligand's atoms,
    affinity, inter, intra, total, n_tors_vina); ``timings`` receives grid_s, search_s, n and the search
    statistics (reference dock.py:113-125)."""
    import time
    cfg = dict(params.V2_DEFAULT if cfg is None else cfg)
    dev = torch.device(device)
    sfp = params.sf_params(sf)
    recs = [{"rec_xyz": np.asarray(c["rec_xyz"], np.float32), "rec_types": np.asarray(c["rec_types"]),
             "center": np.asarray(c["center"], float), "size": np.asarray(c["size"], float)} for c in complexes]
    ligs = [c["lig"] for c in complexes]
    t0 = time.perf_counter()
    gs = make_gridset(recs, sfp, params.GRID_SPACING, params.OUT_OF_BOX_PENALTY, device=dev,
                      lig_types=[np.asarray(l.types)[np.asarray(l.types) >= 0] for l in ligs])
    prob = Problem(gs, LigandBatch(ligs, dev), torch.arange(len(ligs), device=dev), PairPotential(sfp, dev),
                   rec=pad_receptors(recs, dev))
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    bc = torch.tensor(np.array([r["center"] for r in recs]), dtype=torch.float32, device=dev)
    kf = None
    if grid_dtype != "f32":
        from .kernel import B200KernelProblem
        kf = lambda p: B200KernelProblem(p, grid_dtype=grid_dtype)
    if kf is None:
        res = dock_problem(prob, bc, [r["size"] for r in recs], cfg, seed=seed, log=log)
    else:
        LAST_STATS.clear()
        res = dock_problem_kernel(prob, bc, [r["size"] for r in recs], cfg, seed=seed, log=log, stats=LAST_STATS,
                                  kernel_factory=kf)
    t2 = time.perf_counter()
    if timings is not None:
        timings.update({"grid_s": t1 - t0, "search_s": t2 - t1, "n": len(complexes), **LAST_STATS})
    for lig, r in zip(ligs, res):
        r["n_tors_vina"] = lig.n_tors_vina
        r["coords"] = r["coords"][:, :lig.n]
    return res
