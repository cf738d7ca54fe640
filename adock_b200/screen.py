"""One pocket x many ligands with one shared grid set (reference ``src/adock/screen.py:39-78``).

``dock_screen(receptor, box, ligands, ...)`` builds the receptor maps once on the GPU for the union of the
ligands' types (plus C_H, the Stage-A probe type), then docks the ligands in batches against receptor 0 with
``dock_problem_kernel``. Inputs are host data (receptor coordinates/types, ligand preps); results come back as
host numpy arrays. This is the public call the end-to-end benchmark times.
"""
from __future__ import annotations

import numpy as np
import torch

from . import params
from .grid import make_gridset
from .ligand import LigandBatch
from .problem import PairPotential, Problem, pad_receptors
from .search import dock_problem_kernel


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
