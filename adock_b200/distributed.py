"""Screening across GPUs: one process per GPU, ligands sharded, no collective on the data path.

Ligands are independent and every GPU builds the same read-only maps (a few ms), so a screen shards the ligand list
across ranks and each rank docks its shard with ``dock_screen`` on its own GPU. The only collective is the gather of
the results (top poses and affinities, a few KB per ligand) to rank 0 at the end. The reference has no multi-GPU
path; this is the sharded form of its one-pocket screening call (``src/adock/screen.py:39-78``).
"""
from __future__ import annotations

import numpy as np


def shard_indices(costs, rank, world):
    """Indices of the ligands rank ``rank`` of ``world`` docks. Ligands are sorted by cost (heavy atoms, most first)
    and dealt in a snake order (0..w-1, w-1..0, ...), so every rank gets a similar total cost; each rank's indices
    come back in ascending order."""
    costs = np.asarray(costs)
    order = np.argsort(-costs, kind="stable")
    mine = []
    for pos, i in enumerate(order):
        rnd, k = divmod(pos, world)
        r = k if rnd % 2 == 0 else world - 1 - k
        if r == rank:
            mine.append(int(i))
    return sorted(mine)


def _host(r):
    return {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in r.items()}


def dock_screen_sharded(receptor, box, ligands, group=None, dock_fn=None, **kw):
    """Dock ``ligands`` across the ranks of the default process group (or ``group``). Every rank passes the same
    ligand list; rank r docks ``shard_indices`` of it with ``dock_fn`` (default ``screen.dock_screen``) on its
    current device. Rank 0 returns the results of all ligands in input order; the other ranks return None."""
    import torch.distributed as dist
    if dock_fn is None:
        from .screen import dock_screen as dock_fn
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    idx = shard_indices([int(np.asarray(p.heavy).sum()) for p in ligands], rank, world)
    res = dock_fn(receptor, box, [ligands[i] for i in idx], **kw) if idx else []
    payload = [(i, _host(r)) for i, r in zip(idx, res)]
    parts = [None] * world if rank == 0 else None
    dist.gather_object(payload, parts, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(ligands)
    for part in parts:
        for i, r in part:
            out[i] = r
    assert all(r is not None for r in out), "a ligand's result is missing after the gather"
    return out


def max_over_ranks(value, group=None, device=None):
    """The maximum of a per-rank float over the ranks (the job time of a synchronous multi-GPU step)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t)
