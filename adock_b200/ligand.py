"""Ligand batches: the padded, device-resident view of L ligand preparations.

A preparation carries the fields of the reference ``LigandPrep`` (``src/adock/ligand.py:18-119``): ``n`` atoms,
ligand-frame coordinates ``ref [n, 3]``, scoring types ``types [n]`` (-1 = hydrogen), ``heavy [n]``, the torsion
tree (``tors_axis [nt, 2]`` axis atoms, ``tors_mask [nt, n]`` moved atoms, leaf -> root), intra-ligand pairs
``pairs [np, 2]``, ``rg``, ``n_tors`` and ``n_tors_vina``. ``LigandBatch`` keeps the attribute names of the
reference batch (``ligand.py:122-182``: ``ref``, ``types``, ``heavy``, ``amask``, ``axis``, ``tmask``, ``tvalid``,
``pairs``, ``pmask``, ``rg``, ``n_tors_vina``, ``axis_p``, ``axis_u``, sizes ``L, A, K, P``) because callers and
the packing read them; the torsion count is padded to a multiple of 8 as there.

Each padded array is one scatter of the concatenated per-ligand arrays (``_scatter_rows``). There is no host-side
kinematics: poses are turned into coordinates on the device (``adock_pose_atoms`` for all atoms, the search kernels
and ``adock_rescore64`` for heavy atoms).
"""
from __future__ import annotations

import numpy as np
import torch

TORSION_BUCKET = 8


def _counts(preps, field):
    return np.array([len(getattr(p, field)) for p in preps], np.int64)


def _scatter_rows(blocks, counts, width, tail, dtype, fill):
    """[L, width, *tail] array holding block l (counts[l] rows of shape tail) in rows 0..counts[l]-1 of slot l."""
    out = np.full((len(blocks), width) + tail, fill, dtype)
    total = int(counts.sum())
    if total:
        owner = np.repeat(np.arange(len(blocks)), counts)
        row = np.arange(total) - np.repeat(np.cumsum(counts) - counts, counts)
        out[owner, row] = np.concatenate([np.asarray(b, dtype).reshape((-1,) + tail) for b, c in zip(blocks, counts)
                                          if c])
    return out


def _round_up(x, step):
    return step * max(1, -(-int(x) // step))


class LigandBatch:
    """L ligand preparations padded to A atoms, K torsions (multiple of 8) and P intra pairs, as torch tensors on
    ``device``. ``preps`` is kept: the search packs its kernel arrays from it."""

    def __init__(self, preps, device="cpu"):
        self.preps = list(preps)
        ps = self.preps
        n_at = np.array([p.n for p in ps], np.int64)
        n_tor = np.array([p.n_tors for p in ps], np.int64)
        n_pair = _counts(ps, "pairs")
        L, A = len(ps), int(n_at.max())
        K = _round_up(n_tor.max(), TORSION_BUCKET)
        P = max(1, int(n_pair.max()))
        ref = _scatter_rows([p.ref for p in ps], n_at, A, (3,), np.float32, 0.0)
        types = _scatter_rows([p.types for p in ps], n_at, A, (), np.int64, -1)
        axis = _scatter_rows([np.reshape(p.tors_axis, (-1, 2)) for p in ps], n_tor, K, (2,), np.int64, 0)
        pairs = _scatter_rows([np.reshape(p.pairs, (-1, 2)) for p in ps], n_pair, P, (2,), np.int64, 0)
        # moved-atom table [L, K, A]: scatter the (torsion, atom) coordinates of every mask's set entries
        tmask = np.zeros((L, K, A), bool)
        hits = [np.nonzero(np.asarray(p.tors_mask, bool).reshape(p.n_tors, p.n)) for p in ps]
        if any(len(h[0]) for h in hits):
            owner = np.concatenate([np.full(len(h[0]), l) for l, h in enumerate(hits)])
            tmask[owner, np.concatenate([h[0] for h in hits]), np.concatenate([h[1] for h in hits])] = True
        slot = np.arange(max(A, K, P))
        amask = slot[None, :A] < n_at[:, None]
        tvalid = slot[None, :K] < n_tor[:, None]
        pmask = slot[None, :P] < n_pair[:, None]
        # torsion axes from the reference conformer: point = first axis atom, unit vector towards the second
        owner = np.arange(L)[:, None]
        a0, a1 = ref[owner, axis[..., 0]], ref[owner, axis[..., 1]]
        d = a1 - a0
        axis_u = d / np.maximum(np.linalg.norm(d, axis=-1, keepdims=True), np.float32(1e-6))
        self.L, self.A, self.K, self.P = L, A, K, P
        to = lambda a: torch.as_tensor(a, device=device)
        self.ref, self.types, self.amask = to(ref), to(types), to(amask)
        self.heavy = self.types >= 0
        self.axis, self.tmask, self.tvalid = to(axis), to(tmask), to(tvalid)
        self.pairs, self.pmask = to(pairs), to(pmask)
        self.rg = to(np.array([p.rg for p in ps], np.float32))
        self.n_tors_vina = to(np.array([p.n_tors_vina for p in ps], np.float32))
        self.axis_p, self.axis_u = to(a0.astype(np.float32)), to(axis_u.astype(np.float32))
        self._mask_bits = (tmask.astype(np.uint64) << np.arange(K, dtype=np.uint64)[None, :, None]).sum(1)

    def atom_masks(self):
        """[L, A] uint32: bit k set when torsion k moves the atom (K <= 32)."""
        assert self.K <= 32, "at most 32 torsions"
        return self._mask_bits.astype(np.uint32)

    def subset(self, idx):
        """Batch of the ligands ``idx`` (a 1-D index tensor or sequence), same padded sizes."""
        idx_t = torch.as_tensor(idx, dtype=torch.long)
        sel = idx_t.tolist()
        new = LigandBatch.__new__(LigandBatch)
        new.preps = [self.preps[i] for i in sel]
        new.L, new.A, new.K, new.P = len(sel), self.A, self.K, self.P
        for name in ("ref", "types", "heavy", "amask", "axis", "tmask", "tvalid", "pairs", "pmask", "rg",
                     "n_tors_vina", "axis_p", "axis_u"):
            t = getattr(self, name)
            setattr(new, name, t[idx_t.to(t.device)])
        new._mask_bits = self._mask_bits[np.asarray(sel, np.int64)]
        return new

    def to(self, dtype):
        """Copy whose floating-point tensors are in ``dtype``."""
        new = self.subset(range(self.L))
        for name in ("ref", "axis_p", "axis_u", "rg"):
            setattr(new, name, getattr(new, name).to(dtype))
        return new
