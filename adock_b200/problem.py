"""Docking problems and their packing into the search kernels' arrays.

``Problem(gridset, lb, rec_idx, pot, rec=None)`` is the reference container (``src/adock/search.py:65-72``): maps,
ligand batch, receptor of each ligand, pair potential and, for exact energies, the padded receptor atoms
``(xyz [R, N, 3], types [R, N], mask [R, N])`` of ``pad_receptors`` (``search.py:369-379``).

``pack_host`` produces the kernel input layout of the reference ``mckernel.pack_host`` (``mckernel.py:547-599``):
heavy atoms only, AM = 64 when the largest ligand has <= 64 heavy atoms else a multiple of 32, KM = a multiple of
8 >= the largest torsion count, P = the largest pair count; every array is one scatter over the concatenated
ligands, with atom indices renumbered to heavy-atom order.

``PairPotential`` carries the Vina-family parameters; its ``terms``/``energy`` evaluate the published pair terms
(``scoring.py:18-31``) in torch, which the tests use as a float64 check of the kernels' constants.
"""
from __future__ import annotations

import numpy as np
import torch

_PRM_KEYS = ("g1_off", "g1_w", "g2_off", "g2_w", "rep_off", "hyd_good", "hyd_bad", "hb_good", "hb_bad", "cutoff")
_W_KEYS = ("w_g1", "w_g2", "w_rep", "w_hyd", "w_hb")


def _ramp(d, good, bad):
    """1 at d <= good, 0 at d >= bad, linear between (either orientation of good/bad)."""
    return ((bad - d) / (bad - good)).clamp(0.0, 1.0)


def pair_terms(r, ti, tj, radius, hyd, don, acc, prm):
    """Unweighted Vina-family terms [..., 5] = gauss1, gauss2, repulsion, hydrophobic, H-bond of pairs at distance
    r with types ti, tj; zero at r >= cutoff. The surface distance is d = r - R_i - R_j."""
    p = dict(zip(_PRM_KEYS, prm))
    d = r - radius.to(r.dtype)[ti] - radius.to(r.dtype)[tj]
    gauss = lambda off, w: torch.exp(-torch.square((d - off) / w))
    rep = torch.square(torch.clamp(d - p["rep_off"], max=0.0))
    hyd_pair = hyd[ti] & hyd[tj]
    hb_pair = (don[ti] & acc[tj]) | (acc[ti] & don[tj])
    zero = torch.zeros_like(d)
    terms = torch.stack([gauss(p["g1_off"], p["g1_w"]), gauss(p["g2_off"], p["g2_w"]), rep,
                         torch.where(hyd_pair, _ramp(d, p["hyd_good"], p["hyd_bad"]), zero),
                         torch.where(hb_pair, _ramp(d, p["hb_good"], p["hb_bad"]), zero)], -1)
    return terms * (r < p["cutoff"]).unsqueeze(-1).to(terms.dtype)


class PairPotential:
    """Vina-family pair potential (reference interface ``scoring.py:34-61``); ``p`` holds the flat parameters
    (``params.sf_params``)."""

    def __init__(self, sfp, device="cpu"):
        self.p = sfp
        self.radius = torch.tensor(np.asarray(sfp["radius"], np.float32), device=device)
        self.hyd = torch.tensor(np.asarray(sfp["hydrophobic"]), device=device).bool()
        self.don = torch.tensor(np.asarray(sfp["donor"]), device=device).bool()
        self.acc = torch.tensor(np.asarray(sfp["acceptor"]), device=device).bool()

    def prm(self):
        return tuple(self.p[k] for k in _PRM_KEYS)

    def weights(self, device=None):
        return torch.tensor([self.p[k] for k in _W_KEYS], device=device or self.radius.device)

    def terms(self, r, ti, tj):
        return pair_terms(r, ti, tj, self.radius.to(r.device), self.hyd.to(r.device), self.don.to(r.device),
                          self.acc.to(r.device), self.prm())

    def energy(self, r, ti, tj):
        return self.terms(r, ti, tj) @ self.weights(r.device).to(r.dtype)


class Problem:
    """Maps + ligand batch + receptor index per ligand + pair potential (+ receptor atoms for exact energies)."""

    def __init__(self, gridset, lb, rec_idx, pot, rec=None):
        self.gs, self.lb, self.rec_idx, self.pot, self.rec = gridset, lb, rec_idx, pot, rec

    def subset(self, idx):
        return Problem(self.gs, self.lb.subset(idx), self.rec_idx[idx], self.pot, self.rec)


def pad_receptors(receptors, device):
    """(xyz [R, N, 3] f32, types [R, N] i64, mask [R, N] bool) of receptor dicts padded to the largest."""
    counts = np.array([len(r["rec_xyz"]) for r in receptors], np.int64)
    N = int(counts.max())
    owner = np.repeat(np.arange(len(receptors)), counts)
    row = np.arange(counts.sum()) - np.repeat(np.cumsum(counts) - counts, counts)
    xyz = np.zeros((len(receptors), N, 3), np.float32)
    typ = np.zeros((len(receptors), N), np.int64)
    xyz[owner, row] = np.concatenate([np.asarray(r["rec_xyz"], np.float32).reshape(-1, 3) for r in receptors])
    typ[owner, row] = np.concatenate([np.asarray(r["rec_types"], np.int64) for r in receptors])
    mask = np.arange(N)[None, :] < counts[:, None]
    return tuple(torch.as_tensor(a, device=device) for a in (xyz, typ, mask))


def _multiple(x, step):
    return step * max(1, -(-int(x) // step))


def pack_host(prob):
    """Kernel arrays of a Problem: (AM, KM, lig, sf) with
    lig = [ref, typ, tm, ax, axp, axu, pr, na, nt, np, rg, P, gslot] and sf = [prm (15), radius, hyd, don, acc]."""
    preps = prob.lb.preps
    L = len(preps)
    heavy = [np.flatnonzero(np.asarray(p.heavy, bool)) for p in preps]
    na = np.array([len(h) for h in heavy], np.int32)
    nt = np.array([p.n_tors for p in preps], np.int32)
    npr = np.array([len(p.pairs) for p in preps], np.int32)
    AM = 64 if na.max() <= 64 else _multiple(na.max(), 32)
    KM = _multiple(max(int(nt.max()), 1), 8)
    P = max(1, int(npr.max()))
    # heavy-atom renumbering: new[l][old atom] = position among the ligand's heavy atoms (-1 for hydrogens)
    new = []
    for p, h in zip(preps, heavy):
        m = np.full(p.n, -1, np.int64)
        m[h] = np.arange(len(h))
        new.append(m)
    own_a = np.repeat(np.arange(L), na)
    pos_a = np.arange(na.sum()) - np.repeat(np.cumsum(na) - na, na)
    ref = np.zeros((L, AM, 3), np.float32)
    typ = np.zeros((L, AM), np.int32)
    ref[own_a, pos_a] = np.concatenate([np.asarray(p.ref, np.float32)[h] for p, h in zip(preps, heavy)])
    typ[own_a, pos_a] = np.concatenate([np.asarray(p.types)[h] for p, h in zip(preps, heavy)])
    # torsions: moved-atom table over heavy atoms, axis atoms renumbered, axis point and unit vector
    tm = np.zeros((L, KM, AM), np.uint8)
    ax = np.zeros((L, KM, 2), np.int32)
    axp = np.zeros((L, KM, 3), np.float32)
    axu = np.zeros((L, KM, 3), np.float32)
    own_t = np.repeat(np.arange(L), nt)
    pos_t = np.arange(nt.sum()) - np.repeat(np.cumsum(nt) - nt, nt)
    if nt.sum():
        tors = [(np.asarray(p.tors_axis, np.int64).reshape(-1, 2), np.asarray(p.tors_mask, bool).reshape(p.n_tors, p.n))
                for p in preps]
        ax_new = np.concatenate([m[a] for (a, _), m in zip(tors, new)])
        assert (ax_new >= 0).all(), "torsion axis atom is not a heavy atom"
        ax[own_t, pos_t] = ax_new
        pa = np.concatenate([np.asarray(p.ref, np.float32)[a[:, 0]] for (a, _), p in zip(tors, preps)])
        pb = np.concatenate([np.asarray(p.ref, np.float32)[a[:, 1]] for (a, _), p in zip(tors, preps)])
        axp[own_t, pos_t] = pa
        axu[own_t, pos_t] = (pb - pa) / np.maximum(np.linalg.norm(pb - pa, axis=1, keepdims=True), np.float32(1e-6))
        hit = [np.nonzero(msk[:, h]) for (_, msk), h in zip(tors, heavy)]
        own_h = np.concatenate([np.full(len(k), l) for l, (k, _) in enumerate(hit)])
        tm[own_h, np.concatenate([k for k, _ in hit]), np.concatenate([a for _, a in hit])] = 1
    pr = np.zeros((L, P, 2), np.int32)
    if npr.sum():
        own_p = np.repeat(np.arange(L), npr)
        pos_p = np.arange(npr.sum()) - np.repeat(np.cumsum(npr) - npr, npr)
        pr[own_p, pos_p] = np.concatenate([m[np.asarray(p.pairs, np.int64).reshape(-1, 2)]
                                           for p, m in zip(preps, new) if len(p.pairs)])
    rg = np.array([p.rg for p in preps], np.float32)
    # grid slot of each heavy atom in its receptor's maps
    slot = prob.gs.slot.cpu().numpy() if torch.is_tensor(prob.gs.slot) else np.asarray(prob.gs.slot)
    rec = np.asarray(prob.rec_idx.cpu() if torch.is_tensor(prob.rec_idx) else prob.rec_idx, np.int64)
    gsl = np.zeros((L, AM), np.int32)
    gsl[own_a, pos_a] = slot[rec[own_a], typ[own_a, pos_a]]
    assert (gsl >= 0).all(), "a ligand atom type has no grid"
    lig = [ref, typ, tm, ax, axp, axu, pr, na, nt, npr, rg, np.int32(P), gsl]
    sp = prob.pot.p
    prm = np.array([sp[k] for k in _PRM_KEYS + _W_KEYS], np.float32)
    sf = [prm, np.asarray(sp["radius"], np.float32), np.asarray(sp["hydrophobic"], np.int32),
          np.asarray(sp["donor"], np.int32), np.asarray(sp["acceptor"], np.int32)]
    return AM, KM, lig, sf


__all__ = ["Problem", "PairPotential", "pair_terms", "pad_receptors", "pack_host"]
