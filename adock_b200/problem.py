"""Docking problem container and the host packing of a ligand batch for the search kernels.

``Problem`` mirrors ``src/adock/search.py:65-132`` (grid set, ligand batch, receptor index per ligand, pair
potential, optional receptor atoms for exact energies). ``pack_host`` restates ``src/adock/mckernel.py:547-599``:
heavy atoms only, AM = 64 if the largest ligand has <= 64 heavy atoms else a multiple of 32, KM = a multiple
of 8 >= the largest torsion count, P = the largest pair count.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .ligand import internal_coords, pose_coords


class PairPotential:
    """Vina-family pair potential (``src/adock/scoring.py:34-61``): ``p`` holds the flat parameters."""

    def __init__(self, sfp, device="cpu"):
        self.p = sfp
        self.radius = torch.tensor(sfp["radius"], device=device)
        self.hyd = torch.tensor(sfp["hydrophobic"], device=device).bool()
        self.don = torch.tensor(sfp["donor"], device=device).bool()
        self.acc = torch.tensor(sfp["acceptor"], device=device).bool()

    def prm(self):
        p = self.p
        return (p["g1_off"], p["g1_w"], p["g2_off"], p["g2_w"], p["rep_off"], p["hyd_good"], p["hyd_bad"],
                p["hb_good"], p["hb_bad"], p["cutoff"])

    def weights(self, device=None):
        p = self.p
        return torch.tensor([p["w_g1"], p["w_g2"], p["w_rep"], p["w_hyd"], p["w_hb"]],
                            device=device or self.radius.device)

    def terms(self, r, ti, tj):
        return pair_terms(r, ti, tj, self.radius, self.hyd, self.don, self.acc, self.prm())

    def energy(self, r, ti, tj):
        return (self.terms(r, ti, tj) * self.weights(r.device).to(r.dtype)).sum(-1)


def _slope_step(x, good, bad):
    if bad < good:
        return torch.clamp((x - bad) / (good - bad), 0.0, 1.0)
    return torch.clamp((bad - x) / (bad - good), 0.0, 1.0)


def pair_terms(r, ti, tj, radius, hyd, don, acc, prm):
    """Unweighted Vina-family terms [..., 5] (``scoring.py:18-31``)."""
    g1_off, g1_w, g2_off, g2_w, rep_off, hyd_good, hyd_bad, hb_good, hb_bad, cutoff = prm
    radius = radius.to(r.dtype)
    d = r - radius[ti] - radius[tj]
    g1 = torch.exp(-((d - g1_off) / g1_w) ** 2)
    g2 = torch.exp(-((d - g2_off) / g2_w) ** 2)
    dr = d - rep_off
    rep = torch.where(dr < 0, dr * dr, torch.zeros_like(dr))
    hy = torch.where(hyd[ti] & hyd[tj], _slope_step(d, hyd_good, hyd_bad), torch.zeros_like(d))
    hb = torch.where((don[ti] & acc[tj]) | (acc[ti] & don[tj]), _slope_step(d, hb_good, hb_bad), torch.zeros_like(d))
    out = torch.stack([g1, g2, rep, hy, hb], -1)
    return torch.where((r < cutoff).unsqueeze(-1), out, torch.zeros_like(out))


class Problem:
    def __init__(self, gridset, lb, rec_idx, pot, rec=None):
        self.gs, self.lb, self.rec_idx, self.pot = gridset, lb, rec_idx, pot
        self.rec = rec  # optional (xyz [R,N,3], types [R,N], mask [R,N]) for exact (grid-free) energies

    def subset(self, idx):
        return Problem(self.gs, self.lb.subset(idx), self.rec_idx[idx], self.pot, self.rec)

    def inter(self, X):
        lb = self.lb
        L, M, A, _ = X.shape
        t = lb.types[:, None, :].expand(L, M, A)
        ri = self.rec_idx[:, None, None].expand(L, M, A)
        return self.gs.lookup(X, t, ri, mask=lb.heavy[:, None, :].expand(L, M, A)).sum(-1)

    def inter_exact(self, X):
        """Direct pairwise ligand-receptor energy (no grid) [L, M] (search.py:73-90)."""
        rx, rt, rm = self.rec
        lb = self.lb
        L, M, A, _ = X.shape
        out = torch.zeros(L, M, device=X.device, dtype=X.dtype)
        for l in range(L):
            ri = int(self.rec_idx[l])
            hv = lb.heavy[l]
            xl = X[l][:, hv]
            tl = lb.types[l][hv]
            xr, trr = rx[ri][rm[ri]].to(X.dtype), rt[ri][rm[ri]]
            r = torch.cdist(xl.reshape(-1, 3), xr).reshape(M, xl.shape[1], len(xr))
            e = self.pot.energy(r, tl[None, :, None].expand_as(r), trr[None, None, :].expand_as(r))
            out[l] = e.sum((-1, -2))
        return out

    def intra(self, X):
        lb = self.lb
        L, M, A, _ = X.shape
        pi = lb.pairs[:, None, :, :].expand(L, M, lb.P, 2)
        xi = torch.gather(X, 2, pi[..., 0:1].expand(L, M, lb.P, 3))
        xj = torch.gather(X, 2, pi[..., 1:2].expand(L, M, lb.P, 3))
        r = (xi - xj).norm(dim=-1)
        ti = torch.gather(lb.types, 1, lb.pairs[..., 0])[:, None].expand(L, M, lb.P)
        tj = torch.gather(lb.types, 1, lb.pairs[..., 1])[:, None].expand(L, M, lb.P)
        e = self.pot.energy(r, ti.clamp(min=0), tj.clamp(min=0))
        e = torch.where(lb.pmask[:, None, :], e, torch.zeros_like(e))
        return e.sum(-1)

    def energy(self, t, q0, r, theta):
        """Pose -> (total, inter, intra, coords), torch reference path (search.py:121-126)."""
        X = pose_coords(self.lb, t, q0, r, theta)
        ei, ea = self.inter(X), self.intra(X)
        return ei + ea, ei, ea, X


def pad_receptors(receptors, device):
    """(xyz [R,N,3], types [R,N], mask [R,N]) padded to the largest receptor (search.py:369-379)."""
    N = max(len(r["rec_xyz"]) for r in receptors)
    R = len(receptors)
    xyz = np.zeros((R, N, 3), np.float32)
    typ = np.zeros((R, N), np.int64)
    msk = np.zeros((R, N), bool)
    for i, r in enumerate(receptors):
        n = len(r["rec_xyz"])
        xyz[i, :n], typ[i, :n], msk[i, :n] = r["rec_xyz"], r["rec_types"], True
    T = lambda a: torch.as_tensor(a, device=device)
    return T(xyz), T(typ), T(msk)


def _bucket(x, step):
    return max(step, step * math.ceil(x / step))


def pack_host(prob):
    """Numpy packing of a Problem for the search kernels. Returns (AM, KM, lig_arrays, sf_arrays) with
    lig_arrays = [ref, typ, tm, ax, axp, axu, pr, na, nt, np, rg, P, gslot] (mckernel.py:547-599)."""
    lb, gs, pot = prob.lb, prob.gs, prob.pot
    preps = lb.preps
    L = len(preps)
    nh = [int(p.heavy.sum()) for p in preps]
    AM = 64 if max(nh) <= 64 else _bucket(max(nh), 32)
    KM = _bucket(max(max(p.n_tors for p in preps), 1), 8)
    P = max(1, max(len(p.pairs) for p in preps))
    ref = np.zeros((L, AM, 3), np.float32)
    typ = np.zeros((L, AM), np.int32)
    tm = np.zeros((L, KM, AM), np.uint8)
    ax = np.zeros((L, KM, 2), np.int32)
    axp = np.zeros((L, KM, 3), np.float32)
    axu = np.zeros((L, KM, 3), np.float32)
    pr = np.zeros((L, P, 2), np.int32)
    na = np.zeros(L, np.int32)
    nt = np.zeros(L, np.int32)
    npairs = np.zeros(L, np.int32)
    rg = np.zeros(L, np.float32)
    for l, p in enumerate(preps):
        hv = np.where(p.heavy)[0]
        remap = -np.ones(p.n, np.int64)
        remap[hv] = np.arange(len(hv))
        na[l], nt[l], npairs[l], rg[l] = len(hv), p.n_tors, len(p.pairs), p.rg
        ref[l, :len(hv)] = p.ref[hv]
        typ[l, :len(hv)] = p.types[hv]
        if p.n_tors:
            tm[l, :p.n_tors, :len(hv)] = p.tors_mask[:, hv]
            ax[l, :p.n_tors] = remap[p.tors_axis]
            assert (ax[l, :p.n_tors] >= 0).all(), "torsion axis atom is not a heavy atom"
            pa, pb = p.ref[p.tors_axis[:, 0]], p.ref[p.tors_axis[:, 1]]
            u = pb - pa
            axp[l, :p.n_tors] = pa
            axu[l, :p.n_tors] = u / np.maximum(np.linalg.norm(u, axis=1, keepdims=True), 1e-6)
        if len(p.pairs):
            pr[l, :len(p.pairs)] = remap[p.pairs]
    slot = gs.slot.cpu().numpy()
    ri_np = prob.rec_idx.cpu().numpy()
    gsl = np.zeros((L, AM), np.int32)
    for l in range(L):
        gsl[l, :na[l]] = slot[ri_np[l], typ[l, :na[l]]]
    assert (gsl >= 0).all(), "a ligand atom type has no grid"
    lig = [ref, typ, tm, ax, axp, axu, pr, na, nt, npairs, rg, np.int32(P), gsl]
    sp = pot.p
    prm = np.array([sp["g1_off"], sp["g1_w"], sp["g2_off"], sp["g2_w"], sp["rep_off"], sp["hyd_good"],
                    sp["hyd_bad"], sp["hb_good"], sp["hb_bad"], sp["cutoff"], sp["w_g1"], sp["w_g2"],
                    sp["w_rep"], sp["w_hyd"], sp["w_hb"]], np.float32)
    sf = [prm, np.asarray(sp["radius"], np.float32), np.asarray(sp["hydrophobic"], np.int32),
          np.asarray(sp["donor"], np.int32), np.asarray(sp["acceptor"], np.int32)]
    return AM, KM, lig, sf


def heavy_index(lb, AM):
    """[L, AM] index of each packed heavy atom in the LigandBatch atom order (0 past the end)."""
    L = lb.L
    hidx = torch.zeros(L, AM, dtype=torch.long, device=lb.ref.device)
    for l, p in enumerate(lb.preps):
        hv = torch.as_tensor(np.where(p.heavy)[0], device=lb.ref.device)
        hidx[l, :len(hv)] = hv
    return hidx


__all__ = ["Problem", "PairPotential", "pair_terms", "pad_receptors", "pack_host", "heavy_index", "internal_coords",
           "pose_coords"]
