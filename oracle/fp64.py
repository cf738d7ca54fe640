"""Float64 restatement of the pose energy on the packed arrays (numpy).

TEST INFRASTRUCTURE ONLY: the float64 yardstick of tests/ (map-precision errors, the float64 re-score, neighbour
lists, all-atom coordinates). The product never imports it.

Restates, in float64 and vectorised over poses:
  pose_heavy   src/adock/mckernel.py:121-139  torsions k = 0..nt-1 (leaf -> root) applied to the reference
                                              coordinates about the reference axes (Rodrigues), then rotation by
                                              the normalised quaternion (w, x, y, z) and translation
  pair_energy  src/adock/scoring.py:18-31     Vina-family terms x weights, zero at r >= cutoff
  grid_inter   src/adock/grid.py:169-194      trilinear interpolation with the clamp min(max(f, 0), n - 1 - 1e-4)
                                              plus the quadratic out-of-box penalty
  exact_inter  src/adock/search.py:73-90      pairwise ligand-receptor sum (+ the out-of-box penalty, as the
                                              kernels' exact mode adds it)
  intra        src/adock/search.py:108-120    intra-ligand pairs
The inputs are the ``pack_host`` arrays (src/adock/mckernel.py:547-599): heavy atoms only.
"""
from __future__ import annotations

import numpy as np


def quat_matrix(q):
    """[..., 4] (w, x, y, z), normalised here -> rotation matrices [..., 3, 3]."""
    q = np.asarray(q, np.float64)
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    w, x, y, z = np.moveaxis(q, -1, 0)
    return np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                     np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                     np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], -2)


def rotate_about(P, a, u, ang):
    """Rodrigues rotation of points P [..., 3] by ang [...] about the axis through a [3] along unit u [3]."""
    v = P - a
    c, s = np.cos(ang)[..., None], np.sin(ang)[..., None]
    return a + v * c + np.cross(u, v) * s + u * (v @ u)[..., None] * (1 - c)


def internal(ref, masks, axp, axu, nt, theta):
    """Ligand-frame coordinates [N, n, 3] of n atoms (ref [n, 3]) for torsion angles theta [N, >= nt]; masks
    [nt, n] bool: torsion k moves atom a."""
    X = np.broadcast_to(np.asarray(ref, np.float64), (len(theta),) + np.shape(ref)).copy()
    for k in range(nt):
        sel = np.asarray(masks[k], bool)
        if sel.any():
            X[:, sel] = rotate_about(X[:, sel], np.asarray(axp[k], np.float64), np.asarray(axu[k], np.float64),
                                     np.asarray(theta, np.float64)[:, k][:, None])
    return X


def world(Xi, state):
    """Ligand-frame coordinates [N, n, 3] -> world coordinates with states [N, >= 7] (t, q)."""
    state = np.asarray(state, np.float64)
    return np.einsum("nij,naj->nai", quat_matrix(state[:, 3:7]), Xi) + state[:, None, :3]


class Packed:
    """Float64 energy model of one pack_host batch (lig = the 13 ligand arrays, sf = the 5 scoring arrays)."""

    def __init__(self, lig, sf):
        self.ref, self.typ, self.tm, self.ax, self.axp, self.axu, self.pr, self.na, self.nt, self.np, _, _, \
            self.gslot = lig
        prm = np.asarray(sf[0], np.float64)
        (self.g1_off, self.g1_w, self.g2_off, self.g2_w, self.rep_off, self.hyd_good, self.hyd_bad, self.hb_good,
         self.hb_bad, self.cutoff, *self.w) = prm
        self.radius = np.asarray(sf[1], np.float64)
        self.hyd, self.don, self.acc = (np.asarray(a, bool) for a in sf[2:5])

    def pose_heavy(self, l, state):
        """Heavy-atom world coordinates [N, na, 3] of states [N, 7 + KM] of ligand l."""
        na, nt = int(self.na[l]), int(self.nt[l])
        Xi = internal(self.ref[l, :na], self.tm[l, :nt, :na], self.axp[l], self.axu[l], nt,
                      np.asarray(state, np.float64)[:, 7:])
        return world(Xi, state)

    def pair_energy(self, r, ti, tj):
        d = r - self.radius[ti] - self.radius[tj]
        e = self.w[0] * np.exp(-((d - self.g1_off) / self.g1_w) ** 2)
        e = e + self.w[1] * np.exp(-((d - self.g2_off) / self.g2_w) ** 2)
        e = e + self.w[2] * np.minimum(d - self.rep_off, 0.0) ** 2
        ramp = lambda good, bad: np.clip((bad - d) / (bad - good), 0.0, 1.0)
        e = e + self.w[3] * np.where(self.hyd[ti] & self.hyd[tj], ramp(self.hyd_good, self.hyd_bad), 0.0)
        hb = (self.don[ti] & self.acc[tj]) | (self.acc[ti] & self.don[tj])
        e = e + self.w[4] * np.where(hb, ramp(self.hb_good, self.hb_bad), 0.0)
        return np.where(r < self.cutoff, e, 0.0)

    def intra(self, l, X):
        npairs = int(self.np[l])
        if npairs == 0:
            return np.zeros(len(X))
        i, j = self.pr[l, :npairs, 0], self.pr[l, :npairs, 1]
        r = np.linalg.norm(X[:, i] - X[:, j], axis=-1)
        return self.pair_energy(r, self.typ[l, i], self.typ[l, j]).sum(-1)

    @staticmethod
    def penalty(X, lo, hi, pen):
        lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
        return pen * ((np.maximum(lo - X, 0) ** 2 + np.maximum(X - hi, 0) ** 2).sum(-1)).sum(-1)

    def exact_inter(self, l, X, rec_xyz, rec_types):
        rx = np.asarray(rec_xyz, np.float64)
        rt = np.asarray(rec_types, np.int64)
        ta = self.typ[l, :X.shape[1]]
        out = np.zeros(len(X))
        for n in range(len(X)):
            r = np.linalg.norm(X[n][:, None] - rx[None], axis=-1)
            out[n] = self.pair_energy(r, ta[:, None], rt[None, :]).sum()
        return out

    def grid_inter(self, l, X, maps, origin, spacing):
        """maps [T, nx, ny, nz] (values taken as float64), X [N, na, 3] -> [N] (no penalty)."""
        G = np.asarray(maps, np.float64)
        dims = np.array(G.shape[1:])
        f = (X - np.asarray(origin, np.float64)) / spacing
        fc = np.minimum(np.maximum(f, 0.0), dims - 1 - 1e-4)
        i0 = np.floor(fc).astype(np.int64)
        w = fc - i0
        slots = self.gslot[l, :X.shape[1]]
        e = np.zeros(X.shape[:2])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    ww = ((w[..., 0] if dx else 1 - w[..., 0]) * (w[..., 1] if dy else 1 - w[..., 1]) *
                          (w[..., 2] if dz else 1 - w[..., 2]))
                    e += ww * G[slots[None, :], i0[..., 0] + dx, i0[..., 1] + dy, i0[..., 2] + dz]
        return e.sum(-1)

    def grid_magnitude(self, l, X, maps, origin, spacing):
        """Sum over atoms of the trilinear weights times |map value| at the 8 corners: the scale of a relative
        storage error of the maps in the grid energy."""
        return self.grid_inter(l, X, np.abs(np.asarray(maps, np.float64)), origin, spacing)
