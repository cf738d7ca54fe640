"""Padded ligand batches, forward kinematics and quaternion helpers (torch, host side).

Mirrors ``src/adock/ligand.py:122-237``: ``LigandBatch`` field names and padding, ``K`` bucketed to a
multiple of 8; pose = translation of the reference heavy-atom centroid + rotation (quaternion w,x,y,z) +
torsion angles applied leaf -> root about axes taken from the reference conformer (Rodrigues).
These functions serve finalize, neighbour lists and the float64 test oracle; the search itself runs in CUDA.
"""
from __future__ import annotations

import math

import numpy as np
import torch

K_BUCKET = 8


class LigandBatch:
    """Padded tensors for L ligands (one per complex)."""

    def __init__(self, preps, device="cpu"):
        self.preps = list(preps)
        L = len(self.preps)
        A = max(p.n for p in self.preps)
        K = max(max(p.n_tors for p in self.preps), 1)
        K = K_BUCKET * math.ceil(K / K_BUCKET)
        P = max(max(len(p.pairs) for p in self.preps), 1)
        ref = np.zeros((L, A, 3), np.float32)
        types = -np.ones((L, A), np.int64)
        amask = np.zeros((L, A), bool)
        axis = np.zeros((L, K, 2), np.int64)
        tmask = np.zeros((L, K, A), bool)
        tvalid = np.zeros((L, K), bool)
        pairs = np.zeros((L, P, 2), np.int64)
        pmask = np.zeros((L, P), bool)
        for l, p in enumerate(self.preps):
            ref[l, :p.n] = p.ref
            types[l, :p.n] = p.types
            amask[l, :p.n] = True
            axis[l, :p.n_tors] = p.tors_axis
            tmask[l, :p.n_tors, :p.n] = p.tors_mask
            tvalid[l, :p.n_tors] = True
            pairs[l, :len(p.pairs)] = p.pairs
            pmask[l, :len(p.pairs)] = True
        T = lambda a, dt=None: torch.as_tensor(a, device=device, dtype=dt)
        self.L, self.A, self.K, self.P = L, A, K, P
        self.ref, self.types = T(ref), T(types)
        self.heavy = self.types >= 0
        self.amask, self.axis, self.tmask, self.tvalid = T(amask), T(axis), T(tmask), T(tvalid)
        self.pairs, self.pmask = T(pairs), T(pmask)
        self.rg = T(np.array([p.rg for p in self.preps], np.float32))
        self.n_tors_vina = T(np.array([p.n_tors_vina for p in self.preps], np.float32))
        li = torch.arange(L, device=device)[:, None]
        pa, pb = self.ref[li, self.axis[..., 0]], self.ref[li, self.axis[..., 1]]
        u = pb - pa
        self.axis_p = pa
        self.axis_u = u / u.norm(dim=-1, keepdim=True).clamp(min=1e-6)

    def subset(self, idx):
        new = LigandBatch.__new__(LigandBatch)
        new.preps = [self.preps[i] for i in idx.tolist()]
        for k in ("A", "K", "P"):
            setattr(new, k, getattr(self, k))
        new.L = len(idx)
        for k in ("ref", "types", "heavy", "amask", "axis", "tmask", "tvalid", "pairs", "pmask", "rg",
                  "n_tors_vina", "axis_p", "axis_u"):
            setattr(new, k, getattr(self, k)[idx])
        return new

    def to(self, dtype):
        """Copy with floating-point fields in ``dtype`` (float64 for the test oracle)."""
        new = self.subset(torch.arange(self.L, device=self.ref.device))
        for k in ("ref", "axis_p", "axis_u", "rg"):
            setattr(new, k, getattr(new, k).to(dtype))
        return new


def quat_to_mat(q):
    q = q / q.norm(dim=-1, keepdim=True)
    w, x, y, z = q.unbind(-1)
    return torch.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1).reshape(q.shape[:-1] + (3, 3))


def rotvec_to_quat(r):
    ang = r.norm(dim=-1, keepdim=True)
    half = 0.5 * ang
    k = torch.where(ang > 1e-6, torch.sin(half) / ang.clamp(min=1e-6), 0.5 - ang * ang / 48.0)
    return torch.cat([torch.cos(half), r * k], -1)


def quat_mul(a, b):
    aw, ax, ay, az = a.unbind(-1)
    bw, bx, by, bz = b.unbind(-1)
    return torch.stack([aw * bw - ax * bx - ay * by - az * bz,
                        aw * bx + ax * bw + ay * bz - az * by,
                        aw * by - ax * bz + ay * bw + az * bx,
                        aw * bz + ax * by - ay * bx + az * bw], -1)


def random_quat(shape, gen, device):
    q = torch.randn(shape + (4,), generator=gen, device=device)
    return q / q.norm(dim=-1, keepdim=True)


def internal_coords(lb, theta):
    """theta [L, M, K] -> ligand-frame coordinates [L, M, A, 3] (torsions k = 0..K-1, leaf -> root)."""
    L, M, K = theta.shape
    X = lb.ref[:, None].expand(L, M, lb.A, 3)
    for k in range(lb.K):
        p = lb.axis_p[:, k][:, None, None]
        u = lb.axis_u[:, k][:, None, None]
        th = theta[:, :, k][..., None, None]
        v = X - p
        c, s = torch.cos(th), torch.sin(th)
        uu = u.expand_as(v)
        vr = v * c + torch.cross(uu, v, dim=-1) * s + uu * (v * uu).sum(-1, keepdim=True) * (1 - c)
        X = torch.where(lb.tmask[:, k][:, None, :, None], p + vr, X)
    return X


def pose_coords(lb, t, q0, r, theta):
    """World coordinates [L, M, A, 3] of poses (t [L,M,3], q0 [L,M,4], rotation vector r [L,M,3], theta [L,M,K])."""
    X = internal_coords(lb, theta)
    R = quat_to_mat(quat_mul(rotvec_to_quat(r), q0))
    return torch.einsum("lmij,lmaj->lmai", R, X) + t[:, :, None, :]
