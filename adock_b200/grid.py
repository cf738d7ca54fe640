"""Receptor grid maps and their storage contract (reference ``src/adock/grid.py``, ``src/adock/fit/gridfit.py``).

``build_grid`` / ``build_grid_fit`` keep the reference signatures (grid.py:132, gridfit.py:71) and run the
sm_100a kernels of ``libadock_b200.so`` over a receptor cell list built here (``CellList``). ``GridSet`` keeps the reference storage contract (flat concatenation of
per-receptor ``[T_r, nx, ny, nz]`` maps, ``offs``, ``dims``, ``slot``, ``origin``, ``lo``, ``hi``) and can carry an
FP16/BF16 copy of ``flat`` for the search kernels (FP32 interpolation and accumulation either way).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from .params import grid_prm

MAX_TYPES = 24   # grid.py:74
MAX_LT = 64      # gridfit.py:61


def _cuda_device(device):
    dev = torch.device(device)
    if dev.type != "cuda":
        raise RuntimeError("adock_b200 grid builders run on CUDA devices only (no CPU path)")
    return dev


CELL_MIN = 4.0   # A, edge of the receptor cell list's cells (at least)


class CellList:
    """Receptor atoms sorted by cell of a uniform grid (cubic cells of edge ``size`` from ``origin``), with the start
    of every cell; cell (cx, cy, cz) = index (cx * ny + cy) * nz + cz. ``order`` is the sorting permutation (stable,
    so atoms of one cell stay in receptor order)."""

    def __init__(self, xyz, cutoff, spacing):
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        self.size = max(CELL_MIN, (4 * spacing + 2 * cutoff) / 7.0)
        lo = xyz.min(0) if len(xyz) else np.zeros(3, np.float32)
        hi = xyz.max(0) if len(xyz) else np.zeros(3, np.float32)
        self.origin = (lo - 1e-3).astype(np.float32)
        self.dims = np.maximum(np.ceil((hi - self.origin + 1e-3) / self.size).astype(np.int32), 1)
        c = np.minimum(((xyz - self.origin) / self.size).astype(np.int64), self.dims - 1)
        cid = (c[:, 0] * self.dims[1] + c[:, 1]) * self.dims[2] + c[:, 2]
        self.order = np.argsort(cid, kind="stable")
        self.start = np.concatenate([[0], np.cumsum(np.bincount(cid, minlength=int(self.dims.prod())))]).astype(np.int32)

    def args(self, device):
        """(start tensor on device, dims, origin, size) for the *_cells entry points."""
        return (torch.as_tensor(self.start, device=device), np.ascontiguousarray(self.dims, np.int32),
                np.ascontiguousarray(self.origin, np.float32), float(self.size))


def build_grid(rec_xyz, rec_types, sfp, origin, spacing, n, lig_types=None, per_term=False, device="cuda"):
    """Return torch tensor [T, nx, ny, nz] (or [5, T, nx, ny, nz] unweighted if per_term) on ``device``.

    n: int or (nx, ny, nz). lig_types: XS type indices to build (default: all types)."""
    if np.isscalar(n):
        n = (int(n),) * 3
    nx, ny, nz = map(int, n)
    T = len(sfp["radius"])
    lig_types = np.arange(T, dtype=np.int32) if lig_types is None else np.asarray(lig_types, dtype=np.int32)
    assert len(lig_types) <= MAX_TYPES
    dev = _cuda_device(device)
    xyz = np.ascontiguousarray(rec_xyz, np.float32).reshape(-1, 3)
    cells = CellList(xyz, float(sfp["cutoff"]), float(spacing))
    rx = torch.as_tensor(xyz[cells.order], device=dev)
    rt = torch.as_tensor(np.ascontiguousarray(np.asarray(rec_types)[cells.order], np.int32), device=dev)
    cstart, cdims, corg, csize = cells.args(dev)
    nlt = len(lig_types)
    out = torch.empty(((5 if per_term else 1) * nlt * nx * ny * nz,), dtype=torch.float32, device=dev)
    tabs = [np.ascontiguousarray(sfp[k], np.int32) for k in ("hydrophobic", "donor", "acceptor")]
    rad = np.ascontiguousarray(sfp["radius"], np.float32)
    prm = grid_prm(sfp)
    with torch.cuda.device(dev):
        _lib.call("adock_grid_vina_cells", _lib.ptr(rx), _lib.ptr(rt), len(rx), _lib.ptr(cstart), _lib.ptr(cdims),
                  _lib.ptr(corg), csize, _lib.ptr(rad), _lib.ptr(tabs[0]),
                  _lib.ptr(tabs[1]), _lib.ptr(tabs[2]), T, _lib.ptr(lig_types), nlt, float(origin[0]),
                  float(origin[1]), float(origin[2]), float(spacing), nx, ny, nz, _lib.ptr(prm), int(per_term),
                  _lib.ptr(out), _lib.stream_ptr())
    shape = ((5, nlt) if per_term else (nlt,)) + (nx, ny, nz)
    return out.view(shape)


def build_grid_fit(rec_xyz, rec_ext, pot, origin, spacing, n, device="cuda"):
    """Grid [TL, n, n, n] of the fitted inter energy for the compact ligand types of ``pot`` (FittedPotential)."""
    spec = pot.spec
    nlt = pot.TL
    assert nlt <= MAX_LT
    if np.isscalar(n):
        n = (int(n),) * 3
    nx, ny, nz = map(int, n)
    dev = _cuda_device(device)
    xyz = np.ascontiguousarray(rec_xyz, np.float32).reshape(-1, 3)
    cells = CellList(xyz, float(spec.cutoff), float(spacing))
    rx = torch.as_tensor(xyz[cells.order], device=dev)
    re = torch.as_tensor(np.ascontiguousarray(np.asarray(rec_ext)[cells.order], np.int32), device=dev)
    cstart, cdims, corg, csize = cells.args(dev)
    W = torch.as_tensor(np.ascontiguousarray(np.asarray(pot.W, np.float32)), device=dev)
    rad_rec = torch.as_tensor(np.ascontiguousarray(spec.rec_radius, np.float32), device=dev)
    rad_lig = np.ascontiguousarray(pot.radius, np.float32)
    prm = spec.grid_prm()
    out = torch.empty((nlt * nx * ny * nz,), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        _lib.call("adock_grid_fit_cells", _lib.ptr(rx), _lib.ptr(re), len(rx), _lib.ptr(cstart), _lib.ptr(cdims),
                  _lib.ptr(corg), csize, _lib.ptr(rad_rec), int(W.shape[0]),
                  _lib.ptr(rad_lig), nlt, _lib.ptr(W), float(origin[0]), float(origin[1]), float(origin[2]),
                  float(spacing), nx, ny, nz, _lib.ptr(prm), _lib.ptr(out), _lib.stream_ptr())
    return out.view(nlt, nx, ny, nz)


def trilinear(flat, origin, lo, hi, x, t, rec_idx, mask, dims, offs, slot, spacing: float, penalty: float):
    """Torch trilinear lookup + quadratic out-of-box penalty (grid.py:169-194); differentiable w.r.t. x."""
    o = origin[rec_idx]
    dm = dims[rec_idx]
    f = (x - o) / spacing
    fc = torch.minimum(f.clamp(min=0.0), (dm - 1).to(f.dtype) - 1e-4)
    i0 = fc.detach().floor().long()
    w = fc - i0
    ny, nz = dm[..., 1], dm[..., 2]
    base = offs[rec_idx] + slot[rec_idx, t.clamp(min=0)].clamp(min=0) * (dm[..., 0] * ny * nz)
    e = 0.0
    for dx in (0, 1):
        wx = w[..., 0] if dx else 1 - w[..., 0]
        for dy in (0, 1):
            wy = w[..., 1] if dy else 1 - w[..., 1]
            for dz in (0, 1):
                wz = w[..., 2] if dz else 1 - w[..., 2]
                idx = base + ((i0[..., 0] + dx) * ny + (i0[..., 1] + dy)) * nz + (i0[..., 2] + dz)
                e = e + wx * wy * wz * flat[idx].to(wx.dtype)
    out = (lo[rec_idx] - x).clamp(min=0) ** 2 + (x - hi[rec_idx]).clamp(min=0) ** 2
    e = e + penalty * out.sum(-1)
    if mask is not None:
        e = torch.where(mask, e, torch.zeros_like(e))
    return e


class GridSet:
    """Batch of receptor grids with per-receptor origin and box (grid.py:197-248).

    grids: stacked tensor [R, T, n, n, n] (common cube) or a list of per-receptor tensors [T, nx, ny, nz].
    slot: optional [R, n_types] (global type -> grid slot, -1 = not built); default identity."""

    def __init__(self, grids, origins, box_lo, box_hi, spacing, penalty, slot=None, n_types=None):
        dev = origins.device
        if torch.is_tensor(grids):
            self.G = grids
            self.R, self.T, self.n = grids.shape[0], grids.shape[1], grids.shape[2]
            self.flat = grids.reshape(-1)
            sz = self.T * self.n ** 3
            self.dims = torch.full((self.R, 3), self.n, dtype=torch.long, device=dev)
            self.offs = torch.arange(self.R, device=dev, dtype=torch.long) * sz
        else:
            self.G = None
            self.R, self.T = len(grids), grids[0].shape[0]
            self.flat = torch.cat([g.reshape(-1) for g in grids])
            self.dims = torch.tensor([list(g.shape[1:]) for g in grids], dtype=torch.long, device=dev)
            sizes = torch.tensor([g.numel() for g in grids], dtype=torch.long, device=dev)
            self.offs = torch.cumsum(sizes, 0) - sizes
            self.n = int(self.dims.max())
        if slot is None:
            slot = torch.arange(self.T, device=dev).expand(self.R, self.T).contiguous()
        else:
            self.T = n_types
        self.slot = slot
        self.origin = origins
        self.lo, self.hi = box_lo, box_hi
        self.spacing = spacing
        self.penalty = penalty
        self._lowp = {}

    def lookup(self, x, t, rec_idx, mask=None):
        return trilinear(self.flat, self.origin, self.lo, self.hi, x, t, rec_idx, mask, self.dims, self.offs,
                         self.slot, self.spacing, self.penalty)

    def lookup_nearest(self, x, t, rec_idx):
        """Nearest-grid-point energy (no gradient), grid.py:238-247."""
        dm = self.dims[rec_idx]
        f = torch.minimum(((x - self.origin[rec_idx]) / self.spacing).round().clamp(min=0).long(), dm - 1)
        ny, nz = dm[..., 1], dm[..., 2]
        base = self.offs[rec_idx] + self.slot[rec_idx, t.clamp(min=0)].clamp(min=0) * (dm[..., 0] * ny * nz)
        e = self.flat[base + (f[..., 0] * ny + f[..., 1]) * nz + f[..., 2]]
        lo, hi = self.lo[rec_idx], self.hi[rec_idx]
        out = (lo - x).clamp(min=0) ** 2 + (x - hi).clamp(min=0) ** 2
        return e + self.penalty * out.sum(-1)

    def storage(self, dtype: str = "f32"):
        """(flat tensor, ADOCK_GRID_* code) of the maps in ``dtype`` ('f32', 'f16', 'bf16'); low-precision copies
        are made once (round to nearest) and kept."""
        if dtype == "f32":
            return self.flat.float().contiguous(), _lib.ADOCK_GRID_F32
        if dtype not in self._lowp:
            code = {"f16": _lib.ADOCK_GRID_F16, "bf16": _lib.ADOCK_GRID_BF16}[dtype]
            tdt = {"f16": torch.float16, "bf16": torch.bfloat16}[dtype]
            src = self.flat.float().contiguous()
            dst = torch.empty(src.shape, dtype=tdt, device=src.device)
            with torch.cuda.device(src.device):
                _lib.call("adock_grid_convert", _lib.ptr(src), _lib.ptr(dst), src.numel(), code, _lib.stream_ptr())
            self._lowp[dtype] = (dst, code)
        return self._lowp[dtype]


def grid_dims(size, spacing):
    return tuple(int(math.ceil(x / spacing)) + 1 for x in size)


def make_gridset(receptors, sfp, spacing, penalty, device="cuda", per_term=False, cubic=None, lig_types=None,
                 builder=None):
    """receptors: list of dicts with rec_xyz, rec_types, center, size (grid.py:250-282).

    cubic=True: common cube n for all receptors (stacked .G). cubic=False (default unless per_term): each receptor
    gets n_d = ceil(size_d / spacing) + 1 points per axis and, with lig_types, only the ligand's own types plus
    type 0 (C_H, the Stage-A probe type). ``builder`` replaces ``build_grid`` (same signature)."""
    builder = builder or build_grid
    cubic = per_term if cubic is None else cubic
    T_all = len(sfp["radius"])
    if lig_types is not None and not cubic:
        sel = [np.unique(np.concatenate([[0], np.asarray(lt, dtype=np.int64)])) for lt in lig_types]
    else:
        sel = [np.arange(T_all)] * len(receptors)
    slot = -np.ones((len(receptors), T_all), np.int64)
    for i, st in enumerate(sel):
        slot[i, st] = np.arange(len(st))
    n = int(math.ceil(max(max(r["size"]) for r in receptors) / spacing)) + 1
    grids, origins, lo, hi = [], [], [], []
    for r, st in zip(receptors, sel):
        c, s = np.asarray(r["center"], float), np.asarray(r["size"], float)
        origin = c - s / 2.0
        nn = n if cubic else grid_dims(s, spacing)
        grids.append(builder(r["rec_xyz"], r["rec_types"], sfp, origin, spacing, nn, per_term=per_term, device=device,
                             lig_types=None if cubic else st))
        origins.append(origin)
        lo.append(c - s / 2.0)
        hi.append(c + s / 2.0)
    tt = lambda a: torch.tensor(np.array(a), dtype=torch.float32, device=device)
    if cubic:
        return GridSet(torch.stack(grids), tt(origins), tt(lo), tt(hi), spacing, penalty)
    return GridSet(grids, tt(origins), tt(lo), tt(hi), spacing, penalty, slot=torch.as_tensor(slot, device=device),
                   n_types=T_all)


def make_gridset_fit(preps, pot, spacing, penalty, device="cuda", builder=None):
    """preps: dicts with rec_xyz, rec_ext, center, size; common cube n (gridfit.py:96-108)."""
    builder = builder or build_grid_fit
    n = int(math.ceil(max(max(r["size"]) for r in preps) / spacing)) + 1
    grids, origins, lo, hi = [], [], [], []
    for r in preps:
        c, s = np.asarray(r["center"], float), np.asarray(r["size"], float)
        origin = c - s / 2.0
        grids.append(builder(r["rec_xyz"], r["rec_ext"], pot, origin, spacing, n, device=device))
        origins.append(origin)
        lo.append(c - s / 2.0)
        hi.append(c + s / 2.0)
    tt = lambda a: torch.tensor(np.array(a), dtype=torch.float32, device=device)
    return GridSet(torch.stack(grids), tt(origins), tt(lo), tt(hi), spacing, penalty)
