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


def _dims3(n):
    return tuple(map(int, (n,) * 3 if np.isscalar(n) else n))


def prepare_grid(rec_xyz, rec_types, sfp, origin, spacing, n, lig_types=None, per_term=False, device="cuda"):
    """The Vina map build split into its host preparation (cell list, device copies of the receptor and tables)
    and a ``launch(out)`` that only issues the kernel into ``out`` (flat float32 tensor of ``size`` elements).
    Returns (launch, size, shape)."""
    nx, ny, nz = _dims3(n)
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
    tabs = [np.ascontiguousarray(sfp[k], np.int32) for k in ("hydrophobic", "donor", "acceptor")]
    rad = np.ascontiguousarray(sfp["radius"], np.float32)
    prm = grid_prm(sfp)
    o = [float(x) for x in origin]

    def launch(out):
        with torch.cuda.device(dev):
            _lib.call("adock_grid_vina_cells", _lib.ptr(rx), _lib.ptr(rt), len(rx), _lib.ptr(cstart),
                      _lib.ptr(cdims), _lib.ptr(corg), csize, _lib.ptr(rad), _lib.ptr(tabs[0]), _lib.ptr(tabs[1]),
                      _lib.ptr(tabs[2]), T, _lib.ptr(lig_types), nlt, o[0], o[1], o[2], float(spacing), nx, ny, nz,
                      _lib.ptr(prm), int(per_term), _lib.ptr(out), _lib.stream_ptr())
        return out

    shape = ((5, nlt) if per_term else (nlt,)) + (nx, ny, nz)
    return launch, int(np.prod(shape)), shape


def build_grid(rec_xyz, rec_types, sfp, origin, spacing, n, lig_types=None, per_term=False, device="cuda"):
    """Return torch tensor [T, nx, ny, nz] (or [5, T, nx, ny, nz] unweighted if per_term) on ``device``.

    n: int or (nx, ny, nz). lig_types: XS type indices to build (default: all types)."""
    launch, size, shape = prepare_grid(rec_xyz, rec_types, sfp, origin, spacing, n, lig_types, per_term, device)
    return launch(torch.empty(size, dtype=torch.float32, device=_cuda_device(device))).view(shape)


def prepare_grid_fit(rec_xyz, rec_ext, pot, origin, spacing, n, device="cuda"):
    """``build_grid_fit`` split like ``prepare_grid``: returns (launch, size, shape)."""
    spec = pot.spec
    nlt = pot.TL
    assert nlt <= MAX_LT
    nx, ny, nz = _dims3(n)
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
    o = [float(x) for x in origin]

    def launch(out):
        with torch.cuda.device(dev):
            _lib.call("adock_grid_fit_cells", _lib.ptr(rx), _lib.ptr(re), len(rx), _lib.ptr(cstart), _lib.ptr(cdims),
                      _lib.ptr(corg), csize, _lib.ptr(rad_rec), int(W.shape[0]), _lib.ptr(rad_lig), nlt, _lib.ptr(W),
                      o[0], o[1], o[2], float(spacing), nx, ny, nz, _lib.ptr(prm), _lib.ptr(out), _lib.stream_ptr())
        return out

    return launch, nlt * nx * ny * nz, (nlt, nx, ny, nz)


def build_grid_fit(rec_xyz, rec_ext, pot, origin, spacing, n, device="cuda"):
    """Grid [TL, n, n, n] of the fitted inter energy for the compact ligand types of ``pot`` (FittedPotential)."""
    launch, size, shape = prepare_grid_fit(rec_xyz, rec_ext, pot, origin, spacing, n, device)
    return launch(torch.empty(size, dtype=torch.float32, device=_cuda_device(device))).view(shape)


class GridSet:
    """Maps of R receptors in the reference's storage contract (``grid.py:197-248``): ``flat`` concatenates every
    receptor's ``[T_r, nx, ny, nz]`` block (z fastest), with ``offs`` [R] element offsets, ``dims`` [R, 3], ``slot``
    [R, n_types] (global XS type -> map index, -1 = not built), ``origin``, ``lo``, ``hi`` [R, 3], ``spacing`` and
    ``penalty``. ``grids`` is either a stacked tensor [R, T, n, n, n] (a common cube, kept as ``G``) or a list of
    per-receptor tensors. Without ``slot`` every receptor holds all T types in order."""

    def __init__(self, grids, origins, box_lo, box_hi, spacing, penalty, slot=None, n_types=None):
        dev = origins.device
        blocks = list(grids.unbind(0)) if torch.is_tensor(grids) else list(grids)
        self.G = grids if torch.is_tensor(grids) else None
        self.R = len(blocks)
        self.flat = grids.reshape(-1) if self.G is not None else torch.cat([b.reshape(-1) for b in blocks])
        self.dims = torch.tensor([list(b.shape[1:]) for b in blocks], dtype=torch.long, device=dev)
        sizes = torch.tensor([b.numel() for b in blocks], dtype=torch.long, device=dev)
        self.offs = torch.cumsum(sizes, 0) - sizes
        self.n = int(self.dims.max())
        built = blocks[0].shape[0]
        self.T = built if slot is None else n_types
        self.slot = (torch.arange(built, device=dev).repeat(self.R, 1) if slot is None else slot)
        self.origin, self.lo, self.hi = origins, box_lo, box_hi
        self.spacing, self.penalty = spacing, penalty
        self._lowp = {}

    def storage(self, dtype: str = "f32"):
        """(flat tensor, ADOCK_GRID_* code) of the maps in ``dtype`` ('f32', 'f16', 'bf16'); low-precision copies
        are made once (round to nearest) and kept."""
        if dtype == "f32":
            return self.flat.float().contiguous(), _lib.ADOCK_GRID_F32
        if dtype not in self._lowp:
            code = {"f16": _lib.ADOCK_GRID_F16, "bf16": _lib.ADOCK_GRID_BF16}[dtype]
            src = self.flat.float().contiguous()
            dst = torch.empty(src.shape, dtype={"f16": torch.float16, "bf16": torch.bfloat16}[dtype], device=src.device)
            with torch.cuda.device(src.device):
                _lib.call("adock_grid_convert", _lib.ptr(src), _lib.ptr(dst), src.numel(), code, _lib.stream_ptr())
            self._lowp[dtype] = (dst, code)
        return self._lowp[dtype]


def grid_dims(size, spacing):
    return tuple(int(math.ceil(x / spacing)) + 1 for x in size)


def _boxes(receptors):
    """(centre, size, origin = low corner) of every receptor's box, float64."""
    c = np.array([np.asarray(r["center"], float) for r in receptors])
    s = np.array([np.asarray(r["size"], float) for r in receptors])
    return c, s, c - s / 2.0


def _f32(a, device):
    return torch.as_tensor(np.asarray(a, np.float32), device=device)


def make_gridset(receptors, sfp, spacing, penalty, device="cuda", per_term=False, cubic=None, lig_types=None,
                 builder=None):
    """GridSet of receptor dicts (rec_xyz, rec_types, center, size), reference ``grid.py:250-282``.

    cubic (default: per_term): one common cube of n = ceil(max size / spacing) + 1 points per axis for all receptors
    and all types (stacked ``G``). Otherwise each receptor gets ceil(size_d / spacing) + 1 points per axis and, with
    ``lig_types`` (one list per receptor), only those types plus type 0 (C_H, the Stage-A probe). ``builder``
    replaces ``build_grid`` (same signature)."""
    builder = builder or build_grid
    cubic = per_term if cubic is None else cubic
    n_types = len(sfp["radius"])
    centre, size, origin = _boxes(receptors)
    if cubic:
        n = int(math.ceil(size.max() / spacing)) + 1
        G = torch.stack([builder(r["rec_xyz"], r["rec_types"], sfp, o, spacing, n, per_term=per_term, device=device,
                                 lig_types=None) for r, o in zip(receptors, origin)])
        return GridSet(G, _f32(origin, device), _f32(origin, device), _f32(centre + size / 2, device), spacing,
                       penalty)
    types = [np.union1d([0], np.asarray(t, np.int64)) if lig_types is not None else np.arange(n_types)
             for t in (lig_types if lig_types is not None else [None] * len(receptors))]
    slot = np.full((len(receptors), n_types), -1, np.int64)
    for r, t in enumerate(types):
        slot[r, t] = np.arange(len(t))
    maps = [builder(r["rec_xyz"], r["rec_types"], sfp, o, spacing, grid_dims(sz, spacing), per_term=per_term,
                    device=device, lig_types=t) for r, o, sz, t in zip(receptors, origin, size, types)]
    return GridSet(maps, _f32(origin, device), _f32(origin, device), _f32(centre + size / 2, device), spacing,
                   penalty, slot=torch.as_tensor(slot, device=device), n_types=n_types)


def make_gridset_fit(preps, pot, spacing, penalty, device="cuda", builder=None):
    """GridSet of the fitted function's maps (reference ``gridfit.py:96-108``): preps with rec_xyz, rec_ext, center,
    size; one common cube for all receptors, the compact ligand types of ``pot``."""
    builder = builder or build_grid_fit
    centre, size, origin = _boxes(preps)
    n = int(math.ceil(size.max() / spacing)) + 1
    G = torch.stack([builder(r["rec_xyz"], r["rec_ext"], pot, o, spacing, n, device=device)
                     for r, o in zip(preps, origin)])
    return GridSet(G, _f32(origin, device), _f32(origin, device), _f32(centre + size / 2, device), spacing, penalty)
