"""Shared builders for the tests: synthetic problems, packed arrays for the oracle, random poses."""
from __future__ import annotations

import functools

import numpy as np
import torch

from adock_b200 import params, synth
from adock_b200.grid import GridSet, grid_dims
from adock_b200.ligand import LigandBatch
from adock_b200.problem import PairPotential, Problem, pack_host, pad_receptors

SPACING = params.GRID_SPACING
PENALTY = params.OUT_OF_BOX_PENALTY


@functools.lru_cache(maxsize=4)
def receptor(kind="small"):
    """small: 300 atoms in an 18 A cube, 12 A box (33^3 points); cfg0: the 1,500-atom config-0 receptor."""
    if kind == "cfg0":
        return synth.config_receptor(0)
    xyz, types = synth.receptor(300, 18.0, seed=7)
    return synth.receptor_dict(xyz, types, np.full(3, 9.0), np.full(3, 12.0))


@functools.lru_cache(maxsize=8)
def ligands(kind="mixed"):
    if kind == "cfg0":
        return (synth.ligand(24, 5, 0),)
    if kind == "mixed":
        return (synth.ligand(24, 5, 0), synth.ligand(12, 0, 11), synth.ligand(45, 9, 3), synth.ligand(60, 15, 5))
    if kind == "big":
        return (synth.ligand(80, 20, 21), synth.ligand(70, 17, 22))
    raise ValueError(kind)


def lig_types(ligs):
    return np.unique(np.concatenate([[0]] + [np.asarray(l.types) for l in ligs]))


def oracle_grid(rec, sfp, lt):
    """Maps from the reference CPU builder (oracle)."""
    from oracle import ref as R
    o = rec["center"] - rec["size"] / 2
    return R.build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, SPACING, grid_dims(rec["size"], SPACING), lt)


def make_problem(rec, ligs, sfp, G, lt, device):
    """Problem over one receptor with maps G [T, nx, ny, nz] for types lt (numpy or torch)."""
    c, s = rec["center"], rec["size"]
    o = c - s / 2
    slot = -np.ones((1, params.N_XS), np.int64)
    slot[0, lt] = np.arange(len(lt))
    f32 = lambda a: torch.tensor(np.asarray(a, np.float32)[None], device=device)
    Gt = torch.as_tensor(G, device=device, dtype=torch.float32)
    gs = GridSet([Gt], f32(o), f32(o), f32(c + s / 2), SPACING, PENALTY, slot=torch.tensor(slot, device=device),
                 n_types=params.N_XS)
    lb = LigandBatch(list(ligs), device)
    return Problem(gs, lb, torch.zeros(len(ligs), dtype=torch.long, device=device), PairPotential(sfp, device),
                   rec=pad_receptors([rec], device))


def oracle_problem(prob):
    """RefProblem (reference CPU kernels) over the same packed arrays as the product."""
    from oracle import ref as R
    AM, KM, lig, sf = pack_host(prob)
    gs = prob.gs
    grid = dict(flat=gs.flat.float().cpu().numpy(), origin=gs.origin.cpu().numpy(), lo=gs.lo.cpu().numpy(),
                hi=gs.hi.cpu().numpy(), rec_idx=prob.rec_idx.cpu().numpy(), offs=gs.offs.cpu().numpy(),
                dims=gs.dims.cpu().numpy(), T=gs.T, spacing=gs.spacing, penalty=gs.penalty)
    rx, rt, rm = prob.rec
    return R.RefProblem(AM, KM, lig, sf, grid, rec=(rx.cpu().numpy(), rt.cpu().numpy(), rm.sum(1).cpu().numpy()))


def random_quat(shape, gen, device="cpu"):
    """Unit quaternions [*shape, 4] (w, x, y, z), uniform on the 3-sphere (normalised Gaussians)."""
    q = torch.randn(tuple(shape) + (4,), generator=gen, device=device)
    return q / q.norm(dim=-1, keepdim=True)


def random_states(prob, n_per_lig, seed=0, sigma=1.5):
    """Random poses around the box centre (t ~ N(c, sigma), uniform q, theta ~ U(-pi, pi) on real torsions):
    returns (chain_lig int32 [N], state float32 [N, 7+KM]) as numpy."""
    AM, KM, _, _ = pack_host(prob)
    lb = prob.lb
    L = lb.L
    g = torch.Generator().manual_seed(seed)
    c = prob.gs.lo[0].cpu() + (prob.gs.hi[0].cpu() - prob.gs.lo[0].cpu()) / 2
    t = c + torch.randn((L, n_per_lig, 3), generator=g) * sigma
    q = random_quat((L, n_per_lig), g, "cpu")
    th = (torch.rand((L, n_per_lig, lb.K), generator=g) * 2 - 1) * np.pi * lb.tvalid.cpu()[:, None]
    st = np.zeros((L * n_per_lig, 7 + KM), np.float32)
    st[:, :3] = t.reshape(-1, 3).numpy()
    st[:, 3:7] = q.reshape(-1, 4).numpy()
    k = min(lb.K, KM)
    st[:, 7:7 + k] = th.reshape(-1, lb.K)[:, :k].numpy()
    cl = np.repeat(np.arange(L), n_per_lig).astype(np.int32)
    return cl, st


def rel_close(a, b, rel=1e-4, floor=1e-4):
    """max |a - b| / max(|b|, floor / rel) (the reference's _rel_close metric, tests/test_cpukernel.py:50-53)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor / rel)).max())


def vec_rel(a, b, floor=1e-4):
    """max over rows of ||a - b|| / max(||b||, floor) (tests/test_cpukernel.py:43-47)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float((np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), floor)).max())
