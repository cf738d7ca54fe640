"""Map-precision report: per-pose energy error of FP32 / FP16 / BF16 map storage against float64 evaluation.

The search interpolates and accumulates in FP32 whatever the map storage; this measures what the storage costs.
For N random poses (t ~ N(box centre, 1.5 A), uniform q, theta ~ U(-pi, pi)) of a ligand batch, the batched
energy kernel (adock_eg) runs on each storage, and the reference value is the float64 device evaluation of the
same energy (adock_rescore64 in grid mode: float64 kinematics, float64 trilinear interpolation of the FP32-built
maps, float64 penalty and intra-pair terms). Reported per storage: evaluations/s and |E - E64| quantiles.
"""
from __future__ import annotations

import numpy as np
import torch

from . import params
from .grid import make_gridset
from .kernel import B200KernelProblem
from .ligand import LigandBatch
from .problem import PairPotential, Problem, pad_receptors


def random_poses(prob, kp, n_poses, seed=0, sigma=1.5):
    """(chain_lig int32 [N], state [N, SD]) on the device: poses spread evenly over the batch's ligands."""
    dev = kp.device
    L = prob.lb.L
    g = torch.Generator(device=dev).manual_seed(seed)
    cl = (torch.arange(n_poses, device=dev) % L).to(torch.int32)
    c = (prob.gs.lo[0] + prob.gs.hi[0]) / 2
    t = c + torch.randn((n_poses, 3), generator=g, device=dev) * sigma
    q = torch.randn((n_poses, 4), generator=g, device=dev)
    q = q / q.norm(dim=1, keepdim=True)                 # uniform on the unit 3-sphere
    th = (torch.rand((n_poses, prob.lb.K), generator=g, device=dev) * 2 - 1) * np.pi
    th = th * prob.lb.tvalid[cl.long()]
    return cl, kp.pack(t, q, th)


def _time(fn, reps=10, warmup=2):
    """(last output, median ms per call): each call bracketed by its own events, so a one-off host delay (an
    allocation, a module load) in one call does not enter the figure."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for e0, e1 in ev:
        e0.record()
        out = fn()
        e1.record()
    torch.cuda.synchronize()
    return out, float(np.median([e0.elapsed_time(e1) for e0, e1 in ev]))


def precision_report(rec, ligs, n_poses=100_000, device="cuda", dtypes=("f32", "f16", "bf16"), seed=0):
    """rec: receptor dict (rec_xyz, rec_types, center, size); ligs: preps. Returns a dict per storage dtype."""
    dev = torch.device(device)
    sfp = params.sf_params("vina")
    types = np.unique(np.concatenate([l.types for l in ligs]))
    gs = make_gridset([rec], sfp, params.GRID_SPACING, params.OUT_OF_BOX_PENALTY, device=dev, lig_types=[types])
    lb = LigandBatch(ligs, dev)
    prob = Problem(gs, lb, torch.zeros(len(ligs), dtype=torch.long, device=dev), PairPotential(sfp, dev),
                   rec=pad_receptors([rec], dev))
    kp32 = B200KernelProblem(prob, grid_dtype="f32")
    cl, st = random_poses(prob, kp32, n_poses, seed=seed)
    e64, _, _ = kp32.rescore64(cl, st, exact=False)
    e64 = e64.cpu().numpy()
    out = {"poses": int(n_poses), "ligands": len(ligs), "reference": "float64 device evaluation (grid mode)"}
    for dt in dtypes:
        kp = kp32 if dt == "f32" else B200KernelProblem(prob, grid_dtype=dt)
        (e, _), ms = _time(lambda: kp.energy_grad(cl, st))
        err = np.abs(e.cpu().numpy().astype(np.float64) - e64)
        rel = err / np.maximum(np.abs(e64), 1.0)
        out[dt] = {"evals_per_s": n_poses / (ms / 1e3), "ms": ms,
                   "abs_err": {"median": float(np.median(err)), "p99": float(np.quantile(err, 0.99)),
                               "max": float(err.max())},
                   "rel_err_floor1": {"median": float(np.median(rel)), "p99": float(np.quantile(rel, 0.99)),
                                      "max": float(rel.max())}}
    return out
