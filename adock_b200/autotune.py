"""Autotuner for the persistent Monte-Carlo kernel's launch shape.

The MC kernel trades registers per thread for resident warps per SM (``adock_mc_args_t.variant``: 4, 6 or 8
resident 128-thread blocks per SM, i.e. 128, 80 or 64 registers). Which is fastest depends on the atom bucket
(AM), the torsion bucket (KM), the map storage type and the GPU. ``tune_mc`` brings the batch's chains (up to 16,384)
into the regime of a running search (optimised starts + 8 MC steps), then times 8 and 32 MC steps under each
variant and keeps the one with the least time per step between the two; results are cached per (device name, AM,
KM, map dtype) for the life of the process and in ``$ADOCK_TUNE_CACHE`` (a JSON file) if set. A launch of the
80-register variant has about 5 ms more fixed cost than the 128-register one and less per step (2.79 vs 2.93 ms on
the 256-ligand batch), so the time of one short sample picked the variant that a 2,000-step search ran 8 % slower.
"""
from __future__ import annotations

import json
import os
import threading

import torch

VARIANTS = (1, 2, 3)
_cache = {}
_lock = threading.Lock()


def _key(kp):
    return f"{torch.cuda.get_device_name(kp.device)}|AM{kp.AM}|KM{kp.KM}|{kp.grid_dtype}"


def _load_file():
    path = os.environ.get("ADOCK_TUNE_CACHE")
    if path and os.path.exists(path):
        try:
            with open(path) as fh:
                _cache.update(json.load(fh))
        except (OSError, ValueError):
            pass


def _save_file():
    path = os.environ.get("ADOCK_TUNE_CACHE")
    if path:
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as fh:
            json.dump(_cache, fh, indent=1)
        os.replace(tmp, path)


def tune_mc(kp, chain_lig, state, max_chains=16384, steps=32, reps=1):
    """Return the fastest MC launch variant for this kernel object (cached). Each variant runs ``steps`` and
    ``steps // 4`` MC steps from the same starts; the time per step between the two (the best of ``reps``) counts.
    The sample is the whole batch up to ``max_chains`` chains: a chain's time scales with its step count, so a short
    run over the batch has the waves and the tail of the full persistent launch (a sample of about one wave would
    be decided by its tail instead)."""
    key = _key(kp)
    with _lock:
        if not _cache:
            _load_file()
        if key in _cache:
            return int(_cache[key]["variant"])
    dev = kp.device
    N = state.shape[0]
    if N <= max_chains:
        idx = torch.arange(N, device=dev, dtype=torch.long)
    else:
        # the most expensive chains plus an even spread of the rest
        order = kp.chain_order(chain_lig).long()
        take = order[: max_chains // 4].tolist() + order[max_chains // 4:: max(1, N // max_chains)].tolist()
        idx = torch.tensor(sorted(set(take))[:max_chains], device=dev, dtype=torch.long)
    cl = chain_lig[idx].to(torch.int32)
    ci = torch.arange(len(idx), device=dev, dtype=torch.int32)
    times = {}
    # bring the chains from their start poses into the regime of a running search (optimised start + 8 steps)
    # before timing: the first steps from unoptimised starts run longer local optimisations than the steady state
    start, best0 = state[idx].contiguous(), state[idx].contiguous()
    start_e = torch.zeros(len(idx), device=dev)
    best0_e = torch.full((len(idx),), float("inf"), device=dev)
    kp.run_mc(cl, ci, start, start_e, best0, best0_e, True, 8, 0, 1.2, 2.0, 2.0, 1, 0, variant=VARIANTS[0])
    def timed(v, n):
        cur, best = start.clone(), start.clone()
        ce = start_e.clone()
        be = torch.full((len(idx),), float("inf"), device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        kp.run_mc(cl, ci, cur, ce, best, be, False, n, 0, 1.2, 2.0, 2.0, 1, 0, variant=v)
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1)

    for v in VARIANTS:
        timed(v, 1)   # warm-up / module load
        # milliseconds per MC step from two run lengths: a launch also has a fixed part (ramp-up and tail) that
        # differs between variants by a few ms and would decide a short sample, but not a 2,000-step search
        short = max(1, steps // 4)
        times[v] = min((timed(v, steps) - timed(v, short)) / (steps - short) for _ in range(reps))
    best_v = min(times, key=times.get)
    with _lock:
        _cache[key] = {"variant": best_v, "ms_per_step": {str(k): round(t, 4) for k, t in times.items()},
                       "chains": len(idx)}
        _save_file()
    return best_v


def cached():
    return dict(_cache)
