"""adock_mc_noalloc: the Monte-Carlo entry point for callers that cannot allocate device memory.

Such callers (a framework capturing a stream into a CUDA graph that forbids allocation during capture, an
embedder whose memory pool owns the device, a host application that hands over only raw input/output pointers)
cannot provide the scratch adock_mc needs. The no-allocation variant keeps that scratch in a fixed device array
inside the library. Here it must give the same chains as adock_mc on the same inputs, on two calls in a row
(the second call reuses the scratch the first call left behind), and reject a batch that does not fit.

This file is collected last so that a run stopping at the first failure has already run every other test.
"""
import numpy as np
import pytest
import torch

from helpers import ligands, lig_types, make_problem, random_states, receptor, rel_close

pytestmark = pytest.mark.gpu


def _problem(dev):
    from adock_b200 import params
    from adock_b200.grid import build_grid, grid_dims
    sfp = params.sf_params("vina")
    rec = receptor("small")
    ligs = ligands("mixed")
    lt = lig_types(ligs)
    o = rec["center"] - rec["size"] / 2
    G = build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, params.GRID_SPACING,
                   grid_dims(rec["size"], params.GRID_SPACING), lt, device=dev)
    return make_problem(rec, ligs, sfp, G.cpu().numpy(), lt, dev)


def test_mc_noalloc_matches_mc_on_two_calls():
    from adock_b200 import _lib
    from adock_b200.kernel import B200KernelProblem
    assert torch.cuda.is_available()
    dev = torch.device("cuda:0")
    prob = _problem(dev)
    kp = B200KernelProblem(prob)
    for call in range(2):
        cl, st = random_states(prob, 24, seed=10 + call, sigma=1.0)
        M = len(cl)
        clg = torch.as_tensor(cl, device=dev)
        cig = torch.arange(M, dtype=torch.int32, device=dev) * 3 + call
        e0, _ = kp.energy_grad(clg, torch.as_tensor(st, device=dev))
        # existing entry point (caller-allocated scratch)
        cur1, best1 = torch.as_tensor(st, device=dev).clone(), torch.as_tensor(st, device=dev).clone()
        ce1, be1 = e0.clone(), torch.full((M,), float("inf"), device=dev)
        kp.run_mc(clg, cig, cur1, ce1, best1, be1, call == 0, 3, 4, 1.2, 2.0, 2.0, 777 + call, 2 * call)
        # no-allocation entry point through the C-ABI
        cur2, best2 = torch.as_tensor(st, device=dev).clone(), torch.as_tensor(st, device=dev).clone()
        ce2, be2 = e0.clone(), torch.full((M,), float("inf"), device=dev)
        a = _lib.McArgs()
        a.chain_lig, a.chain_id, a.n_chains = _lib.ptr(clg), _lib.ptr(cig), M
        a.nbr = a.nbr_n = None
        a.nb_max = 0
        a.cur, a.cur_e, a.best, a.best_e = _lib.ptr(cur2), _lib.ptr(ce2), _lib.ptr(best2), _lib.ptr(be2)
        a.init_opt, a.mc_steps, a.bfgs_iters = int(call == 0), 3, 4
        a.temp, a.amp_pos, a.amp_rot = 1.2, 2.0, 2.0
        a.seed, a.step_offset, a.exact = 777 + call, 2 * call, 0
        a.order = a.queue = a.evals = None
        with torch.cuda.device(dev):
            _lib.call("adock_mc_noalloc", kp.c_lig, kp.c_grids, kp.c_sf, kp.c_rec, a, _lib.stream_ptr())
        torch.cuda.synchronize(dev)
        assert rel_close(ce2.cpu().numpy(), ce1.cpu().numpy(), 1e-5, 1e-5) < 1e-5
        assert rel_close(be2.cpu().numpy(), be1.cpu().numpy(), 1e-5, 1e-5) < 1e-5
        assert rel_close(cur2.cpu().numpy(), cur1.cpu().numpy(), 1e-5, 1e-5) < 1e-5
        assert rel_close(best2.cpu().numpy(), best1.cpu().numpy(), 1e-5, 1e-5) < 1e-5


def test_mc_noalloc_rejects_batches_beyond_its_scratch():
    from adock_b200 import _lib
    lib = _lib.load()
    big = _lib.Ligands()
    big.L, big.AM, big.KM, big.P = 4096, 128, 32, 4000
    assert lib.adock_mc_noalloc_scratch_bytes(big.L, big.AM, big.KM, big.P) > 16 << 20
    with pytest.raises(RuntimeError, match="scratch"):
        _lib.call("adock_mc_noalloc", big, _lib.Grids(), _lib.SF(), _lib.Receptors(), _lib.McArgs(), None)
