"""FP16 / BF16 map storage (the search's low-precision path) against float64.

- adock_grid_convert rounds to nearest like torch's conversions, bit for bit (FP16 saturating at +-65504).
- The energy/gradient kernel on FP16 and BF16 maps equals the float64 oracle evaluated on the same stored (decoded)
  map values: rel 1e-4 with a 1e-4 floor, the FP32 bar; so interpolation and accumulation stay FP32-exact and the
  only error of a low-precision search is the storage rounding.
- That storage error, against the float64 evaluation of the FP32 maps (the yardstick of precision.py, itself pinned
  to the oracle in test_gpu_parity.py), stays inside its bound: per pose |E - E64| <= u * sum_atoms sum_corners
  w |v| + 1e-4 (1 + |E64|) with u = 2^-11 (FP16) or 2^-8 (BF16), the unit roundoff of the storage format; and the
  FP16 p99 stays under the 0.1 kcal/mol accuracy bar of the screening comparison.
- One MC step on FP16 / BF16 maps keeps best energies equal to a re-evaluation of the returned states.
"""
import numpy as np
import pytest
import torch

from helpers import ligands, lig_types, make_problem, oracle_grid, random_states, receptor, rel_close

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
UNIT_ROUNDOFF = {"f16": 2.0 ** -11, "bf16": 2.0 ** -8}
TORCH = {"f16": torch.float16, "bf16": torch.bfloat16}


def test_grid_convert_matches_round_to_nearest():
    from adock_b200 import _lib
    g = torch.Generator(device=DEV).manual_seed(0)
    x = torch.randn(1 << 20, generator=g, device=DEV) * torch.exp(torch.randn(1 << 20, generator=g, device=DEV) * 4)
    x[:6] = torch.tensor([0.0, -0.0, 65504.0, 70000.0, -1e9, 1e-8], device=DEV)
    for dt, code in (("f16", _lib.ADOCK_GRID_F16), ("bf16", _lib.ADOCK_GRID_BF16)):
        out = torch.empty(x.shape, dtype=TORCH[dt], device=DEV)
        _lib.call("adock_grid_convert", _lib.ptr(x), _lib.ptr(out), x.numel(), code, _lib.stream_ptr())
        want = (x.clamp(-65504.0, 65504.0) if dt == "f16" else x).to(TORCH[dt])
        assert torch.equal(out.view(torch.int16), want.view(torch.int16)), dt


def _setup(kind):
    from adock_b200 import params
    from adock_b200.kernel import B200KernelProblem
    sfp = params.sf_params("vina")
    rec = receptor("cfg0")
    ligs = ligands(kind)
    lt = lig_types(ligs)
    G = oracle_grid(rec, sfp, lt)
    pg, pc = make_problem(rec, ligs, sfp, G, lt, DEV), make_problem(rec, ligs, sfp, G, lt, "cpu")
    return pg, pc, G, B200KernelProblem


@pytest.mark.parametrize("dt", ["f16", "bf16"])
@pytest.mark.parametrize("kind", ["mixed", "big"])
def test_low_precision_maps_against_fp64(dt, kind):
    from adock_b200.problem import pack_host
    from oracle.fp64 import Packed
    pg, pc, G32, KP = _setup(kind)
    kp = KP(pg, grid_dtype=dt)
    cl, st = random_states(pc, 64, seed=5, sigma=1.5)
    e, g = kp.energy_grad(torch.as_tensor(cl, device=DEV), torch.as_tensor(st, device=DEV))
    e = e.cpu().numpy().astype(np.float64)
    stored = pg.gs.storage(dt)[0].float().cpu().numpy().astype(np.float64).reshape(G32.shape)
    model = Packed(*pack_host(pc)[2:])
    gs = pc.gs
    lo, hi, org = gs.lo[0].numpy(), gs.hi[0].numpy(), gs.origin[0].numpy()
    want_lp, want_32, scale = np.zeros(len(cl)), np.zeros(len(cl)), np.zeros(len(cl))
    for l in range(pc.lb.L):
        sel = np.where(cl == l)[0]
        X = model.pose_heavy(l, st[sel])
        rest = model.penalty(X, lo, hi, gs.penalty) + model.intra(l, X)
        want_lp[sel] = model.grid_inter(l, X, stored, org, gs.spacing) + rest
        want_32[sel] = model.grid_inter(l, X, G32, org, gs.spacing) + rest
        scale[sel] = model.grid_magnitude(l, X, G32, org, gs.spacing)
    # the kernel is exact (FP32 arithmetic) on the values it stores
    assert rel_close(e, want_lp) < 1e-4
    # the storage error is within the roundoff bound of the format
    err = np.abs(e - want_32)
    bound = UNIT_ROUNDOFF[dt] * scale + 1e-4 * (1 + np.abs(want_32))
    assert np.all(err <= bound), (err.max(), (err / bound).max())
    if dt == "f16":
        assert np.quantile(err, 0.99) < 0.1


@pytest.mark.parametrize("dt", ["f16", "bf16"])
def test_mc_on_low_precision_maps_is_consistent(dt):
    pg, pc, G32, KP = _setup("mixed")
    kp = KP(pg, grid_dtype=dt)
    cl, st = random_states(pc, 16, seed=3, sigma=1.0)
    M = len(cl)
    clg = torch.as_tensor(cl, device=DEV)
    cur = torch.as_tensor(st, device=DEV).clone()
    best = cur.clone()
    e0, _ = kp.energy_grad(clg, cur)
    cur_e, best_e = torch.zeros(M, device=DEV), torch.full((M,), float("inf"), device=DEV)
    kp.run_mc(clg, torch.arange(M, device=DEV), cur, cur_e, best, best_e, True, 10, 0, 1.2, 2.0, 2.0, 7, 0)
    e1, _ = kp.energy_grad(clg, best)
    torch.testing.assert_close(e1, best_e, rtol=1e-4, atol=1e-4)
    assert (best_e <= e0 + 1e-4).all()
