"""Host-side logic of the learned proposal: the training targets built from the MC kernel's state log."""
import math

import numpy as np
import torch

from adock_b200.proposal import moves_to


def _qmul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


def _rotvec_quat(r):
    ang = np.linalg.norm(r)
    if ang < 1e-12:
        return np.array([1.0, 0, 0, 0])
    return np.concatenate([[math.cos(ang / 2)], math.sin(ang / 2) * r / ang])


def test_moves_to_reaches_target():
    g = torch.Generator().manual_seed(3)
    n = 64
    states = torch.zeros(n, 32)
    states[:, :3] = torch.randn(n, 3, generator=g) * 3
    q = torch.randn(n, 4, generator=g)
    states[:, 3:7] = q / q.norm(dim=1, keepdim=True)
    nt = torch.randint(0, 21, (n,), generator=g)
    th = (torch.rand(n, 20, generator=g) * 2 - 1) * math.pi
    th[torch.arange(20)[None, :] >= nt[:, None]] = 0
    states[:, 7:27] = th
    states[:, 27] = nt.float()
    states[:, 28] = torch.arange(n).float()
    target = torch.zeros(n, 7 + 24)
    target[:, :3] = torch.randn(n, 3, generator=g) * 3
    qt = torch.randn(n, 4, generator=g)
    target[:, 3:7] = qt / qt.norm(dim=1, keepdim=True)
    target[:, 7:] = (torch.rand(n, 24, generator=g) * 2 - 1) * 3 * math.pi
    y = moves_to(states, target).double().numpy()
    S, T = states.double().numpy(), target.double().numpy()
    for i in range(n):
        assert np.allclose(S[i, :3] + y[i, :3], T[i, :3], atol=1e-5)
        assert np.linalg.norm(y[i, 3:6]) <= math.pi + 1e-5    # shortest rotation
        qn = _qmul(_rotvec_quat(y[i, 3:6]), S[i, 3:7])
        assert min(np.abs(qn - T[i, 3:7]).max(), np.abs(qn + T[i, 3:7]).max()) < 1e-4
        k = int(nt[i])
        d = y[i, 6:6 + k]
        assert np.all(np.abs(d) <= math.pi + 1e-5)
        diff = S[i, 7:7 + k] + d - T[i, 7:7 + k]
        assert np.allclose(np.remainder(diff + math.pi, 2 * math.pi) - math.pi, 0, atol=1e-4)
        assert np.all(y[i, 6 + k:26] == 0) and y[i, 26] == k and np.all(y[i, 27:] == 0)


def test_moves_to_identity_is_zero():
    states = torch.zeros(4, 32)
    states[:, 3] = 1.0
    states[:, 27] = 5
    target = torch.zeros(4, 27)
    target[:, 3] = 1.0
    y = moves_to(states, target)
    assert torch.all(y[:, :26] == 0) and torch.all(y[:, 26] == 5)


def test_ligand_best_chain():
    from adock_b200.proposal import ligand_best_chain
    chain_lig = torch.tensor([0, 0, 0, 1, 1, 2, 2, 2], dtype=torch.int32)
    best_e = torch.tensor([3.0, -1.0, 2.0, 5.0, 4.0, 1.0, 1.0, 7.0])
    assert ligand_best_chain(chain_lig, best_e).tolist() == [1, 4, 6]


def test_interp_to_gap():
    from adock_b200.proposal import interp_to_gap
    rows = [{"steps": 500, "median_gap": 0.4, "ligands_per_s": 100.0},
            {"steps": 1000, "median_gap": 0.05, "ligands_per_s": 50.0},
            {"steps": 2000, "median_gap": 0.01, "ligands_per_s": 25.0}]
    r = interp_to_gap(rows, 0.1)
    # log-log: 0.4 -> 0.05 over a doubling is a factor 8 = 2^3; 0.1 is 2^2 below 0.4, so 2/3 of the doubling
    assert abs(r["steps"] - 500 * 2 ** (2 / 3)) < 1e-6
    w = (r["steps"] - 500) / 500
    assert abs(1 / r["ligands_per_s"] - ((1 - w) / 100 + w / 50)) < 1e-12
    assert interp_to_gap(rows, 0.5) == {"steps": 500, "ligands_per_s": 100.0}
    assert interp_to_gap(rows, 0.001) is None


def test_learned_fraction_schedule():
    from adock_b200.proposal import frac_at, parse_frac
    assert parse_frac("0.3") == 0.3
    sched = parse_frac("0.5>0.3@128")
    assert sched == (0.5, 0.3, 128)
    assert [frac_at(sched, s) for s in (0, 96, 128, 500)] == [0.5, 0.5, 0.3, 0.3]
    assert frac_at(0.3, 1000) == 0.3


def test_interp_to_gap_between_budgets():
    """Steps to a median gap by log-log interpolation between the two bracketing budgets, ligands/s from the time
    per ligand interpolated linearly in steps; the first budget when it already reaches the gap; None when none
    does."""
    from adock_b200.proposal import interp_to_gap
    rows = [{"steps": 250, "median_gap": 0.4, "ligands_per_s": 160.0},
            {"steps": 500, "median_gap": 0.1 / 4, "ligands_per_s": 80.0},
            {"steps": 1000, "median_gap": 0.01, "ligands_per_s": 40.0}]
    r = interp_to_gap(rows, 0.1)
    # log gap falls by log(16) over log(2) steps: 0.1 is a quarter of that way
    assert math.isclose(r["steps"], 250 * 2 ** 0.5, rel_tol=1e-9)
    w = (r["steps"] - 250) / 250
    assert math.isclose(r["ligands_per_s"], 1 / ((1 - w) / 160 + w / 80), rel_tol=1e-9)
    assert interp_to_gap(rows, 0.5) == {"steps": 250, "ligands_per_s": 160.0}
    assert interp_to_gap(rows, 0.001) is None


def test_parse_learned_and_bench_specs():
    import importlib.util
    import pathlib
    from adock_b200.proposal import parse_learned
    v = parse_learned([("a", 32, 0.3), ("b", 32, (0.6, 0.3, 64), "dagger2", 4, False, 3)])
    assert v["a"] == (32, 0.3, "chain", 1, False, 1)
    assert v["b"] == (32, (0.6, 0.3, 64), "dagger2", 4, False, 3)
    path = pathlib.Path(__file__).resolve().parents[1] / "bench.py"
    spec = importlib.util.spec_from_file_location("bench_for_test", path)
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    got = bench.parse_variants("learned_dagger2:32:0.6>0.3@64:dagger2:4:0:3,x:16:0.5:chain:1:hint")
    assert got == [("learned_dagger2", 32, (0.6, 0.3, 64), "dagger2", 4, False, 3), ("x", 16, 0.5, "chain", 1, True)]
