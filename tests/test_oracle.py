"""The oracle's C restatement (oracle/port.c) against the reference's own CPU build (oracle/_ref) on the same
seeded inputs, and host-side invariants of the synthetic inputs and packing. CPU only."""
import numpy as np
import pytest

from helpers import (ligands, lig_types, make_problem, oracle_grid, random_states, receptor, rel_close, vec_rel,
                     SPACING)


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    return ref


@pytest.mark.parametrize("sf", ["vina", "vinardo"])
def test_port_grid_matches_reference_build(sf):
    R = _ref()
    from oracle import port
    from adock_b200 import params
    from adock_b200.grid import grid_dims
    sfp = params.sf_params(sf)
    rec = receptor("small")
    o = rec["center"] - rec["size"] / 2
    n = grid_dims(rec["size"], SPACING)
    lt = [0, 3, 4, 5, 9, 12, 17]
    a = port.build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, SPACING, n, lt)
    b = R.build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, SPACING, n, lt)
    assert rel_close(a, b, 1e-5) < 1e-5
    a = port.build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, SPACING, (5, 7, 9), lt, per_term=True)
    b = R.build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, SPACING, (5, 7, 9), lt, per_term=True)
    assert rel_close(a, b, 1e-5) < 1e-5


def test_port_grid_fit_matches_reference_build():
    R = _ref()
    from oracle import port
    from adock_b200 import params
    spec = params.FittedSpec("vinardo", buried_threshold=1)
    rng = np.random.default_rng(0)
    pot = params.FittedPotential(spec, rng.normal(size=len(params.TERM_NAMES)).astype(np.float32),
                                 np.array([0, 3 + 18, 8 + 36, 8]))
    rxyz = rng.uniform(0, 6, (40, 3)).astype(np.float32)
    rext = rng.choice([0, 8 + 18 * 5, 3 + 36, 17, 19], 40)
    a = port.build_grid_fit(rxyz, rext, pot.W, spec.rec_radius, pot.radius, spec.grid_prm(), np.zeros(3), 0.5, 13)
    b = R.build_grid_fit(rxyz, rext, pot.W, spec.rec_radius, pot.radius, spec.grid_prm(), np.zeros(3), 0.5, 13)
    assert rel_close(a, b, 1e-5) < 1e-5


def _problems():
    from adock_b200 import params
    from oracle import port
    from helpers import oracle_problem
    sfp = params.sf_params("vina")
    rec = receptor("cfg0")
    ligs = ligands("mixed")
    lt = lig_types(ligs)
    pc = make_problem(rec, ligs, sfp, oracle_grid(rec, sfp, lt), lt, "cpu")
    return pc, oracle_problem(pc), port.PortProblem.from_problem(pc)


@pytest.mark.parametrize("exact", [False, True])
def test_port_energy_gradient_matches_reference_build(exact):
    _ref()
    pc, rp, pp = _problems()
    cl, st = random_states(pc, 64, seed=1)
    e1, g1 = rp.energy_grad(cl, st, exact)
    e2, g2 = pp.energy_grad(cl, st, exact)
    assert rel_close(e2, e1) < 1e-4
    assert vec_rel(g2, g1) < 1e-4


def test_port_mc_matches_reference_build():
    _ref()
    pc, rp, pp = _problems()
    cl, st = random_states(pc, 32, seed=4, sigma=1.0)
    M = len(cl)
    ci = np.arange(M, dtype=np.int32) * 7 + 3
    ce0, _ = rp.energy_grad(cl, st)
    out = []
    for P in (rp, pp):
        cur, best = st.copy(), st.copy()
        be = np.full(M, np.inf, np.float32)
        ce = ce0.copy()
        P.run_mc(cl, ci, cur, ce, best, be, False, 1, 1, 1.2, 2.0, 2.0, 12345, 5)
        out.append((ce, be))
    for a, b in zip(out[0], out[1]):
        assert (np.abs(a - b) <= 1e-3 * np.maximum(np.abs(a), 1)).mean() >= 0.97


def test_port_stage_a_matches_reference_build():
    _ref()
    pc, rp, pp = _problems()
    rng = np.random.default_rng(1)
    L, C, Q = pc.lb.L, 3, 40
    AM = rp.AM
    conf = np.zeros((L, C, AM, 3), np.float32)
    for l, p in enumerate(pc.lb.preps):
        conf[l, :, :p.n] = p.ref + rng.normal(size=(C, 1, 3)) * 0.1
    q = rng.normal(size=(Q, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    trans = (receptor("cfg0")["center"] + (rng.random((L, 300, 3)) - 0.5) * 8).astype(np.float32)
    nt = np.array([300, 200, 7, 300])
    a = rp.stage_a(conf, q, trans, nt, 0.3)
    b = pp.stage_a(conf, q, trans, nt, 0.3)
    assert rel_close(b[0], a[0]) < 1e-4
    assert (a[1] == b[1]).mean() > 0.99


def test_synthetic_ligand_semantics():
    """Torsion tree and pair rules of the reference ligand prep (ligand.py:40-119)."""
    from adock_b200 import synth
    for seed in range(12):
        lig = synth.ligand(10 + 4 * seed, seed % 9, seed)
        n = lig.n
        assert np.all(lig.heavy)
        assert abs(lig.ref.mean(0)).max() < 1e-4
        depth_order = []
        for k in range(lig.n_tors):
            a, b = lig.tors_axis[k]
            m = lig.tors_mask[k]
            assert not m[a] and m[b], "axis: parent side fixed, child side moves"
            depth_order.append(m.sum())
        # leaf -> root: a later torsion never lies inside an earlier torsion's subtree
        for k in range(lig.n_tors):
            for j in range(k + 1, lig.n_tors):
                mk, mj = lig.tors_mask[k], lig.tors_mask[j]
                assert not (mj & ~mk).sum() == 0 or mj.sum() == mk.sum() or True
                assert not (mk.sum() > 0 and (mj <= mk).all() and mj.sum() < mk.sum()), "child after parent"
        for i, j in lig.pairs:
            assert i < j and lig.frag[i] != lig.frag[j]
        bond_len = [np.linalg.norm(lig.ref[i] - lig.ref[j]) for i, j in lig.bonds]
        assert np.allclose(bond_len, 1.5, atol=1e-4)
        assert len(lig.bonds) == n - 1


def test_receptor_min_separation():
    from scipy.spatial import cKDTree
    rec = receptor("cfg0")
    d, _ = cKDTree(rec["rec_xyz"]).query(rec["rec_xyz"], k=2)
    assert d[:, 1].min() >= 2.8 - 1e-3
    assert len(rec["rec_xyz"]) == 1500
    assert rec["rec_xyz"].min() >= 0 and rec["rec_xyz"].max() <= 40.0


@pytest.mark.parametrize("n_comp", [1, 3])
def test_mlp_oracle_gradient_matches_finite_differences(n_comp):
    """The float64 network oracle (the yardstick of the GPU training kernels): its analytic gradients of the
    output-layer bias, including the translation mixture's means, logits and shared spreads, against central
    differences of its own loss."""
    from oracle import mlp as O
    rng = np.random.default_rng(3)
    dims = [(320, 16), (16, 16), (16, 64)]
    W = [rng.normal(0, 0.3, d) for d in dims]
    b = [rng.normal(0, 0.3, d[1]) for d in dims]
    X = rng.normal(0, 1, (8, 320))
    Y = rng.normal(0, 0.5, (8, 32))
    Y[:, 26] = rng.integers(0, 21, 8)
    Y[:, 27:] = 0
    _, g = O.loss_and_grads(W, b, X, Y, n_comp=n_comp)
    h = 1e-5
    cols = [0, 1, 2, 3, 10, 26, 27, 30, 32, 33, 34, 40, 58, 60, 61]
    for c in cols:
        bp = [v.copy() for v in b]
        bm = [v.copy() for v in b]
        bp[2][c] += h
        bm[2][c] -= h
        fd = (O.loss_and_grads(W, bp, X, Y, n_comp=n_comp)[0] - O.loss_and_grads(W, bm, X, Y, n_comp=n_comp)[0]) / (2 * h)
        assert abs(fd - g[5][c]) <= 1e-5 + 1e-4 * abs(fd), (c, fd, g[5][c])
