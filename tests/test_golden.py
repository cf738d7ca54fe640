"""The oracle and the host-side restatements against golden vectors recorded from the reference itself
(tests/golden/make_golden.py): pack_host, pair terms, the fitted pair table, CPU grid maps, and the search
kernels (energy/gradient in grid and exact mode, Stage A, one MC step). CPU only."""
from pathlib import Path

import numpy as np
import pytest
import torch

from helpers import rel_close, vec_rel

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    return dict(np.load(GOLD / name))


def _golden_ligands():
    from adock_b200 import synth
    return [synth.ligand(24, 5, 0), synth.ligand(13, 2, 9), synth.ligand(41, 11, 4)]


def _golden_problem():
    """Problem over the golden receptor / ligands with maps from the oracle's C restatement."""
    from oracle import port
    from adock_b200 import params, synth
    from adock_b200.grid import make_gridset
    from adock_b200.ligand import LigandBatch
    from adock_b200.problem import PairPotential, Problem, pad_receptors
    g = _load("grid.npz")
    rec = synth.receptor_dict(g["rec_xyz"], g["rec_types"], np.full(3, 10.0), np.full(3, 12.0))
    ligs = _golden_ligands()
    sfp = params.sf_params("vina")
    lt = np.unique(np.concatenate([[0]] + [l.types for l in ligs]))

    def builder(rx, rt, sfp_, origin, spacing, n, per_term=False, device="cpu", lig_types=None):
        return torch.as_tensor(port.build_grid(rx, rt, sfp_, origin, spacing, n, lig_types, per_term))

    gs = make_gridset([rec], sfp, 0.375, 10.0, device="cpu", lig_types=[lt], builder=builder)
    prob = Problem(gs, LigandBatch(ligs), torch.zeros(3, dtype=torch.long), PairPotential(sfp),
                   rec=pad_receptors([rec], "cpu"))
    return prob


def test_ligand_batch_matches_reference():
    """LigandBatch's padded arrays equal the reference LigandBatch's on the golden ligands (and its per-atom torsion
    bitmasks, the all-atom kinematics' input, encode the same moved-atom table)."""
    from adock_b200.ligand import LigandBatch
    gold = _load("batch.npz")
    lb = LigandBatch(_golden_ligands())
    for k, v in gold.items():
        got = getattr(lb, k).numpy()
        assert got.shape == v.shape, k
        if v.dtype.kind == "f":
            np.testing.assert_allclose(got, v, rtol=1e-6, atol=1e-7, err_msg=k)
        else:
            np.testing.assert_array_equal(got, v, err_msg=k)
    bits = lb.atom_masks()
    table = (bits[:, None, :] >> np.arange(lb.K, dtype=np.uint32)[None, :, None]) & 1
    np.testing.assert_array_equal(table.astype(bool), gold["tmask"])
    sub = lb.subset(torch.tensor([2, 0]))
    np.testing.assert_array_equal(sub.ref.numpy(), gold["ref"][[2, 0]])
    np.testing.assert_array_equal(sub.atom_masks(), bits[[2, 0]])


def test_search_host_tables():
    """The search driver's host tables: one lattice per distinct (receptor, box), its point counts per axis (those
    of arange(-s/2 + 1, s/2 - 1 + 1e-6, step)), the box of each ligand, and the chain widening rule."""
    from adock_b200.search import _boxes, _widen
    from adock_b200 import params

    class _Prob:
        class lb:
            L = 4
        rec_idx = torch.tensor([0, 0, 1, 0])

    c = torch.tensor([[1.0, 2, 3], [1.0, 2, 3], [1.0, 2, 3], [0.0, 0, 0]])
    s = [np.array([22.5, 22.5, 22.5])] * 3 + [np.array([10.0, 12.0, 14.5])]
    table, rec, n, lig_box = _boxes(_Prob, c, s, 1.5)
    assert len(table) == 3 and lig_box[0] == lig_box[1] and len({lig_box[0], lig_box[2], lig_box[3]}) == 3
    for b in range(3):
        l = int(np.flatnonzero(lig_box == b)[0])
        np.testing.assert_allclose(table[b], np.concatenate([c[l].numpy(), s[l]]))
        assert rec[b] == int(_Prob.rec_idx[l])
        want = [len(np.arange(-x / 2 + 1.0, x / 2 - 1.0 + 1e-6, 1.5)) for x in s[l]]
        np.testing.assert_array_equal(n[b], want)
    cfg = dict(params.V2_DEFAULT)
    wide, f = _widen(cfg, 4)
    assert f == 4 and wide["n_chains"] == 1024 and wide["mc_steps"] == 32 and wide["mc_segment"] == 8
    assert _widen(cfg, 64)[1] == 1


def test_pack_host_matches_reference():
    from adock_b200.problem import pack_host
    gold = _load("pack.npz")
    prob = _golden_problem()
    AM, KM, lig, sf = pack_host(prob)
    assert AM == int(gold["AM"]) and KM == int(gold["KM"])
    names = ["ref", "typ", "tm", "ax", "axp", "axu", "pr", "na", "nt", "np", "rg", "P", "gslot"]
    for n, a in zip(names, lig):
        np.testing.assert_array_equal(np.asarray(a), gold[n], err_msg=n)
    for n, a in zip(["prm", "radius", "hyd", "don", "acc"], sf):
        np.testing.assert_array_equal(a, gold[n], err_msg=n)
    np.testing.assert_array_equal(prob.gs.dims.numpy(), gold["grid_dims"])
    np.testing.assert_array_equal(prob.gs.slot.numpy(), gold["grid_slot"])


@pytest.mark.parametrize("sf", ["vina", "vinardo"])
def test_pair_terms_match_reference(sf):
    from adock_b200 import params
    from adock_b200.problem import PairPotential
    gold = _load("pair_terms.npz")
    pot = PairPotential(params.sf_params(sf))
    r = torch.tensor(np.repeat(gold[f"{sf}_r"][None], len(gold[f"{sf}_ti"]), 0), dtype=torch.float64)
    ti = torch.as_tensor(gold[f"{sf}_ti"])[:, None].expand(r.shape)
    tj = torch.as_tensor(gold[f"{sf}_tj"])[:, None].expand(r.shape)
    np.testing.assert_allclose(pot.energy(r, ti, tj).numpy(), gold[f"{sf}_energy"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(pot.terms(r, ti, tj).numpy(), gold[f"{sf}_terms"], rtol=1e-12, atol=1e-15)


def test_two_atom_known_answers():
    """Closed-form Vina terms at fixed distances (the reference's KAT, tests/test_scoring_grid.py:16-51)."""
    import math
    from adock_b200 import params
    from adock_b200.problem import PairPotential
    sfp = params.sf_params("vina")
    pot = PairPotential(sfp)
    i = params.XS_INDEX
    for a, b, r in (("C_H", "C_H", 4.0), ("N_D", "O_A", 2.9), ("O_DA", "O_DA", 3.3), ("Met_D", "O_A", 2.0)):
        d = r - sfp["radius"][i[a]] - sfp["radius"][i[b]]
        d = float(np.float32(r) - np.float32(sfp["radius"][i[a]]) - np.float32(sfp["radius"][i[b]]))
        e = sfp["w_g1"] * math.exp(-(d / 0.5) ** 2) + sfp["w_g2"] * math.exp(-((d - 3.0) / 2.0) ** 2)
        e += sfp["w_rep"] * (d * d if d < 0 else 0.0)
        if sfp["hydrophobic"][i[a]] and sfp["hydrophobic"][i[b]]:
            e += sfp["w_hyd"] * (1.0 if d < 0.5 else 0.0 if d > 1.5 else (1.5 - d))
        if (sfp["donor"][i[a]] and sfp["acceptor"][i[b]]) or (sfp["acceptor"][i[a]] and sfp["donor"][i[b]]):
            e += sfp["w_hb"] * (1.0 if d < -0.7 else 0.0 if d > 0 else -d / 0.7)
        got = float(pot.energy(torch.tensor([r], dtype=torch.float64), torch.tensor([i[a]]), torch.tensor([i[b]])))
        assert got == pytest.approx(e, rel=2e-5, abs=1e-7)


def test_fitted_table_matches_reference():
    from adock_b200 import params
    gold = _load("fitted.npz")
    spec = params.fitted_spec()
    pot = params.FittedPotential(spec, gold["weights"], gold["lig_list"])
    np.testing.assert_array_equal(pot.W, gold["W"])
    np.testing.assert_array_equal(pot.radius, gold["rad_lig"])
    np.testing.assert_array_equal(spec.rec_radius, gold["rec_radius"])
    np.testing.assert_array_equal(spec.indicator().sum((2, 3)), gold["indicator_sum"])
    np.testing.assert_array_equal(params.fitted_weights(), gold["weights"])


def test_fitted_known_answers():
    """Salt bridge / buried carbons / metal-acceptor features (reference tests/test_fit_features.py:34-73) through
    the pair table: W[rec, lig] . basis reproduces the closed forms."""
    from adock_b200 import params
    X = params.N_XS
    spec = params.FittedSpec("vina", buried_threshold=100)
    I = spec.indicator()
    ti = {n: k for k, (n, _, _) in enumerate(params.INTER_TERMS)}
    # buried C_H - C_H: hydrophobic, hyd_buried and gauss1_buried active; no hbond / ionic
    m = I[0 + X, 0]
    assert m[params.B_HYD, ti["hyd_buried"]] == 1 and m[params.B_G1, ti["gauss1_buried"]] == 1
    assert m[:, ti["hbond"]].sum() == 0 and m[:, ti["ionic"]].sum() == 0
    # cation donor (lig N_D, class 1) - anion acceptor (rec O_A, charge 2 -> -1): ionic indicator = 1 * -1
    m = I[8 + X * 4, 3 + X]
    assert m[params.B_ION, ti["ionic"]] == -1 and m[params.B_HB, ti["hbond_charged"]] == 1
    assert m[params.B_HB, ti["hbond_ligdonor"]] == 1
    # metal (rec Met_D) - acceptor (lig O_A): metal_acceptor, hbond, not ligdonor
    m = I[17, 8]
    assert m[params.B_HB, ti["metal_acceptor"]] == 1 and m[params.B_HB, ti["hbond"]] == 1
    assert m[params.B_HB, ti["hbond_ligdonor"]] == 0
    gold = _load("fitted.npz")
    # features of the three recorded pairs from the basis values and the indicator
    for f, (lt, rt, r) in zip(gold["feats"], gold["feat_pairs"]):
        lt, rt = int(lt), int(rt)
        d = r - spec.xs_radius[spec.lig_xs[lt]] - spec.rec_radius[rt]
        basis = np.array([math_exp(-(d / 0.5) ** 2), math_exp(-((d - 3.0) / 2.0) ** 2), d * d if d < 0 else 0.0,
                          np.clip((1.5 - d) / 1.0, 0, 1), np.clip((0.0 - d) / 0.7, 0, 1),
                          1.0 / max(r, 2.0) ** 2 - 1.0 / 64.0])
        np.testing.assert_allclose(basis @ I[rt, lt], f, rtol=1e-6, atol=1e-7)


def math_exp(x):
    import math
    return math.exp(x)


def test_oracle_grid_matches_reference():
    from oracle import port
    from adock_b200 import params
    g = _load("grid.npz")
    sfp = params.sf_params("vina")
    a = port.build_grid(g["rec_xyz"], g["rec_types"], sfp, g["origin"], 0.375, (13, 15, 17), g["lig_types"])
    assert rel_close(a, g["grid"], 1e-5) < 1e-5
    a = port.build_grid(g["rec_xyz"], g["rec_types"], sfp, g["origin"], 0.375, (5, 6, 7), g["lig_types"], per_term=True)
    assert rel_close(a, g["grid_per_term"], 1e-5) < 1e-5


def test_oracle_search_kernels_match_reference():
    from oracle import port
    gold = _load("search.npz")
    pp = port.PortProblem.from_problem(_golden_problem())
    cl, st = gold["chain_lig"], gold["state"]
    e, g = pp.energy_grad(cl, st)
    assert rel_close(e, gold["e"]) < 1e-4
    assert vec_rel(g, gold["g"]) < 1e-4
    e, g = pp.energy_grad(cl, st, exact=True)
    assert rel_close(e, gold["e_exact"]) < 1e-4
    assert vec_rel(g, gold["g_exact"]) < 1e-4
    be, bi = pp.stage_a(gold["conf"], gold["quats"], gold["trans"], gold["ntrans"], 0.3)
    assert rel_close(be, gold["stage_e"]) < 1e-4
    assert (bi == gold["stage_i"]).mean() > 0.99
    cur, best = st.copy(), st.copy()
    ce = gold["e"].copy()
    bst = np.full(len(cl), np.inf, np.float32)
    pp.run_mc(cl, gold["mc_chain_id"], cur, ce, best, bst, False, 1, 1, 1.2, 2.0, 2.0, 4242, 3)
    ok = np.abs(ce - gold["mc_cur_e"]) <= 1e-3 * np.maximum(np.abs(gold["mc_cur_e"]), 1)
    assert ok.mean() >= 0.97
