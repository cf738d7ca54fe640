"""The whole search on the B200 through its callers (reference search.py:544-671 via dock_screen, screen.py:39-78,
and dock_batch, dock.py:69-125): well-formed, reproducible results, and each complex docked against its own
receptor and box. The comparison with the reference's own search is in test_gpu_pipeline.py (fixture dock.npz)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    from adock_b200 import params, synth
    rec = synth.config_receptor(0)
    ligs = [synth.ligand(n, r, seed) for n, r, seed in ((12, 2, 101), (16, 3, 102), (20, 4, 103))]
    cfg = params.workload_preset(16, 300)
    return rec, ligs, cfg


def test_dock_screen_results_are_well_formed_and_reproducible(case):
    from adock_b200.screen import dock_screen
    rec, ligs, cfg = case
    box = {"center": rec["center"], "size": rec["size"]}
    a = dock_screen(rec, box, ligs, cfg, device="cuda:0", seed=3)
    b = dock_screen(rec, box, ligs, cfg, device="cuda:0", seed=3)
    assert len(a) == len(ligs)
    lo, hi = rec["center"] - rec["size"] / 2 - 2.0, rec["center"] + rec["size"] / 2 + 2.0
    for p, ra, rb in zip(ligs, a, b):
        aff = np.asarray(ra["affinity"])
        X = np.asarray(ra["coords"])
        assert 1 <= len(aff) <= cfg["n_out"] and np.isfinite(aff).all()
        assert np.all(np.diff(aff) >= -1e-6), "poses are ranked by affinity"
        assert X.shape[0] == len(aff) and X.shape[-1] == 3 and np.isfinite(X).all()
        heavy = X[:, np.asarray(p.heavy, bool)] if X.shape[1] == len(p.heavy) else X
        assert np.all(heavy >= lo) and np.all(heavy <= hi), "returned poses lie in the box"
        np.testing.assert_array_equal(aff, np.asarray(rb["affinity"]))
        np.testing.assert_array_equal(X, np.asarray(rb["coords"]))


def test_dock_batch_routes_each_ligand_to_its_receptor():
    """dock_batch (reference dock.py:69-125): three receptors with different boxes, one ligand each, one search.
    Every returned pose lies in its own complex's box, and its total energy equals a float64 re-evaluation
    against its own receptor's atoms (exact pair terms + out-of-box penalty + intra pairs)."""
    from adock_b200 import params, synth
    from adock_b200.problem import pack_host
    from adock_b200.screen import dock_batch
    from helpers import make_problem
    from oracle.fp64 import Packed
    complexes = []
    for i, (n, r, sd) in enumerate(((12, 2, 201), (16, 3, 202), (20, 4, 203))):
        xyz, ty = synth.receptor(500, 24.0, seed=30 + i)
        box = synth.receptor_dict(xyz, ty, np.full(3, 12.0) + i, np.array([14.0, 16.0, 15.0]) + 2 * i)
        complexes.append(dict(box, lig=synth.ligand(n, r, sd)))
    cfg = params.workload_preset(16, 150)
    res = dock_batch(complexes, cfg, device="cuda:0", seed=1)
    sfp = params.sf_params("vina")
    for c, r in zip(complexes, res):
        lig = c["lig"]
        lo, hi = c["center"] - c["size"] / 2, c["center"] + c["size"] / 2
        X = np.asarray(r["coords"], np.float64)
        assert X.shape[1] == lig.n and np.all(X >= lo - 2.0) and np.all(X <= hi + 2.0)
        lt = np.unique(np.concatenate([[0], lig.types]))
        G = np.zeros((len(lt),) + tuple(int(np.ceil(s / params.GRID_SPACING)) + 1 for s in c["size"]), np.float32)
        model = Packed(*pack_host(make_problem(c, [lig], sfp, G, lt, "cpu"))[2:])
        want = (model.exact_inter(0, X, c["rec_xyz"], c["rec_types"]) + model.penalty(X, lo, hi, 10.0)
                + model.intra(0, X))
        np.testing.assert_allclose(r["total"], want, rtol=1e-3, atol=1e-2)
