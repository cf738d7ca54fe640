"""Result files: the per-complex CSV (the reference batch runner's columns, scripts/run_adock.py:3-6) and SD files
of ranked poses with the reference's properties (src/adock/dock.py:128-141), written and read back. CPU only."""
import csv

import numpy as np


def _result(lig, n_poses=3, seed=0):
    g = np.random.default_rng(seed)
    X = lig.ref[None] + g.normal(size=(n_poses, lig.n, 3)).astype(np.float32)
    aff = np.sort(g.normal(size=n_poses)) - 5
    return {"coords": X, "affinity": aff, "inter": aff - 1, "intra": np.full(n_poses, 1.0), "total": aff}


def test_csv_rows_and_file(tmp_path):
    from adock_b200 import synth
    from adock_b200.output import CSV_COLUMNS, result_rows, write_results_csv
    ligs = [synth.ligand(12, 2, 1), synth.ligand(20, 4, 2)]
    res = [_result(ligs[0]), None]
    ref = [res[0]["coords"][0] + 0.5, None]
    rows = result_rows(["a", "b"], res, ligs, wall_s=3.0, ref_coords=ref)
    p = tmp_path / "out.csv"
    write_results_csv(p, rows)
    got = list(csv.DictReader(open(p)))
    assert list(got[0].keys()) == CSV_COLUMNS
    assert got[0]["status"] == "ok" and got[1]["status"] == "failed"
    assert float(got[0]["affinity_top1"]) == round(float(res[0]["affinity"][0]), 4)
    assert abs(float(got[0]["rmsd_top1"]) - np.sqrt(3 * 0.25)) < 1e-3 and got[0]["success_top1"] == "1"
    assert got[0]["wall_s_amortised"] == "1.5000" and got[0]["n_poses"] == "3"


def test_sdf_round_trip(tmp_path):
    from adock_b200 import synth
    from adock_b200.output import read_sdf_coords, write_poses_sdf
    lig = synth.ligand(24, 5, 0)
    r = _result(lig, 4)
    p = tmp_path / "poses.sdf"
    write_poses_sdf(p, r, lig)
    recs = read_sdf_coords(p)
    assert len(recs) == 4
    for i, (X, props) in enumerate(recs):
        np.testing.assert_allclose(X, r["coords"][i], atol=1e-4)
        assert props["adock_rank"] == str(i + 1)
        assert props["adock_affinity"] == f"{r['affinity'][i]:.3f}"
    text = open(p).read()
    assert text.count("V2000") == 4 and text.count("M  END") == 4
    assert f"{lig.n:3d}{len(lig.bonds):3d}" in text
