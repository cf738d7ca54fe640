"""Result files of a docking run: the per-complex CSV of the batch runner and SD files of the ranked poses.

CSV (``write_results_csv``): one row per complex with the columns of the reference's batch runner
(``scripts/run_adock.py:3-6``: id, rmsd_top1, rmsd_best5, success_top1, affinity_top1, wall_s_amortised, status)
plus the top pose's inter, intra and total energies and the number of poses returned. RMSDs are filled when a
reference pose of the ligand is given (heavy atoms in the prep's atom order, no symmetry correction), else empty;
success = top-1 RMSD < 2 A.

SDF (``write_poses_sdf``): one V2000 record per pose, best first, with the properties the reference writes
(``src/adock/dock.py:128-141``: adock_affinity, adock_inter, adock_intra to 3 decimals, adock_rank). The reference
copies an RDKit molecule; here the record is written from the prep itself: element of each atom from its scoring
type (hydrogens have type -1), bonds from ``prep.bonds`` when the prep carries them.
"""
from __future__ import annotations

import csv

import numpy as np

from .params import XS_NAMES

CSV_COLUMNS = ["id", "rmsd_top1", "rmsd_best5", "success_top1", "affinity_top1", "inter_top1", "intra_top1",
               "total_top1", "n_poses", "wall_s_amortised", "status"]
SUCCESS_RMSD = 2.0


def _element(xs_type):
    if xs_type < 0:
        return "H"
    name = XS_NAMES[int(xs_type)].split("_")[0]
    return "Zn" if name == "Met" else name


def pose_rmsd(coords, ref_coords, heavy):
    """RMSD over heavy atoms between each pose [n, A, 3] and a reference pose [A, 3] (same atom order)."""
    X = np.asarray(coords, np.float64)[:, :len(heavy)][:, np.asarray(heavy, bool)]
    R = np.asarray(ref_coords, np.float64)[np.asarray(heavy, bool)]
    return np.sqrt(((X - R[None]) ** 2).sum(-1).mean(-1))


def result_rows(ids, results, preps, wall_s, ref_coords=None, status=None):
    """CSV rows of a batch: wall_s is the batch's wall time (amortised over its complexes); ref_coords[i] an optional
    reference pose per complex; status[i] an optional status ('ok' where a result exists)."""
    rows = []
    n = max(len(results), 1)
    for i, (cid, r, p) in enumerate(zip(ids, results, preps)):
        row = {k: "" for k in CSV_COLUMNS}
        row.update(id=cid, wall_s_amortised=f"{wall_s / n:.4f}")
        st = (status[i] if status is not None else None) or ("ok" if r is not None and len(r["affinity"]) else "failed")
        row["status"] = st
        if st == "ok":
            row.update(affinity_top1=f"{float(r['affinity'][0]):.4f}", inter_top1=f"{float(r['inter'][0]):.4f}",
                       intra_top1=f"{float(r['intra'][0]):.4f}", total_top1=f"{float(r['total'][0]):.4f}",
                       n_poses=str(len(r["affinity"])))
            if ref_coords is not None and ref_coords[i] is not None:
                d = pose_rmsd(r["coords"], ref_coords[i], np.asarray(p.types) >= 0)
                row.update(rmsd_top1=f"{d[0]:.4f}", rmsd_best5=f"{d[:5].min():.4f}",
                           success_top1=str(int(d[0] < SUCCESS_RMSD)))
        rows.append(row)
    return rows


def write_results_csv(path, rows):
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=CSV_COLUMNS)
        w.writeheader()
        for r in rows:
            w.writerow({k: r.get(k, "") for k in CSV_COLUMNS})


def _molblock(name, elements, X, bonds, props):
    lines = [name, "  adock_b200", ""]
    lines.append(f"{len(elements):3d}{len(bonds):3d}  0  0  0  0  0  0  0  0999 V2000")
    for el, (x, y, z) in zip(elements, X):
        lines.append(f"{x:10.4f}{y:10.4f}{z:10.4f} {el:<3} 0  0  0  0  0  0  0  0  0  0  0  0")
    for i, j in bonds:
        lines.append(f"{i + 1:3d}{j + 1:3d}  1  0  0  0  0")
    lines.append("M  END")
    for k, v in props:
        lines += [f">  <{k}>", v, ""]
    lines.append("$$$$")
    return "\n".join(lines) + "\n"


def write_poses_sdf(path, result, prep, name="pose"):
    """The ranked poses of one complex (a search result dict) as an SD file."""
    n = int(prep.n)
    elements = [_element(t) for t in np.asarray(prep.types)[:n]]
    bonds = [tuple(map(int, b)) for b in getattr(prep, "bonds", [])]
    with open(path, "w") as f:
        for i, X in enumerate(np.asarray(result["coords"])[:, :n]):
            if not np.isfinite(X).all():
                continue
            props = [("adock_affinity", f"{float(result['affinity'][i]):.3f}"),
                     ("adock_inter", f"{float(result['inter'][i]):.3f}"),
                     ("adock_intra", f"{float(result['intra'][i]):.3f}"), ("adock_rank", str(i + 1))]
            f.write(_molblock(f"{name}_{i + 1}", elements, X, bonds, props))


def read_sdf_coords(path):
    """(coordinates [n_atoms, 3], properties dict) of every record of an SD file written by write_poses_sdf."""
    out = []
    for block in open(path).read().split("$$$$\n"):
        if not block.strip():
            continue
        lines = block.split("\n")
        na = int(lines[3][:3])
        X = np.array([[float(l[0:10]), float(l[10:20]), float(l[20:30])] for l in lines[4:4 + na]])
        props, k = {}, None
        for l in lines[4 + na:]:
            if l.startswith(">  <"):
                k = l[4:l.index(">", 4)]
            elif k is not None:
                props[k] = l
                k = None
        out.append((X, props))
    return out
