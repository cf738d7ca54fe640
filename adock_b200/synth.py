"""Seeded synthetic receptors and ligands with the shapes of the benchmark configurations.

The reference prepares receptors from PDB files and ligands with RDKit/meeko (``src/adock/typing.py``,
``src/adock/ligand.py:18-119``); neither toolkit is part of the hot path. This module emits objects with exactly
the fields the search consumes (``LigandPrep``: n, ref, types, heavy, tors_axis, tors_mask, pairs, rg, n_tors,
n_tors_vina, center) with the same semantics:

- fragments are the connected components after cutting the rotatable bonds;
- the root fragment minimises the tree depth, then maximises its heavy-atom count (``ligand.py:81-82``);
- torsions are ordered leaf -> root (deepest first, ties in breadth-first order); the mask of a torsion is the
  set of atoms of the subtree it moves; the axis is (atom in the parent fragment, atom in the child fragment);
- intra pairs are heavy-atom pairs in different fragments with topological distance > 3 (``ligand.py:111-119``).

Receptor: heavy atoms uniformly placed in a cube with a minimum separation (dart throwing, then pairwise
push-apart relaxation where dart throwing cannot reach the requested density), XS types drawn from the
configured mix.
"""
from __future__ import annotations

import math
from collections import deque

import numpy as np

from .params import XS_INDEX

# XS type mix of the synthetic workloads: C_H .45 / C_P .20 / N_P .08 / N_D .06 / N_A .06 / O_A .08 / O_DA .05 / S_P .02
TYPE_MIX = (("C_H", 0.45), ("C_P", 0.20), ("N_P", 0.08), ("N_D", 0.06), ("N_A", 0.06), ("O_A", 0.08),
            ("O_DA", 0.05), ("S_P", 0.02))
MIX_TYPES = np.array([XS_INDEX[n] for n, _ in TYPE_MIX], np.int64)
MIX_P = np.array([p for _, p in TYPE_MIX], np.float64)

BOND = 1.5                      # A
TETRA = math.acos(-1.0 / 3.0)   # 109.47 deg


# ------------------------------------------------------------------------------------------------ receptor
def receptor(n_atoms: int, extent: float, min_sep: float = 2.8, seed: int = 0):
    """Return (xyz [N,3] float32, types [N] int64) with all pairwise distances >= min_sep (to 1e-3 A)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    pts = np.empty((0, 3))
    # dart throwing in batches
    for _ in range(60):
        need = n_atoms - len(pts)
        if need <= 0:
            break
        cand = rng.uniform(0.0, extent, (max(4 * need, 256), 3))
        if len(pts):
            d, _ = cKDTree(pts).query(cand, k=1)
            cand = cand[d >= min_sep]
        keep = []
        if len(cand):
            # resolve conflicts inside the batch greedily in draw order
            tree = cKDTree(cand)
            taken = np.zeros(len(cand), bool)
            blocked = np.zeros(len(cand), bool)
            for i in range(len(cand)):
                if blocked[i]:
                    continue
                taken[i] = True
                keep.append(i)
                if len(keep) >= need:
                    break
                for j in tree.query_ball_point(cand[i], min_sep):
                    blocked[j] = True
        if keep:
            pts = np.concatenate([pts, cand[keep]])
    if len(pts) < n_atoms:
        # the requested density is above the dart-throwing limit: add random points and relax
        pts = np.concatenate([pts, rng.uniform(0.0, extent, (n_atoms - len(pts), 3))])
        pts = _relax(pts, extent, min_sep, rng)
    pts = pts[:n_atoms]
    types = MIX_TYPES[rng.choice(len(MIX_TYPES), size=n_atoms, p=MIX_P)]
    return pts.astype(np.float32), types.astype(np.int64)


def _relax(pts, extent, min_sep, rng, max_iter=2000):
    from scipy.spatial import cKDTree
    target = min_sep * 1.0005
    for _ in range(max_iter):
        pairs = cKDTree(pts).query_pairs(target, output_type="ndarray")
        if len(pairs) == 0:
            return pts
        i, j = pairs[:, 0], pairs[:, 1]
        d = pts[j] - pts[i]
        r = np.linalg.norm(d, axis=1)
        small = r < 1e-6
        if small.any():
            d[small] = rng.normal(size=(int(small.sum()), 3))
            r[small] = np.linalg.norm(d[small], axis=1)
        push = ((target - r) * 0.5 + 1e-4)[:, None] * d / r[:, None]
        np.add.at(pts, i, -push)
        np.add.at(pts, j, push)
        np.clip(pts, 0.0, extent, out=pts)
    raise RuntimeError("receptor relaxation did not converge")


def receptor_dict(xyz, types, center, size):
    return {"rec_xyz": xyz, "rec_types": types, "center": np.asarray(center, float), "size": np.asarray(size, float)}


# ------------------------------------------------------------------------------------------------ ligand
class _Mol:
    """Stand-in for the RDKit molecule the reference keeps on a prep (only the conformer count is read)."""

    def GetNumConformers(self):
        return 1


class SynthLigand:
    """Fields of the reference ``LigandPrep`` (``src/adock/ligand.py:18-119``); all atoms are heavy atoms."""

    def __init__(self, xyz, types, bonds, rot_bonds):
        n = len(xyz)
        self.n = n
        self.types = np.asarray(types, np.int64)
        self.heavy = self.types >= 0
        self.center = xyz[self.heavy].mean(0)
        self.ref = (xyz - self.center).astype(np.float32)
        self.bonds = [tuple(sorted(b)) for b in bonds]
        self.rot_bonds = sorted(tuple(sorted(b)) for b in rot_bonds)
        self.mol = _Mol()
        self._build_tree()
        self._build_pairs()
        self.n_tors_vina = self.n_tors
        h = self.ref[self.heavy]
        self.rg = float(np.sqrt(((h - h.mean(0)) ** 2).sum(1).mean())) if len(h) > 1 else 1.0

    def _build_tree(self):
        n = self.n
        rot = set(self.rot_bonds)
        adj = [[] for _ in range(n)]
        for i, j in self.bonds:
            if (i, j) not in rot:
                adj[i].append(j)
                adj[j].append(i)
        frag = -np.ones(n, dtype=np.int64)
        nf = 0
        for s in range(n):
            if frag[s] >= 0:
                continue
            frag[s] = nf
            dq = deque([s])
            while dq:
                u = dq.popleft()
                for v in adj[u]:
                    if frag[v] < 0:
                        frag[v] = nf
                        dq.append(v)
            nf += 1
        self.frag = frag
        fadj = [[] for _ in range(nf)]
        for i, j in self.rot_bonds:
            fadj[frag[i]].append((frag[j], i, j))
            fadj[frag[j]].append((frag[i], j, i))

        def bfs(root):
            depth, par = {root: 0}, {root: None}
            dq = deque([root])
            while dq:
                u = dq.popleft()
                for v, a, b in fadj[u]:
                    if v not in depth:
                        depth[v] = depth[u] + 1
                        par[v] = (u, a, b)
                        dq.append(v)
            return depth, par

        nheavy = np.bincount(frag[self.heavy], minlength=nf)
        root = min(range(nf), key=lambda f: (max(bfs(f)[0].values()), -nheavy[f]))
        depth, par = bfs(root)
        assert len(depth) == nf, "ligand graph is disconnected"
        self.root = root
        children = {f: [] for f in range(nf)}
        for f, p in par.items():
            if p is not None:
                children[p[0]].append(f)

        def subtree(f):
            out, st = [], [f]
            while st:
                g = st.pop()
                out.extend(np.where(frag == g)[0].tolist())
                st.extend(children[g])
            return out

        tors = []
        for f, p in par.items():
            if p is None:
                continue
            _, a, b = p
            mask = np.zeros(n, bool)
            mask[subtree(f)] = True
            tors.append((depth[f], a, b, mask))
        tors.sort(key=lambda x: -x[0])
        self.tors_axis = np.array([[a, b] for _, a, b, _ in tors], np.int64).reshape(-1, 2)
        self.tors_mask = np.array([m for *_, m in tors], bool).reshape(-1, n)
        self.n_tors = len(tors)

    def _build_pairs(self):
        n = self.n
        # topological distances by BFS over all bonds
        adj = [[] for _ in range(n)]
        for i, j in self.bonds:
            adj[i].append(j)
            adj[j].append(i)
        dist = np.full((n, n), 10 ** 6, np.int64)
        for s in range(n):
            dist[s, s] = 0
            dq = deque([s])
            while dq:
                u = dq.popleft()
                for v in adj[u]:
                    if dist[s, v] > dist[s, u] + 1:
                        dist[s, v] = dist[s, u] + 1
                        dq.append(v)
        hv = np.where(self.heavy)[0]
        pairs = [(i, j) for ii, i in enumerate(hv) for j in hv[ii + 1:]
                 if self.frag[i] != self.frag[j] and dist[i, j] > 3]
        self.pairs = np.array(pairs, np.int64).reshape(-1, 2)


def _unit(v):
    return v / np.linalg.norm(v)


def _perp(v, rng):
    while True:
        w = np.cross(v, rng.normal(size=3))
        nw = np.linalg.norm(w)
        if nw > 1e-3:
            return w / nw


def _new_direction(nbr_dirs, rng):
    """Unit bond direction at tetrahedral angles to the existing bond directions of the parent atom."""
    k = len(nbr_dirs)
    if k == 0:
        return _unit(rng.normal(size=3))
    if k == 1:
        v = nbr_dirs[0]
        return math.cos(TETRA) * v + math.sin(TETRA) * _perp(v, rng)
    if k == 2:
        v1, v2 = nbr_dirs
        b = -(v1 + v2)
        nb = np.linalg.norm(b)
        b = b / nb if nb > 1e-6 else _perp(v1, rng)
        n = np.cross(v1, v2)
        nn = np.linalg.norm(n)
        n = n / nn if nn > 1e-6 else _perp(b, rng)
        half = 0.5 * TETRA
        return _unit(b * math.cos(half) + (1 if rng.random() < 0.5 else -1) * n * math.sin(half))
    return _unit(-(nbr_dirs[0] + nbr_dirs[1] + nbr_dirs[2]))


def ligand(n_heavy: int, n_rot: int, seed: int, min_nonbonded: float = 2.9, max_tries: int = 200):
    """Random-tree ligand: bond length 1.5 A, tetrahedral bond angles, valence <= 4, no non-bonded contact
    closer than ``min_nonbonded`` (1-2 and 1-3 neighbours excepted), ``n_rot`` rotatable bonds chosen among the
    non-terminal bonds (capped at the number available), types from the XS mix."""
    rng = np.random.default_rng(seed)
    for _attempt in range(max_tries):
        xyz = np.zeros((n_heavy, 3))
        nbrs = [[] for _ in range(n_heavy)]
        bonds = []
        ok = True
        for a in range(1, n_heavy):
            placed = False
            # prefer chain-like growth (parents with one neighbour) so enough non-terminal bonds exist
            cand = [p for p in range(a) if len(nbrs[p]) < 4]
            w = np.array([3.0 if len(nbrs[p]) == 1 else 1.0 for p in cand])
            order = rng.choice(len(cand), size=len(cand), replace=False, p=w / w.sum())
            for oi in order[:12]:
                p = cand[oi]
                dirs = [_unit(xyz[q] - xyz[p]) for q in nbrs[p]]
                excl = set([p] + nbrs[p])
                for _ in range(12):
                    pos = xyz[p] + BOND * _new_direction(dirs, rng)
                    others = [q for q in range(a) if q not in excl]
                    if not others or np.min(np.linalg.norm(xyz[others] - pos, axis=1)) >= min_nonbonded:
                        xyz[a] = pos
                        nbrs[p].append(a)
                        nbrs[a].append(p)
                        bonds.append((p, a))
                        placed = True
                        break
                if placed:
                    break
            if not placed:
                ok = False
                break
        if not ok:
            continue
        inner = [(i, j) for i, j in bonds if len(nbrs[i]) > 1 and len(nbrs[j]) > 1]
        k = min(n_rot, len(inner))
        pick = rng.choice(len(inner), size=k, replace=False) if k else []
        rot = [inner[i] for i in pick]
        types = MIX_TYPES[rng.choice(len(MIX_TYPES), size=n_heavy, p=MIX_P)]
        return SynthLigand(xyz, types, bonds, rot)
    raise RuntimeError(f"could not grow a ligand with {n_heavy} atoms (seed {seed})")


def ligand_set(n: int, heavy_range, rot_range, seed0: int = 0, workers: int = 1):
    """Ligands from seeds seed0..seed0+n-1; sizes drawn uniformly from the inclusive ranges with the same seed.
    workers > 1: the seeds are split over that many processes (started with spawn, so a caller that has already
    initialised CUDA can use it); every ligand depends on its seed alone, so the list is the same."""
    if workers > 1 and n >= 4 * workers:
        # a pool that fails to start its workers (e.g. a caller script without a __main__ guard, which spawned
        # workers re-import) raises BrokenProcessPool instead of waiting for them
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        per = -(-n // workers)
        parts = [(min(per, n - a), tuple(heavy_range), tuple(rot_range), seed0 + a) for a in range(0, n, per)]
        with ProcessPoolExecutor(len(parts), mp_context=mp.get_context("spawn")) as pool:
            chunks = list(pool.map(ligand_set, *zip(*parts)))
        return [x for c in chunks for x in c]
    out = []
    for s in range(seed0, seed0 + n):
        r = np.random.default_rng(10_000 + s)
        nh = int(r.integers(heavy_range[0], heavy_range[1] + 1))
        nr = int(r.integers(rot_range[0], rot_range[1] + 1))
        out.append(ligand(nh, nr, s))
    return out


# ------------------------------------------------------------------------------------------------ configurations
def config_receptor(cfg: int):
    """(receptor dict, box center, box size) of the benchmark configurations.

    cfg 0/1: 1,500 atoms in a 40 A cube, seed 0, 22.5 A box at the centre (61^3 points at 0.375 A).
    cfg 2/4: 8,000 atoms in a 60 A cube, seed 0, 30 A box at the centre (81^3 points)."""
    if cfg in (0, 1):
        xyz, types = receptor(1500, 40.0, seed=0)
        c, s = np.full(3, 20.0), np.full(3, 22.5)
    elif cfg in (2, 4):
        xyz, types = receptor(8000, 60.0, seed=0)
        c, s = np.full(3, 30.0), np.full(3, 30.0)
    else:
        raise ValueError(cfg)
    return receptor_dict(xyz, types, c, s)


def config_ligands(cfg: int, n=None):
    if cfg == 0:
        return [ligand(24, 5, 0)]
    if cfg in (1, 2):
        return ligand_set(256 if n is None else n, (10, 60), (0, 15))
    if cfg == 4:
        return ligand_set(16384 if n is None else n, (8, 80), (0, 20))
    raise ValueError(cfg)
