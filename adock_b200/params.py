"""Scoring-function parameters for the docking hot path.

Holds the X-Score (XS) atom-type table, the Vina / Vinardo pair-term constants, the search presets used by the
synthetic workloads, and the fitted (linear-in-weights) scoring function's pair table.

The numbers are the published AutoDock Vina 1.2 / Vinardo constants as the reference records them in
``config/adock.json`` ("xs_types", "scoring") and ``config/adock_fitted.json`` ("nonlinear", "weights"); the
fitted-table construction restates ``src/adock/fit/terms.py:58-155`` (``Spec``, ``indicator``, ``pair_table``).
"""
from __future__ import annotations

import numpy as np

# ------------------------------------------------------------------------------------------------ XS atom types
# name: (radius_vina, radius_vinardo, hydrophobic, donor, acceptor)   -- config/adock.json "xs_types"
XS_TABLE = [
    ("C_H", 1.9, 2.0, 1, 0, 0),
    ("C_P", 1.9, 2.0, 0, 0, 0),
    ("N_P", 1.8, 1.7, 0, 0, 0),
    ("N_D", 1.8, 1.7, 0, 1, 0),
    ("N_A", 1.8, 1.7, 0, 0, 1),
    ("N_DA", 1.8, 1.7, 0, 1, 1),
    ("O_P", 1.7, 1.6, 0, 0, 0),
    ("O_D", 1.7, 1.6, 0, 1, 0),
    ("O_A", 1.7, 1.6, 0, 0, 1),
    ("O_DA", 1.7, 1.6, 0, 1, 1),
    ("S_P", 2.0, 2.0, 0, 0, 0),
    ("P_P", 2.1, 2.1, 0, 0, 0),
    ("F_H", 1.5, 1.5, 1, 0, 0),
    ("Cl_H", 1.8, 1.8, 1, 0, 0),
    ("Br_H", 2.0, 2.0, 1, 0, 0),
    ("I_H", 2.2, 2.2, 1, 0, 0),
    ("Si", 2.2, 2.2, 0, 0, 0),
    ("Met_D", 1.2, 1.2, 0, 1, 0),
]
XS_NAMES = [r[0] for r in XS_TABLE]
XS_INDEX = {n: i for i, n in enumerate(XS_NAMES)}
N_XS = len(XS_TABLE)

# Vina / Vinardo pair terms (config/adock.json "scoring")
_SCORING = {
    "vina": dict(radius_col=1, cutoff=8.0, g1=(0.0, 0.5, -0.035579), g2=(3.0, 2.0, -0.005156), rep=(0.0, 0.840245),
                 hyd=(0.5, 1.5, -0.035069), hb=(-0.7, 0.0, -0.587439), rot_weight=0.05846),
    "vinardo": dict(radius_col=2, cutoff=8.0, g1=(0.0, 0.8, -0.045), g2=(3.0, 2.0, 0.0), rep=(0.0, 0.8),
                    hyd=(0.0, 2.5, -0.035), hb=(-0.6, 0.0, -0.6), rot_weight=0.05846),
}

GRID_SPACING = 0.375          # config/adock.json grid.spacing (Vina default)
OUT_OF_BOX_PENALTY = 10.0     # config/adock.json grid.out_of_box_penalty (kcal/mol/A^2)


def sf_params(sf: str = "vina") -> dict:
    """Flat scoring-function parameters + per-type arrays (same keys as ``src/adock/config.py:45-62``)."""
    p = _SCORING[sf]
    col = p["radius_col"]
    return {
        "name": sf, "cutoff": p["cutoff"],
        "g1_off": p["g1"][0], "g1_w": p["g1"][1], "w_g1": p["g1"][2],
        "g2_off": p["g2"][0], "g2_w": p["g2"][1], "w_g2": p["g2"][2],
        "rep_off": p["rep"][0], "w_rep": p["rep"][1],
        "hyd_good": p["hyd"][0], "hyd_bad": p["hyd"][1], "w_hyd": p["hyd"][2],
        "hb_good": p["hb"][0], "hb_bad": p["hb"][1], "w_hb": p["hb"][2],
        "rot_weight": p["rot_weight"],
        "radius": np.array([r[col] for r in XS_TABLE], np.float32),
        "hydrophobic": np.array([r[3] for r in XS_TABLE], np.int32),
        "donor": np.array([r[4] for r in XS_TABLE], np.int32),
        "acceptor": np.array([r[5] for r in XS_TABLE], np.int32),
    }


def grid_prm(sfp: dict) -> np.ndarray:
    """15-float vector of the grid builder (order of ``src/adock/grid.py:84-87``):
    cutoff, g1_off, g1_w, g2_off, g2_w, rep_off, hyd_good, hyd_bad, hb_good, hb_bad, w_g1, w_g2, w_rep, w_hyd, w_hb."""
    keys = ["cutoff", "g1_off", "g1_w", "g2_off", "g2_w", "rep_off", "hyd_good", "hyd_bad", "hb_good", "hb_bad",
            "w_g1", "w_g2", "w_rep", "w_hyd", "w_hb"]
    return np.array([sfp[k] for k in keys], np.float32)


def search_prm(sfp: dict) -> np.ndarray:
    """15-float vector of the search kernels (order of ``src/adock/mckernel.py:594-596``):
    g1_off, g1_w, g2_off, g2_w, rep_off, hyd_good, hyd_bad, hb_good, hb_bad, cutoff, w_g1, w_g2, w_rep, w_hyd, w_hb."""
    keys = ["g1_off", "g1_w", "g2_off", "g2_w", "rep_off", "hyd_good", "hyd_bad", "hb_good", "hb_bad", "cutoff",
            "w_g1", "w_g2", "w_rep", "w_hyd", "w_hb"]
    return np.array([sfp[k] for k in keys], np.float32)


# ------------------------------------------------------------------------------------------------ search presets
# v2_default of config/adock.json "search", plus the synthetic-workload settings (fixed MC budget, no widening,
# no size scaling, no early stop) under which the benchmark configurations are defined.
V2_DEFAULT = {
    "engine": "kernel", "n_chains": 256, "stageA_conformers": 8, "stageA_conformer_trials": 64,
    "stageA_rotations": 384, "stageA_translation_step": 1.5, "stageA_atom_cap": 0.3,
    "mc_steps": 128, "mc_segment": 32, "mc_size_ref": 25, "bfgs_iters": 0, "final_bfgs_iters": 100,
    "polish_top": 32, "polish_iters": 100, "mc_temperature": 1.2, "mc_amp_pos": 2.0, "mc_amp_rot": 2.0,
    "early_stop_rounds": 0, "early_stop_tol": 0.01, "min_total_chains": 4096, "min_chain_steps": 32,
    "polish_nbr_margin": 2.0, "cluster_rmsd": 2.0, "n_out": 9,
}


def workload_preset(n_chains: int, mc_steps: int, **kw) -> dict:
    """v2_default with a fixed budget: n_chains x mc_steps per ligand in one segment, no widening/size scaling."""
    cfg = dict(V2_DEFAULT, n_chains=n_chains, mc_steps=mc_steps, mc_segment=mc_steps, mc_size_ref=0,
               min_total_chains=0)
    cfg.update(kw)
    return cfg


# ------------------------------------------------------------------------------------------------ fitted function
# basis functions and inter terms (src/adock/fit/terms.py:21-43)
B_G1, B_G2, B_REP, B_HYD, B_HB, B_ION = range(6)
N_BASIS = 6
INTER_TERMS = [
    ("gauss1", B_G1, "all"), ("gauss2", B_G2, "all"), ("repulsion", B_REP, "all"),
    ("hydrophobic", B_HYD, "hyd"), ("hbond", B_HB, "hb"), ("hyd_buried", B_HYD, "hyd_bur"),
    ("hbond_buried", B_HB, "hb_bur"), ("hbond_ligdonor", B_HB, "hb_ligdon"), ("hbond_charged", B_HB, "hb_chg"),
    ("metal_acceptor", B_HB, "metal"), ("ionic", B_ION, "ion"), ("polar_apolar", B_HYD, "mismatch"),
    ("gauss1_buried", B_G1, "bur"),
]
INTRA_TERMS = ["intra_gauss1", "intra_gauss2", "intra_repulsion", "intra_hydrophobic", "intra_hbond"]
TERM_NAMES = [t[0] for t in INTER_TERMS] + INTRA_TERMS
N_INTER = len(INTER_TERMS)

# config/adock_fitted.json
FITTED_NONLINEAR = dict(base="vina", buried_threshold=177.0, buried_radius=10.0, ion_rmin=2.0)
FITTED_WEIGHTS = {
    "gauss1": -0.04205807783159489, "gauss2": -0.004991743991543715, "repulsion": 0.8156755426614062,
    "hydrophobic": -0.037384251945279, "hbond": -0.5992849056216177, "hyd_buried": -0.010445834116223103,
    "hbond_buried": -0.033401801182270895, "hbond_ligdonor": 0.04364980965614507,
    "hbond_charged": -0.05896339457313388, "metal_acceptor": -0.2891157216623504, "ionic": 0.5160035204995856,
    "polar_apolar": -0.019994960794392377, "gauss1_buried": -0.009641505343954668,
    "intra_gauss1": -0.025311347297737166, "intra_gauss2": -0.004635982193796613,
    "intra_repulsion": 0.7775323047062759, "intra_hydrophobic": -0.023113067408981426,
    "intra_hbond": -0.2059719834408973,
}


def fitted_weights() -> np.ndarray:
    return np.array([FITTED_WEIGHTS[k] for k in TERM_NAMES], np.float32)


class FittedSpec:
    """Extended atom types of the fitted function (``src/adock/fit/terms.py:58-107``).

    ligand ext type = xs + N_XS * charge_class (0 neutral, 1 cation, 2 anion);
    receptor ext type = xs + N_XS * (buried + 2 * charge_class). No side-chain split (the stock fitted preset)."""

    def __init__(self, base="vina", buried_threshold=1e9, buried_radius=10.0, ion_rmin=2.0, rep_cap=None):
        sfp = sf_params(base)
        self.base = base
        self.cutoff = float(sfp["cutoff"])
        self.buried_threshold, self.buried_radius, self.ion_rmin = float(buried_threshold), float(buried_radius), float(ion_rmin)
        self.rep_cap = None if rep_cap is None else float(rep_cap)
        self.prm = {k: sfp[k] for k in ("g1_off", "g1_w", "g2_off", "g2_w", "rep_off", "hyd_good", "hyd_bad",
                                        "hb_good", "hb_bad")}
        self.rot_weight = sfp["rot_weight"]
        X = N_XS
        self.nxs = X
        self.xs_radius = sfp["radius"].astype(np.float32)
        self.xs_hyd = sfp["hydrophobic"].astype(bool)
        self.xs_don = sfp["donor"].astype(bool)
        self.xs_acc = sfp["acceptor"].astype(bool)
        self.xs_polar = np.array([n.split("_")[0] in ("N", "O") for n in XS_NAMES])
        self.xs_metal = np.array([n == "Met_D" for n in XS_NAMES])
        self.lig_xs = np.tile(np.arange(X), 3)
        self.lig_chg = np.repeat([0, 1, -1], X)
        blk = np.repeat(np.arange(6), X)
        self.rec_xs = np.tile(np.arange(X), 6)
        self.rec_bur = blk % 2 == 1
        self.rec_chg = np.array([0, 1, -1])[(blk // 2) % 3]
        self.n_lt, self.n_rt = 3 * X, 6 * X
        self.rec_radius = self.xs_radius[self.rec_xs].astype(np.float32)

    def indicator(self) -> np.ndarray:
        """I[n_rt, n_lt, N_BASIS, N_INTER]: contribution of basis k to term m for a (receptor, ligand) type pair."""
        lx, rx = self.lig_xs, self.rec_xs
        Lh, Ld, La, Lp = self.xs_hyd[lx], self.xs_don[lx], self.xs_acc[lx], self.xs_polar[lx]
        Rh, Rd, Ra, Rp, Rm = self.xs_hyd[rx], self.xs_don[rx], self.xs_acc[rx], self.xs_polar[rx], self.xs_metal[rx]
        both = lambda l, r: r[:, None] & l[None, :]
        shape = (self.n_rt, self.n_lt)
        bur = np.broadcast_to(self.rec_bur[:, None], shape)
        hb = both(Ld, Ra) | both(La, Rd)
        hyd = both(Lh, Rh)
        anychg = (self.rec_chg != 0)[:, None] | (self.lig_chg != 0)[None, :]
        ind = {
            "all": np.ones(shape, bool), "hyd": hyd, "hb": hb, "hyd_bur": hyd & bur, "hb_bur": hb & bur,
            "hb_ligdon": both(Ld, Ra) & ~np.broadcast_to(Rm[:, None], shape), "hb_chg": hb & anychg,
            "metal": both(La, Rm), "ion": (self.rec_chg[:, None] * self.lig_chg[None, :]).astype(np.float32),
            "mismatch": both(Lh, Rp) | both(Lp, Rh), "bur": bur,
        }
        I = np.zeros(shape + (N_BASIS, N_INTER), np.float32)
        for m, (_, k, iid) in enumerate(INTER_TERMS):
            I[:, :, k, m] = ind[iid]
        return I

    def pair_table(self, w_inter) -> np.ndarray:
        """W[n_rt, n_lt, N_BASIS] = sum_m w_m I_m (``terms.py:153-155``)."""
        return np.einsum("rlkm,m->rlk", self.indicator(), np.asarray(w_inter, np.float32)).astype(np.float32)

    def grid_prm(self) -> np.ndarray:
        """12-float vector of the fitted grid builder (``src/adock/fit/gridfit.py:78-81``)."""
        p = self.prm
        cap = np.float32(3.0e38) if self.rep_cap is None else self.rep_cap
        return np.array([self.cutoff, p["g1_off"], p["g1_w"], p["g2_off"], p["g2_w"], p["rep_off"], p["hyd_good"],
                         p["hyd_bad"], p["hb_good"], p["hb_bad"], self.ion_rmin, cap], np.float32)


def fitted_spec() -> FittedSpec:
    return FittedSpec(**FITTED_NONLINEAR)


class FittedPotential:
    """Fitted function restricted to a compact ligand-type list (``terms.py:300-328``): ``W [n_rt, TL, 6]``,
    ligand radii per compact type, and the intra-ligand Vina form with the fitted intra weights (``p``)."""

    def __init__(self, spec: FittedSpec, weights, lig_ext_list):
        w = np.asarray(weights, np.float32)
        self.spec = spec
        self.lig_ext_list = np.asarray(lig_ext_list, np.int64)
        self.TL = len(self.lig_ext_list)
        xs = spec.lig_xs[self.lig_ext_list]
        self.W = np.ascontiguousarray(spec.pair_table(w[:N_INTER])[:, self.lig_ext_list, :])
        self.radius = spec.xs_radius[xs].astype(np.float32)
        self.rad_rec = spec.rec_radius
        sfp = sf_params(spec.base)
        self.p = {**{k: sfp[k] for k in ("cutoff", "g1_off", "g1_w", "g2_off", "g2_w", "rep_off", "hyd_good",
                                        "hyd_bad", "hb_good", "hb_bad")},
                  "name": "fitted", "rot_weight": spec.rot_weight,
                  "w_g1": float(w[N_INTER]), "w_g2": float(w[N_INTER + 1]), "w_rep": float(w[N_INTER + 2]),
                  "w_hyd": float(w[N_INTER + 3]), "w_hb": float(w[N_INTER + 4]),
                  "radius": self.radius, "hydrophobic": spec.xs_hyd[xs].astype(np.int32),
                  "donor": spec.xs_don[xs].astype(np.int32), "acceptor": spec.xs_acc[xs].astype(np.int32)}


def receptor_ext_types(rec_xyz, rec_types, spec: FittedSpec, rec_chg=None):
    """Receptor ext types from buriedness (heavy-atom count within ``buried_radius``, self excluded) and charge
    class (``terms.py:204-231``). Synthetic receptors carry no charges unless ``rec_chg`` is given."""
    from scipy.spatial import cKDTree
    xyz = np.asarray(rec_xyz, np.float64)
    tree = cKDTree(xyz)
    cnt = np.array([len(x) for x in tree.query_ball_point(xyz, spec.buried_radius)]) - 1
    bur = (cnt >= spec.buried_threshold).astype(np.int64)
    chg = np.zeros(len(xyz), np.int64) if rec_chg is None else np.asarray(rec_chg, np.int64)
    return (np.asarray(rec_types, np.int64) + spec.nxs * (bur + 2 * chg)).astype(np.int64)
