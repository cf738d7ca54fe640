"""Analytic pose gradient of the CUDA energy (adock_eg) against central finite differences of the energy.

The differences are taken in float64 on the device (adock_rescore64: the same energy as adock_eg, float64
kinematics, the same maps or receptor atoms; the test first checks that the two energies agree), with steps of
2e-5 A / 2e-5 rad on every state component: translation, rotation (a rotation vector composed on the left of the
quaternion, the convention of the torque components) and each torsion. The state is float32, so each difference
is divided by the perturbation actually stored (for the rotation: the rotation vector between the two stored
quaternions, and the gradient is projected on it).

Components whose perturbation moves an atom across a grid cell (grid mode), or a ligand-receptor (exact mode) or
intra-ligand pair across the 8 A cutoff or an end of its hydrophobic or H-bond ramp, are masked: there the energy
has a step or a kink. This follows the
reference's checks of the lookup gradient (tests/test_scoring_grid.py:122-140) and of the pose gradient
(tests/test_ligand.py:74-110). Bar: per pose ||fd - g|| / max(||g||, 1) < 1e-3 over the unmasked components.
"""
import numpy as np
import pytest
import torch

from helpers import ligands, lig_types, make_problem, oracle_grid, random_states, receptor, rel_close

pytestmark = pytest.mark.gpu
H = 2e-5


def _qmul(a, b):
    aw, ax, ay, az = np.moveaxis(a, -1, 0)
    bw, bx, by, bz = np.moveaxis(b, -1, 0)
    return np.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], -1)


def _rotvec_between(qa, qb):
    """Rotation vector r with quat(r) * qb = qa (unit quaternions, float64)."""
    qa = qa / np.linalg.norm(qa, axis=-1, keepdims=True)
    qb = qb / np.linalg.norm(qb, axis=-1, keepdims=True)
    r = _qmul(qa, qb * np.array([1, -1, -1, -1]))
    r = r * np.where(r[..., :1] < 0, -1.0, 1.0)
    s = np.linalg.norm(r[..., 1:], axis=-1, keepdims=True)
    return r[..., 1:] * 2 * np.arctan2(s, r[..., :1]) / np.maximum(s, 1e-300)


def _perturbations(st, nt):
    """(plus, minus) float32 states [N, D, SD] and the stored perturbation [N, D, 3 or 1] per component."""
    N, SD = st.shape
    D = 6 + nt
    plus = np.repeat(st[:, None].astype(np.float64), D, 1)
    minus = plus.copy()
    for d in range(3):
        plus[:, d, d] += H
        minus[:, d, d] -= H
        v = np.zeros(3)
        v[d] = 1.0
        dq = np.concatenate([[np.cos(H / 2)], np.sin(H / 2) * v])
        dqi = dq * np.array([1, -1, -1, -1])
        plus[:, 3 + d, 3:7] = _qmul(dq, st[:, 3:7].astype(np.float64))
        minus[:, 3 + d, 3:7] = _qmul(dqi, st[:, 3:7].astype(np.float64))
    for k in range(nt):
        plus[:, 6 + k, 7 + k] += H
        minus[:, 6 + k, 7 + k] -= H
    plus, minus = plus.astype(np.float32), minus.astype(np.float32)
    step = np.zeros((N, D, 3))
    for d in range(3):
        step[:, d, 0] = plus[:, d, d].astype(np.float64) - minus[:, d, d]
        step[:, 3 + d] = _rotvec_between(plus[:, 3 + d, 3:7].astype(np.float64), minus[:, 3 + d, 3:7].astype(np.float64))
    for k in range(nt):
        step[:, 6 + k, 0] = plus[:, 6 + k, 7 + k].astype(np.float64) - minus[:, 6 + k, 7 + k]
    return plus, minus, step


def _crossing(model, dp, dm, rp, rm, ti, tj):
    """True where a pair's perturbation crosses a point where its energy has a step or a kink: the cutoff, the ends
    of the hydrophobic ramp (hydrophobic pairs) or of the H-bond ramp (donor-acceptor pairs)."""
    bad = (rp < model.cutoff) != (rm < model.cutoff)
    hyd = model.hyd[ti] & model.hyd[tj]
    hb = (model.don[ti] & model.acc[tj]) | (model.acc[ti] & model.don[tj])
    for edge, on in ((model.hyd_good, hyd), (model.hyd_bad, hyd), (model.hb_good, hb), (model.hb_bad, hb)):
        bad |= on & ((dp < edge) != (dm < edge))
    return bad


def _kinks(model, l, plus, minus, exact, gs, rec_xyz, rec_types):
    """[N, D] True where the perturbation crosses a grid cell (grid mode), or a pair (intra, and ligand-receptor in
    exact mode) crosses its cutoff or a ramp end (float64 oracle kinematics)."""
    N, D, SD = plus.shape
    Xp = model.pose_heavy(l, plus.reshape(-1, SD)).reshape(N, D, -1, 3)
    Xm = model.pose_heavy(l, minus.reshape(-1, SD)).reshape(N, D, -1, 3)
    na = Xp.shape[2]
    tl = model.typ[l, :na]
    bad = np.zeros((N, D), bool)
    npairs = int(model.np[l])
    if npairs:
        i, j = model.pr[l, :npairs, 0], model.pr[l, :npairs, 1]
        rp = np.linalg.norm(Xp[..., i, :] - Xp[..., j, :], axis=-1)
        rm = np.linalg.norm(Xm[..., i, :] - Xm[..., j, :], axis=-1)
        rs = model.radius[tl[i]] + model.radius[tl[j]]
        bad |= _crossing(model, rp - rs, rm - rs, rp, rm, tl[i], tl[j]).any(-1)
    if exact:
        rt = np.asarray(rec_types, np.int64)
        rs = model.radius[tl][:, None] + model.radius[rt][None, :]
        for n in range(N):
            rp = np.linalg.norm(Xp[n][:, :, None] - rec_xyz[None, None], axis=-1)
            rm = np.linalg.norm(Xm[n][:, :, None] - rec_xyz[None, None], axis=-1)
            bad[n] |= _crossing(model, rp - rs, rm - rs, rp, rm, tl[:, None], rt[None, :]).any((-1, -2))
    else:
        dims = gs.dims[0].numpy()
        cell = lambda X: np.floor(np.minimum(np.maximum((X - gs.origin[0].numpy()) / gs.spacing, 0), dims - 1 - 1e-4))
        bad |= (cell(Xp) != cell(Xm)).any((-1, -2))
    return bad


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("kind", ["mixed", "big"])
def test_gradient_matches_central_differences(exact, kind):
    from adock_b200 import params
    from adock_b200.kernel import B200KernelProblem
    from adock_b200.problem import pack_host
    from oracle.fp64 import Packed
    dev = torch.device("cuda:0")
    sfp = params.sf_params("vina")
    rec = receptor("cfg0")
    ligs = ligands(kind)
    lt = lig_types(ligs)
    G = oracle_grid(rec, sfp, lt)
    pg, pc = make_problem(rec, ligs, sfp, G, lt, dev), make_problem(rec, ligs, sfp, G, lt, "cpu")
    kp = B200KernelProblem(pg)
    model = Packed(*pack_host(pc)[2:])
    cl, st = random_states(pc, 16, seed=21, sigma=1.5)
    e, g = kp.energy_grad(torch.as_tensor(cl, device=dev), torch.as_tensor(st, device=dev), exact=exact)
    e, g = e.cpu().numpy(), g.cpu().numpy()
    e64, _, _ = kp.rescore64(torch.as_tensor(cl, device=dev), torch.as_tensor(st, device=dev), exact=exact)
    assert rel_close(e, e64.cpu().numpy()) < 1e-4, "adock_eg and the float64 re-score compute different energies"
    checked = 0
    for l in range(pc.lb.L):
        sel = np.where(cl == l)[0]
        nt = int(model.nt[l])
        D = 6 + nt
        plus, minus, step = _perturbations(st[sel], nt)
        SD = st.shape[1]
        both = np.concatenate([plus.reshape(-1, SD), minus.reshape(-1, SD)])
        clb = torch.full((len(both),), l, dtype=torch.int32, device=dev)
        E, _, _ = kp.rescore64(clb, torch.as_tensor(both, device=dev), exact=exact)
        E = E.cpu().numpy().reshape(2, len(sel), D)
        dE = E[0] - E[1]
        gl = g[sel, :D].astype(np.float64)
        # analytic change along the stored perturbation: translation / torsion components 1-D, rotation 3-D
        pred = np.concatenate([gl[:, :3] * step[:, :3, 0],
                               np.einsum("ndk,nk->nd", step[:, 3:6], gl[:, 3:6]),
                               gl[:, 6:] * step[:, 6:, 0]], 1)
        size = np.linalg.norm(step, axis=-1)
        fd, an = dE / size, pred / size
        bad = _kinks(model, l, plus, minus, exact, pc.gs, rec["rec_xyz"].astype(np.float64), rec["rec_types"])
        fd, an = np.where(bad, 0.0, fd), np.where(bad, 0.0, an)
        err = np.linalg.norm(fd - an, axis=1) / np.maximum(np.linalg.norm(an, axis=1), 1.0)
        assert err.max() < 1e-3, (l, err.max(), bad.mean())
        checked += int((~bad).sum())
    assert checked > 0.8 * sum(16 * (6 + int(model.nt[l])) for l in range(pc.lb.L))
