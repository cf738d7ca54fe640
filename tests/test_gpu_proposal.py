"""Learned proposal on the B200: tensor-core GEMM against torch, network gradients against the float64 oracle
(oracle/mlp.py), feature rows and the training-data log of the MC kernel, training, and the proposal-driven MC
with its plain-MC fallback."""
import numpy as np
import pytest
import torch

from helpers import ligands, lig_types, make_problem, oracle_grid, receptor, random_states

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    assert torch.cuda.is_available()
    return torch.device("cuda:0")


@pytest.mark.parametrize("M,N,K,ta,tb", [(64, 64, 32, 0, 0), (100, 72, 40, 0, 0), (257, 256, 288, 1, 0),
                                         (256, 64, 1000, 1, 0), (333, 256, 64, 0, 1), (1, 7, 5, 1, 1)])
def test_gemm_bf16_matches_torch(dev, M, N, K, ta, tb):
    from adock_b200.proposal import _gemm
    g = torch.Generator(device=dev).manual_seed(M * 7 + N)
    A = torch.randn(K, M, device=dev, generator=g).to(torch.bfloat16) if ta else \
        torch.randn(M, K, device=dev, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device=dev, generator=g).to(torch.bfloat16) if tb else \
        torch.randn(K, N, device=dev, generator=g).to(torch.bfloat16)
    Am = A.t() if ta else A
    Bm = B.t() if tb else B
    sA = (1, M) if ta else (K, 1)
    sB = (1, K) if tb else (N, 1)
    C = torch.empty(M, N, device=dev)
    bias = torch.randn(N, device=dev, generator=g)
    with torch.cuda.device(dev):
        _gemm(A, sA, B, sB, M, N, K, C=C, bias=bias)
    ref = Am.float() @ Bm.float() + bias
    torch.testing.assert_close(C, ref, rtol=1e-4, atol=1e-3)
    from adock_b200 import _lib
    assert _lib.load().adock_gemm_status() == 0


def _gemm_call(name, A, sA, B, sB, M, N, K, C=None, beta=0.0, bias=None, act=0, pre=None, Cb=None):
    from adock_b200 import _lib
    _lib.call(name, M, N, K, _lib.ptr(A), sA[0], sA[1], _lib.ptr(B), sB[0], sB[1], _lib.ptr(C),
              N if C is not None else 0, float(beta), _lib.ptr(bias), int(act), _lib.ptr(pre), _lib.ptr(Cb),
              N if Cb is not None else 0, _lib.stream_ptr())


@pytest.mark.parametrize("M,N,K", [(8192, 256, 288), (300, 200, 70), (129, 65, 16), (1, 1, 1), (5, 130, 0)])
def test_gemm_tcgen05_epilogue_matches_mma_sync(dev, M, N, K):
    """The tcgen05 GEMM against the independent mma.sync kernel: beta accumulation, bias, pre-activation copy,
    SiLU and the BF16 copy, on sizes that are not tile multiples (and K = 0)."""
    from adock_b200 import _lib
    g = torch.Generator(device=dev).manual_seed(M + 3 * N + 7 * K)
    A = torch.randn(M, max(K, 1), device=dev, generator=g).to(torch.bfloat16)
    B = torch.randn(max(K, 1), N, device=dev, generator=g).to(torch.bfloat16)
    C0 = torch.randn(M, N, device=dev, generator=g)
    bias = torch.randn(N, device=dev, generator=g)
    out = {}
    for name in ("adock_gemm_bf16", "adock_gemm_bf16_mma"):
        C, pre = C0.clone(), torch.empty(M, N, device=dev)
        Cb = torch.empty(M, N, dtype=torch.bfloat16, device=dev)
        with torch.cuda.device(dev):
            _gemm_call(name, A, (max(K, 1), 1), B, (N, 1), M, N, K, C=C, beta=0.5, bias=bias, act=1, pre=pre, Cb=Cb)
        out[name] = (C, pre, Cb)
    torch.cuda.synchronize(dev)
    assert _lib.load().adock_gemm_status() == 0
    ref_pre = (A[:, :K].float() @ B[:K].float() if K > 0 else torch.zeros(M, N, device=dev)) + 0.5 * C0 + bias
    for name, (C, pre, Cb) in out.items():
        torch.testing.assert_close(pre, ref_pre, rtol=1e-4, atol=2e-3, msg=name)
        torch.testing.assert_close(C, torch.nn.functional.silu(ref_pre), rtol=1e-4, atol=2e-3, msg=name)
        torch.testing.assert_close(Cb.float(), C, rtol=1e-2, atol=1e-2, msg=name)
    a, b = out["adock_gemm_bf16"][1], out["adock_gemm_bf16_mma"][1]
    torch.testing.assert_close(a, b, rtol=1e-5, atol=1e-4)


@pytest.mark.parametrize("n_comp", [1, 3])
def test_network_gradients_match_float64_oracle(dev, n_comp):
    from oracle import mlp as O
    from adock_b200.proposal import ProposalNet
    net = ProposalNet(dev, seed=3, n_comp=n_comp)
    for w in net.W:   # a non-trivial network
        w.add_(torch.randn_like(w) * 0.05)
    net.Wb = [w.to(torch.bfloat16).contiguous() for w in net.W]
    g = torch.Generator(device=dev).manual_seed(1)
    B = 512
    from adock_b200.proposal import IN
    X = torch.randn(B, IN, device=dev, generator=g).to(torch.bfloat16)
    Y = torch.randn(B, 32, device=dev, generator=g) * 0.5
    Y[:, 26] = torch.randint(0, 21, (B,), device=dev, generator=g).float()
    Y[:, 27:] = 0
    loss, grads = net.loss_grad(X, Y)
    Wr = [w.to(torch.bfloat16).double().cpu().numpy() for w in net.W]
    lo, go = O.loss_and_grads(Wr, [b.double().cpu().numpy() for b in net.b], X.double().cpu().numpy(),
                              Y.double().cpu().numpy(), n_comp=n_comp)
    assert abs(float(loss) - lo) <= 1e-2 * max(1.0, abs(lo))
    for gg, gr in zip(grads, go):
        gg = gg.double().cpu().numpy()
        assert np.linalg.norm(gg - gr) <= 2e-2 * np.linalg.norm(gr) + 1e-6


def _problem(dev):
    from adock_b200 import params
    sfp = params.sf_params("vina")
    rec = receptor("cfg0")
    ligs = ligands("mixed")
    lt = lig_types(ligs)
    G = oracle_grid(rec, sfp, lt) if _have_ref() else None
    if G is None:
        from adock_b200.grid import build_grid, grid_dims
        o = rec["center"] - rec["size"] / 2
        G = build_grid(rec["rec_xyz"], rec["rec_types"], sfp, o, params.GRID_SPACING,
                       grid_dims(rec["size"], params.GRID_SPACING), lt, device=dev).cpu().numpy()
    return make_problem(rec, ligs, sfp, G, lt, dev)


def _have_ref():
    from oracle import ref
    return ref.available()


def test_features_log_training_and_proposal_mc(dev):
    from adock_b200 import params
    from adock_b200.kernel import B200KernelProblem
    from adock_b200.proposal import ProposalNet, collect, run_mc_segments
    prob = _problem(dev)
    kp = B200KernelProblem(prob)
    cl, st = random_states(prob, 32, seed=7, sigma=1.0)
    cl = torch.as_tensor(cl, device=dev)
    st = torch.as_tensor(st, device=dev)
    M = len(cl)
    ci = torch.arange(M, dtype=torch.int32, device=dev)
    # feature rows: finite, torsion sin/cos zero beyond each ligand's count, descriptors as documented
    F = kp.prop_features(cl, st).float().cpu().numpy()
    assert F.shape == (M, 320) and np.isfinite(F).all()
    for i in range(M):
        p = prob.lb.preps[int(cl[i])]
        assert abs(F[i, 263] - p.n / 64) < 1e-2 and abs(F[i, 264] - p.n_tors / 20) < 1e-2
        assert np.all(F[i, 223 + 2 * p.n_tors:263] == 0) and np.all(F[i, 275:] == 0)
        assert abs(np.linalg.norm(F[i, 219:223]) - 1) < 2e-2 and F[i, 219] >= 0
    # training-data log of the plain search
    cfg = params.workload_preset(32, 6)
    cur, best = st.clone(), st.clone()
    ce, be = torch.zeros(M, device=dev), torch.full((M,), float("inf"), device=dev)
    X, Y = collect(kp, cl, ci, cur, ce, best, be, cfg, seed=5, cap=100000)
    assert X.shape[0] > M  # several improving moves per chain
    Yn = Y.cpu().numpy()
    assert np.isfinite(Yn).all() and np.all(np.abs(Yn[:, 6:26]) <= np.pi + 1e-4)
    nt = Yn[:, 26].astype(int)
    for i in range(len(Yn)):
        assert np.all(Yn[i, 6 + nt[i]:26] == 0)
    # training lowers the loss
    net = ProposalNet(dev, seed=0)
    l0 = float(net.loss_grad(X, Y)[0])
    net.fit(X, Y, epochs=30, batch=min(256, X.shape[0]), lr=3e-3)
    l1 = float(net.loss_grad(X, Y)[0])
    assert l1 < l0
    # proposal-driven MC: energies are consistent and the fallback accounting adds up
    cur, best = st.clone(), st.clone()
    ce, be = torch.zeros(M, device=dev), torch.full((M,), float("inf"), device=dev)
    stats = {}
    run_mc_segments(kp, net, cl, ci, cur, ce, best, be, cfg, seed=9, prop_k=4, stats=stats)
    e_best, _ = kp.energy_grad(cl, best)
    torch.testing.assert_close(e_best, be, rtol=1e-4, atol=1e-4)
    assert stats["prop_steps"] + stats["plain_steps"] == M * cfg["mc_steps"]
    assert stats["prop_steps"] > 0
    # a second round of training data from the learned search itself: moves logged across its segments
    from adock_b200.proposal import collect_learned
    X2, Y2 = collect_learned(kp, net, cl, ci, st.clone(), cfg, seed=11, cap=100000, prop_k=4)
    assert X2.shape[0] > M and X2.shape[0] == Y2.shape[0]
    Y2n = Y2.cpu().numpy()
    assert np.isfinite(Y2n).all() and np.all(np.abs(Y2n[:, 6:26]) <= np.pi + 1e-4)


def _wrap(d):
    return d - 2 * np.pi * np.floor((d + np.pi) / (2 * np.pi))


def test_ligand_best_hint(dev):
    """adock_prop_hint picks, per ligand, the chain with the lowest finite best energy (ties: the lowest chain
    index; non-finite energies never win) and copies its state; the feature row's hint columns equal a float64
    restatement (translation / rotation-vector / torsion differences, energy terms); segmenting the plain search
    for the hint leaves its moves unchanged."""
    from adock_b200 import params
    from adock_b200.kernel import B200KernelProblem
    from adock_b200.proposal import HINT_COLS, collect, without_hint
    prob = _problem(dev)
    kp = B200KernelProblem(prob)
    L = prob.lb.L
    cl, st = random_states(prob, 12, seed=4, sigma=1.5)
    M = len(cl)
    cln = np.asarray(cl)
    rng = np.random.default_rng(3)
    be = rng.normal(-5, 2, M).astype(np.float32)
    be[rng.random(M) < 0.1] = np.inf
    be[rng.random(M) < 0.05] = np.nan
    l0 = np.where(cln == 0)[0]
    be[l0] = np.inf                      # ligand 0: no finite energy -> no hint
    l1 = np.where(cln == 1)[0]
    be[l1[1]] = be[l1[3]] = -50.0        # tie: the lower chain index wins
    clg, stg = torch.as_tensor(cl, device=dev), torch.as_tensor(st, device=dev)
    hint = kp.prop_hint(clg, stg, torch.as_tensor(be, device=dev)).cpu().numpy()
    for l in range(L):
        ch = np.where((cln == l) & np.isfinite(be))[0]
        if len(ch) == 0:
            assert np.all(hint[l] == 0), l
            continue
        w = ch[np.argmin(be[ch])]
        assert l != 1 or w == l1[1]
        K = min(20, st.shape[1] - 7)
        np.testing.assert_array_equal(hint[l, :7 + K], st[w, :7 + K])
        assert hint[l, 27] == be[w] and hint[l, 28] == 1.0
    # hint columns of the feature rows
    ce = rng.normal(-3, 2, M).astype(np.float32)
    F = kp.prop_features(clg, stg, torch.as_tensor(ce, device=dev), torch.as_tensor(hint, device=dev))
    F = F.float().cpu().numpy()
    F0 = kp.prop_features(clg, stg).float().cpu().numpy()
    other = [c for c in range(320) if c not in HINT_COLS]
    np.testing.assert_array_equal(F[:, other], F0[:, other])
    assert np.all(F0[:, HINT_COLS] == 0)
    slog = lambda v: np.sign(v) * np.log1p(np.abs(v))
    for i in range(M):
        h = hint[cln[i]].astype(np.float64)
        s = st[i].astype(np.float64)
        if h[28] == 0:
            assert np.all(F[i, HINT_COLS] == 0)
            continue
        qa = s[3:7] / np.linalg.norm(s[3:7])
        qb = h[3:7] / np.linalg.norm(h[3:7])
        aw, av = qa[0], -qa[1:]
        r = np.concatenate([[qb[0] * aw - qb[1:] @ av], qb[0] * av + aw * qb[1:] + np.cross(qb[1:], av)])
        r = r if r[0] >= 0 else -r
        sn = np.linalg.norm(r[1:])
        rv = r[1:] * 2 * np.arctan2(sn, r[0]) / max(sn, 1e-300) / np.pi
        nt = prob.lb.preps[cln[i]].n_tors
        want = np.concatenate([(h[:3] - s[:3]) / 10, rv, [slog(ce[i] - h[27]), slog(ce[i]), 1.0]])
        tw = np.zeros(20)
        tw[:nt] = _wrap(h[7:7 + nt] - s[7:7 + nt]) / np.pi
        got = F[i, HINT_COLS]
        # BF16 rows: 2^-8 relative; wrapped torsion differences near +-pi may land on either end
        assert np.all(np.abs(got[:9] - want) <= 1e-2 * np.maximum(np.abs(want), 0.1)), (i, got[:9], want)
        dt = np.abs(got[9:] - tw)
        assert np.all((dt <= 1e-2) | (np.abs(dt - 2) <= 1e-2)), (i, got[9:], tw)
    np.testing.assert_array_equal(without_hint(torch.as_tensor(F)).numpy()[:, HINT_COLS], 0)
    # the segmented plain search (hint in the logged features) makes the same moves as one launch
    cfg = params.workload_preset(32, 12)
    res = []
    for hs in (0, 4):
        cur, best = stg.clone(), stg.clone()
        c_e, b_e = torch.zeros(M, device=dev), torch.full((M,), float("inf"), device=dev)
        X, Y = collect(kp, clg, torch.arange(M, dtype=torch.int32, device=dev), cur, c_e, best, b_e, cfg, seed=5,
                       cap=100000, hint_segment=hs)
        res.append((best.cpu(), b_e.cpu(), X))
    torch.testing.assert_close(res[0][1], res[1][1], rtol=0, atol=0)
    torch.testing.assert_close(res[0][0], res[1][0], rtol=0, atol=0)
    assert (res[1][2][:, HINT_COLS[-20:]] != 0).any() and (res[0][2][:, HINT_COLS] == 0).all()


def test_trained_proposal_beats_plain_mc_at_equal_budget(dev):
    """What the trained network gains: on the screening shapes (8,000-atom receptor, 8-80-atom ligands), a proposal
    trained on the plain search's moves from 96 fresh ligands, then FP16 maps + learned proposal vs plain FP32 MC
    on 64 held-out ligands x 32 chains from the same Stage-A starts at an equal budget of 500 steps. The gap is a
    ligand's best energy minus the lowest any run found for it (a 2,000-step plain run included). Bar: the learned
    search's median gap is below 0.7 x plain MC's."""
    from adock_b200 import synth
    from adock_b200.proposal import ab_compare
    rec = synth.config_receptor(2)
    train = synth.ligand_set(96, (8, 80), (0, 20), seed0=500_000)
    held = synth.ligand_set(64, (8, 80), (0, 20), seed0=600_000)
    ab = ab_compare(rec, train, held, device=dev, budgets=(500,), ref_steps=2000, log_cap=1_000_000,
                    learned=[("learned", 32, 0.3, "chain")], plain_f16=False)
    gap = {m: next(r["median_gap"] for r in rs if r["steps"] == 500) for m, rs in ab["methods"].items()}
    assert gap["learned"] < 0.7 * gap["plain_f32"], gap
