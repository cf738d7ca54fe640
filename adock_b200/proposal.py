"""Learned Monte-Carlo proposal (no reference counterpart).

A small MLP proposes the MC move of each chain: x [320 features of the chain's current state] -> SiLU(256) ->
SiLU(256) -> 64 outputs = Gaussian means (columns 0..25) and log standard deviations (32..57) of the move
(translation 3 A, rotation vector 3 rad, torsion deltas 20 rad). Weights are BF16 on the tensor cores with FP32
accumulation; training keeps FP32 master weights and Adam moments. Every kernel is the library's own
(adock_gemm_bf16, adock_mlp_nll, adock_silu_backward, adock_bias_grad, adock_adam).

Training data come from the plain search itself (``collect``): the MC kernel logs, for each accepted move that
lowered the chain's energy, the features of the pre-move state and the state; the target is the move from that
state to the chain's best state at the end of the run. In the search (``run_mc_segments``) a fraction of the
steps take the network's move instead of the random perturbation (the sampled spread has floors so the moves keep
exploring); the Vina-form energy with BFGS and the Metropolis test still decide every move, and a chain whose
learned moves are rejected 8 times in a row falls back to plain MC until it accepts a move.

A network with ``uses_hint`` also reads the ligand-best hint: before each segment, the best state over the chain's
ligand's chains (``B200KernelProblem.prop_hint``), given relative to the chain's state (translation, rotation and
torsion differences, energy difference). Without it those columns (``HINT_COLS``) are 0, in training and search.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib

IN, HID, OUT = 320, 256, 64
HINT_COLS = list(range(275, 284)) + list(range(288, 308))   # ligand-best hint columns of the feature row


def _gemm(A, sA, B, sB, M, N, K, C=None, beta=0.0, bias=None, act=0, pre=None, Cb=None):
    """C[M,N] = A[M,K] B[K,N] (BF16 operands with (row, col) strides sA, sB; FP32 accumulation)."""
    _lib.call("adock_gemm_bf16", M, N, K, _lib.ptr(A), sA[0], sA[1], _lib.ptr(B), sB[0], sB[1], _lib.ptr(C),
              N if C is not None else 0, float(beta), _lib.ptr(bias), int(act), _lib.ptr(pre), _lib.ptr(Cb),
              N if Cb is not None else 0, _lib.stream_ptr())


def check_gemm(where):
    """Raise if a tensor-core GEMM gave up waiting for its MMAs since the last check (its output tile was then not
    written, so the network's outputs or gradients are unusable). Synchronises the device."""
    if _lib.load().adock_gemm_status() != 0:
        raise RuntimeError(f"{where}: a tcgen05 GEMM timed out waiting for its tensor-core work; results discarded")


class ProposalNet:
    """320 -> 256 -> 256 -> 64 MLP; weights W_i stored [K, N] row-major (x @ W). uses_hint: the network reads the
    ligand-best hint columns (else they are 0 in its inputs)."""

    def __init__(self, device="cuda", seed=0, init_log_sd=(0.0, -1.0, -0.5), uses_hint=False, n_comp=1):
        dev = torch.device(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        dims = [(IN, HID), (HID, HID), (HID, OUT)]
        self.W = [(torch.randn(k, n, generator=g) * math.sqrt(2.0 / k)).to(dev) for k, n in dims]
        self.W[2].mul_(0.01)
        self.n_comp = int(n_comp)
        assert self.n_comp in (1, 3)
        if self.n_comp == 3:
            # translation mixture: the extra means (columns 27-29, 58-60) start further apart than the 0.01 scale
            # of the other outputs, so that the components can take different basins
            for c in (27, 28, 29, 58, 59, 60):
                self.W[2][:, c] *= 30.0
        self.b = [torch.zeros(n, device=dev) for _, n in dims]
        # initial spread: log sd for translation, rotation, torsion columns
        self.b[2][32:35] = init_log_sd[0]
        self.b[2][35:38] = init_log_sd[1]
        self.b[2][38:58] = init_log_sd[2]
        self.params = self.W + self.b
        self.Wb = [w.to(torch.bfloat16).contiguous() for w in self.W]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step = 0
        self.device = dev
        self.uses_hint = bool(uses_hint)

    def state_dict(self):
        return {"W": [w.cpu() for w in self.W], "b": [b.cpu() for b in self.b], "step": self.step,
                "uses_hint": self.uses_hint, "n_comp": self.n_comp}

    def load_state_dict(self, d):
        for dst, src in zip(self.W + self.b, d["W"] + d["b"]):
            dst.copy_(src.to(self.device))
        self.Wb = [w.to(torch.bfloat16).contiguous() for w in self.W]
        self.step = int(d.get("step", 0))
        self.uses_hint = bool(d.get("uses_hint", False))
        self.n_comp = int(d.get("n_comp", 1))

    def forward(self, x, save=False):
        """x: BF16 [B, 320] -> out FP32 [B, 64] (and saved activations when save)."""
        B = x.shape[0]
        dev = self.device
        pre1 = torch.empty(B, HID, device=dev)
        h1 = torch.empty(B, HID, dtype=torch.bfloat16, device=dev)
        pre2 = torch.empty(B, HID, device=dev)
        h2 = torch.empty(B, HID, dtype=torch.bfloat16, device=dev)
        out = torch.empty(B, OUT, device=dev)
        c1 = torch.empty(B, HID, device=dev)
        c2 = torch.empty(B, HID, device=dev)
        with torch.cuda.device(dev):
            _gemm(x, (IN, 1), self.Wb[0], (HID, 1), B, HID, IN, C=c1, bias=self.b[0], act=1, pre=pre1, Cb=h1)
            _gemm(h1, (HID, 1), self.Wb[1], (HID, 1), B, HID, HID, C=c2, bias=self.b[1], act=1, pre=pre2, Cb=h2)
            _gemm(h2, (HID, 1), self.Wb[2], (OUT, 1), B, OUT, HID, C=out, bias=self.b[2])
        if save:
            return out, (x, pre1, h1, pre2, h2)
        return out

    def loss_grad(self, x, y):
        """Mean Gaussian NLL of moves y [B, 32] and the parameter gradients (list matching self.params)."""
        B = x.shape[0]
        dev = self.device
        out, (x, pre1, h1, pre2, h2) = self.forward(x, save=True)
        dout = torch.empty(B, OUT, dtype=torch.bfloat16, device=dev)
        loss = torch.zeros(1, device=dev)
        gW = [torch.empty_like(w) for w in self.W]
        gb = [torch.empty_like(b) for b in self.b]
        dH2 = torch.empty(B, HID, device=dev)
        dA2 = torch.empty(B, HID, dtype=torch.bfloat16, device=dev)
        dH1 = torch.empty(B, HID, device=dev)
        dA1 = torch.empty(B, HID, dtype=torch.bfloat16, device=dev)
        s = _lib.stream_ptr
        with torch.cuda.device(dev):
            _lib.call("adock_mlp_nll", _lib.ptr(out), _lib.ptr(y), B, self.n_comp, _lib.ptr(dout), _lib.ptr(loss), s())
            # layer 3: dW3 = h2^T dout, db3, dH2 = dout W3^T
            _gemm(h2, (1, HID), dout, (OUT, 1), HID, OUT, B, C=gW[2])
            _lib.call("adock_bias_grad", _lib.ptr(dout), B, OUT, _lib.ptr(gb[2]), s())
            _gemm(dout, (OUT, 1), self.Wb[2], (1, OUT), B, HID, OUT, C=dH2)
            _lib.call("adock_silu_backward", _lib.ptr(dH2), _lib.ptr(pre2), B * HID, _lib.ptr(dA2), s())
            # layer 2
            _gemm(h1, (1, HID), dA2, (HID, 1), HID, HID, B, C=gW[1])
            _lib.call("adock_bias_grad", _lib.ptr(dA2), B, HID, _lib.ptr(gb[1]), s())
            _gemm(dA2, (HID, 1), self.Wb[1], (1, HID), B, HID, HID, C=dH1)
            _lib.call("adock_silu_backward", _lib.ptr(dH1), _lib.ptr(pre1), B * HID, _lib.ptr(dA1), s())
            # layer 1
            _gemm(x, (1, IN), dA1, (HID, 1), IN, HID, B, C=gW[0])
            _lib.call("adock_bias_grad", _lib.ptr(dA1), B, HID, _lib.ptr(gb[0]), s())
        return loss / B, gW + gb

    def train_step(self, x, y, lr=1e-3, wd=0.0):
        loss, grads = self.loss_grad(x, y)
        self.step += 1
        with torch.cuda.device(self.device):
            for i, (p, g_, m, v) in enumerate(zip(self.params, grads, self.m, self.v)):
                pb = self.Wb[i] if i < 3 else None
                _lib.call("adock_adam", _lib.ptr(p), _lib.ptr(g_), _lib.ptr(m), _lib.ptr(v), _lib.ptr(pb), p.numel(),
                          float(lr), 0.9, 0.999, 1e-8, self.step, float(wd), _lib.stream_ptr())
        return loss

    def fit(self, X, Y, epochs=3, batch=4096, lr=1e-3, seed=0, log=None):
        """Minibatch Adam over (X BF16 [n, 320], Y [n, 32]); returns the mean loss of the last epoch."""
        n = X.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        last = float("nan")
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g, device=self.device)
            tot = torch.zeros(1, device=self.device)
            nb = 0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                tot += self.train_step(X[idx].contiguous(), Y[idx].contiguous(), lr=lr)
                nb += 1
            last = float(tot) / max(nb, 1)
            check_gemm(f"training epoch {ep}")
            if log is not None:
                log(f"epoch {ep}: loss {last:.4f}")
        return last


def moves_to(states, target):
    """Moves (proposal coordinates, [n, 32]) from logged states [n, 32] (t, q, torsions 0..19, count at 27) to
    target states [n, >= 7] (t, q, torsions): translation difference, rotation vector of q_target q^-1 (w >= 0),
    torsion differences wrapped to [-pi, pi) for torsions below the count (0 above); the count goes to entry 26."""
    n = states.shape[0]
    y = torch.zeros(n, 32, device=states.device)
    y[:, :3] = target[:, :3] - states[:, :3]
    qa = states[:, 3:7] / states[:, 3:7].norm(dim=1, keepdim=True)
    qb = target[:, 3:7] / target[:, 3:7].norm(dim=1, keepdim=True)
    aw, av = qa[:, :1], -qa[:, 1:]
    bw, bv = qb[:, :1], qb[:, 1:]
    w = bw * aw - (bv * av).sum(1, keepdim=True)
    v = bw * av + aw * bv + torch.cross(bv, av, dim=1)
    sgn = torch.where(w < 0, -1.0, 1.0)
    w, v = w * sgn, v * sgn
    sn = v.norm(dim=1, keepdim=True)
    ang = 2.0 * torch.atan2(sn, w)
    y[:, 3:6] = torch.where(sn > 1e-7, v * ang / sn.clamp_min(1e-12), 2.0 * v)
    nt = states[:, 27]
    K = min(20, target.shape[1] - 7)
    th = torch.zeros(n, 20, device=states.device)
    th[:, :K] = target[:, 7:7 + K]
    d = th - states[:, 7:27]
    d = d - 2 * math.pi * torch.floor((d + math.pi) / (2 * math.pi))
    d = torch.where(torch.arange(20, device=states.device)[None, :] < nt[:, None], d, torch.zeros_like(d))
    y[:, 6:26] = d
    y[:, 26] = nt
    return y


def ligand_best_chain(chain_lig, best_e):
    """Per ligand (0..max), the index of its chain with the lowest best energy (the highest index among ties;
    -1 for a ligand without chains)."""
    lig = chain_lig.long()
    L = int(lig.max()) + 1
    lo = torch.full((L,), float("inf"), device=best_e.device).scatter_reduce(0, lig, best_e, "amin")
    idx = torch.arange(len(lig), device=best_e.device)
    cand = torch.where(best_e <= lo[lig], idx, torch.full_like(idx, -1))
    return torch.full((L,), -1, dtype=torch.long, device=best_e.device).scatter_reduce(0, lig, cand, "amax")


def without_hint(X):
    """Feature rows with the ligand-best hint columns set to 0 (the inputs of a network without the hint)."""
    X = X.clone()
    X[:, HINT_COLS] = 0
    return X


def collect(kp, chain_lig, chain_id, cur, cur_e, best, best_e, cfg, seed, cap, init_opt=True, target="chain",
            hint_segment=0):
    """Run the plain MC search on the given chains with the training-data log on; returns (X BF16 [n, 320],
    Y [n, 32]): the features of the pre-move state of each accepted improving move and, as its target, the move
    from that state to a low-energy minimum the run found (n <= cap). target "chain": the chain's own best state
    at the end of the run; "ligand": the best state over all chains of the chain's ligand; "both": returns
    (X, Y_chain, Y_ligand). hint_segment > 0: the run is cut into launches of that many steps (the same moves:
    the random streams are indexed by step) and the logged features carry the ligand-best hint taken before each
    launch; 0: one launch, hint columns 0."""
    dev = kp.device
    lx = torch.empty(cap, IN, dtype=torch.bfloat16, device=dev)
    ly = torch.empty(cap, 32, device=dev)
    ln = torch.zeros(1, dtype=torch.int32, device=dev)
    steps = cfg["mc_steps"]
    seg = hint_segment if hint_segment > 0 else max(steps, 1)
    for sg in range(max(1, math.ceil(steps / seg))):
        k = min(seg, steps - sg * seg)
        hint = kp.prop_hint(chain_lig, best, best_e) if hint_segment > 0 and sg > 0 else None
        kp.run_mc(chain_lig, chain_id, cur, cur_e, best, best_e, init_opt and sg == 0, k, cfg["bfgs_iters"],
                  cfg["mc_temperature"], cfg["mc_amp_pos"], cfg["mc_amp_rot"], seed, sg * seg, log=(lx, ly, ln),
                  hint=hint)
    n = min(int(ln), cap)
    states = ly[:n]
    ch = states[:, 28].long()
    ok = torch.isfinite(states[:, :27]).all(1) & torch.isfinite(best[ch]).all(1)
    y_chain = y_lig = None
    if target in ("chain", "both"):
        y_chain = moves_to(states, best[ch])
    if target in ("ligand", "both"):
        y_lig = moves_to(states, best[ligand_best_chain(chain_lig, best_e)[chain_lig.long()[ch]]])
    keep = _finite_rows(lx[:n], ok, y_chain, y_lig)
    if target == "both":
        return lx[:n][keep], y_chain[keep], y_lig[keep]
    return lx[:n][keep], (y_chain if target == "chain" else y_lig)[keep]


def _finite_rows(X, ok, *Ys):
    """Rows of a training batch whose features, state and targets are all finite (a row with a non-finite value
    would turn the whole network into NaN at the first gradient step)."""
    keep = ok & torch.isfinite(X.float()).all(1)
    for Y in Ys:
        if Y is not None:
            keep &= torch.isfinite(Y).all(1)
    return keep


def collect_learned(kp, net, chain_lig, chain_id, cur, cfg, seed, cap, prop_k=32, prop_frac=0.3, prop_tries=1):
    """The learned search (``run_mc_segments`` with ``net``) from the states ``cur`` with the training-data log on;
    returns (X, Y) as ``collect`` does, the targets being the learned search's own final minima of each chain."""
    dev = kp.device
    N = cur.shape[0]
    best = cur.clone()
    ce, be = torch.zeros(N, device=dev), torch.full((N,), float("inf"), device=dev)
    lx = torch.empty(cap, IN, dtype=torch.bfloat16, device=dev)
    ly = torch.empty(cap, 32, device=dev)
    ln = torch.zeros(1, dtype=torch.int32, device=dev)
    run_mc_segments(kp, net, chain_lig, chain_id, cur, ce, best, be, cfg, seed, prop_k=prop_k, prop_frac=prop_frac,
                    log=(lx, ly, ln), prop_tries=prop_tries)
    n = min(int(ln), cap)
    states = ly[:n]
    tgt = best[states[:, 28].long()]
    Y = moves_to(states, tgt)
    keep = _finite_rows(lx[:n], torch.isfinite(states[:, :27]).all(1) & torch.isfinite(tgt).all(1), Y)
    return lx[:n][keep], Y[keep]


def _starts(prob, kp, cfg, seed):
    """Stage-A start poses of every chain (the search driver's first stage), packed as MC states."""
    from .search import stage_a_starts
    dev = kp.device
    L, M = prob.lb.L, cfg["n_chains"]
    lo, hi = prob.gs.lo[0].cpu().numpy(), prob.gs.hi[0].cpu().numpy()
    cur, _ = stage_a_starts(prob, kp, np.tile((lo + hi) / 2, (L, 1)), [hi - lo] * L, cfg, seed)
    chain_lig = torch.arange(L, device=dev, dtype=torch.int32).repeat_interleave(M)
    chain_id = torch.arange(L * M, device=dev, dtype=torch.int32)
    return chain_lig, chain_id, cur


def _problem_for(rec, ligs, dev, grid_dtype="f32"):
    import numpy as np
    from . import params
    from .grid import make_gridset
    from .kernel import B200KernelProblem
    from .ligand import LigandBatch
    from .problem import PairPotential, Problem, pad_receptors
    sfp = params.sf_params("vina")
    types = np.unique(np.concatenate([l.types for l in ligs]))
    gs = make_gridset([rec], sfp, params.GRID_SPACING, params.OUT_OF_BOX_PENALTY, device=dev, lig_types=[types])
    prob = Problem(gs, LigandBatch(ligs, dev), torch.zeros(len(ligs), dtype=torch.long, device=dev),
                   PairPotential(sfp, dev), rec=pad_receptors([rec], dev))
    return prob, B200KernelProblem(prob, grid_dtype=grid_dtype)


def _best_per_ligand(best_e, L, M):
    return best_e.view(L, M).min(1).values


def parse_learned(learned):
    """Learned variants (name, segment steps, learned fraction[, training "chain" | "ligand" | "dagger" |
    "daggerN"[, tries[, hint[, n_comp]]]]) -> {name: (prop_k, prop_frac, target, tries, hint, n_comp)}: the
    chain's or the ligand's best pose as target, or the chain network fine-tuned N times on its own search's
    moves; tries candidate targets per learned step; hint: the network reads the ligand-best hint; n_comp: 1, or 3
    for a translation mixture."""
    return {v[0]: (v[1], v[2], v[3] if len(v) > 3 else "chain", int(v[4]) if len(v) > 4 else 1,
                   bool(v[5]) if len(v) > 5 else False, int(v[6]) if len(v) > 6 else 1) for v in learned}


def _rounds(t):   # "dagger" = 1 self-training round on top of "chain", "dagger2" = 2, ...
    return int(t[6:] or 1) if t.startswith("dagger") else 0


def _dagger_name(n):
    return "chain" if n == 0 else ("dagger" if n == 1 else f"dagger{n}")


def train_variants(rec, train_ligs, variants, device="cuda", chains=32, train_steps=500, log_cap=2_000_000,
                   epochs=3, seed=0, log=None):
    """Train the networks the learned variants need (values of ``parse_learned``) on fresh ligands: the plain FP32
    search (Stage-A starts, ``train_steps`` MC steps) logs its improving moves, a network is fitted to them, and
    each self-training round lets the previous round's network drive the search on the training ligands and
    fine-tunes a copy on that search's moves. Returns ({(target, hint): net}, training record)."""
    from . import params
    dev = torch.device(device)
    variants = list(variants)
    cfg_tr = params.workload_preset(chains, train_steps)
    prob_t, kp_t = _problem_for(rec, train_ligs, dev)
    cl, ci, cur = _starts(prob_t, kp_t, cfg_tr, seed)
    N = cur.shape[0]
    best = cur.clone()
    ce, be = torch.zeros(N, device=dev), torch.full((N,), float("inf"), device=dev)
    torch.cuda.synchronize(dev)
    any_hint = any(v[4] for v in variants)
    X, Yc, Yl = collect(kp_t, cl, ci, cur, ce, best, be, cfg_tr, seed=seed + 1, cap=log_cap, target="both",
                        hint_segment=32 if any_hint else 0)
    nets = {}
    rec_out = {"moves": int(X.shape[0]), "epochs": epochs}
    # one network family per (hint, n_comp); each family trains the rounds its targets need
    targets = {(v[2], v[4], v[5]) for v in variants}
    for (t, h, m) in list(targets):
        for n in range(_rounds(t)):
            targets.add((_dagger_name(n), h, m))

    def label(tgt, hint, mix):
        return tgt + ("_hint" if hint else "") + ("_mix3" if mix > 1 else "")

    for (tgt, hint, mix) in sorted(targets, key=lambda th: (th[1], th[2], th[0] == "ligand", _rounds(th[0]))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        n = _rounds(tgt)
        if n > 0:
            # self-training round n: the previous round's network drives the search on the training ligands with
            # the log on; a copy of it is fine-tuned on those moves (targets: that search's own final minima)
            prev = nets[(_dagger_name(n - 1), hint, mix)]
            net = ProposalNet(dev, seed=seed, uses_hint=hint, n_comp=mix)
            net.load_state_dict(prev.state_dict())
            cl2, ci2, cur2 = _starts(prob_t, kp_t, cfg_tr, seed + 5 * n)
            X2, Y2 = collect_learned(kp_t, prev, cl2, ci2, cur2, cfg_tr, seed + 5 * n + 1, log_cap)
            loss = net.fit(X2, Y2, epochs=epochs, batch=4096, lr=5e-4, seed=seed + n, log=log)
            rec_out[label(tgt, hint, mix) + "_moves"] = int(X2.shape[0])
            del X2, Y2
        else:
            Y = Yc if tgt == "chain" else Yl
            net = ProposalNet(dev, seed=seed, uses_hint=hint, n_comp=mix)
            loss = net.fit(X if hint else without_hint(X), Y, epochs=epochs, batch=4096, lr=1e-3, seed=seed, log=log)
        e1.record()
        torch.cuda.synchronize(dev)
        nets[(tgt, hint, mix)] = net
        rec_out[label(tgt, hint, mix)] = {"final_loss": loss, "train_ms": e0.elapsed_time(e1)}
    return nets, rec_out


def ab_compare(rec, train_ligs, eval_ligs, device="cuda", chains=32, budgets=(125, 250, 500, 1000, 2000),
               ref_steps=8000, train_steps=500, log_cap=2_000_000, epochs=3, learned=(("learned_f16", 32, 0.3),),
               seed=0, log=None, learned_budgets=None, plain_f16=True):
    """Learned proposal vs plain MC at equal step budget (config-3 style evaluation).

    1. Training data: plain FP32 search (Stage-A starts, ``train_steps`` MC steps) on ``train_ligs`` with the
       move log on; the network is trained on it (``epochs`` of Adam).
    2. Reference: plain FP32 search with ``ref_steps`` steps on the held-out ``eval_ligs``; E_ref(l) = the lowest
       best energy over the ligand's chains (also over all runs below, so gaps are >= 0). The long run is also
       reported as the plain FP32 search's row at ``ref_steps``.
    3. For each budget S: plain FP32, plain FP16 and each learned FP16 variant (name, segment length prop_k,
       learned fraction prop_frac; proposals with plain fallback) from the same Stage-A starts;
       gap(l) = E(l) - E_ref(l); reported: median and mean gap, ligands/s of Stage A + MC, evaluations per step
       and per second. ``learned_budgets`` limits the learned variants' budgets; ``plain_f16=False`` skips the plain
       FP16 rows.
    """
    from . import params
    dev = torch.device(device)
    out = {"chains": chains, "budgets": list(budgets), "ref_steps": ref_steps, "train_ligands": len(train_ligs),
           "eval_ligands": len(eval_ligs)}
    variants = parse_learned(learned)
    # 1. data + training
    nets, out["train"] = train_variants(rec, train_ligs, variants.values(), dev, chains=chains,
                                        train_steps=train_steps, log_cap=log_cap, epochs=epochs, seed=seed, log=log)
    # 2./3. evaluation on held-out ligands
    probs = {"f32": _problem_for(rec, eval_ligs, dev, "f32")}
    probs["f16"] = (probs["f32"][0], type(probs["f32"][1])(probs["f32"][0], grid_dtype="f16"))
    L = len(eval_ligs)

    def run(method, steps):
        prob, kp = probs["f16" if method != "plain_f32" else "f32"]
        ev0 = int(kp.evals[0])
        cfg = params.workload_preset(chains, steps)
        cfg["autotune"] = False
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        cl, ci, cur = _starts(prob, kp, cfg, seed + 2)
        best = cur.clone()
        ce, be = torch.zeros(cur.shape[0], device=dev), torch.full((cur.shape[0],), float("inf"), device=dev)
        st = {}
        if method in variants:
            k, frac, tgt, tries, hint, mix = variants[method]
            run_mc_segments(kp, nets[(tgt, hint, mix)], cl, ci, cur, ce, best, be, cfg, seed + 3, prop_k=k,
                            prop_frac=frac, stats=st, prop_tries=tries)
        else:
            kp.run_mc(cl, ci, cur, ce, best, be, True, steps, cfg["bfgs_iters"], cfg["mc_temperature"],
                      cfg["mc_amp_pos"], cfg["mc_amp_rot"], seed + 3, 0)
        ev[1].record()
        torch.cuda.synchronize(dev)
        ms = ev[0].elapsed_time(ev[1])
        st["evals_per_step"] = (int(kp.evals[0]) - ev0) / (cur.shape[0] * steps)
        st["evals_per_s"] = (int(kp.evals[0]) - ev0) / (ms / 1e3)
        return _best_per_ligand(be, L, chains), ms, st

    ref, ref_ms, ref_st = run("plain_f32", ref_steps)
    results = {}
    out["learned_variants"] = {n: {"prop_k": k, "prop_frac": f, "target": t, "tries": r, "hint": h, "n_comp": m}
                               for n, (k, f, t, r, h, m) in variants.items()}
    for m in ("plain_f32", *(("plain_f16",) if plain_f16 else ()), *variants):
        for S in (learned_budgets or budgets if m in variants else budgets):
            results[(m, S)] = run(m, S)
    floor = ref.clone()
    for (e, _, _) in results.values():
        floor = torch.minimum(floor, e)
    out["reference"] = {"ms": ref_ms, "median_best": float(ref.median())}
    results[("plain_f32", ref_steps)] = (ref, ref_ms, ref_st)   # the long run is also the plain search's last budget
    rows = {}
    for (m, S), (e, ms, st) in sorted(results.items(), key=lambda kv: (kv[0][0], kv[0][1])):
        gap = (e - floor).cpu()
        rows.setdefault(m, []).append({"steps": S, "median_gap": float(gap.median()), "mean_gap": float(gap.mean()),
                                       "ligands_per_s": L / (ms / 1e3), "ms": ms, **st})
    out["methods"] = rows
    # equal-gap comparison: the budget each method needs to reach the plain FP32 median gap at its largest budget
    target = next(r["median_gap"] for r in rows["plain_f32"] if r["steps"] == max(budgets))
    out["target_gap"] = target
    for m, rs in rows.items():
        ok = [r for r in rs if r["median_gap"] <= target + 1e-6]
        out.setdefault("at_target_gap", {})[m] = ({"steps": ok[0]["steps"], "ligands_per_s": ok[0]["ligands_per_s"]}
                                                  if ok else None)
    a = out["at_target_gap"]
    for m in variants:
        if a.get(m) and a.get("plain_f32"):
            out[f"speedup_at_equal_gap_{m}"] = a[m]["ligands_per_s"] / a["plain_f32"]["ligands_per_s"]
    # the same at a fixed median-gap bar of 0.1 kcal/mol (the accuracy bar of the screening comparison)
    for m, rs in rows.items():
        ok = [r for r in rs if r["median_gap"] <= 0.1]
        out.setdefault("at_gap_0.1", {})[m] = ({"steps": ok[0]["steps"], "ligands_per_s": ok[0]["ligands_per_s"]}
                                               if ok else None)
    b = out["at_gap_0.1"]
    for m in ("plain_f16", *variants):
        if b.get(m) and b.get("plain_f32"):
            out[f"speedup_at_gap_0.1_{m}"] = b[m]["ligands_per_s"] / b["plain_f32"]["ligands_per_s"]
    # the same between budgets: steps to a 0.1 median gap by log-log interpolation of the gap between the two
    # budgets that bracket it, ligands/s there by linear interpolation of the time per ligand
    c = out["interp_at_gap_0.1"] = {m: interp_to_gap(rs, 0.1) for m, rs in rows.items()}
    for m in ("plain_f16", *variants):
        if c.get(m) and c.get("plain_f32"):
            out[f"speedup_interp_at_gap_0.1_{m}"] = c[m]["ligands_per_s"] / c["plain_f32"]["ligands_per_s"]
    return out


def full_screen(rec, train_ligs, screen_ligs, variant, device="cuda", chains=32, learned_steps=(400, 600),
                plain_steps=3000, ref_steps=8000, n_sub=1024, train_steps=500, log_cap=4_000_000, epochs=3, seed=0,
                log=None):
    """The full-form screening run: all of ``screen_ligs`` docked in one batch by the learned FP16 search
    (``variant`` as in ``parse_learned``) at each budget of ``learned_steps`` and by the plain FP32 search at
    ``plain_steps``, each timed with CUDA events from Stage A to the end of the MC phase, with the launch variant
    the autotuner picks for the batch (tuned before the timed runs). The median best-energy gap of every run is
    measured on the first ``n_sub`` ligands against a ``ref_steps`` plain FP32 run of that subset (floor: the lowest
    energy any run found for the ligand). At equal gap: the learned budget that reaches the plain run's median gap
    (and the 0.1 kcal/mol bar), interpolated between the learned budgets as in ``interp_to_gap``."""
    from . import params
    dev = torch.device(device)
    v = parse_learned([variant])
    name, (k, frac, tgt, tries, hint, mix) = next(iter(v.items()))
    t_train = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_train[0].record()
    nets, train_rec = train_variants(rec, train_ligs, v.values(), dev, chains=chains, train_steps=train_steps,
                                     log_cap=log_cap, epochs=epochs, seed=seed, log=log)
    t_train[1].record()
    net = nets[(tgt, hint, mix)]
    del nets
    L = len(screen_ligs)
    n_sub = min(n_sub, L)
    prob, kp32 = _problem_for(rec, screen_ligs, dev, "f32")
    kp16 = type(kp32)(prob, grid_dtype="f16")

    def run(kp, steps, learned):
        cfg = params.workload_preset(chains, steps)
        cfg["autotune"] = False
        ev0 = int(kp.evals[0])
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        cl, ci, cur = _starts(prob, kp, cfg, seed + 2)
        ev[1].record()
        best = cur.clone()
        ce, be = torch.zeros(cur.shape[0], device=dev), torch.full((cur.shape[0],), float("inf"), device=dev)
        st = {}
        if learned:
            run_mc_segments(kp, net, cl, ci, cur, ce, best, be, cfg, seed + 3, prop_k=k, prop_frac=frac, stats=st,
                            prop_tries=tries)
        else:
            kp.run_mc(cl, ci, cur, ce, best, be, True, steps, cfg["bfgs_iters"], cfg["mc_temperature"],
                      cfg["mc_amp_pos"], cfg["mc_amp_rot"], seed + 3, 0)
        ev[2].record()
        torch.cuda.synchronize(dev)
        ms = ev[0].elapsed_time(ev[2])
        n_ev = int(kp.evals[0]) - ev0
        row = {"steps": steps, "ms": ms, "stage_a_ms": ev[0].elapsed_time(ev[1]), "ligands_per_s": L / (ms / 1e3),
               "evals_per_s": n_ev / (ev[1].elapsed_time(ev[2]) / 1e3), "evals_per_step": n_ev / (cur.shape[0] * steps),
               "mc_variant": int(getattr(kp, "mc_variant", 0)), **st}
        return _best_per_ligand(be, L, chains), row

    # the launch variant for this batch (autotuner samples on the Stage-A starts, untimed)
    for kp in (kp32, kp16):
        cl, _, cur = _starts(prob, kp, params.workload_preset(chains, 1), seed + 2)
        kp.tune(cl, cur)
    learned = [run(kp16, S, True) for S in sorted(learned_steps)]
    e_p, row_p = run(kp32, plain_steps, False)
    # gap floor on the subset: a long plain FP32 run of its ligands
    prob_s, kp_s = _problem_for(rec, screen_ligs[:n_sub], dev, "f32")
    cfg_r = params.workload_preset(chains, ref_steps)
    cfg_r["autotune"] = False
    cl, ci, cur = _starts(prob_s, kp_s, cfg_r, seed + 4)
    best = cur.clone()
    ce, be = torch.zeros(cur.shape[0], device=dev), torch.full((cur.shape[0],), float("inf"), device=dev)
    kp_s.run_mc(cl, ci, cur, ce, best, be, True, ref_steps, cfg_r["bfgs_iters"], cfg_r["mc_temperature"],
                cfg_r["mc_amp_pos"], cfg_r["mc_amp_rot"], seed + 5, 0)
    e_ref = _best_per_ligand(be, n_sub, chains)
    floor = torch.minimum(e_ref, e_p[:n_sub])
    for e, _ in learned:
        floor = torch.minimum(floor, e[:n_sub])
    for e, row in learned + [(e_p, row_p)]:
        gap = (e[:n_sub] - floor).cpu()
        row.update(median_gap=float(gap.median()), mean_gap=float(gap.mean()))
    torch.cuda.synchronize(dev)
    rows_l = [r for _, r in learned]
    at_plain = interp_to_gap(rows_l, row_p["median_gap"])
    at_bar = interp_to_gap(rows_l, 0.1)
    out = {"ligands": L, "chains": chains, "gap_subset": n_sub, "ref_steps": ref_steps,
           "train_ligands": len(train_ligs), "train": train_rec, "train_ms": t_train[0].elapsed_time(t_train[1]),
           "learned_variant": {"name": name, "prop_k": k, "prop_frac": frac, "target": tgt, "tries": tries,
                               "hint": hint, "n_comp": mix},
           "learned_f16": rows_l, "plain_f32": row_p,
           "learned_at_plain_gap": at_plain, "learned_at_gap_0.1": at_bar}
    if at_plain:
        out["speedup_at_equal_gap"] = at_plain["ligands_per_s"] / row_p["ligands_per_s"]
    return out


def interp_to_gap(rows, gap):
    """Steps and ligands/s at which a method's median gap reaches ``gap``, interpolated between the two budgets
    that bracket it (log gap linear in log steps; time per ligand linear in steps); None if no budget reaches it,
    the first budget itself if it already does."""
    rs = sorted(rows, key=lambda r: r["steps"])
    for lo, hi in zip([None] + rs[:-1], rs):
        if hi["median_gap"] <= gap:
            if lo is None or lo["median_gap"] <= gap or hi["median_gap"] <= 0:
                return {"steps": hi["steps"], "ligands_per_s": hi["ligands_per_s"]}
            f = (math.log(gap) - math.log(lo["median_gap"])) / (math.log(hi["median_gap"]) - math.log(lo["median_gap"]))
            s = math.exp(math.log(lo["steps"]) + f * (math.log(hi["steps"]) - math.log(lo["steps"])))
            w = (s - lo["steps"]) / (hi["steps"] - lo["steps"])
            t = (1 - w) / lo["ligands_per_s"] + w / hi["ligands_per_s"]
            return {"steps": s, "ligands_per_s": 1.0 / t}
    return None


def frac_at(prop_frac, step):
    """The learned-step fraction of the segment that starts at ``step``: a number, or (early, late, until)."""
    if isinstance(prop_frac, (tuple, list)):
        early, late, until = prop_frac
        return float(early if step < until else late)
    return float(prop_frac)


def parse_frac(text):
    """A learned-fraction field of a variant spec: "0.3", or "0.5>0.3@128" for 0.5 before step 128 and 0.3 after."""
    if ">" in text:
        a, rest = text.split(">")
        b, c = rest.split("@")
        return (float(a), float(b), int(c))
    return float(text)


def run_mc_segments(kp, net, chain_lig, chain_id, cur, cur_e, best, best_e, cfg, seed, prop_k=32, init_opt=True,
                    stats=None, prop_frac=0.3, log=None, prop_tries=1):
    """MC with learned proposals: the run is cut into segments of prop_k steps; before each segment the network
    reads every chain's current state and draws prop_k target states per chain around it (adock_prop_sample); a
    step proposes the next of them with probability prop_frac, else it takes the plain random move (and plain MC
    after 8 consecutive rejections of learned proposals). log: the training-data log of run_mc, kept across the
    segments. prop_tries > 1: each learned step draws that many targets, evaluates each once and optimises the
    lowest-energy one. prop_frac may be a schedule (early, late, until): the fraction ``early`` for the segments that
    start before step ``until``, ``late`` after."""
    steps = cfg["mc_steps"]
    pst = torch.zeros(4, dtype=torch.int64, device=kp.device)
    marks = []   # per segment: events before the network launches and before the MC launch
    for sg in range(math.ceil(steps / prop_k)):
        k = min(prop_k, steps - sg * prop_k)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)] if stats is not None else None
        if ev:
            ev[0].record()
        hint = kp.prop_hint(chain_lig, best, best_e) if net.uses_hint and sg > 0 else None
        feat = kp.prop_features(chain_lig, cur, cur_e, hint)
        out = net.forward(feat)
        moves = kp.prop_sample(chain_lig, chain_id, out, cur, k * prop_tries, seed ^ 0x5EEDBA5E, sg, net.n_comp)
        if ev:
            ev[1].record()
            marks.append(ev)
        kp.run_mc(chain_lig, chain_id, cur, cur_e, best, best_e, init_opt and sg == 0, k, cfg["bfgs_iters"],
                  cfg["mc_temperature"], cfg["mc_amp_pos"], cfg["mc_amp_rot"], seed, sg * prop_k, prop=moves,
                  prop_stats=pst, prop_frac=frac_at(prop_frac, sg * prop_k), log=log, prop_tries=prop_tries,
                  hint=hint)
    check_gemm("learned-proposal search")
    if stats is not None:
        p, pa, q, qa = pst.tolist()
        stats.update(prop_steps=p, prop_accepted=pa, plain_steps=q, plain_accepted=qa)
        if marks:
            end = torch.cuda.Event(enable_timing=True)
            end.record()
            end.synchronize()
            net_ms = sum(a.elapsed_time(b) for a, b in marks)
            total = marks[0][0].elapsed_time(end)
            # the network's share of the learned search: features, the three GEMMs with their epilogues, sampling
            stats.update(net_ms=net_ms, mc_segments_ms=total - net_ms, segments=len(marks))
    return pst
