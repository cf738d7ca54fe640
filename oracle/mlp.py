"""Float64 restatement of the proposal network's forward pass, Gaussian NLL and backward pass (numpy).

TEST INFRASTRUCTURE ONLY: the gradient oracle for the library's BF16 tensor-core kernels (tests/). The network
has no reference counterpart; this is the project's own CPU restatement of adock_b200/proposal.py.

out = SiLU(SiLU(x W1 + b1) W2 + b2) W3 + b3; means = out[:, 0:26], log sd = clip(out[:, 32:58], -4, 2);
loss = mean over rows of sum over active dims (translation, rotation, torsions < count) of
0.5 ((y - mean) / sd)^2 + log sd (clipped entries pass no gradient to the log sd).
n_comp = 3: the translation term is -log sum_k softmax(logits)_k N(y_t | mean_k, sd) + const, with means at
columns 0, 27, 58, logits at 26, 30, 61 and the per-axis sd of columns 32-34.
"""
import numpy as np


def _silu(a):
    return a / (1.0 + np.exp(-a))


def _dsilu(a):
    s = 1.0 / (1.0 + np.exp(-a))
    return s * (1.0 + a * (1.0 - s))


MIX_MEAN = (0, 27, 58)
MIX_LOGIT = (26, 30, 61)


def _lse(a, axis):
    m = a.max(axis, keepdims=True)
    return (m + np.log(np.exp(a - m).sum(axis, keepdims=True))).squeeze(axis)


def loss_and_grads(W, b, X, Y, n_comp=1):
    """W: 3 arrays [K, N]; b: 3 arrays [N]; X [B, 320]; Y [B, 32]. Returns (loss, [dW1, dW2, dW3, db1, db2, db3])."""
    W = [np.asarray(w, np.float64) for w in W]
    b = [np.asarray(v, np.float64) for v in b]
    X = np.asarray(X, np.float64)
    Y = np.asarray(Y, np.float64)
    B = X.shape[0]
    a1 = X @ W[0] + b[0]
    h1 = _silu(a1)
    a2 = h1 @ W[1] + b[1]
    h2 = _silu(a2)
    out = h2 @ W[2] + b[2]
    nt = Y[:, 26].astype(int)
    d = np.arange(26)
    active = (d[None, :] < 6) | (d[None, :] - 6 < nt[:, None])
    mu, ls_raw = out[:, :26], out[:, 32:58]
    ls = np.clip(ls_raw, -4.0, 2.0)
    z = (Y[:, :26] - mu) * np.exp(-ls)
    loss = float(np.sum(np.where(active, 0.5 * z * z + ls, 0.0)) / B)
    dout = np.zeros_like(out)
    dout[:, :26] = np.where(active, -z * np.exp(-ls), 0.0) / B
    inside = (ls_raw > -4.0) & (ls_raw < 2.0)
    dout[:, 32:58] = np.where(active & inside, 1.0 - z * z, 0.0) / B
    if n_comp == 3:
        # the translation columns of the single-Gaussian term are replaced by the mixture
        loss -= float(np.sum(0.5 * z[:, :3] ** 2 + ls[:, :3]) / B)
        dout[:, :3] = 0.0
        isd = np.exp(-ls[:, :3])                                              # [B, 3]
        mu_k = np.stack([out[:, c:c + 3] for c in MIX_MEAN], 1)               # [B, K, 3]
        lg = out[:, list(MIX_LOGIT)]                                          # [B, K]
        zk = (Y[:, None, :3] - mu_k) * isd[:, None, :]
        lp = lg - 0.5 * (zk ** 2).sum(2)
        lse_g, lse_p = _lse(lg, 1), _lse(lp, 1)
        loss += float(np.sum(lse_g - lse_p + ls[:, :3].sum(1)) / B)
        r = np.exp(lp - lse_p[:, None])
        p = np.exp(lg - lse_g[:, None])
        for k, (cm, cl) in enumerate(zip(MIX_MEAN, MIX_LOGIT)):
            dout[:, cl] = (p[:, k] - r[:, k]) / B
            dout[:, cm:cm + 3] = -r[:, k, None] * zk[:, k] * isd / B
        dls = (r[:, :, None] * (1.0 - zk ** 2)).sum(1)
        dout[:, 32:35] = np.where(inside[:, :3], dls, 0.0) / B
    dW3, db3 = h2.T @ dout, dout.sum(0)
    dA2 = (dout @ W[2].T) * _dsilu(a2)
    dW2, db2 = h1.T @ dA2, dA2.sum(0)
    dA1 = (dA2 @ W[1].T) * _dsilu(a1)
    dW1, db1 = X.T @ dA1, dA1.sum(0)
    return loss, [dW1, dW2, dW3, db1, db2, db3]
