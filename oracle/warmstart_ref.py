"""CPU (NumPy FP64) restatement of the learned warm-start network's forward and
backward passes -- TEST INFRASTRUCTURE ONLY: the checker for the device kernels
(mstm_b200/csrc/warmstart.cu composed by mstm_b200/warmstart.py).  Only tests/
use it.  MSTM has no such network; this file restates the project's own
definition (encoder, three message-passing layers with residual node updates,
linear head, masked mean-square loss) so the device gradients can be checked.
"""
import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_d(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(P, X, ef, dst, src, target, mask, layers=3):
    """P: dict name -> float64 array (shapes as WarmStartNet).  Returns (loss, grads)."""
    G = {k: np.zeros_like(v) for k, v in P.items()}
    Nn = X.shape[0]
    Z0 = X @ P["enc_w"] + P["enc_b"]
    h = silu(Z0)
    cache = []
    for t in range(layers):
        Ze = np.concatenate([h[dst], h[src], ef], axis=1)
        Zm = Ze @ P[f"m{t}_w"] + P[f"m{t}_b"]
        M = silu(Zm)
        agg = np.zeros((Nn, M.shape[1]))
        np.add.at(agg, dst, M)
        Zu = h @ P[f"u{t}_w1"] + agg @ P[f"u{t}_w2"] + P[f"u{t}_b"]
        cache.append((h, Ze, Zm, agg, Zu))
        h = h + silu(Zu)
    y = h @ P["out_w"] + P["out_b"]
    msum = mask.sum()
    d = (y - target) * mask
    loss = (d * d).sum() / msum
    dy = 2.0 * d / msum
    G["out_w"] = h.T @ dy
    G["out_b"] = dy.sum(axis=0)
    dh = dy @ P["out_w"].T
    H = P["enc_b"].shape[0]
    for t in reversed(range(layers)):
        h_t, Ze, Zm, agg, Zu = cache[t]
        dZu = dh * silu_d(Zu)
        G[f"u{t}_b"] = dZu.sum(axis=0)
        G[f"u{t}_w1"] = h_t.T @ dZu
        G[f"u{t}_w2"] = agg.T @ dZu
        dh_t = dh + dZu @ P[f"u{t}_w1"].T
        dagg = dZu @ P[f"u{t}_w2"].T
        dM = dagg[dst]
        dZm = dM * silu_d(Zm)
        G[f"m{t}_b"] = dZm.sum(axis=0)
        G[f"m{t}_w"] = Ze.T @ dZm
        dZe = dZm @ P[f"m{t}_w"].T
        np.add.at(dh_t, dst, dZe[:, :H])
        np.add.at(dh_t, src, dZe[:, H:2 * H])
        dh = dh_t
    dZ0 = dh * silu_d(Z0)
    G["enc_b"] = dZ0.sum(axis=0)
    G["enc_w"] = X.T @ dZ0
    return loss, G


def knn(pos, k):
    """k nearest neighbours (ties by index) of every point."""
    d = ((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d, np.inf)
    return np.argsort(d, axis=1, kind="stable")[:, :k]
