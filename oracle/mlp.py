"""ORACLE — test infrastructure only.

numpy restatement of the learned schedule selector's model and loss, used to
check the gradients computed by the CUDA forward/backward kernels
(b2p_selector_grad).  Parameter layout: W1[64][11], b1[64], W2[64][64],
b2[64], W3[48][64], b3[48], concatenated.
"""
import numpy as np

F, H, C = 11, 64, 48


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((H, F), (H,), (H, H), (H,), (C, H), (C,)):
        k = int(np.prod(shape))
        out.append(p[o:o + k].reshape(shape))
        o += k
    return out


def loss_and_grad(params, X, T, ce_weight):
    """Mean over samples of  sum_c p_c t_c / t_min  - ce_weight log p_best,
    softmax over the configurations with finite time."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    m = X.shape[0]
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    z = h2 @ W3.T + b3
    valid = np.isfinite(T)
    zm = np.where(valid, z, -np.inf)
    zmax = zm.max(axis=1, keepdims=True)
    e = np.where(valid, np.exp(z - zmax), 0.0)
    p = e / e.sum(axis=1, keepdims=True)
    tmin = np.where(valid, T, np.inf).min(axis=1, keepdims=True)
    r = np.where(valid, T / tmin, 0.0)
    er = (p * r).sum(axis=1, keepdims=True)
    best = np.argmin(np.where(valid, T, np.inf), axis=1)
    onehot = np.zeros_like(p)
    onehot[np.arange(m), best] = 1.0
    pbest = p[np.arange(m), best]
    loss = float(np.mean(er[:, 0] - ce_weight * np.log(np.maximum(pbest, 1e-30))))
    dz = np.where(valid, p * (r - er) + ce_weight * (p - onehot), 0.0) / m
    gW3 = dz.T @ h2
    gb3 = dz.sum(axis=0)
    dh2 = (dz @ W3) * (a2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(axis=0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    gW1 = dh1.T @ X
    gb1 = dh1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def predict(params, X, masks):
    W1, b1, W2, b2, W3, b3 = unpack(params)
    h1 = np.maximum(np.asarray(X, np.float64) @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    z = h2 @ W3.T + b3
    z = np.where(masks, z, -np.inf)
    return np.argmax(z, axis=1)
