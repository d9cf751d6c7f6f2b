"""CPU oracle for the path-guiding MLP (no counterpart in the reference
renderer): forward pass, the vMF-mixture negative log-likelihood and its
gradient, backpropagation and Adam, in float64 numpy.

TEST INFRASTRUCTURE ONLY: tests/ use it to check the GPU kernels
(bulbit_b200/csrc/guide.cu); nothing in the product imports it.

With bf16=True, weights, input features and hidden activations are rounded to
bfloat16 (round to nearest even) where the GPU rounds them, so the GPU's
results can be compared tightly; with bf16=False it is the exact network.
"""
import math

import numpy as np

N_IN, N_HID, N_OUT, N_LOBES = 80, 64, 40, 8
KAPPA_LOG_MIN, KAPPA_LOG_MAX = -2.0, 7.0

# Parameter offsets: W0 b0 W1 b1 W2 b2 W3 b3, W [out][in].
SHAPES = [(N_HID, N_IN), (N_HID,), (N_HID, N_HID), (N_HID,), (N_HID, N_HID), (N_HID,), (N_OUT, N_HID), (N_OUT,)]
N_PARAMS = sum(int(np.prod(s)) for s in SHAPES)


def unpack(params):
    out, at = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(params[at:at + n], np.float64).reshape(s))
        at += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(p, np.float64).ravel() for p in parts])


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def features(raw, aabb):
    """The 80 inputs of a raw query (p, n, wo, roughness): sin/cos(2^k pi p_a)
    of the position scaled to [0, 1] by aabb, k = 0..11, then n, wo,
    roughness and a constant 1."""
    raw = np.asarray(raw, np.float64)
    lo = np.asarray(aabb[:3], np.float64)
    ext = np.asarray(aabb[3:], np.float64) - lo
    inv = np.where(ext > 0, 1.0 / np.where(ext > 0, ext, 1.0), 0.0)
    pn = (raw[:, 0:3] - lo) * inv
    cols = []
    for a in range(3):
        for k in range(12):
            x = pn[:, a] * (2.0 ** k)
            cols.append(np.sin(math.pi * x))
            cols.append(np.cos(math.pi * x))
    f = np.stack(cols, axis=1)
    return np.concatenate([f, raw[:, 3:6], raw[:, 6:9], raw[:, 9:10], np.ones((raw.shape[0], 1))], axis=1)


def forward(params, x, bf=False):
    """Returns the outputs and the list of layer inputs (for backprop)."""
    W0, b0, W1, b1, W2, b2, W3, b3 = unpack(params)
    q = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    acts = [q(x)]
    h = acts[0]
    for W, b in ((W0, b0), (W1, b1), (W2, b2)):
        h = np.maximum(h @ q(W).T + b, 0.0)
        h = q(h)
        acts.append(h)
    y = h @ q(W3).T + b3
    return y, acts


def mixture(y):
    y = np.asarray(y, np.float64).reshape(-1, N_LOBES, 5)
    logits = y[:, :, 0]
    logw = logits - logits.max(1, keepdims=True)
    logw = logw - np.log(np.exp(logw).sum(1, keepdims=True))
    m = y[:, :, 1:4]
    ln = np.maximum(np.linalg.norm(m, axis=2, keepdims=True), 1e-6)
    mu = m / ln
    r = y[:, :, 4]
    kappa = np.exp(np.clip(r, KAPPA_LOG_MIN, KAPPA_LOG_MAX))
    return logw, mu, kappa, ln, r


def vmf_log_norm(k):
    return np.log(k) - np.log(2 * math.pi) - np.log1p(-np.exp(-2 * k))


def mixture_pdf(y, d):
    logw, mu, kappa, _, _ = mixture(y)
    cos = np.einsum("blk,bk->bl", mu, np.asarray(d, np.float64))
    return np.exp(logw + vmf_log_norm(kappa) + kappa * (cos - 1)).sum(1)


def nll_grad(y, d, w):
    """Per-sample loss -w log q(d) and its gradient w.r.t. the 40 outputs."""
    d = np.asarray(d, np.float64)
    w = np.asarray(w, np.float64)
    logw, mu, kappa, ln, r = mixture(y)
    cos = np.einsum("blk,bk->bl", mu, d)
    lp = logw + vmf_log_norm(kappa) + kappa * (cos - 1)
    mx = lp.max(1, keepdims=True)
    logq = (mx + np.log(np.exp(lp - mx).sum(1, keepdims=True)))[:, 0]
    gamma = np.exp(lp - logq[:, None])
    pi = np.exp(logw)
    g = np.zeros((y.shape[0], N_LOBES, 5))
    g[:, :, 0] = -w[:, None] * (gamma - pi)
    dm = (d[:, None, :] - mu * cos[:, :, None]) * (gamma * kappa / ln[:, :, 0])[:, :, None]
    g[:, :, 1:4] = -w[:, None, None] * dm
    two_k = 2 * kappa
    dlog = 1 - two_k / np.expm1(two_k) + kappa * (cos - 1)
    clamped = (r < KAPPA_LOG_MIN) | (r > KAPPA_LOG_MAX)
    g[:, :, 4] = np.where(clamped, 0.0, -w[:, None] * gamma * dlog)
    return -w * logq, g.reshape(-1, N_OUT)


def gradient(params, raw, dirs, weights, aabb, bf=False):
    """Gradient of sum_i -w_i log q_i(d_i) w.r.t. all parameters, and the sum."""
    W0, b0, W1, b1, W2, b2, W3, b3 = unpack(params)
    q = bf16 if bf else (lambda v: np.asarray(v, np.float64))
    x = features(raw, aabb)
    y, acts = forward(params, x, bf)
    loss, gy = nll_grad(y, dirs, weights)
    if bf:
        gy_q = bf16(gy)
    else:
        gy_q = gy
    grads = [None] * 8
    grads[7] = gy.sum(0)
    grads[6] = gy_q.T @ acts[3]
    dz = (gy_q @ q(W3)) * (acts[3] > 0)
    for li, W in ((2, W2), (1, W1), (0, W0)):
        grads[2 * li + 1] = dz.sum(0)
        dzq = q(dz)
        grads[2 * li] = dzq.T @ acts[li]
        if li > 0:
            dz = (dzq @ q(W)) * (acts[li] > 0)
    return pack(grads), float(loss.sum())


def adam(params, grad, m, v, step, lr, b1=0.9, b2=0.99, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
