"""The path-guiding MLP's GPU kernels (bulbit_b200/csrc/guide.cu) against the
float64 CPU oracle (oracle/mlp_ref.py): forward outputs, parameter gradients
of the vMF-mixture negative log-likelihood, the Adam update, and that online
training fits a known directional distribution.

Tolerances: BF16 weights and activations with FP32 accumulation. Against the
oracle with the same BF16 roundings: outputs within 1e-2 absolute, gradients
within 3 % relative L2 per layer. Against the exact float64 network: outputs
within 5e-2, gradients cosine similarity >= 0.99."""
import numpy as np
import pytest

from bulbit_b200 import lib
from oracle import mlp_ref

pytestmark = pytest.mark.gpu

AABB = np.array([-1, -1, -1, 1, 1, 1], np.float32)
LAYERS = ["W0", "b0", "W1", "b1", "W2", "b2", "W3", "b3"]


def random_batch(n, seed):
    rng = np.random.default_rng(seed)
    raw = np.zeros((n, 10), np.float32)
    raw[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    nrm = rng.normal(size=(n, 3))
    raw[:, 3:6] = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    raw[:, 6:9] = wo / np.linalg.norm(wo, axis=1, keepdims=True)
    raw[:, 9] = rng.uniform(0, 1, n)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    w = rng.uniform(0.1, 2.0, n).astype(np.float32)
    return raw, d, w


def trained_params(g):
    """Parameters with non-trivial output weights (the initial output layer is
    near zero), so every layer's gradient is exercised."""
    p = g.params().astype(np.float64)
    rng = np.random.default_rng(3)
    at = mlp_ref.N_PARAMS - 40 - 40 * 64
    p[at:at + 40 * 64] = rng.uniform(-0.3, 0.3, 40 * 64)
    return p.astype(np.float32)


def test_forward_matches_oracle():
    g = lib.GpuGuide(AABB, seed=7)
    p = trained_params(g)
    g.set_params(p)
    raw, _, _ = random_batch(1000, 1)
    out = g.forward(raw)
    x = mlp_ref.features(raw, AABB)
    y_bf, _ = mlp_ref.forward(p, x, bf=True)
    y, _ = mlp_ref.forward(p, x, bf=False)
    assert np.abs(out - y_bf).max() < 1e-2
    assert np.abs(out - y).max() < 5e-2


def test_gradient_matches_oracle():
    g = lib.GpuGuide(AABB, seed=7)
    p = trained_params(g)
    g.set_params(p)
    raw, d, w = random_batch(4096, 2)
    grad, loss = g.gradient(raw, d, w)
    ref_bf, loss_bf = mlp_ref.gradient(p, raw, d, w, AABB, bf=True)
    ref, _ = mlp_ref.gradient(p, raw, d, w, AABB, bf=False)
    assert abs(loss - loss_bf) / abs(loss_bf) < 1e-3
    at = 0
    for name, shape in zip(LAYERS, mlp_ref.SHAPES):
        k = int(np.prod(shape))
        a, b, c = grad[at:at + k], ref_bf[at:at + k], ref[at:at + k]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = float(a @ c / (np.linalg.norm(a) * np.linalg.norm(c) + 1e-30))
        print(f"{name}: rel L2 vs bf16 oracle {rel:.2e}, cosine vs float64 oracle {cos:.5f}")
        assert rel < 3e-2, name
        assert cos > 0.99, name
        at += k


def test_adam_step_matches_oracle():
    g = lib.GpuGuide(AABB, seed=9)
    raw, d, w = random_batch(2048, 4)
    p0 = g.params().astype(np.float64)
    grad, _ = g.gradient(raw, d, w)
    g.train_step(raw, d, w, lr=1e-2)
    p1 = g.params()
    ref, _, _ = mlp_ref.adam(p0, grad.astype(np.float64) / len(raw), np.zeros_like(p0), np.zeros_like(p0), 1, 1e-2)
    assert np.abs(p1 - ref).max() < 1e-5


def test_training_fits_a_directional_distribution():
    """Samples whose directions cluster around a position-dependent axis:
    the mean negative log-likelihood must fall well below that of the
    initial broad mixture."""
    g = lib.GpuGuide(AABB, seed=11)
    rng = np.random.default_rng(5)
    losses = []
    for it in range(300):
        raw, _, _ = random_batch(1 << 14, 100 + it)
        axis = np.stack([np.sign(raw[:, 0]), 0.5 * np.ones(len(raw)), np.sign(raw[:, 2])], 1)
        axis /= np.linalg.norm(axis, axis=1, keepdims=True)
        d = axis + 0.15 * rng.normal(size=axis.shape)
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        losses.append(g.train_step(raw, d, np.ones(len(raw), np.float32), lr=1e-2))
    print("loss first/last", losses[0], np.mean(losses[-10:]))
    assert np.mean(losses[-10:]) < losses[0] - 2.0


def test_mixture_sampling_matches_its_density():
    """Directions the device draws from a vMF mixture follow the density it
    evaluates: on 800 equal-area bins of the sphere, observed counts agree
    with the oracle density's integral within Poisson noise (|z| < 6); the
    returned pdf matches the oracle's density at the sampled direction."""
    rng = np.random.default_rng(8)
    y = rng.normal(size=(1, 40)).astype(np.float32)
    y[0, 4::5] = rng.uniform(-1, 4, 8)  # log kappa: kappas from 0.4 to 55
    n = 1 << 21
    outs = np.repeat(y, n, 0)
    d, pdf = lib.mixture_sample(outs, rng.uniform(0, 1, (n, 3)).astype(np.float32))
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-5)
    ref_pdf = mlp_ref.mixture_pdf(outs[:4096].astype(np.float64), d[:4096].astype(np.float64))
    assert np.allclose(pdf[:4096], ref_pdf, rtol=2e-3, atol=1e-6)
    assert np.allclose(lib.mixture_pdf(outs[:4096], d[:4096]), pdf[:4096])
    nz, nphi = 20, 40
    zi = np.clip(((d[:, 2] + 1) / 2 * nz).astype(int), 0, nz - 1)
    pi_ = np.clip(((np.arctan2(d[:, 1], d[:, 0]) + np.pi) / (2 * np.pi) * nphi).astype(int), 0, nphi - 1)
    counts = np.bincount(zi * nphi + pi_, minlength=nz * nphi)
    sub = 16  # midpoint rule, 16 x 16 points per bin
    zz = -1 + (np.arange(nz * sub) + 0.5) * 2 / (nz * sub)
    pp = -np.pi + (np.arange(nphi * sub) + 0.5) * 2 * np.pi / (nphi * sub)
    Z, PH = np.meshgrid(zz, pp, indexing="ij")
    R = np.sqrt(1 - Z ** 2)
    dirs = np.stack([R * np.cos(PH), R * np.sin(PH), Z], -1).reshape(-1, 3)
    dens = mlp_ref.mixture_pdf(np.repeat(y.astype(np.float64), len(dirs), 0), dirs)
    area = (2 / (nz * sub)) * (2 * np.pi / (nphi * sub))
    expect = dens.reshape(nz, sub, nphi, sub).sum(axis=(1, 3)) * area * n
    z = (counts.reshape(nz, nphi) - expect) / np.sqrt(np.maximum(expect, 1))
    assert abs(expect.sum() / n - 1) < 1e-3
    assert np.abs(z).max() < 6
