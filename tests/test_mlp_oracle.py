"""Pins the path-guiding MLP's CPU oracle (oracle/mlp_ref.py) before the GPU
kernels are checked against it: its analytic parameter gradient of the vMF-mixture
negative log-likelihood agrees with central finite differences, its mixture
density integrates to 1 over the sphere, and Adam reduces to the published
update (Kingma & Ba, 2015)."""
import numpy as np

from oracle import mlp_ref

AABB = np.array([-1, -1, -1, 1, 1, 1], np.float64)


def batch(n, seed):
    rng = np.random.default_rng(seed)
    raw = np.concatenate([rng.uniform(-1, 1, (n, 3)), rng.normal(size=(n, 6)), rng.uniform(0, 1, (n, 1))], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return raw, d, rng.uniform(0.5, 1.5, n)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(size=mlp_ref.N_PARAMS) * 0.1
    raw, d, w = batch(8, 1)
    g, _ = mlp_ref.gradient(p, raw, d, w, AABB)
    for i in rng.choice(mlp_ref.N_PARAMS, 40, replace=False):
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        fd = (mlp_ref.gradient(pp, raw, d, w, AABB)[1] - mlp_ref.gradient(pm, raw, d, w, AABB)[1]) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_mixture_density_normalised():
    rng = np.random.default_rng(2)
    y = rng.normal(size=(3, mlp_ref.N_OUT))
    # Midpoint rule on a fine (theta, phi) grid.
    nt, nphi = 400, 800
    th = (np.arange(nt) + 0.5) * np.pi / nt
    ph = (np.arange(nphi) + 0.5) * 2 * np.pi / nphi
    T, P = np.meshgrid(th, ph, indexing="ij")
    dirs = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    dA = (np.pi / nt) * (2 * np.pi / nphi) * np.sin(T).ravel()
    for k in range(3):
        pdf = mlp_ref.mixture_pdf(np.repeat(y[k:k + 1], len(dirs), 0), dirs)
        assert abs((pdf * dA).sum() - 1.0) < 2e-3


def test_adam_first_step():
    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.3, -0.1, 0.0])
    p1, m, v = mlp_ref.adam(p, g, np.zeros(3), np.zeros(3), 1, 0.01)
    # First step: m_hat = g, v_hat = g^2, so each moves by lr * sign(g).
    assert np.allclose(p1, p - 0.01 * g / (np.abs(g) + 1e-8))
