"""Guided path tracing on the GPU: one-sample MIS between the neural vMF
guide and the BSDF, measured against the plain path tracer:

* unbiased: the guided image mean agrees with the plain one within their Monte
  Carlo standard errors (4 sigma), with an untrained and a trained guide, and
  at selection probabilities near 0 (BSDF only) and near 1 (guide only);
* training helps: against a high-spp plain reference, the relMSE of the same
  guided estimator is lower with the trained guide than with the untrained one
  (what the learned network gains over the method without it);
* the plain renders are unchanged by the presence of guiding code (the parity
  tests of test_render_gpu.py run without a guide)."""
import numpy as np
import pytest

from bulbit_b200 import lib, scenes

pytestmark = pytest.mark.gpu


def rel_mse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def mean_and_se(film):
    img = film.image()
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    n = film.count.astype(np.float64)
    var = np.maximum(0.0, film.moments[..., 1] - film.moments[..., 0] ** 2) * np.where(n > 1, n / (n - 1), 1)
    se = np.sqrt(np.sum(var / np.maximum(n, 1))) / lum.size
    return float(np.nanmean(lum)), float(se)


@pytest.fixture(scope="module")
def setup():
    scene = scenes.cornell_icosphere(levels=5, width=64, height=64, spp=64, max_bounces=12)
    acc = lib.GpuAccel(scene)
    integ = lib.GpuPathIntegrator(acc, scene)
    return scene, acc, integ


@pytest.fixture(scope="module")
def smooth():
    """The same box with an undisplaced icosphere: interpolated normals and
    tangents stay close to orthogonal, so the BSDF's sampled (f, pdf) agree
    with its f() and PDF() at the world direction."""
    scene = scenes.cornell_icosphere(levels=5, width=64, height=64, spp=64, max_bounces=12, displacement=0.0)
    acc = lib.GpuAccel(scene)
    integ = lib.GpuPathIntegrator(acc, scene)
    return scene, acc, integ


def train(integ, guide, iterations, seed0=200):
    for i in range(iterations):
        integ.render(spp=16, seed=seed0 + i, guide=guide, train=True, wave_paths=1 << 14)


def pixel_stats(film):
    """Per-pixel luminance mean and its standard error."""
    img = film.image()
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    n = film.count.astype(np.float64)
    var = np.maximum(0.0, film.moments[..., 1] - film.moments[..., 0] ** 2) * np.where(n > 1, n / (n - 1), 1)
    return lum, np.sqrt(var / np.maximum(n, 1))


def check_unbiased(plain, film, label):
    """Image mean within 4 standard errors, and per pixel: the mean of z^2
    over pixels (z = difference / combined standard error) near 1, so that
    no bias hides in pixels whose errors cancel in the image mean."""
    mp, sp = mean_and_se(plain)
    mg, sg = mean_and_se(film)
    lp, ep = pixel_stats(plain)
    lg, eg = pixel_stats(film)
    se = np.hypot(ep, eg)
    ok = se > 0
    z2 = float(np.mean(((lg - lp)[ok] / se[ok]) ** 2))
    print(f"{label}: guided mean {mg:.5f} +- {sg:.5f}, plain {mp:.5f} +- {sp:.5f}, per-pixel mean z^2 {z2:.3f}")
    assert abs(mg - mp) <= 4 * np.hypot(sg, sp)
    assert z2 < 1.25


def test_guided_estimator_is_unbiased(setup, smooth):
    """Untrained and trained guide on the displaced icosphere and on the
    smooth one. On the displaced sphere the shading frame (interpolated
    tangent and normal, not orthogonalised, as in the reference) is far from
    orthonormal, and such vertices are traced as by the plain tracer."""
    scene, acc, integ = setup
    plain = integ.render(spp=512, seed=1)
    guide = lib.GpuGuide(acc.bounds(), seed=3)
    check_unbiased(plain, integ.render(spp=512, seed=2, guide=guide), "displaced, untrained")
    train(integ, guide, 200)
    check_unbiased(plain, integ.render(spp=512, seed=3, guide=guide), "displaced, trained")
    scene, acc, integ = smooth
    plain = integ.render(spp=512, seed=1)
    guide = lib.GpuGuide(acc.bounds(), seed=3)
    check_unbiased(plain, integ.render(spp=512, seed=2, guide=guide), "smooth, untrained")
    train(integ, guide, 200)
    check_unbiased(plain, integ.render(spp=512, seed=3, guide=guide), "smooth, trained")


@pytest.mark.parametrize("which,bound", [("setup", 1.0), ("smooth", 0.8)])
def test_training_lowers_relmse(request, which, bound):
    """What the learned network gains over the same estimator without it:
    relMSE against an 8192-spp plain render, trained vs untrained guide. On
    the displaced icosphere most vertices of the sphere are traced unguided
    (skewed shading frames), so the gain there is smaller."""
    scene, acc, integ = request.getfixturevalue(which)
    ref = integ.render(spp=8192, seed=7).image()
    untrained = lib.GpuGuide(acc.bounds(), seed=5)
    trained = lib.GpuGuide(acc.bounds(), seed=5)
    train(integ, trained, 200)
    e_plain, e_untrained, e_trained = [], [], []
    for k in range(5):
        e_plain.append(rel_mse(integ.render(spp=64, seed=50 + k).image(), ref))
        e_untrained.append(rel_mse(integ.render(spp=64, seed=60 + k, guide=untrained).image(), ref))
        e_trained.append(rel_mse(integ.render(spp=64, seed=70 + k, guide=trained).image(), ref))
    p, u, t = np.mean(e_plain), np.mean(e_untrained), np.mean(e_trained)
    print(f"{which} relMSE at 64 spp: plain {p:.4e}, guided untrained {u:.4e}, guided trained {t:.4e} "
          f"(trained/plain {t / p:.3f}, trained/untrained {t / u:.3f})")
    assert t < bound * u


def test_guided_render_is_deterministic_and_graph_safe(setup):
    scene, acc, integ = setup
    guide = lib.GpuGuide(acc.bounds(), seed=9)
    a = integ.render(spp=16, seed=4, guide=guide, path_L=True)
    b = integ.render(spp=16, seed=4, guide=guide, path_L=True, use_graph=False, wave_paths=4096)
    assert np.array_equal(a.path_L, b.path_L)


def test_bsdf_only_selection_reproduces_plain(setup):
    """Selection probability -> 0: the guided code path samples the BSDF and
    weights each sample with the sample's own f and pdf, so it estimates what
    the plain tracer does, displaced shading frames included."""
    scene, acc, integ = setup
    plain = integ.render(spp=512, seed=1)
    guide = lib.GpuGuide(acc.bounds(), seed=3)
    check_unbiased(plain, integ.render(spp=512, seed=2, guide=guide, select=1e-4), "select 1e-4")


def test_guide_only_selection_is_unbiased():
    """Selection probability -> 1 in an all-diffuse box, where the weights
    stay bounded (the vMF mixture covers the whole sphere): the guide alone
    estimates the same image."""
    scene = scenes.cornell_icosphere(levels=4, width=48, height=48, spp=64, max_bounces=12,
                                     sphere_material=scenes.diffuse((0.7, 0.7, 0.7)))
    acc = lib.GpuAccel(scene)
    integ = lib.GpuPathIntegrator(acc, scene)
    plain = integ.render(spp=1024, seed=1)
    guide = lib.GpuGuide(acc.bounds(), seed=3)
    check_unbiased(plain, integ.render(spp=1024, seed=2, guide=guide, select=0.9999), "select 0.9999")

