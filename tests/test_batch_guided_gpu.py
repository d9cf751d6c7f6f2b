"""Guided batches: bbg_batch_render with one guide per scene. Each bounce
level buckets the guide queries by scene (chunks of 128 queries, padded) and
runs every scene's MLP in one grouped forward launch; with training, each
scene's guide takes Adam steps on that scene's own records of the wave.

Bars:
* fixed guides: each scene's film and every path's radiance equal rendering
  that scene alone with its guide, bit for bit (the grouped forward gives each
  query its own scene's weights and bounds, the single-guide forward's
  arithmetic), with the CUDA graph, without it, and with waves that straddle
  scene boundaries;
* training: every scene's guide changes, each differently, and the trained
  batch's images agree with plain renders of the same scenes within their
  Monte Carlo errors (the estimator stays unbiased);
* a guide for some scenes only, or one guide shared by two scenes, is
  refused, and the batch stays usable."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu


def small(scene, w, h):
    scene.camera.width = w
    scene.camera.height = h
    return scene


@pytest.fixture(scope="module")
def guided_batch():
    out = []
    for seed, (w, h) in zip((2, 0, 1, 11), ((40, 32), (24, 24), (56, 40), (16, 48))):
        out.append(small(scenes.cornell_batch_variant(seed), w, h))
    out.append(small(scenes.readme_sphere(), 64, 36))
    items = []
    for k, s in enumerate(out):
        acc = lib.GpuAccel(s)
        items.append((s, acc, lib.GpuPathIntegrator(acc, s), lib.GpuGuide(acc.bounds(), seed=20 + k)))
    return items


def check_equal(films, items, spp):
    for film, (scene, _, integ, guide) in zip(films, items):
        alone = integ.render(spp=spp, seed=scene.seed, path_L=True, guide=guide)
        assert np.array_equal(film.count, alone.count), scene.name
        assert np.array_equal(film.rgb_sum, alone.rgb_sum), scene.name
        assert np.array_equal(film.moments, alone.moments), scene.name
        assert np.array_equal(film.path_L, alone.path_L), scene.name


def test_guided_batch_equals_individual_guided_renders(guided_batch):
    integs = [it for _, _, it, _ in guided_batch]
    guides = [g for _, _, _, g in guided_batch]
    b = lib.GpuBatch()
    films, stats = b.render(integs, spp=4, path_L=True, guides=guides)
    assert stats.paths == sum(it.scene.camera.width * it.scene.camera.height * 4 for it in integs)
    check_equal(films, guided_batch, 4)
    films, _ = b.render(integs, spp=4, path_L=True, guides=guides)  # the captured graph, replayed
    check_equal(films, guided_batch, 4)
    films, _ = b.render(integs, spp=4, path_L=True, guides=guides, use_graph=False, wave_paths=1000)
    check_equal(films, guided_batch, 4)
    # A batch of one scene.
    films, _ = lib.GpuBatch().render(integs[:1], spp=4, path_L=True, guides=guides[:1])
    check_equal(films, guided_batch[:1], 4)
    # A plain render of the same batch after the guided ones.
    films, _ = b.render(integs, spp=4, path_L=True)
    for film, integ in zip(films, integs):
        alone = integ.render(spp=4, seed=integ.scene.seed, path_L=True)
        assert np.array_equal(film.path_L, alone.path_L), integ.scene.name


def pixel_stats(film):
    img = film.image()
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    n = film.count.astype(np.float64)
    var = np.maximum(0.0, film.moments[..., 1] - film.moments[..., 0] ** 2) * np.where(n > 1, n / (n - 1), 1)
    return lum, np.sqrt(var / np.maximum(n, 1))


def test_guided_batch_training_is_per_scene_and_unbiased():
    scs = [small(scenes.cornell_batch_variant(seed, spp=64), 48, 48) for seed in (3, 5, 8)]
    accs = [lib.GpuAccel(s) for s in scs]
    integs = [lib.GpuPathIntegrator(a, s) for a, s in zip(accs, scs)]
    guides = [lib.GpuGuide(a.bounds(), seed=7) for a in accs]  # the same start for all
    start = guides[0].params()
    b = lib.GpuBatch()
    for it in range(6):
        b.render(integs, spp=16, seeds=[100 + it] * 3, guides=guides, train=True, batch=4096, steps=2,
                 wave_paths=1 << 15)
    after = [g.params() for g in guides]
    for k, p in enumerate(after):
        assert np.all(np.isfinite(p)) and not np.array_equal(p, start), k
    assert not np.array_equal(after[0], after[1]) and not np.array_equal(after[1], after[2])
    guided, _ = b.render(integs, spp=256, seeds=[7] * 3, guides=guides)
    for film, integ in zip(guided, integs):
        plain = integ.render(spp=256, seed=8)
        lp, ep = pixel_stats(plain)
        lg, eg = pixel_stats(film)
        se = np.hypot(ep, eg)
        ok = se > 0
        z2 = float(np.mean(((lg - lp)[ok] / se[ok]) ** 2))
        d = float(np.nanmean(lg) - np.nanmean(lp))
        sd = float(np.sqrt(np.sum(se[ok] ** 2)) / lg.size)
        print(integ.scene.name, "mean diff", d, "se", sd, "per-pixel z^2", z2)
        assert abs(d) <= 4 * sd and z2 < 1.3, integ.scene.name


def test_guided_batch_rejects_partial_or_shared_guides(guided_batch):
    integs = [it for _, _, it, _ in guided_batch[:3]]
    guides = [g for _, _, _, g in guided_batch[:3]]
    b = lib.GpuBatch()
    n = len(integs)
    ints = (lib.C.c_void_p * n)(*[it.h.value for it in integs])
    cams = (abi.Camera * n)(*[lib.camera(it.scene.camera) for it in integs])
    films = [lib.Film(c.width, c.height, 2) for c in cams]
    fstructs = (abi.Film * n)(*[f.struct() for f in films])

    def call(guide_list):
        params = (abi.RenderParams * n)()
        for i in range(n):
            params[i].spp = 2
            params[i].seed = i
            params[i].guide = guide_list[i].h if guide_list[i] is not None else None
        stats = abi.RenderStats()
        return lib.get_lib().bbg_batch_render(b.h, n, ints, cams, params, fstructs, abi.BBG_MEM_HOST,
                                              lib.C.byref(stats))

    assert call([guides[0], None, guides[2]]) == abi.BBG_ERR_INVALID_ARG
    assert call([guides[0], guides[1], guides[0]]) == abi.BBG_ERR_INVALID_ARG
    assert call(guides) == abi.BBG_OK
