"""Several scenes rendered in one batch (bbg_batch_render): every stage runs
once per bounce level over the paths of all scenes. Each path keeps its
scene's sampler stream and arithmetic, so each scene's film and every
path's radiance must equal rendering that scene alone, bit for bit: with
uneven sizes, mixed materials and primitive kinds, waves that straddle
scene boundaries, and with or without the CUDA graph."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu


def small(scene, w, h):
    scene.camera.width = w
    scene.camera.height = h
    return scene


@pytest.fixture(scope="module")
def batch_scenes():
    out = []
    for seed, (w, h) in zip((2, 0, 1, 11), ((40, 32), (24, 24), (56, 40), (16, 48))):
        s = scenes.cornell_batch_variant(seed)
        out.append(small(s, w, h))
    out.append(small(scenes.readme_sphere(), 64, 36))  # spheres, spot and infinite light
    items = []
    for s in out:
        acc = lib.GpuAccel(s)
        items.append((s, acc, lib.GpuPathIntegrator(acc, s)))
    return items


def check_equal(batch_films, integs, spp, wave_paths=0):
    for film, integ in zip(batch_films, integs):
        alone = integ.render(spp=spp, seed=integ.scene.seed, path_L=True, wave_paths=wave_paths)
        assert np.array_equal(film.count, alone.count), integ.scene.name
        assert np.array_equal(film.rgb_sum, alone.rgb_sum), integ.scene.name
        assert np.array_equal(film.moments, alone.moments), integ.scene.name
        assert np.array_equal(film.path_L, alone.path_L), integ.scene.name


def test_batch_equals_individual_renders(batch_scenes):
    integs = [it for _, _, it in batch_scenes]
    b = lib.GpuBatch()
    films, stats = b.render(integs, spp=4, path_L=True)
    assert stats.paths == sum(it.scene.camera.width * it.scene.camera.height * 4 for it in integs)
    check_equal(films, integs, 4)
    # Twice more: the captured graph is replayed; then without the graph and
    # with waves of 1000 paths, which straddle scene boundaries.
    films, _ = b.render(integs, spp=4, path_L=True)
    check_equal(films, integs, 4)
    films, _ = b.render(integs, spp=4, path_L=True, use_graph=False, wave_paths=1000)
    check_equal(films, integs, 4)


def test_batch_rejects_what_it_cannot_render(batch_scenes):
    integs = [it for _, _, it in batch_scenes[:2]]
    b = lib.GpuBatch()
    with pytest.raises(lib.BbgError) as e:
        b.render(integs, spp=[4, 8])
    assert e.value.status == abi.BBG_ERR_INVALID_ARG
    acc = batch_scenes[0][1]
    acc.set_traversal(abi.BBG_TRAVERSAL_REFERENCE)
    try:
        with pytest.raises(lib.BbgError) as e:
            b.render(integs, spp=4)
        assert e.value.status == abi.BBG_ERR_UNSUPPORTED
    finally:
        acc.set_traversal(abi.BBG_TRAVERSAL_WIDE)
    films, _ = b.render(integs, spp=2)  # still usable after the rejections
    assert all(f.count.sum() > 0 for f in films)
