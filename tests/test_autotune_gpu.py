"""The autotuner (bbg_integrator_autotune, bbg_batch_autotune): it picks a
traversal launch shape (threads per block, stack entries in shared memory)
and a wave size by timing probe renders, caches the choice per scene
signature, and -- since every configuration schedules the same per-path
arithmetic -- changes no result: films and per-path radiance stay
bit-identical under every launch shape and wave size."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu

SHAPES = [(128, 16), (128, 0), (128, 8), (256, 16)]


@pytest.fixture(scope="module")
def setup():
    scene = scenes.cornell_icosphere(levels=5, width=96, height=80, spp=8, max_bounces=8)
    acc = lib.GpuAccel(scene)
    return scene, acc, lib.GpuPathIntegrator(acc, scene)


def test_every_launch_shape_gives_the_same_paths(setup):
    scene, acc, integ = setup
    ref = integ.render(spp=8, seed=3, path_L=True)
    for block, short in SHAPES:
        for wave in (0, 4096 * 8 + 8):
            integ.set_tuning(block, short, wave)
            f = integ.render(spp=8, seed=3, path_L=True)
            assert np.array_equal(f.path_L, ref.path_L), (block, short, wave)
            assert np.array_equal(f.rgb_sum, ref.rgb_sum)
    integ.set_tuning()
    with pytest.raises(lib.BbgError):
        integ.set_tuning(64, 16)


def test_autotune_picks_a_candidate_and_caches_it(setup):
    scene, acc, integ = setup
    t = integ.autotune(spp=8)
    assert (t.block, t.short_stack) in SHAPES
    assert t.wave_paths > 0 and t.probe_ms > 0 and t.from_cache == 0
    again = lib.GpuPathIntegrator(acc, scene).autotune(spp=8)  # an identical scene
    assert again.from_cache == 1 and (again.block, again.short_stack, again.wave_paths) == (
        t.block, t.short_stack, t.wave_paths)
    ref = lib.GpuPathIntegrator(acc, scene).render(spp=8, seed=3, path_L=True)
    assert np.array_equal(integ.render(spp=8, seed=3, path_L=True).path_L, ref.path_L)


def test_batch_autotune(setup):
    scene, acc, integ = setup
    others = []
    for seed, (w, h) in ((3, (32, 24)), (11, (24, 40))):
        s = scenes.cornell_batch_variant(seed)
        s.camera.width, s.camera.height = w, h
        a = lib.GpuAccel(s)
        others.append((a, lib.GpuPathIntegrator(a, s)))
    integs = [integ] + [it for _, it in others]
    b = lib.GpuBatch()
    t = b.autotune(integs, spp=8)
    assert (t.block, t.short_stack) in SHAPES and t.from_cache == 0
    films, _ = b.render(integs, spp=8, path_L=True)
    for f, it in zip(films, integs):
        alone = it.render(spp=8, seed=it.scene.seed, path_L=True)
        assert np.array_equal(f.path_L, alone.path_L)
