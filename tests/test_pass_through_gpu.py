"""The pass-through drain's failure path. Paths that cross material-less
surfaces count no bounce (PathIntegrator::Li, src/integrator/path_integrator.cpp:95-100),
so they can outlive a wave's max_bounces + 1 levels; the renderer traces them
on level by level, host-driven and bounded (bbg_render_params.pass_through_levels,
default 4096), and returns BBG_ERR_TIMEOUT when the bound is reached. The
failure is made on the host: a scene of nested material-less spheres around
the camera with the bound lowered below the number of surfaces a camera ray
crosses. No kernel waits on anything, so nothing on the GPU can hang; the
integrator stays usable and the same scene renders under the default bound,
with per-path radiance equal to the reference's."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu


def nested_shells_scene(n_shells=6):
    scene = scenes.cornell_icosphere(levels=1, width=24, height=24, spp=2, max_bounces=1)
    cam = np.array(scene.camera.position[:], np.float32)
    shells = []
    for k in range(n_shells):
        s = abi.Sphere()
        s.p[:] = cam.tolist()
        s.q[:] = [0, 0, 0, 1]
        s.s[:] = [1, 1, 1]
        s.radius = 0.05 + 0.04 * k
        shells.append(s)
    scene.spheres = shells
    scene.prim_kind = np.concatenate([scene.prim_kind, np.ones(n_shells, np.int32)]).astype(np.int32)
    scene.prim_index = np.concatenate([scene.prim_index, np.arange(n_shells)]).astype(np.int32)
    scene.prim_material = np.concatenate([scene.prim_material, -np.ones(n_shells, np.int32)]).astype(np.int32)
    return scene


def test_pass_through_bound_reports_timeout(oracle):
    scene = nested_shells_scene()
    acc = lib.GpuAccel(scene)
    integ = lib.GpuPathIntegrator(acc, scene)
    # Every camera ray leaves through six shells before it reaches a wall:
    # more pass-through levels than a bound of 2 allows.
    with pytest.raises(lib.BbgError) as e:
        integ.render(pass_through_levels=2)
    assert e.value.status == abi.BBG_ERR_TIMEOUT
    assert b"pass-through" in lib.get_lib().bbg_last_error()
    # The handle and the device context stay usable: the default bound lets
    # the paths finish, and they match the reference path for path.
    film = integ.render(path_L=True)
    rs = oracle.RefScene(scene)
    rs.make_integrator()
    ref_L, _ = rs.trace_paths()
    num = np.abs(film.path_L.astype(np.float64) - ref_L).max(axis=1)
    den = np.abs(ref_L.astype(np.float64)).max(axis=1)
    err = np.where(num == 0, 0.0, num / np.maximum(den, 1e-30))
    assert (err <= 1e-4).mean() >= 0.999
    assert film.stats.closest_rays >= 24 * 24 * 2 * 7
