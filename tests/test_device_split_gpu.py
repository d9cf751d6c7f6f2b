"""The SAH tree over references split on the device
(bbg_accel_create_device_split, bulbit_b200/csrc/split_build.cu): early split
clipping in rounds on the device, then the device SAH build over the
references. Checked: a budget of 0 gives the device SAH tree itself (node for
node); the build is deterministic; every triangle is covered by the leaf boxes
of its references (sampled points of every triangle); closest hits agree with
the reference BVH (src/accel/bvh.cpp:299-332) except near-ties, any-hit
agrees, in both layouts; per-path radiance over it agrees with
PathIntegrator::Li (src/integrator/path_integrator.cpp:26-196)."""
import time

import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes
from test_render_gpu import check_paths
from test_trace_gpu import classify_against_brute_force

pytestmark = pytest.mark.gpu


def leaf_boxes_cover_triangles(scene, nodes, slots, grid=6):
    """True where every sampled point (barycentric grid with the corners and
    edges) of every triangle lies in the box of one of the leaves holding it."""
    leaf = nodes["count"] > 0
    first = nodes["offset"][leaf].astype(np.int64)
    count = nodes["count"][leaf].astype(np.int64)
    slot_leaf = np.repeat(np.arange(int(leaf.sum())), count)
    slot_idx = np.concatenate([np.arange(f, f + c) for f, c in zip(first, count)])
    prim = slots[slot_idx]
    lo = nodes["bmin"][leaf][slot_leaf].astype(np.float64)
    hi = nodes["bmax"][leaf][slot_leaf].astype(np.float64)
    tri = scene.tri_indices[scene.prim_index[prim]]
    p = scene.positions.astype(np.float64)
    a, b, c = p[tri[:, 0]], p[tri[:, 1]], p[tri[:, 2]]
    us, vs = np.meshgrid(np.linspace(0, 1, grid), np.linspace(0, 1, grid))
    keep = us + vs <= 1 + 1e-12
    us, vs = us[keep], vs[keep]
    pts = a[:, None, :] + us[None, :, None] * (b - a)[:, None, :] + vs[None, :, None] * (c - a)[:, None, :]
    inside = ((pts >= lo[:, None, :]) & (pts <= hi[:, None, :])).all(axis=2)  # (slots, samples)
    covered = np.zeros((scene.n_prims, len(us)), bool)
    np.logical_or.at(covered, prim, inside)
    return covered


@pytest.mark.parametrize("name,make", [
    ("cornell_ico4", lambda: scenes.cornell_icosphere(levels=4, width=8, height=8)),
    ("soup200k", lambda: scenes.triangle_soup(200_000, seed=5)),
])
def test_budget_zero_is_the_device_sah_tree(name, make):
    scene = make()
    a = lib.GpuAccel(scene, device_sah=True)
    b = lib.GpuAccel(scene, device_sah=True, split=0.0)
    na, sa = a.export()
    nb, sb = b.export()
    assert np.array_equal(na.view(np.uint8), nb.view(np.uint8))
    assert np.array_equal(sa, sb)
    a.close()
    b.close()


def test_deterministic_and_covering():
    scene = scenes.cornell_icosphere(levels=3, width=8, height=8)
    a = lib.GpuAccel(scene, device_sah=True, split=8.0)
    b = lib.GpuAccel(scene, device_sah=True, split=8.0)
    na, sa = a.export()
    nb, sb = b.export()
    assert np.array_equal(na.view(np.uint8), nb.view(np.uint8)) and np.array_equal(sa, sb)
    n = scene.n_prims
    counts = np.bincount(sa, minlength=n)
    print(f"cornell_ico3: {n} primitives, {len(sa)} references (budget {8 * n}), most split: {counts.max()}")
    assert len(sa) > n and len(sa) <= n * 9
    assert counts.min() >= 1  # every primitive is in the tree
    # The box walls are split first: their wasted area dwarfs the sphere's.
    assert counts[:12].min() > 10 * np.median(counts[14:])
    covered = leaf_boxes_cover_triangles(scene, na, sa)
    assert covered.all(), np.argwhere(~covered)[:5]
    a.close()
    b.close()


def test_device_split_tree_parity(oracle):
    cornell = scenes.cornell_icosphere(levels=6, width=8, height=8)
    rng = np.random.default_rng(9)
    n = 200_000
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = rng.uniform(-0.95, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 6], rays[:, 7] = 1e-4, np.inf
    anyq = rays.copy()
    anyq[:, 7] = rng.uniform(0.05, 2.0, n).astype(np.float32)
    soup = scenes.triangle_soup(100_000, seed=5)
    srays, sany = scenes.soup_rays(1 << 18, seed=6)
    for scene, cl, an in ((cornell, rays, anyq), (soup, srays, sany)):
        rs = oracle.RefScene(scene)
        acc = lib.GpuAccel(scene, device_sah=True, split=3.0)
        ref_prim, ref_t, _ = rs.intersect(cl)
        ref_occ, _ = rs.intersect_any(an)
        for mode in (abi.BBG_TRAVERSAL_WIDE, abi.BBG_TRAVERSAL_ORDERED):
            acc.set_traversal(mode)
            prim, t, _, _ = acc.intersect(cl)
            ties, leaks_ref, leaks_dev, unexplained = classify_against_brute_force(rs, cl, prim, t, ref_prim, ref_t)
            print(f"device split tree, {scene.name}: {ties} near-ties, {leaks_ref} + {leaks_dev} leaks")
            assert not unexplained, unexplained[:5]
            assert leaks_ref + leaks_dev <= 1e-3 * len(cl)
            same = (prim == ref_prim) & (ref_prim >= 0)
            assert np.array_equal(t[same].view(np.uint32), ref_t[same].view(np.uint32))
            assert np.array_equal(acc.intersect_any(an), ref_occ)
        acc.close()


def test_device_split_tree_paths(oracle):
    scene = scenes.cornell_icosphere(levels=4, width=48, height=48, spp=8, max_bounces=16)
    rs = oracle.RefScene(scene)
    rs.make_integrator()
    scene.positions, scene.normals, scene.tangents, scene.uvs = rs.mesh_arrays()
    acc = lib.GpuAccel(scene, device_sah=True, split=3.0)
    integ = lib.GpuPathIntegrator(acc, scene)
    film = integ.render(path_L=True)
    ref_L, _ = rs.trace_paths()
    check_paths("cornell, device split tree", film.path_L, ref_L)


def test_full_cornell_device_split_build():
    """The 1,310,734-triangle Cornell scene at budget 3: references, build time,
    and a frame over the tree equal to one over the reference tree within the
    Monte Carlo noise (same sampler streams: the films differ only where a
    path met a near-tie)."""
    scene = scenes.cornell_icosphere(levels=8, width=128, height=128, spp=16, max_bounces=16)
    t0 = time.perf_counter()
    acc = lib.GpuAccel(scene, device_sah=True, split=3.0)
    build_s = time.perf_counter() - t0
    nodes, slots = acc.export()
    print(f"cornell 1,310,734 triangles: {len(slots)} references, build {build_s * 1e3:.0f} ms")
    assert scene.n_prims < len(slots) <= 4 * scene.n_prims
    ref = lib.GpuAccel(scene)
    f_split = lib.GpuPathIntegrator(acc, scene).render()
    f_ref = lib.GpuPathIntegrator(ref, scene).render()
    a, b = f_split.image(), f_ref.image()
    close = np.isclose(a, b, rtol=1e-4, atol=1e-6)
    print(f"frame over the device split tree vs the reference tree: {close.mean():.5f} of values within 1e-4")
    assert close.mean() >= 0.99
    acc.close()
    ref.close()
