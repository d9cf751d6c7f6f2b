"""The reference's SAH tree built on the device (bbg_accel_create_device_sah)
against the host build (bbg_bvh_build), which reproduces BVH::BVH /
BuildRecursive / FlattenBVH (src/accel/bvh.cpp:8-297) node for node: the two
flattened trees are byte-identical (boxes, axes, child offsets, leaf ranges)
and so are the slot orders, on soups and meshes from a few thousand to a
million primitives, spheres, coincident primitives (leaves by zero centroid
extent) and pairs split by nth_element; so are the 8-wide layouts collapsed
from them on the device and on the host. Queries and renders over it then
equal those over the host-built tree bit for bit, in every traversal mode."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu


def coincident_scene():
    s = scenes.triangle_soup(300, seed=9)
    pos = s.positions.copy()
    pos[: 3 * 64] = np.tile(pos[:3], (64, 1))  # 64 coincident triangles: one leaf
    pos[3 * 64: 3 * 66] = pos[3 * 70: 3 * 72] + 1e-3  # near pairs
    s.positions = pos
    return s


CASES = {
    "soup2k": lambda: scenes.triangle_soup(2000, seed=1),
    "soup200k": lambda: scenes.triangle_soup(200_000, seed=5),
    "soup_1048576": lambda: scenes.triangle_soup(1 << 20, seed=1),
    "cornell_ico4": lambda: scenes.cornell_icosphere(levels=4, width=16, height=16),
    "cornell_1310734": lambda: scenes.cornell_icosphere(levels=8, width=16, height=16),
    "readme_spheres": lambda: scenes.readme_sphere(),
    "coincident": coincident_scene,
    "one_triangle": lambda: scenes.triangle_soup(1, seed=2),
    "two_triangles": lambda: scenes.triangle_soup(2, seed=3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_sah_tree_equals_host_build(name):
    scene = CASES[name]()
    host_nodes, host_slots = lib.bvh_build(lib.prim_aabbs(scene))
    acc = lib.GpuAccel(scene, device_sah=True)
    nodes, slots = acc.export()
    print(f"{name}: {scene.n_prims} primitives, {len(nodes)} nodes")
    assert nodes.shape == host_nodes.shape
    assert np.array_equal(nodes.view(np.uint8), host_nodes.view(np.uint8))
    assert np.array_equal(slots, host_slots)
    assert np.array_equal(acc.bounds(), np.concatenate([host_nodes[0]["bmin"], host_nodes[0]["bmax"]]))
    acc.close()


@pytest.mark.parametrize("name", list(CASES))
def test_device_wide_layout_equals_host_collapse(name):
    """The 8-wide layout collapsed on the device (SahPlanKernel and the
    level-by-level collapse, sah_build.cu) equals the host collapse of the
    same tree (BuildWide8, accel.cu) byte for byte: the same surface-area plan
    in the same double-precision arithmetic, the same breadth-first
    numbering, slot assignment and quantisation. Where a leaf holds more
    primitives than the layout encodes (the 64 coincident triangles), both
    leave it unbuilt."""
    scene = CASES[name]()
    host = lib.GpuAccel(scene)
    dev = lib.GpuAccel(scene, device_sah=True)
    wh, wd = host.export_wide8(), dev.export_wide8()
    print(f"{name}: {len(wh)} wide nodes")
    assert (len(wh) > 0) == (name != "coincident")
    assert wh.shape == wd.shape
    assert np.array_equal(wh.view(np.uint32), wd.view(np.uint32))
    host.close()
    dev.close()


def test_device_sah_queries_equal_host_tree():
    scene = scenes.triangle_soup(200_000, seed=5)
    closest, anyq = scenes.soup_rays(1 << 18, seed=6)
    host = lib.GpuAccel(scene)
    dev = lib.GpuAccel(scene, device_sah=True)
    for mode in (abi.BBG_TRAVERSAL_WIDE, abi.BBG_TRAVERSAL_ORDERED, abi.BBG_TRAVERSAL_REFERENCE):
        host.set_traversal(mode)
        dev.set_traversal(mode)
        a, b = host.intersect(closest), dev.intersect(closest)
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        assert np.array_equal(host.intersect_any(anyq), dev.intersect_any(anyq))
    # Counting runs in the reference's order over the same tree.
    host.set_counting(True)
    dev.set_counting(True)
    host.intersect(closest)
    dev.intersect(closest)
    assert host.last_counts() == dev.last_counts()


def test_device_sah_render_equals_host_tree():
    scene = scenes.cornell_icosphere(levels=5, width=48, height=48, spp=8, max_bounces=16)
    films = []
    for kw in ({}, {"device_sah": True}):
        acc = lib.GpuAccel(scene, **kw)
        integ = lib.GpuPathIntegrator(acc, scene)
        films.append(integ.render(path_L=True))
        integ.close()
        acc.close()
    assert np.array_equal(films[0].path_L, films[1].path_L)
    assert np.array_equal(films[0].rgb_sum, films[1].rgb_sum)
