"""The host SAH builder (bbg_bvh_build) reproduces the reference BVH
(src/accel/bvh.cpp:56-297) node for node, and the primitive AABBs match
Triangle::GetAABB / Sphere::GetAABB bit for bit."""
import numpy as np
import pytest

from bulbit_b200 import lib, scenes


def leaf_sets(nodes, slots):
    out = []
    for n in nodes:
        if n["count"] > 0:
            out.append(tuple(slots[n["offset"]:n["offset"] + n["count"]]))
        else:
            out.append(None)
    return out


def assert_same_tree(mine, ref):
    (mn, ms), (rn, rs) = mine, ref
    assert mn.shape == rn.shape
    assert np.array_equal(mn["bmin"].view(np.uint32), rn["bmin"].view(np.uint32))
    assert np.array_equal(mn["bmax"].view(np.uint32), rn["bmax"].view(np.uint32))
    assert np.array_equal(mn["count"], rn["count"])
    interior = mn["count"] == 0
    assert np.array_equal(mn["axis"][interior], rn["axis"][interior])
    assert np.array_equal(mn["offset"][interior], rn["offset"][interior])
    # Leaves: same primitives in the same order (slot offsets may differ only
    # where the reference built subtrees concurrently).
    assert leaf_sets(mn, ms) == leaf_sets(rn, rs)
    assert sorted(ms.tolist()) == list(range(ms.shape[0]))
    # This builder's leaves take consecutive slots in depth-first node order
    # (also where it built subtrees on separate threads).
    leaves = mn[mn["count"] > 0]
    starts = np.concatenate([[0], np.cumsum(leaves["count"].astype(np.int64))[:-1]])
    assert np.array_equal(leaves["offset"], starts)


@pytest.mark.parametrize("make", [
    lambda: scenes.triangle_soup(2000, seed=1),
    lambda: scenes.triangle_soup(100_000, seed=5),
    lambda: scenes.triangle_soup(400_000, seed=6),
    lambda: scenes.cornell_icosphere(levels=4, width=16, height=16),
    lambda: scenes.readme_sphere(),
], ids=["soup2k", "soup100k_parallel_ref_build", "soup400k_parallel_builds", "cornell_ico4", "readme_sphere"])
def test_builder_matches_reference(oracle, make):
    scene = make()
    rs = oracle.RefScene(scene)
    mine = lib.bvh_build(lib.prim_aabbs(scene))
    assert_same_tree(mine, rs.bvh())


def test_duplicate_primitives_build_like_the_reference(oracle):
    # Coincident triangles: zero centroid extent -> one leaf (bvh.cpp:111-123).
    s = scenes.triangle_soup(64, seed=9)
    s.positions = np.tile(s.positions[:3], (64, 1))
    rs = oracle.RefScene(s)
    mine = lib.bvh_build(lib.prim_aabbs(s))
    assert_same_tree(mine, rs.bvh())
    assert mine[0].shape[0] == 1 and mine[0]["count"][0] == 64


def test_prim_aabbs_match_reference_leaf_bounds(oracle):
    s = scenes.triangle_soup(1, seed=3)
    rs = oracle.RefScene(s)
    nodes, _ = rs.bvh()
    a = lib.prim_aabbs(s)
    assert np.array_equal(a[0, :3].view(np.uint32), nodes["bmin"][0].view(np.uint32))
    assert np.array_equal(a[0, 3:].view(np.uint32), nodes["bmax"][0].view(np.uint32))


def test_builder_rejects_bad_input():
    with pytest.raises(lib.BbgError):
        lib.bvh_build(np.zeros((0, 6), np.float32))


def _bad_tree_status(nodes, slots, scene):
    import ctypes
    from bulbit_b200 import abi
    g = scene.geometry()
    b = abi.Bvh()
    b.n_nodes, b.nodes = nodes.shape[0], nodes.ctypes.data
    b.n_slots, b.slot_prims = slots.shape[0], slots.ctypes.data
    h = ctypes.c_void_p()
    st = lib.get_lib().bbg_accel_create(ctypes.byref(g), ctypes.byref(b), ctypes.byref(h))
    assert not h.value
    return st


@pytest.mark.parametrize("corrupt", ["child_out_of_range", "child_backwards", "leaf_past_slots", "slot_prim_range"])
def test_corrupt_trees_are_rejected_before_upload(corrupt):
    """Host-side validation catches malformed input trees (no device work)."""
    from bulbit_b200 import abi
    s = scenes.triangle_soup(500, seed=2)
    nodes, slots = lib.bvh_build(lib.prim_aabbs(s))
    nodes, slots = nodes.copy(), slots.copy()
    interior = np.nonzero(nodes["count"] == 0)[0]
    leaves = np.nonzero(nodes["count"] > 0)[0]
    if corrupt == "child_out_of_range":
        nodes["offset"][interior[3]] = nodes.shape[0] + 5
    elif corrupt == "child_backwards":
        nodes["offset"][interior[3]] = 0  # a cycle back to the root
    elif corrupt == "leaf_past_slots":
        nodes["offset"][leaves[-1]] = slots.shape[0]
    else:
        slots[7] = 10_000
    assert _bad_tree_status(nodes, slots, s) == abi.BBG_ERR_BAD_BVH


def test_oversized_leaf_is_rejected():
    """70000 coincident triangles form one leaf; the reference would truncate
    its uint16 primitive_count (include/bulbit/bvh.h:56), this builder refuses."""
    s = scenes.triangle_soup(70_000, seed=2)
    s.positions = np.tile(s.positions[:3], (70_000, 1))
    with pytest.raises(lib.BbgError) as e:
        lib.bvh_build(lib.prim_aabbs(s))
    assert "65535" in str(e.value)


@pytest.mark.parametrize("make", [
    lambda: scenes.triangle_soup(1 << 20, seed=1),
    lambda: scenes.cornell_icosphere(levels=8, width=16, height=16),
], ids=["microbenchmark_soup_1048576", "cornell_1310734"])
def test_builder_matches_reference_at_full_size(oracle, make):
    """The trees the benchmark workloads use, node for node: the 1,048,576-
    triangle soup and the Cornell box with the 8-level displaced icosphere."""
    scene = make()
    rs = oracle.RefScene(scene)
    mine = lib.bvh_build(lib.prim_aabbs(scene))
    assert_same_tree(mine, rs.bvh())
