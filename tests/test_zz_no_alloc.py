"""bbg_intersect_static: the closest-hit query for callers that cannot
allocate device memory while they trace (allocation forbidden after start-up,
real-time loops, device memory held by another allocator). It stages rays and
hits through one fixed device array instead of library-allocated buffers.

Checked through the C ABI against bbg_intersect on the same accel: identical
primitive ids and bit-identical t (the tolerance these tests use for
traversal), on two calls in a row, the second with different rays, so the
shared array's left-over contents (its work counter in particular) cannot leak
into the next call. The device's free memory (cudaMemGetInfo) is the same
before and after each of the two calls: the array and the query's kernels are
set up when the accel is created, so even the first call allocates nothing.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process."""
import gc

import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu

MAX_RAYS = 1 << 18


def static_intersect(acc, rays):
    rays = np.ascontiguousarray(rays, np.float32)
    hits = np.zeros((rays.shape[0], 4), np.float32)
    st = lib.get_lib().bbg_intersect_static(acc.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data)
    return st, hits


def free_device_memory():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_static_entry_point_matches_intersect_on_two_calls():
    free_device_memory()  # the CUDA context exists before anything is measured
    scene = scenes.triangle_soup(100_000, seed=1)
    acc = lib.GpuAccel(scene)
    first, _ = scenes.soup_rays(MAX_RAYS, seed=2)
    second, _ = scenes.soup_rays(50_000, seed=7)
    # The 8-wide layout (default) on the first call, the binary one on the
    # second; no other library call in between, and no collection of earlier
    # tests' handles (which would free device memory) while measuring.
    gc.collect()
    gc.disable()
    try:
        results, free = [], [free_device_memory()]
        for rays, mode in ((first, abi.BBG_TRAVERSAL_WIDE), (second, abi.BBG_TRAVERSAL_ORDERED)):
            acc.set_traversal(mode)
            st, hits = static_intersect(acc, rays)
            assert st == abi.BBG_OK, lib.get_lib().bbg_last_error()
            results.append(hits)
            free.append(free_device_memory())
    finally:
        gc.enable()
    assert free[0] == free[1] == free[2], f"free device memory changed across the calls: {free}"
    for rays, mode, hits in ((first, abi.BBG_TRAVERSAL_WIDE, results[0]),
                             (second, abi.BBG_TRAVERSAL_ORDERED, results[1])):
        acc.set_traversal(mode)
        prim, t, u, v = acc.intersect(rays)
        assert np.array_equal(hits[:, 0].view(np.int32), prim)
        assert np.array_equal(hits[:, 1].view(np.uint32), t.view(np.uint32))
        assert np.array_equal(hits[:, 2:], np.stack([u, v], 1))
        assert (prim >= 0).mean() > 0.5


def test_static_entry_point_reference_order_counting_and_limit():
    scene = scenes.triangle_soup(20_000, seed=3)
    acc = lib.GpuAccel(scene)
    acc.set_traversal(abi.BBG_TRAVERSAL_REFERENCE)
    rays, _ = scenes.soup_rays(10_000, seed=4)
    st, hits = static_intersect(acc, rays)
    assert st == abi.BBG_OK
    prim, t, _, _ = acc.intersect(rays)
    assert np.array_equal(hits[:, 0].view(np.int32), prim)
    # A counting accel: both queries traverse in the reference's order.
    acc.set_traversal(abi.BBG_TRAVERSAL_WIDE)
    acc.set_counting(True)
    st, hits = static_intersect(acc, rays)
    assert st == abi.BBG_OK
    prim, t, _, _ = acc.intersect(rays)
    assert np.array_equal(hits[:, 0].view(np.int32), prim)
    assert np.array_equal(hits[:, 1].view(np.uint32), t.view(np.uint32))
    acc.set_counting(False)
    # Beyond the fixed array: a clear error, nothing traced.
    big = np.zeros((MAX_RAYS + 1, 8), np.float32)
    st, _ = static_intersect(acc, big)
    assert st == abi.BBG_ERR_INVALID_ARG
    assert b"262144" in lib.get_lib().bbg_last_error()
