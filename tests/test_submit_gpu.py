"""Submitted queries (bbg_intersect_submit, bbg_intersect_any_submit,
bbg_accel_synchronize): batches of BVH::Intersect / IntersectAny
(src/accel/bvh.cpp:299-361) queued back to back through the accel's staging
ring. Results must equal the synchronous calls' bit for bit, whatever the
order of submissions, buffer kinds and sizes (a larger batch after smaller
ones regrows the staging slots while queued work may still use them), and
the closest hits must agree with the reference's."""
import numpy as np
import pytest
import torch

from bulbit_b200 import abi, lib, scenes
from test_trace_gpu import compare_closest

pytestmark = pytest.mark.gpu


def _pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


@pytest.fixture(scope="module")
def soup():
    scene = scenes.triangle_soup(100_000, seed=21)
    closest, anyq = scenes.soup_rays(3_000_000, seed=22)
    return scene, closest, anyq


def test_submitted_host_queries_equal_synchronous(oracle, soup):
    scene, closest, anyq = soup
    acc = lib.GpuAccel(scene)
    want_hits = np.zeros((len(closest), 4), np.float32)
    want_occ = np.zeros(len(anyq), np.uint8)
    check = lib.check
    L = lib.get_lib()
    check(L.bbg_intersect(acc.h, lib._p(closest), len(closest), lib._p(want_hits), abi.BBG_MEM_HOST, None), "sync")
    check(L.bbg_intersect_any(acc.h, lib._p(anyq), len(anyq), lib._p(want_occ), abi.BBG_MEM_HOST, None), "sync")

    small = 300_000  # sizes the staging slots for 300K rays; the full batch then regrows them
    pin_c, pin_a = _pinned(closest), _pinned(anyq)
    hits_small = torch.zeros((small, 4), dtype=torch.float32).pin_memory()
    hits = torch.zeros((len(closest), 4), dtype=torch.float32).pin_memory()
    occ = torch.zeros(len(anyq), dtype=torch.uint8).pin_memory()
    occ_pageable = np.zeros(len(anyq), np.uint8)
    acc.synchronize()  # nothing queued: returns at once
    acc.submit_host_ptr(pin_c.data_ptr(), small, hits_small.data_ptr())
    acc.submit_host_ptr(pin_c.data_ptr(), len(closest), hits.data_ptr())
    acc.submit_any_host_ptr(pin_a.data_ptr(), len(anyq), occ.data_ptr())
    acc.submit_any_host_ptr(pin_a.data_ptr(), len(anyq), occ_pageable.ctypes.data)
    acc.submit_host_ptr(pin_c.data_ptr(), 0, hits.data_ptr())  # an empty batch queues nothing
    acc.synchronize()
    assert np.array_equal(hits_small.numpy().view(np.uint32), want_hits[:small].view(np.uint32))
    assert np.array_equal(hits.numpy().view(np.uint32), want_hits.view(np.uint32))
    assert np.array_equal(occ.numpy(), want_occ)
    assert np.array_equal(occ_pageable, want_occ)

    # A synchronous call after submissions waits for them and answers in place.
    hits.zero_()
    occ.zero_()
    acc.submit_any_host_ptr(pin_a.data_ptr(), len(anyq), occ.data_ptr())
    prim, t, _, _ = acc.intersect(closest)
    assert np.array_equal(occ.numpy(), want_occ)
    assert np.array_equal(t.view(np.uint32), want_hits[:, 1].view(np.uint32))

    # The closest hits (submitted and synchronous alike, shown equal above)
    # against the reference's BVH::Intersect, on a sample.
    rs = oracle.RefScene(scene)
    sample = closest[:200_000]
    ref_prim, ref_t, _ = rs.intersect(sample)
    frac, unexplained, t_bad = compare_closest(rs, sample, want_hits[:200_000, 0].view(np.int32),
                                               want_hits[:200_000, 1], ref_prim, ref_t)
    assert not unexplained and t_bad.size == 0
    acc.close()


def test_submitted_device_queries_and_mixed_order(soup):
    scene, closest, anyq = soup
    acc = lib.GpuAccel(scene)
    want_prim, want_t, _, _ = acc.intersect(closest)
    want_occ = acc.intersect_any(anyq)
    dev = torch.device("cuda")
    rays_d = torch.from_numpy(closest).to(dev)
    any_d = torch.from_numpy(anyq).to(dev)
    hits_d = torch.zeros((len(closest), 4), dtype=torch.float32, device=dev)
    occ_d = torch.zeros(len(anyq), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    pin_a = _pinned(anyq)
    occ_h = torch.zeros(len(anyq), dtype=torch.uint8).pin_memory()
    # Device and host batches interleaved on one accel.
    acc.submit_device(rays_d, hits_d)
    acc.submit_any_host_ptr(pin_a.data_ptr(), len(anyq), occ_h.data_ptr())
    acc.submit_any_device(any_d, occ_d)
    acc.synchronize()
    h = hits_d.cpu().numpy()
    assert np.array_equal(h[:, 0].view(np.int32), want_prim)
    assert np.array_equal(h[:, 1].view(np.uint32), want_t.view(np.uint32))
    assert np.array_equal(occ_d.cpu().numpy(), want_occ)
    assert np.array_equal(occ_h.numpy(), want_occ)
    acc.close()


def test_counting_accel_refuses_submissions(soup):
    scene, closest, _ = soup
    acc = lib.GpuAccel(scene)
    acc.set_counting(True)
    hits = np.zeros((16, 4), np.float32)
    with pytest.raises(lib.BbgError) as e:
        acc.submit_host_ptr(closest.ctypes.data, 16, hits.ctypes.data)
    assert e.value.status == abi.BBG_ERR_UNSUPPORTED
    acc.close()
