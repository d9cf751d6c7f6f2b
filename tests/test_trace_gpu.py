"""GPU traversal parity: bbg_intersect / bbg_intersect_any against the
reference's BVH::Intersect / IntersectAny (src/accel/bvh.cpp:299-361) on the
same scene, tree and rays.

Bar: closest-hit primitive ids bit-exact except on rays whose two nearest hits
lie within 1e-5 relative t (the mismatch fraction is reported), t bit-exact
where the ids agree, any-hit results identical."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu

NEAR_TIE_REL = 1e-5


def compare_closest(rs, rays, prim, t, ref_prim, ref_t):
    mism = np.nonzero(prim != ref_prim)[0]
    unexplained = []
    for i in mism:
        prims, ts = rs.intersect_all(rays[i])
        ok = len(ts) >= 2 and (ts[1] - ts[0]) <= NEAR_TIE_REL * abs(ts[0])
        if not ok:
            unexplained.append((int(i), int(prim[i]), int(ref_prim[i]), float(t[i]), float(ref_t[i])))
    frac = len(mism) / max(1, len(prim))
    same = prim == ref_prim
    hit = same & (ref_prim >= 0)
    t_bad = np.nonzero(t[hit].view(np.uint32) != ref_t[hit].view(np.uint32))[0]
    return frac, unexplained, t_bad


def run_parity(oracle, scene, closest, anyq, use_ref_tree):
    rs = oracle.RefScene(scene)
    tree = rs.bvh() if use_ref_tree else None
    acc = lib.GpuAccel(scene, bvh=tree)
    ref_prim, ref_t, _ = rs.intersect(closest)
    ref_occ, _ = rs.intersect_any(anyq)
    fracs = {}
    names = {abi.BBG_TRAVERSAL_REFERENCE: "reference-order", abi.BBG_TRAVERSAL_ORDERED: "ordered",
             abi.BBG_TRAVERSAL_WIDE: "8-wide"}
    for mode in (abi.BBG_TRAVERSAL_REFERENCE, abi.BBG_TRAVERSAL_ORDERED, abi.BBG_TRAVERSAL_WIDE):
        acc.set_traversal(mode)
        prim, t, _, _ = acc.intersect(closest)
        frac, unexplained, t_bad = compare_closest(rs, closest, prim, t, ref_prim, ref_t)
        name = names[mode]
        print(f"{scene.name} [{name}]: closest mismatch fraction {frac:.2e} ({int(round(frac * len(prim)))} rays), "
              f"hit rate {(ref_prim >= 0).mean():.3f}")
        assert not unexplained, unexplained[:5]
        assert t_bad.size == 0
        occ = acc.intersect_any(anyq)
        assert np.array_equal(occ, ref_occ)
        fracs[name] = frac
    acc.close()
    return fracs


@pytest.mark.parametrize("use_ref_tree", [True, False], ids=["reference_tree", "own_tree"])
def test_soup_parity(oracle, use_ref_tree):
    scene = scenes.triangle_soup(200_000, seed=1)
    closest, anyq = scenes.soup_rays(262_144, seed=2)
    run_parity(oracle, scene, closest, anyq, use_ref_tree)


def test_full_size_soup_parity(oracle):
    """1,048,576 triangles (the microbenchmark scene) on 2M of its rays."""
    scene = scenes.triangle_soup(1 << 20, seed=1)
    closest, anyq = scenes.soup_rays(1 << 21, seed=2)
    run_parity(oracle, scene, closest, anyq, use_ref_tree=False)


def test_cornell_parity(oracle):
    scene = scenes.cornell_icosphere(levels=6, width=8, height=8)
    rng = np.random.default_rng(4)
    n = 200_000
    o = rng.uniform(-0.95, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3], rays[:, 3:6], rays[:, 6], rays[:, 7] = o, d, 1e-4, np.inf
    anyq = rays.copy()
    anyq[:, 7] = rng.uniform(0.05, 2.0, n).astype(np.float32)
    run_parity(oracle, scene, rays, anyq, use_ref_tree=True)


def test_sphere_parity(oracle):
    scene = scenes.readme_sphere()
    # Add a rotated, scaled second sphere.
    sph = scenes.abi.Sphere()
    sph.p[:] = [1.5, 0.2, -0.7]
    q = np.array([0.2, -0.4, 0.1, 0.9], np.float32)
    q /= np.linalg.norm(q)
    sph.q[:] = q.tolist()
    sph.s[:] = [1.0, 1.0, 1.0]
    sph.radius = 0.6
    scene.spheres.append(sph)
    scene.prim_kind = np.array([1, 1], np.int32)
    scene.prim_index = np.array([0, 1], np.int32)
    scene.prim_material = np.array([0, 0], np.int32)
    rng = np.random.default_rng(5)
    n = 100_000
    o = rng.uniform(-4, 4, (n, 3)).astype(np.float32)
    tgt = rng.uniform(-1, 2, (n, 3)).astype(np.float32)
    d = (tgt - o).astype(np.float32)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3], rays[:, 3:6], rays[:, 6], rays[:, 7] = o, d, 1e-4, np.inf  # unnormalised directions
    anyq = rays.copy()
    anyq[:, 7] = rng.uniform(0.1, 3, n).astype(np.float32)
    run_parity(oracle, scene, rays, anyq, use_ref_tree=True)


def test_edge_rays(oracle):
    """Axis-aligned directions (infinite 1/d), origins on slab planes,
    t_max <= t_min, zero-length direction, origin inside a box."""
    scene = scenes.triangle_soup(20_000, seed=3)
    rays = []
    for axis in range(3):
        for sgn in (1.0, -1.0):
            for k in range(200):
                d = [0.0, 0.0, 0.0]
                d[axis] = sgn
                o = list(np.random.default_rng(k).uniform(-1, 1, 3))
                o[axis] = -3.0 * sgn
                rays.append(o + d + [1e-4, np.inf])
    rays.append([0.0, 0.0, -3.0, 0.0, 0.0, 1.0, 1.0, 1.0])      # t_max == t_min
    rays.append([0.0, 0.0, -3.0, 0.0, 0.0, 1.0, 2.0, 1.0])      # t_max < t_min
    rays.append([0.1, 0.2, 0.3, 0.0, 0.0, 0.0, 1e-4, np.inf])   # zero direction
    rays.append([-1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1e-4, np.inf])  # origin on the root box corner
    rays = np.array(rays, np.float32)
    run_parity(oracle, scene, rays, rays, use_ref_tree=True)


def test_empty_batch_and_counts(oracle):
    scene = scenes.triangle_soup(10_000, seed=4)
    acc = lib.GpuAccel(scene)
    prim, t, _, _ = acc.intersect(np.zeros((0, 8), np.float32))
    assert prim.shape == (0,)
    closest, _ = scenes.soup_rays(10_000, seed=6)
    acc.set_counting(True)
    acc.intersect(closest)
    nodes, prims = acc.last_counts()
    assert nodes > 10_000 and prims > 0


def test_closest_and_any_agree_at_full_size():
    """Size-independent property on the full 16M-ray microbenchmark set:
    any-hit over [t_min, t_max] is true exactly when the closest hit over
    [t_min, inf] lies at or before t_max."""
    import torch
    scene = scenes.triangle_soup(1 << 20, seed=1)
    closest, anyq = scenes.soup_rays(1 << 24, seed=2)
    acc = lib.GpuAccel(scene)
    rc = torch.from_numpy(closest).cuda()
    ra = torch.from_numpy(anyq).cuda()
    for mode in (abi.BBG_TRAVERSAL_ORDERED, abi.BBG_TRAVERSAL_WIDE):
        acc.set_traversal(mode)
        hits = torch.empty((rc.shape[0], 4), dtype=torch.float32, device="cuda")
        occ = torch.empty(rc.shape[0], dtype=torch.uint8, device="cuda")
        acc.intersect_device(rc, hits)
        acc.intersect_any_device(ra, occ)
        prim = hits[:, 0].view(torch.int32)
        t = hits[:, 1]
        expect = (prim >= 0) & (t <= ra[:, 7])
        assert torch.equal(expect.to(torch.uint8), occ)
        if mode == abi.BBG_TRAVERSAL_ORDERED:
            ordered_prim = prim.clone()
        else:
            # the two layouts agree except on exact ties
            assert (prim != ordered_prim).float().mean().item() < 1e-5


def classify_against_brute_force(rs, rays, prim, t, ref_prim, ref_t):
    """Mismatches between two trees' closest hits, classified with a brute-force
    test of every primitive: near-ties, and rays one tree would let through (its
    slab test, without a robustness margin as in the reference, missing a box
    that contains the true closest hit). Returns (ties, leaks_ref, leaks_dev,
    unexplained)."""
    ties = leaks_ref = leaks_dev = 0
    unexplained = []
    for i in np.nonzero(prim != ref_prim)[0]:
        prims, ts = rs.intersect_all(rays[i])
        if len(ts) >= 2 and (ts[1] - ts[0]) <= NEAR_TIE_REL * abs(ts[0]):
            ties += 1
        elif len(ts) and prim[i] == prims[0] and t[i] == ts[0]:
            leaks_ref += 1
        elif len(ts) and ref_prim[i] == prims[0] and ref_t[i] == ts[0]:
            leaks_dev += 1
        else:
            unexplained.append((int(i), int(prim[i]), int(ref_prim[i]), float(t[i]), float(ref_t[i])))
    return ties, leaks_ref, leaks_dev, unexplained


def test_split_reference_tree_parity(oracle):
    """The SAH tree over split references (bbg_accel_create_split): closest hits
    agree with the reference BVH except near-ties, any-hit agrees, in both
    layouts."""
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
        acc = lib.GpuAccel(scene, split=1.0)
        ref_prim, ref_t, _ = rs.intersect(cl)
        ref_occ, _ = rs.intersect_any(an)
        for mode in (abi.BBG_TRAVERSAL_WIDE, abi.BBG_TRAVERSAL_ORDERED):
            acc.set_traversal(mode)
            prim, t, _, _ = acc.intersect(cl)
            ties, leaks_ref, leaks_dev, unexplained = classify_against_brute_force(rs, cl, prim, t, ref_prim, ref_t)
            print(f"split-reference tree, {scene.name}: {ties} near-ties, {leaks_ref} + {leaks_dev} leaks")
            assert not unexplained, unexplained[:5]
            assert leaks_ref + leaks_dev <= 1e-3 * len(cl)
            same = (prim == ref_prim) & (ref_prim >= 0)
            assert np.array_equal(t[same].view(np.uint32), ref_t[same].view(np.uint32))
            assert np.array_equal(acc.intersect_any(an), ref_occ)
        acc.close()


def test_device_built_tree_parity(oracle):
    """The linear BVH built on the device: closest hits agree with the
    reference BVH except near-ties (or rays that one tree's boxes would let
    through, counted separately: none were seen), any-hit agrees on the soup;
    the tree has no reference layout (reference traversal, counting and export
    are refused)."""
    soup = scenes.triangle_soup(200_000, seed=1)
    closest, anyq = scenes.soup_rays(1 << 19, seed=2)
    cornell = scenes.cornell_icosphere(levels=6, width=8, height=8)
    rng = np.random.default_rng(4)
    n = 200_000
    crays = np.zeros((n, 8), np.float32)
    crays[:, :3] = rng.uniform(-0.95, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    crays[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    crays[:, 6], crays[:, 7] = 1e-4, np.inf
    for scene, rays, anyq in ((soup, closest, anyq), (cornell, crays, None)):
        rs = oracle.RefScene(scene)
        acc = lib.GpuAccel(scene, device_build=True)
        ref_prim, ref_t, _ = rs.intersect(rays)
        # the 8-wide layout collapsed on the device (the default), then the binary one
        for mode in (abi.BBG_TRAVERSAL_WIDE, abi.BBG_TRAVERSAL_ORDERED):
            acc.set_traversal(mode)
            prim, t, _, _ = acc.intersect(rays)
            ties, leaks_ref, leaks_dev, unexplained = classify_against_brute_force(rs, rays, prim, t, ref_prim,
                                                                                   ref_t)
            print(f"device-built tree ({'8-wide' if mode == abi.BBG_TRAVERSAL_WIDE else 'binary'}), {scene.name}: "
                  f"{len(rays)} rays, mismatches: {ties} near-ties, {leaks_ref} through the reference tree, "
                  f"{leaks_dev} through the device tree")
            assert not unexplained, unexplained[:5]
            assert leaks_ref + leaks_dev <= 1e-3 * len(rays)
            same = (prim == ref_prim) & (ref_prim >= 0)
            assert np.array_equal(t[same].view(np.uint32), ref_t[same].view(np.uint32))
            if anyq is not None:
                ref_occ, _ = rs.intersect_any(anyq)
                assert np.array_equal(acc.intersect_any(anyq), ref_occ)
    for call in (lambda: acc.set_traversal(abi.BBG_TRAVERSAL_REFERENCE), lambda: acc.set_counting(True),
                 lambda: acc.export()):
        with pytest.raises(lib.BbgError) as e:
            call()
        assert e.value.status == abi.BBG_ERR_UNSUPPORTED


def test_oversized_leaf_falls_back_to_the_binary_layout(oracle):
    """64 coincident triangles make one leaf of 64 primitives, more than the
    8-wide layout encodes: the accel keeps the binary layout (WIDE is
    refused), and hits still match the reference."""
    scene = scenes.triangle_soup(2000, seed=9)
    pos = scene.positions.copy()
    pos[: 3 * 64] = np.tile(pos[:3], (64, 1))
    scene.positions = pos
    rs = oracle.RefScene(scene)
    acc = lib.GpuAccel(scene, bvh=rs.bvh())
    with pytest.raises(lib.BbgError) as e:
        acc.set_traversal(abi.BBG_TRAVERSAL_WIDE)
    assert e.value.status == abi.BBG_ERR_UNSUPPORTED
    closest, anyq = scenes.soup_rays(50_000, seed=3)
    ref_prim, ref_t, _ = rs.intersect(closest)
    prim, t, _, _ = acc.intersect(closest)
    frac, unexplained, t_bad = compare_closest(rs, closest, prim, t, ref_prim, ref_t)
    assert not unexplained and t_bad.size == 0
    ref_occ, _ = rs.intersect_any(anyq)
    assert np.array_equal(acc.intersect_any(anyq), ref_occ)


def test_traversal_counts_match_a_replay_of_the_reference():
    """The counting run behind the roofline's algorithmic bytes (nodes popped
    and primitive tests in BVH::RayCast's order) equals the oracle's replay of
    RayCast with the reference's own TestRay and primitive tests, for
    closest-hit and any-hit queries (64K rays each)."""
    from oracle import ref
    soup = scenes.triangle_soup(1 << 20, seed=1)
    closest, anyq = scenes.soup_rays(1 << 16, seed=2)
    cornell = scenes.cornell_icosphere(levels=6, width=8, height=8)
    rng = np.random.default_rng(12)
    n = 1 << 16
    crays = np.zeros((n, 8), np.float32)
    crays[:, :3] = rng.uniform(-0.95, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    crays[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    crays[:, 6], crays[:, 7] = 1e-4, np.inf
    cany = crays.copy()
    cany[:, 7] = rng.uniform(0.05, 2.0, n).astype(np.float32)
    for scene, cl, an in ((soup, closest, anyq), (cornell, crays, cany)):
        rs = ref.RefScene(scene)
        acc = lib.GpuAccel(scene, bvh=rs.bvh())
        acc.set_counting(True)
        acc.intersect(cl)
        gpu_closest = acc.last_counts()
        acc.intersect_any(an)
        gpu_any = acc.last_counts()
        cpu_closest = rs.count_traversal(cl)
        cpu_any = rs.count_traversal(an, any_hit=True)
        print(f"{scene.name}: closest {gpu_closest} vs {cpu_closest}, any {gpu_any} vs {cpu_any}")
        assert tuple(gpu_closest) == cpu_closest
        assert tuple(gpu_any) == cpu_any
        acc.close()
