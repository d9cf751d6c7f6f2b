"""Split-reference build (bbg_split_references, host only): the references'
boxes cover every point of their triangle, lie inside the triangle's own box,
respect the budget, and with no budget are the primitives' own boxes."""
import numpy as np

from bulbit_b200 import lib, scenes


def triangle_points(scene, prim, k, rng):
    v = scene.tri_indices.reshape(-1, 3)[scene.prim_index[prim]]
    p = scene.positions.reshape(-1, 3)[v].astype(np.float64)
    a = rng.random((k, 2))
    flip = a.sum(1) > 1
    a[flip] = 1 - a[flip]
    return p[0] + a[:, :1] * (p[1] - p[0]) + a[:, 1:] * (p[2] - p[0]), p


def test_no_budget_is_the_primitive_boxes():
    scene = scenes.cornell_icosphere(levels=3, width=8, height=8)
    boxes, prims = lib.split_references(scene, 0.0)
    assert np.array_equal(prims, np.arange(scene.n_prims))
    assert np.array_equal(boxes, lib.prim_aabbs(scene))


def test_split_references_cover_their_triangles():
    scene = scenes.cornell_icosphere(levels=4, width=8, height=8)
    n = scene.n_prims
    boxes, prims = lib.split_references(scene, 1.0)
    assert n < len(prims) <= 2 * n
    own = lib.prim_aabbs(scene)
    # inside the primitive's own (padded) box
    assert np.all(boxes[:, :3] >= own[prims, :3]) and np.all(boxes[:, 3:] <= own[prims, 3:])
    rng = np.random.default_rng(1)
    by_prim = {}
    for i, p in enumerate(prims):
        by_prim.setdefault(int(p), []).append(i)
    split = [p for p, r in by_prim.items() if len(r) > 1]
    assert len(split) > 100
    for p in split[:400]:
        pts, verts = triangle_points(scene, p, 200, rng)
        pts = np.concatenate([pts, verts])
        b = boxes[by_prim[p]].astype(np.float64)
        inside = ((pts[:, None, :] >= b[None, :, :3]) & (pts[:, None, :] <= b[None, :, 3:])).all(2).any(1)
        assert inside.all(), p
    # splitting shrinks the total box area
    def area(bx):
        d = bx[:, 3:] - bx[:, :3]
        return 2 * (d[:, 0] * d[:, 1] + d[:, 1] * d[:, 2] + d[:, 2] * d[:, 0])
    assert area(boxes).sum() < area(own).sum()


def test_spheres_are_never_split():
    scene = scenes.readme_sphere()
    boxes, prims = lib.split_references(scene, 4.0)
    assert np.array_equal(prims, np.arange(scene.n_prims))
    assert np.array_equal(boxes, lib.prim_aabbs(scene))


def test_budget_bounds_the_reference_count():
    scene = scenes.triangle_soup(5000, seed=3)
    for budget in (0.25, 0.5, 2.0):
        _, prims = lib.split_references(scene, budget)
        assert len(prims) <= scene.n_prims * (1 + budget) + 1
        assert np.array_equal(np.unique(prims), np.arange(scene.n_prims))
