"""Scene-level instancing (dmap_scene_create_instanced): an object placed by
a rigid to_world transform answers a world-space ray as the object answers
the same ray moved to object space (the displaced surface moves rigidly:
S = R (P + h N) + t): the same hits and texels, t within 1e-7 relative
(the two Newton runs start from differently rounded rays and stop within
the residual tolerance), normals rotated; several instances answer with their nearest.
An affine transform that is not rigid (a scale or shear) keeps the object's
triangles and takes each ray to object space (x = Linv (w - T), t
unchanged, as the reference's instancing hands the instanced geometry its
ray): the same hits and t as the object's query of the moved ray, normals
moved as sign(det L) Linv^T n, surface points moved by L."""
import numpy as np
import pytest

import dmap_b200 as dm
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu


def _rigid(axis, angle, t, mirror=False):
    a = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    R = np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K
    if mirror:
        R = R @ np.diag([1.0, 1.0, -1.0])
    return np.concatenate([R, np.asarray(t, np.float64)[:, None]], 1)


@pytest.fixture(scope="module")
def world():
    ctx = dm.Context(0)
    sc = helpers.small_sphere(32, patches=(0, 1, 5, 16))
    assets = [dm.Asset(ctx, a.nodes, a.scale, a.offset, a.repeat) for a in sc.assets]
    obj = dm.Scene(ctx, assets, sc.tris, sc.tri_asset)
    Ms = [_rigid([0, 0, 1], 0.7, [3.0, 0.0, 0.0]), _rigid([1, 1, 0], -1.1, [-3.0, 0.5, 0.0]),
          _rigid([0.3, 1, 0.2], 2.0, [0.0, 3.0, 1.0], mirror=True)]
    return ctx, sc, assets, obj, Ms


def _rays_at(sc, M, n, seed):
    """World rays at the instance's base-surface points, from 2 units out
    along the normal, jittered."""
    R, t = M[:, :3], M[:, 3]
    p, m = scenes.base_points(sc, n, seed=seed)
    rng = np.random.default_rng(seed)
    pw, mw = p @ R.T + t, m @ R.T
    eye = pw + 2.0 * mw + (rng.random((n, 3)) - 0.5)
    rays = np.zeros((n, 8))
    rays[:, 0:3], rays[:, 3:6], rays[:, 7] = eye, pw - eye, np.inf
    return rays


def test_instance_equals_object_space(world):
    ctx, sc, assets, obj, Ms = world
    n_tri = len(sc.tris)
    for M in Ms:
        inst = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, n_tri], [0], M)
        R, t = M[:, :3], M[:, 3]
        rays = _rays_at(sc, M, 3000, 1)
        local = rays.copy()
        local[:, 0:3] = (rays[:, 0:3] - t) @ R     # R^T (o - t)
        local[:, 3:6] = rays[:, 3:6] @ R           # R^T d
        hw = inst.intersect(rays, dm.TraversalOptions(leaf_precision="f64"), np.float64)
        ho = obj.intersect(local, dm.TraversalOptions(leaf_precision="f64"), np.float64)
        hit = ho["tri"] >= 0
        assert hit.sum() > 500
        same = (hw["tri"] >= 0) == hit
        assert same.mean() > 0.999                  # grazing rays may flip on rounding
        both = hit & (hw["tri"] >= 0)
        assert (hw["tri"][both] == ho["tri"][both]).mean() > 0.999
        assert np.allclose(hw["t"][both], ho["t"][both], rtol=1e-7, atol=0)
        assert (hw["i"][both] == ho["i"][both]).mean() > 0.999
        ng = ho["ng"][both] @ R.T
        if np.linalg.det(R) < 0:
            ng = -ng   # the mirror flips Su x Sv
        assert np.abs(np.sum(ng * hw["ng"][both], axis=1)).min() > 1 - 1e-6


def test_instances_take_the_nearest(world):
    ctx, sc, assets, obj, Ms = world
    n_tri = len(sc.tris)
    M = np.stack(Ms)
    inst = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, n_tri], [0, 0, 0], M)
    assert inst.n_tri == 3 * n_tri
    rays = np.concatenate([_rays_at(sc, m, 1000, 2 + k) for k, m in enumerate(Ms)])
    h = inst.intersect(rays, dm.TraversalOptions(leaf_precision="f64"), np.float64)
    best_t = np.full(len(rays), np.inf)
    best_tri = np.full(len(rays), -1)
    for k, m in enumerate(Ms):
        one = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, n_tri], [0], m)
        hk = one.intersect(rays, dm.TraversalOptions(leaf_precision="f64"), np.float64)
        closer = (hk["tri"] >= 0) & (hk["t"] < best_t)
        best_t[closer] = hk["t"][closer]
        best_tri[closer] = hk["tri"][closer] + k * n_tri
    assert np.array_equal(h["tri"], best_tri)
    hit = best_tri >= 0
    assert hit.sum() > 1000 and np.allclose(h["t"][hit], best_t[hit], rtol=1e-12, atol=0)


def _affine(rigid_part, scale, shear, t):
    """A 3x4 to_world whose linear part is a rotation times a scale and shear."""
    S = np.diag(scale).astype(np.float64)
    S[0, 1] = shear
    L = rigid_part[:, :3] @ S
    return np.concatenate([L, np.asarray(t, np.float64)[:, None]], 1)


def _affine_rays(sc, M, n, seed):
    """World rays at the instance's base-surface points, from about 2 units
    out along the moved normal, jittered."""
    L, t = M[:, :3], M[:, 3]
    Li = np.linalg.inv(L)
    p, m = scenes.base_points(sc, n, seed=seed)
    rng = np.random.default_rng(seed)
    pw = p @ L.T + t
    mw = m @ Li
    mw /= np.linalg.norm(mw, axis=1, keepdims=True)
    eye = pw + 2.0 * mw + (rng.random((n, 3)) - 0.5)
    rays = np.zeros((n, 8))
    rays[:, 0:3], rays[:, 3:6], rays[:, 7] = eye, pw - eye, np.inf
    return rays


NON_RIGID = [(_rigid([0, 0, 1], 0.7, [0, 0, 0]), (1.5, 0.7, 1.0), 0.3, [2.0, -1.0, 0.5]),
             (_rigid([1, 1, 0], -1.1, [0, 0, 0], mirror=True), (0.6, 1.3, 2.0), -0.4, [-2.0, 0.5, 1.0])]


@pytest.mark.parametrize("k", [0, 1])
def test_non_rigid_instance_equals_object_space(world, k):
    ctx, sc, assets, obj, Ms = world
    rot, scale, shear, t = NON_RIGID[k]
    M = _affine(rot, scale, shear, t)
    L, T = M[:, :3], M[:, 3]
    Li = np.linalg.inv(L)
    inst = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, len(sc.tris)], [0], M)
    rays = _affine_rays(sc, M, 3000, 5 + k)
    local = rays.copy()
    local[:, 0:3] = (rays[:, 0:3] - T) @ Li.T
    local[:, 3:6] = rays[:, 3:6] @ Li.T
    for leaf, rtol in (("f64", 1e-9), ("f32", 1e-6)):
        for schedule in ("wavefront", "simple"):
            opt = dm.TraversalOptions(leaf_precision=leaf, schedule=schedule, order="index")
            hw = inst.intersect(rays, opt, np.float64)
            ho = obj.intersect(local, opt, np.float64)
            hit = ho["tri"] >= 0
            assert hit.sum() > 500
            assert ((hw["tri"] >= 0) == hit).mean() > 0.999
            both = hit & (hw["tri"] >= 0)
            assert (hw["tri"][both] == ho["tri"][both]).mean() > 0.999
            assert np.allclose(hw["t"][both], ho["t"][both], rtol=rtol, atol=0)
            assert np.abs(hw["st"][both] - ho["st"][both]).max() < 1e-6
            ng = ho["ng"][both] @ Li * np.sign(np.linalg.det(L))
            ng /= np.linalg.norm(ng, axis=1, keepdims=True)
            assert np.abs(np.sum(ng * hw["ng"][both], axis=1)).min() > 1 - 1e-6
            assert (np.sum(ng * hw["ng"][both], axis=1) > 0).all()
    # surface points are the object's moved by L
    hw = inst.intersect(rays, dm.TraversalOptions(leaf_precision="f64", order="index"), np.float64)
    ho = obj.intersect(local, dm.TraversalOptions(leaf_precision="f64", order="index"), np.float64)
    both = (ho["tri"] >= 0) & (hw["tri"] == ho["tri"])
    sw, so = inst.surface_points(hw[both]), obj.surface_points(ho[both])
    assert np.allclose(sw[:, 0:3], so[:, 0:3] @ L.T + T, rtol=0, atol=1e-7)
    assert np.allclose(sw[:, 6:9], so[:, 6:9] @ L.T, rtol=0, atol=1e-7)


def test_mixed_instances_take_the_nearest(world):
    """A rigid and a non-rigid instance in one scene: each ray's hit is the
    nearer of the two single-instance scenes' hits."""
    ctx, sc, assets, obj, Ms = world
    n_tri = len(sc.tris)
    rot, scale, shear, t = NON_RIGID[0]
    Ma = _affine(rot, scale, shear, t)
    Mr = Ms[1]
    both_M = np.stack([Ma, Mr])
    inst = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, n_tri], [0, 0], both_M)
    rays = np.concatenate([_affine_rays(sc, Ma, 1500, 11), _rays_at(sc, Mr, 1500, 12)])
    opt = dm.TraversalOptions(leaf_precision="f64")
    h = inst.intersect(rays, opt, np.float64)
    best_t = np.full(len(rays), np.inf)
    best_tri = np.full(len(rays), -1)
    for k, m in enumerate([Ma, Mr]):
        # a single non-rigid instance keeps the transform path; the rigid one
        # alone would be flattened, so pair it with an identity-scaled copy
        one = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, n_tri], [0], m) if k == 0 else \
            dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, n_tri], [0, 0],
                               np.stack([_affine(np.eye(3, 4), (1e-3, 1e-3, 1e-3), 0.0, [50.0, 50.0, 50.0]), m]))
        hk = one.intersect(rays, opt, np.float64)
        tri_k = hk["tri"] if k == 0 else np.where(hk["tri"] >= n_tri, hk["tri"] - n_tri, -1)
        closer = (tri_k >= 0) & (hk["t"] < best_t)
        best_t[closer] = hk["t"][closer]
        best_tri[closer] = tri_k[closer] + k * n_tri
    hit = best_tri >= 0
    assert hit.sum() > 1500
    assert (h["tri"] == best_tri).mean() > 0.999
    same = hit & (h["tri"] == best_tri)
    assert np.allclose(h["t"][same], best_t[same], rtol=1e-9, atol=0)


def test_non_rigid_tessellation_refused(world):
    ctx, sc, assets, obj, Ms = world
    rot, scale, shear, t = NON_RIGID[0]
    inst = dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, len(sc.tris)], [0],
                              _affine(rot, scale, shear, t))
    with pytest.raises(dm.DmapError) as e:
        inst.tessellate_uniform(2)
    assert e.value.status == 8
