"""Scene-level instancing (dmap_scene_create_instanced): an object placed by
a rigid to_world transform answers a world-space ray as the object answers
the same ray moved to object space (the displaced surface moves rigidly:
S = R (P + h N) + t): the same hits and texels, t within 1e-7 relative
(the two Newton runs start from differently rounded rays and stop within
the residual tolerance), normals rotated; several instances answer with their nearest;
non-rigid transforms are refused."""
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


def test_non_rigid_refused(world):
    ctx, sc, assets, obj, Ms = world
    M = Ms[0].copy()
    M[:, :3] *= 2.0
    with pytest.raises(dm.DmapError) as e:
        dm.Scene.instanced(ctx, assets, sc.tris, sc.tri_asset, [0, len(sc.tris)], [0], M)
    assert e.value.status == 8
