"""The FP32 path against the oracle: the walk's node tests are FP32 and
widened outward, the leaves are the reference's FP64 leaf, so the hit set
must equal the oracle's and every reported hit record (t, st, bary, ng, i, j)
must be the oracle's, bit for bit; a ray the FP64 walk finds a root for
reaches a leaf here too (conservative bounds)."""
import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return dm.Context(0)


def _check(cpu, dev, rays, bound="both", k=1, order="nearest", **kw):
    ho, so = cpu.intersect(rays, bound, k, stats=True, order=order)
    hd, sd = dev.intersect(rays, dm.TraversalOptions(bound, k, precision="f32", order=order, **kw, leaf_precision="f64"), np.float64,
                           stats=True)
    assert np.array_equal(hd["tri"] >= 0, ho[:, 10] >= 0), "hit/miss set differs"
    hit = ho[:, 10] >= 0
    assert np.array_equal(hd["tri"][hit], ho[hit, 10].astype(np.int32))
    assert np.array_equal(hd["t"][hit], ho[hit, 0]), "t differs from the oracle's FP64 root"
    assert np.array_equal(hd["st"][hit], ho[hit, 1:3]) and np.array_equal(hd["bary"][hit], ho[hit, 3:5])
    assert np.array_equal(hd["ng"][hit], ho[hit, 5:8])
    assert np.array_equal(hd["i"][hit], ho[hit, 8].astype(np.int32))
    assert np.array_equal(hd["j"][hit], ho[hit, 9].astype(np.int32))
    # the FP32 bounds enclose the surface: a ray whose FP64 walk finds a root
    # reaches that root's leaf here too
    got = hd["tri"] >= 0
    assert (sd[got, 2] >= 1).all()
    return hit.sum(), float((sd[:, 1].sum() / max(so[:, 1].sum(), 1)))


@pytest.mark.parametrize("bound,k", [("both", 1), ("box", 1), ("slab", 6)])
def test_f32_quad(ctx, oracle, bound, k):
    sc = scenes.quad_scene(64)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([scenes.quad_camera_rays(64, 64), helpers.near_surface_rays(cpu, 2000),
                           helpers.aimed_rays(cpu, 2000)[0]])
    n, ratio = _check(cpu, dev, rays, bound, k)
    assert n > 1000 and ratio < 1.5


@pytest.mark.parametrize("schedule,rounds,bps,order", [("wavefront", 6, 4, "nearest"), ("wavefront", 0, 1, "nearest"),
                                                       ("wavefront", 1, 2, "nearest"), ("wavefront", 32, 4, "nearest"),
                                                       ("simple", 6, 4, "nearest"), ("wavefront", 6, 4, "index"),
                                                       ("wavefront", 1, 2, "index"), ("simple", 6, 4, "index")])
def test_f32_sphere(ctx, oracle, schedule, rounds, bps, order):
    """Every schedule and both triangle orders give the oracle's hits;
    rounds = 0 runs everything in the inline-leaf walk, rounds = 1 parks
    each ray once."""
    sc = helpers.small_sphere(32)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([scenes.sphere_camera_rays(96, 54), helpers.near_surface_rays(cpu, 2000),
                           helpers.aimed_rays(cpu, 2000)[0]])
    n, ratio = _check(cpu, dev, rays, order=order, schedule=schedule, rounds=rounds, blocks_per_sm=bps)
    assert n > 1000 and ratio < 1.5


def test_f32_schedules_agree_bitwise(ctx, oracle):
    """The wavefront and the simple schedule return the same records."""
    sc = helpers.small_sphere(32)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([scenes.sphere_camera_rays(64, 36), helpers.near_surface_rays(cpu, 1500)])
    a, sa = dev.intersect(rays, dm.TraversalOptions(schedule="wavefront", leaf_precision="f64"), np.float64, stats=True)
    b, sb = dev.intersect(rays, dm.TraversalOptions(schedule="simple", leaf_precision="f64"), np.float64, stats=True)
    assert np.array_equal(a["tri"], b["tri"])
    hit = a["tri"] >= 0
    assert np.array_equal(a["t"][hit], b["t"][hit]) and np.array_equal(a["ng"][hit], b["ng"][hit])
    # the wavefront walk may run leaves past a hit that the simple walk prunes
    assert (sa[:, 2] >= sb[:, 2]).all()


def test_f32_f16_texels_and_offset(ctx, oracle):
    """FP16 texels (the precision variant): the oracle sees them widened to double."""
    sc = helpers.small_sphere(64, patches=(0, 1, 2, 17))
    for a in sc.assets:
        a.nodes = a.nodes.astype(np.float16)
        a.scale, a.offset = 0.9, 0.01
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([helpers.near_surface_rays(cpu, 2000), helpers.aimed_rays(cpu, 2000)[0]])
    _check(cpu, dev, rays)


def test_f32_bf16_texels(ctx, oracle):
    """BF16 texels: the device stores bfloat16, the oracle sees the same
    values widened to double; every hit record equals the oracle's."""
    sc = helpers.small_sphere(64, patches=(0, 1, 2, 17))
    for a in sc.assets:
        a.nodes = dm.from_bf16(dm.to_bf16(a.nodes))
        a.scale, a.offset = 0.9, 0.01
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc, texel="bf16")
    rays = np.concatenate([helpers.near_surface_rays(cpu, 2000), helpers.aimed_rays(cpu, 2000)[0]])
    n, _ = _check(cpu, dev, rays)
    assert n > 1000


def test_f32_never_miss(ctx, oracle):
    sc = helpers.small_sphere(32)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays, t_s, miss_dist, _ = helpers.aimed_rays(cpu, 4000, seed=91)
    h = dev.intersect(rays, dm.TraversalOptions(precision="f32", leaf_precision="f64"))
    ok = miss_dist < 1e-6
    assert (h["tri"][ok] >= 0).all()


def test_f32_occluded(ctx, oracle):
    sc = helpers.small_sphere(32)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = helpers.near_surface_rays(cpu, 3000)
    rays[:, 7] = np.where(np.arange(len(rays)) % 2 == 0, 1.0, np.inf)
    ho, _ = cpu.intersect(rays)
    h = dev.intersect(rays, dm.TraversalOptions(precision="f32", mode="occluded", leaf_precision="f64"))
    assert np.array_equal(h["tri"] >= 0, ho[:, 10] >= 0)


def test_f32_grazing_rays_f16(ctx, oracle):
    """The precision variant's stress case: FP16 texels and rays 0.1-5 deg
    above the tangent plane, aimed at base-surface points, some aimed at
    displaced surface points; every hit record equals the oracle's."""
    sc = helpers.small_sphere(64, patches=(0, 1, 5, 16))
    for a in sc.assets:
        a.nodes = a.nodes.astype(np.float16)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    p, m = scenes.base_points(sc, 3000, seed=77)
    rng = np.random.default_rng(78)
    _, _, S = helpers.surface_points(cpu, rng, 1000)
    nrm = S / np.linalg.norm(S, axis=1, keepdims=True)   # sphere patches: radial normals
    rays = np.concatenate([scenes.grazing_rays(p, m, seed=79), scenes.grazing_rays(S, nrm, seed=80)])
    n, _ = _check(cpu, dev, rays)
    assert n > 1000


@pytest.mark.parametrize("n,k", [(16, 8), (8, 24)])
def test_f32_many_triangles_tree(ctx, oracle, n, k):
    """Scenes of more than 256 triangles (768 and 6912) take their candidates
    from the triangle tree in both orders; hits equal the oracle's loops and
    the simple schedule's."""
    sc = scenes.cube_sphere_scene(n, k)
    assert len(sc.tris) > 256
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([scenes.sphere_camera_rays(96, 54), helpers.near_surface_rays(cpu, 1500),
                           helpers.aimed_rays(cpu, 1500)[0]])
    for order in ("nearest", "index"):
        n_hit, _ = _check(cpu, dev, rays, order=order)
        assert n_hit > 1000
        a = dev.intersect(rays, dm.TraversalOptions(schedule="wavefront", order=order, leaf_precision="f64"), np.float64)
        b = dev.intersect(rays, dm.TraversalOptions(schedule="simple", order=order, leaf_precision="f64"), np.float64)
        assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("k", [30, 40])
def test_f32_many_triangles_large_tree(ctx, oracle, k):
    """Scenes of 10800 and 19200 triangles (deeper trees): hits equal the
    oracle's in both triangle orders, and the simple schedule's; occlusion
    agrees with the closest hits."""
    sc = scenes.cube_sphere_scene(8, k)
    assert len(sc.tris) > 8192
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([scenes.sphere_camera_rays(96, 54), helpers.near_surface_rays(cpu, 1500),
                           helpers.aimed_rays(cpu, 1500)[0]])
    for order in ("nearest", "index"):
        n_hit, _ = _check(cpu, dev, rays, order=order)
        assert n_hit > 1000
        a = dev.intersect(rays, dm.TraversalOptions(schedule="wavefront", order=order, leaf_precision="f64"), np.float64)
        b = dev.intersect(rays, dm.TraversalOptions(schedule="simple", order=order, leaf_precision="f64"), np.float64)
        assert a.tobytes() == b.tobytes()
    occ = dev.intersect(rays, dm.TraversalOptions(mode="occluded", leaf_precision="f64"), np.float64)
    assert np.array_equal(occ["tri"] >= 0, a["tri"] >= 0)


@pytest.mark.parametrize("k", [16, 48])
def test_f32_nearest_tree_refills(ctx, oracle, k):
    """The nearest order over more than 256 triangles takes its candidates
    from the triangle tree, eight at a time: rays grazing a cube sphere of
    small patches (3072 and 27648 triangles) pass over more than eight
    triangle boxes, so the buffer is refilled past its last entry; every
    hit record equals the oracle's nearest-order loop, on both schedules,
    the FP32 leaf within its tolerance of it."""
    sc = scenes.cube_sphere_scene(8, k, amplitude=0.08 * 4 / k)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    p, m = scenes.base_points(sc, 3000, seed=91)
    rays = np.concatenate([scenes.grazing_rays(p, m, seed=92), helpers.near_surface_rays(cpu, 1500),
                           scenes.sphere_camera_rays(64, 36)])
    ho, so = cpu.intersect(rays, stats=True, order="nearest")
    assert so[:, 0].max() > 8, "no ray walked more than eight triangles"
    for schedule in ("wavefront", "simple"):
        n_hit, _ = _check(cpu, dev, rays, order="nearest", schedule=schedule)
        assert n_hit > 1000
    h32 = dev.intersect(rays, dm.TraversalOptions(order="nearest"), np.float64)
    from test_gpu_leaf32 import judge
    judge(h32, ho, rays, sc.extent)


@pytest.mark.parametrize("tree", [False, True])
def test_f32_default_launch_shape(ctx, tree):
    """blocks_per_sm 0 (the default) launches the walk at the occupancy it is
    compiled for (4 CTAs per SM over the candidate mask, 5 over the triangle
    tree); its records equal those of explicit launch shapes, fewer and more
    CTAs than can be resident, bit for bit."""
    assert dm.TraversalOptions().blocks_per_sm == 0
    sc = scenes.cube_sphere_scene(16, 8 if tree else 4)   # 768 or 192 triangles
    assert (len(sc.tris) > 256) == tree
    dev = dm.Scene.from_synthetic(ctx, sc)
    rays = scenes.sphere_camera_rays(128, 72)
    ref = dev.intersect(rays, dm.TraversalOptions(), np.float64)
    assert (ref["tri"] >= 0).sum() > 1000
    for bps in (1, 3, 4, 5, 8):
        got = dev.intersect(rays, dm.TraversalOptions(blocks_per_sm=bps), np.float64)
        assert got.tobytes() == ref.tobytes(), bps
