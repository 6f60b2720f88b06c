"""Parity of the CUDA path with the oracle, through the C ABI.

FP64 precision: the device pyramid and the device walk follow the
reference's double arithmetic operation for operation, so pyramids, setup
records, hits and counters must equal the oracle exactly."""
from pathlib import Path

import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
CHANNELS = dm.CHANNELS


@pytest.fixture(scope="module")
def ctx():
    return dm.Context(0)


@pytest.mark.parametrize("case", ["random_65", "random_33", "step_17", "ramp_17"])
def test_device_pyramid_equals_golden(ctx, case):
    z = np.load(GOLDEN / f"pyramid_{case}.npz")
    a = dm.Asset(ctx, z["values"], float(z["scale"][0]), keep_f64=True)
    for k in range(a.n_levels):
        lv = a.level(k, "f64")
        lf = a.level(k, "f32")
        for ch in CHANNELS:
            assert np.array_equal(lv[ch], z[f"fold/{ch}_L{k}"]), (case, k, ch)
        # the FP32 node encloses the FP64 one
        assert (lf["h_min"] <= lv["h_min"]).all() and (lf["h_max"] >= lv["h_max"]).all()
        for c, rc in (("h0", "r"), ("gu", "ru"), ("gv", "rv")):
            assert (np.abs(lf[c] - lv[c]) + lv[rc] <= lf[rc]).all(), (case, k, c)


@pytest.mark.parametrize("dtype,scale,offset,repeat", [(np.float32, 1.0, 0.0, False), (np.float16, 0.7, -0.2, True),
                                                       (np.float64, 0.013, 0.5, False)])
def test_device_pyramid_equals_oracle(ctx, oracle, dtype, scale, offset, repeat):
    rng = np.random.default_rng(3)
    v = rng.random((129, 129)).astype(dtype)
    a = dm.Asset(ctx, v, scale, offset, repeat, keep_f64=True)
    ref = oracle.pyramid(v.astype(np.float64), scale, offset)
    assert a.n_levels == len(ref)
    for k, lv in enumerate(ref):
        got = a.level(k, "f64")
        for ch in CHANNELS:
            assert np.array_equal(got[ch], lv[ch]), (k, ch)


@pytest.mark.parametrize("build", ["fold", "direct"])
def test_device_pyramid_bf16_equals_oracle(ctx, oracle, build):
    """BF16 texels: the device pyramid of the bfloat16 grid equals the
    oracle's pyramid of the same values widened to double."""
    rng = np.random.default_rng(5)
    v = rng.random((129, 129)) * 2.0 - 1.0
    a = dm.Asset(ctx, v, 0.3, 0.1, True, keep_f64=True, build=build, texel="bf16")
    ref = oracle.pyramid(dm.from_bf16(dm.to_bf16(v)), 0.3, 0.1, build)
    assert a.n_levels == len(ref)
    for k, lv in enumerate(ref):
        got = a.level(k, "f64")
        for ch in CHANNELS:
            assert np.array_equal(got[ch], lv[ch]), (k, ch)


def _compare(cpu, dev, rays, bound="both", k=1, leaf="newton", order="nearest"):
    ho, so = cpu.intersect(rays, bound, k, leaf, stats=True, order=order)
    hd, sd = dev.intersect(rays, dm.TraversalOptions(bound, k, leaf, precision="f64", order=order, leaf_precision="f64"), np.float64,
                           stats=True)
    assert np.array_equal(hd["tri"], ho[:, 10].astype(np.int32))
    hit = ho[:, 10] >= 0
    assert np.array_equal(hd["t"][hit], ho[hit, 0])
    assert np.array_equal(hd["st"][hit], ho[hit, 1:3])
    assert np.array_equal(hd["bary"][hit], ho[hit, 3:5])
    assert np.array_equal(hd["ng"][hit], ho[hit, 5:8])
    assert np.array_equal(hd["i"][hit], ho[hit, 8].astype(np.int32))
    assert np.array_equal(hd["j"][hit], ho[hit, 9].astype(np.int32))
    assert np.isinf(hd["t"][~hit]).all()
    assert np.array_equal(sd[:, :7], so[:, :7])
    return hit.sum()


@pytest.fixture(scope="module")
def quad_pair(ctx, oracle):
    sc = scenes.quad_scene(64)
    return py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc, keep_f64=True)


@pytest.fixture(scope="module")
def sphere_pair(ctx, oracle):
    sc = helpers.small_sphere(32)
    return py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc, keep_f64=True)


def test_setup_equals_oracle(quad_pair, sphere_pair):
    for cpu, dev in (quad_pair, sphere_pair):
        for t in range(cpu.n_tri):
            assert np.array_equal(dev.triangle_info(t), cpu.triangle_info(t)), t


@pytest.mark.parametrize("bound,k", [("both", 1), ("box", 1), ("slab", 6), ("both", 0)])
def test_f64_walk_equals_oracle_quad(quad_pair, bound, k):
    cpu, dev = quad_pair
    rays = np.concatenate([scenes.quad_camera_rays(64, 64), helpers.near_surface_rays(cpu, 1500),
                           helpers.aimed_rays(cpu, 1500)[0]])
    assert _compare(cpu, dev, rays, bound, k) > 1000


@pytest.mark.parametrize("order", ["nearest", "index"])
def test_f64_walk_equals_oracle_sphere(sphere_pair, order):
    """Both triangle orders: the nearest-first one and the reference's flat loop."""
    cpu, dev = sphere_pair
    rays = np.concatenate([scenes.sphere_camera_rays(96, 54), helpers.near_surface_rays(cpu, 1500),
                           helpers.aimed_rays(cpu, 1500)[0]])
    assert _compare(cpu, dev, rays, order=order) > 1000


def test_f64_two_triangle_leaf_equals_oracle(quad_pair):
    cpu, dev = quad_pair
    rays = np.concatenate([scenes.quad_camera_rays(32, 32), helpers.near_surface_rays(cpu, 800)])
    _compare(cpu, dev, rays, leaf="two_triangle")
    _compare(cpu, dev, rays, leaf="two_triangle", order="index")


def test_f64_float64_rays(sphere_pair):
    """Rays in double reach the walk unrounded (the drop-in signature)."""
    cpu, dev = sphere_pair
    rays = helpers.near_surface_rays(cpu, 500).astype(np.float64)
    rays[:, 0:3] += 1e-9  # not representable in float32
    ho, _ = cpu.intersect(rays)
    hd = dev.intersect(rays, dm.TraversalOptions(precision="f64", leaf_precision="f64"), np.float64)
    assert np.array_equal(hd["t"], ho[:, 0])


def test_f64_occluded_matches_closest(sphere_pair):
    """occluded_callback (displaced_geometry.cpp:79-106): a ray is occluded
    iff the closest-hit walk within (t_min, t_max) finds a hit."""
    cpu, dev = sphere_pair
    rays = np.concatenate([scenes.sphere_camera_rays(48, 27), helpers.near_surface_rays(cpu, 800)])
    rays[:, 7] = np.where(np.arange(len(rays)) % 2 == 0, 2.0, np.inf)
    closest = dev.intersect(rays, dm.TraversalOptions(precision="f64", leaf_precision="f64"))
    occl = dev.intersect(rays, dm.TraversalOptions(precision="f64", mode="occluded", leaf_precision="f64"))
    assert np.array_equal(closest["tri"] >= 0, occl["tri"] >= 0)


@pytest.mark.parametrize("n,dtype,scale,offset", [(65, np.float32, 1.0, 0.0), (129, np.float16, 0.7, -0.2),
                                                  (257, np.float64, 0.013, 0.5)])
def test_device_direct_pyramid_equals_oracle(ctx, oracle, n, dtype, scale, offset):
    """The Direct build (every level from the node grid) == the oracle's,
    bit for bit, in FP64; the FP32 levels enclose them."""
    rng = np.random.default_rng(5)
    v = rng.random((n, n)).astype(dtype)
    a = dm.Asset(ctx, v, scale, offset, keep_f64=True, build="direct")
    ref = oracle.pyramid(v.astype(np.float64), scale, offset, build="direct")
    assert a.n_levels == len(ref)
    for k, lv in enumerate(ref):
        got = a.level(k, "f64")
        for ch in CHANNELS:
            assert np.array_equal(got[ch], lv[ch]), (k, ch)
        f = a.level(k, "f32")
        assert (f["h_min"] <= lv["h_min"]).all() and (f["h_max"] >= lv["h_max"]).all()


def test_direct_build_walk_equals_oracle(ctx, oracle):
    """A scene on Direct-built pyramids: the FP64 and FP32 paths' hits == the
    oracle's on the same build."""
    sc = scenes.quad_scene(64)
    cpu = py_oracle.CpuScene(oracle, sc, build="direct")
    dev = dm.Scene.from_synthetic(ctx, sc, keep_f64=True, build="direct")
    rays = np.concatenate([scenes.quad_camera_rays(48, 48), helpers.near_surface_rays(cpu, 1500)])
    _compare(cpu, dev, rays)
    ho, _ = cpu.intersect(rays)
    h32 = dev.intersect(rays, dm.TraversalOptions(precision="f32", leaf_precision="f64"), np.float64)
    assert np.array_equal(h32["tri"], ho[:, 10].astype(np.int32))
    hit = ho[:, 10] >= 0
    assert np.array_equal(h32["t"][hit], ho[hit, 0])
