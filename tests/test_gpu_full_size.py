"""Parity at the benchmark's own sizes: the FP32 product path against the
CPU oracle on the plain-method configurations as the benchmark runs them,
not on reduced maps.

- The small plain-method case exactly: one unit quad displaced by a 512^2
  map, 256 x 256 camera rays (65,536), every ray against the oracle.
- The GPU-scale case's real scene: 96 patches of 2048^2 FP32 maps (L = 11,
  5.59M pyramid cells each). The benchmark's own rays (1920 x 1080 jittered
  primaries and one bounce per primary hit) are answered on the device in
  full; a stride sample of them (primaries and bounces in proportion, every
  patch) goes through the oracle's flat loop over all 96 patches, evaluated
  a group of patches at a time. Every record must be the oracle's, bit for
  bit; on the whole ray list the FP32 path equals the FP64 device path.
- The precision variant: the same scene with FP16 texels (the oracle sees
  them widened to double) and seeded grazing rays 0.1-5 degrees above the
  base surface, which stress the conservative FP32 bounds.
These tests hold up to about 55 GB of device memory and take a few minutes
(the 96 oracle pyramids are built on the host, 16 at a time: about 7 GB)."""
import os

import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
FIELDS = ("t", "st", "bary", "ng", "i", "j")


def _release(ctx, dev):
    """Frees the scene's device memory before the next test builds its own."""
    dev.close()
    for a in dev.assets:
        a.close()
    ctx.close()


def _equal_records(h, ho, what):
    """Device records (HIT64) against oracle records (n x 12 doubles)."""
    assert np.array_equal(h["tri"], ho[:, 10].astype(np.int32)), f"{what}: hit set or triangle differs"
    hit = ho[:, 10] >= 0
    cols = {"t": ho[:, 0], "st": ho[:, 1:3], "bary": ho[:, 3:5], "ng": ho[:, 5:8], "i": ho[:, 8], "j": ho[:, 9]}
    for f in FIELDS:
        got = h[f][hit]
        want = cols[f][hit]
        if f in ("i", "j"):
            want = want.astype(np.int32)
        assert np.array_equal(got, want), f"{what}: {f} differs from the oracle"
    return int(hit.sum())


def test_quad_512_all_camera_rays(oracle):
    sc = scenes.quad_scene(512)
    rays = scenes.quad_camera_rays(256, 256)
    assert len(rays) == 65536
    ctx = dm.Context(0)
    dev = dm.Scene.from_synthetic(ctx, sc)
    cpu = py_oracle.CpuScene(oracle, sc)
    for order in ("index", "nearest"):
        ho, _ = cpu.intersect(rays, order=order, threads=THREADS)
        h = dev.intersect(rays, dm.TraversalOptions(precision="f32", order=order, leaf_precision="f64"))
        n = _equal_records(h, ho, f"quad 512, {order} order")
        assert n > 20000  # the 45 degree view sees the quad in about a third of its pixels
    _release(ctx, dev)


@pytest.fixture(scope="module")
def sphere():
    return scenes.sphere_benchmark_scene(2048, np.float32, min(16, THREADS))


def _bench_rays(dev, prim):
    """The benchmark's ray list: primaries, then one bounce per primary hit
    from the FP64 path's hits in the flat loop's order."""
    h0 = dev.intersect(prim, dm.TraversalOptions(precision="f64", order="index", leaf_precision="f64"))
    hit = h0["tri"] >= 0
    bounce = scenes.bounce_rays(prim[hit], h0["t"][hit], h0["ng"][hit])
    return np.concatenate([prim, bounce]).astype(np.float32), int(hit.sum())


def test_sphere_2048_benchmark_rays(oracle, sphere):
    ctx = dm.Context(0)
    dev = dm.Scene.from_synthetic(ctx, sphere, keep_f64=True)
    prim = scenes.sphere_camera_rays(1920, 1080)
    rays, n_prim_hits = _bench_rays(dev, prim)
    assert len(rays) == len(prim) + n_prim_hits
    # every ray: the product path (both orders) equals the FP64 device path
    for order in ("nearest", "index"):
        h32 = dev.intersect(rays, dm.TraversalOptions(precision="f32", order=order, leaf_precision="f64"))
        h64 = dev.intersect(rays, dm.TraversalOptions(precision="f64", order=order, leaf_precision="f64"))
        assert np.array_equal(h32["tri"], h64["tri"]), f"{order}: FP32 and FP64 hit sets differ"
        hit = h64["tri"] >= 0
        for f in FIELDS:
            assert np.array_equal(h32[f][hit], h64[f][hit]), f"{order}: {f} differs between FP32 and FP64"
    # a stride sample through the CPU oracle's flat loop over all 96 patches
    sample = np.ascontiguousarray(rays[::97])
    ho = helpers.oracle_flat_loop_by_groups(oracle, sphere, sample, group=16, threads=THREADS)
    h = dev.intersect(sample, dm.TraversalOptions(precision="f32", order="index", leaf_precision="f64"))
    n = _equal_records(h, ho, "sphere 96 x 2048^2")
    assert n > len(sample) // 4 and len(sample) > 25000
    _release(ctx, dev)


def test_sphere_2048_f16_grazing_rays(oracle, sphere):
    sc16 = scenes.Scene([scenes.Asset(a.nodes.astype(np.float16), a.scale, a.offset, a.repeat)
                         for a in sphere.assets], sphere.tris, sphere.tri_asset, name=sphere.name + "_f16",
                        extent=sphere.extent)
    ctx = dm.Context(0)
    dev = dm.Scene.from_synthetic(ctx, sc16)
    p, m = scenes.base_points(sc16, 60_000, seed=scenes.SEED + 7)
    rays = scenes.grazing_rays(p, m, seed=scenes.SEED + 8)
    h = dev.intersect(rays, dm.TraversalOptions(precision="f32", order="index", leaf_precision="f64"))
    ho = helpers.oracle_flat_loop_by_groups(oracle, sc16, rays, group=16, threads=THREADS)
    n = _equal_records(h, ho, "sphere 96 x 2048^2 FP16, grazing")
    # rays aimed at the base surface mostly find the displaced one
    assert n > len(rays) // 2
    _release(ctx, dev)
