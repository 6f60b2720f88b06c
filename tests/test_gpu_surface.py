"""Hit records to surface points (dmap_surface_points) against the oracle's
restatement of DisplacedGeometry::surface_point (displaced_geometry.cpp:
126-152): position, winding-oriented normal, uv-scaled tangents and object
uv, bit for bit, for FP64 and FP32 hit records, with and without a uv map."""
import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world(oracle):
    ctx = dm.Context(0)
    sc = helpers.small_sphere(32)
    return ctx, py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)


@pytest.mark.parametrize("hit_dtype", [np.float64, np.float32])
@pytest.mark.parametrize("uvmap", [((1.0, 1.0), (0.0, 0.0), False), ((4.0, 2.5), (0.25, -0.5), True)])
def test_surface_points_equal_oracle(world, hit_dtype, uvmap):
    ctx, cpu, dev = world
    rays = np.concatenate([scenes.sphere_camera_rays(64, 36), helpers.near_surface_rays(cpu, 1500)])
    hits = dev.intersect(rays, dm.TraversalOptions(leaf_precision="f64"), hit_dtype)
    sp = dev.surface_points(hits, *uvmap)
    hit = hits["tri"] >= 0
    assert hit.sum() > 300
    assert (sp[~hit] == 0).all()
    want = np.array([cpu.surface_point(int(h["tri"]), float(h["bary"][0]), float(h["bary"][1]), *uvmap)
                     for h in hits[hit]])
    assert np.array_equal(sp[hit], want)
    # the normal is unit and agrees with the hit's own geometric normal up to orientation
    assert np.allclose(np.linalg.norm(sp[hit, 3:6], axis=1), 1.0)
    assert (np.abs(np.sum(sp[hit, 3:6] * hits["ng"][hit], axis=1)) > 0.999).all()
