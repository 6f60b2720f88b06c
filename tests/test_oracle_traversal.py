"""The oracle's traversal against the reference compiled here (bit for bit),
and the invariants the reference's validate_traversal.cpp checks."""
import numpy as np
import pytest

import py_oracle
from dmap_b200 import scenes
import helpers


@pytest.fixture(scope="module")
def quad():
    return scenes.quad_scene(64)


@pytest.fixture(scope="module")
def sphere():
    return helpers.small_sphere(32)


def _all_rays(cpu, scene, camera):
    return np.concatenate([camera, helpers.near_surface_rays(cpu, 800), helpers.aimed_rays(cpu, 800)[0]])


@pytest.mark.parametrize("bound,k", [("both", 1), ("box", 1), ("slab", 3), ("both", 0)])
def test_oracle_equals_reference_quad(oracle, reference, quad, bound, k):
    so, sr = py_oracle.CpuScene(oracle, quad), py_oracle.CpuScene(reference, quad)
    for t in range(so.n_tri):
        assert np.array_equal(so.triangle_info(t), sr.triangle_info(t))
        assert np.array_equal(so.triangle_frame(t), sr.triangle_frame(t))
    rays = _all_rays(so, quad, scenes.quad_camera_rays(48, 48))
    ho, sto = so.intersect(rays, bound, k, stats=True, order="index")
    hr, st_r = sr.intersect(rays, bound, k, stats=True, order="index")
    assert np.array_equal(ho, hr)
    cols = [0, 1, 2, 3, 5, 6]
    assert np.array_equal(sto[:, cols], st_r[:, cols])
    assert np.isfinite(ho[:, 0]).sum() > 500


def test_oracle_equals_reference_two_triangle_leaf(oracle, reference, quad):
    so, sr = py_oracle.CpuScene(oracle, quad), py_oracle.CpuScene(reference, quad)
    rays = _all_rays(so, quad, scenes.quad_camera_rays(32, 32))
    assert np.array_equal(so.intersect(rays, leaf="two_triangle", order="index")[0],
                          sr.intersect(rays, leaf="two_triangle", order="index")[0])


def test_oracle_equals_reference_sphere(oracle, reference, sphere):
    so, sr = py_oracle.CpuScene(oracle, sphere), py_oracle.CpuScene(reference, sphere)
    for t in range(so.n_tri):
        assert np.array_equal(so.triangle_info(t), sr.triangle_info(t))
    rays = np.concatenate([scenes.sphere_camera_rays(64, 36), helpers.near_surface_rays(so, 600),
                           helpers.aimed_rays(so, 600)[0]])
    ho, sto = so.intersect(rays, stats=True, order="index")
    hr, st_r = sr.intersect(rays, stats=True, order="index")
    assert np.array_equal(ho, hr)
    assert np.array_equal(sto[:, [0, 1, 2, 3, 5, 6]], st_r[:, [0, 1, 2, 3, 5, 6]])


def test_node_bound_equals_reference(oracle, reference, sphere):
    so, sr = py_oracle.CpuScene(oracle, sphere), py_oracle.CpuScene(reference, sphere)
    rng = np.random.default_rng(5)
    rays = helpers.near_surface_rays(so, 50)
    for r in rays:
        tri = int(rng.integers(so.n_tri))
        level = int(rng.integers(0, 6))
        m = 32 >> level
        i, j = int(rng.integers(m)), int(rng.integers(m))
        a = so.node_bound(tri, level, i, j, r.astype(np.float64))
        b = sr.node_bound(tri, level, i, j, r.astype(np.float64))
        assert np.array_equal(a, b, equal_nan=True)


def test_mode_invariance(oracle, sphere):
    """validate_traversal.cpp:313-388 (3): every bound mode and level policy
    gives the same hits, t within 4 residual tolerances."""
    so = py_oracle.CpuScene(oracle, sphere)
    rays = np.concatenate([scenes.sphere_camera_rays(48, 27), helpers.near_surface_rays(so, 600)])
    ref, _ = so.intersect(rays)
    tol = np.array([so.triangle_info(t)[2] for t in range(so.n_tri)])
    for bound, k in [("box", 5), ("slab", 5), ("both", 5), ("both", 0), ("both", 2)]:
        got, _ = so.intersect(rays, bound, k)
        hit = np.isfinite(ref[:, 0])
        assert np.array_equal(hit, np.isfinite(got[:, 0])), (bound, k)
        tri = ref[hit, 10].astype(int)
        assert (np.abs(ref[hit, 0] - got[hit, 0]) <= 4 * tol[tri] + 1e-12 * (ref[hit, 0] + 4)).all()


def test_never_miss_and_residual(oracle, sphere):
    """validate_traversal.cpp:392-461 (4) and :210-237 (2): rays aimed at
    surface points hit at or before them; Newton hits lie within 2
    tolerances of the surface, inside their leaf and the domain."""
    so = py_oracle.CpuScene(oracle, sphere)
    rays, t_s, miss_dist, _ = helpers.aimed_rays(so, 1500, seed=77)
    hits, _ = so.intersect(rays)
    tol = np.array([so.triangle_info(t)[2] for t in range(so.n_tri)])
    ok = miss_dist < 1e-6   # float32 rounding of the ray moved it off the point
    hit = np.isfinite(hits[:, 0])
    assert hit[ok].all()
    d = rays[:, 3:6].astype(np.float64)
    cos = np.abs(np.sum(d * hits[:, 5:8], axis=1)) / np.linalg.norm(d, axis=1)
    slack = 1e-9 * (t_s + 4) + 4 * tol[np.maximum(hits[:, 10].astype(int), 0)] / np.maximum(cos, 1e-3)
    slack += miss_dist / np.maximum(cos, 1e-3)
    assert (hits[hit, 0] <= t_s[hit] + slack[hit]).all()
    for r in np.nonzero(hit)[0][:300]:
        tri = int(hits[r, 10])
        S = so.displaced_position(tri, hits[r, 1], hits[r, 2])
        p = rays[r, 0:3].astype(np.float64) + hits[r, 0] * rays[r, 3:6].astype(np.float64)
        assert np.linalg.norm(S - p) <= 2 * tol[tri] + 1e-12


@pytest.mark.parametrize("name", ["quad", "sphere"])
def test_nearest_order_same_hits(oracle, quad, sphere, name):
    """The nearest-first triangle order finds the flat loop's hits: the same
    hit set and triangles, t within the Newton tolerance (bit-identical on
    almost every ray), and it walks fewer triangles and nodes."""
    sc = quad if name == "quad" else sphere
    so = py_oracle.CpuScene(oracle, sc)
    cam = scenes.quad_camera_rays(48, 48) if name == "quad" else scenes.sphere_camera_rays(64, 36)
    rays = np.concatenate([cam, helpers.near_surface_rays(so, 800), helpers.aimed_rays(so, 800)[0]])
    hi, si = so.intersect(rays, stats=True, order="index")
    hn, sn = so.intersect(rays, stats=True, order="nearest")
    hit = hi[:, 10] >= 0
    assert np.array_equal(hit, hn[:, 10] >= 0)
    assert np.array_equal(hi[hit, 10], hn[hit, 10])
    tol = np.array([so.triangle_info(t)[2] for t in range(so.n_tri)])
    tri = hi[hit, 10].astype(int)
    assert (np.abs(hi[hit, 0] - hn[hit, 0]) <= 4 * tol[tri]).all()
    assert (hi[hit, 0] == hn[hit, 0]).mean() > 0.99
    assert sn[:, 0].sum() <= si[:, 0].sum() and sn[:, 1].sum() <= si[:, 1].sum()


def test_flat_loop_by_groups_equals_the_whole_loop(oracle):
    """The chained evaluation the full-size tests use (a group of assets at
    a time, each group's loop starting from the t_max the earlier groups
    left) is the whole flat loop, record for record."""
    sc = helpers.small_sphere(16)
    cpu = py_oracle.CpuScene(oracle, sc)
    rays = np.concatenate([helpers.near_surface_rays(cpu, 1500), scenes.sphere_camera_rays(40, 30)])
    whole, _ = cpu.intersect(rays, order="index")
    for g in (1, 2, 4):
        chained = helpers.oracle_flat_loop_by_groups(oracle, sc, rays, group=g)
        assert np.array_equal(chained.tobytes(), whole.tobytes())
    assert (whole[:, 10] >= 0).sum() > 300
