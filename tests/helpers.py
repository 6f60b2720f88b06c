"""Ray sets of the reference's traversal tests, generated through the CPU
oracle (test infrastructure): near-surface rays
(traversal_test_util.cpp:101-109) and rays aimed at surface points
(validate_traversal.cpp:392-410). Rays are rounded to float32 so the GPU
paths and the oracle see the same numbers."""
import math

import numpy as np

from dmap_b200 import scenes


def _uniform_bary(rng, n):
    r = np.sqrt(rng.random(n))
    return np.stack([1.0 - r, r * rng.random(n)], axis=1)


def _edges(scene):
    t = scene.tris
    p0, p1, p2 = t[:, 0:3], t[:, 3:6], t[:, 6:9]
    return (np.linalg.norm(p1 - p0, axis=1) + np.linalg.norm(p2 - p0, axis=1)
            + np.linalg.norm(p2 - p1, axis=1)) / 3.0


def surface_points(cpu, rng, n):
    """Uniform points of random triangles: (tri, st, S)."""
    sc = cpu.scene
    n_tri = len(sc.tris)
    tri = np.minimum((rng.random(n) * n_tri).astype(np.int64), n_tri - 1)
    b = _uniform_bary(rng, n)
    st = np.empty((n, 2))
    S = np.empty((n, 3))
    for k in range(n):
        t = sc.tris[tri[k]]
        t0, t1, t2 = t[18:20], t[20:22], t[22:24]
        st[k] = t0 + b[k, 0] * (t1 - t0) + b[k, 1] * (t2 - t0)
        S[k] = cpu.displaced_position(int(tri[k]), st[k, 0], st[k, 1])
    return tri, st, S


def near_surface_rays(cpu, n, seed=2027):
    rng = np.random.default_rng(seed)
    tri, _, S = surface_points(cpu, rng, n)
    edges = _edges(cpu.scene)[tri]
    r = edges * 10.0 ** (-1.0 + 1.5 * rng.random(n))
    o = S + r[:, None] * scenes.uniform_direction(rng, n)
    d = scenes.uniform_direction(rng, n)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3:6], rays[:, 7] = o, d, np.inf
    return rays


def aimed_rays(cpu, n, seed=2028):
    """Rays that must hit at or before t_s (the never-miss check)."""
    rng = np.random.default_rng(seed)
    tri, st, S = surface_points(cpu, rng, n)
    d = scenes.uniform_direction(rng, n)
    t_s = _edges(cpu.scene)[tri] * 10.0 ** (-1.5 + 2.0 * rng.random(n))
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3:6], rays[:, 7] = S - t_s[:, None] * d, d, np.inf
    # the float32 ray no longer passes exactly through S: recompute t_s along it
    o32, d32 = rays[:, 0:3].astype(np.float64), rays[:, 3:6].astype(np.float64)
    t_s = np.sum((S - o32) * d32, axis=1) / np.sum(d32 * d32, axis=1)
    miss_dist = np.linalg.norm(o32 + t_s[:, None] * d32 - S, axis=1)
    return rays, t_s, miss_dist, tri


def small_sphere(n=32, patches=(0, 1, 5, 16, 40, 95)):
    return scenes.cube_sphere_scene(n, 4, patches=list(patches))


def chart_scene(n=32, seed=7):
    """Triangles with general charts (texture coordinates off the cell
    lattice), one of them mirrored, and a repeat-wrapped object whose chart
    leaves the unit tile: the cases the texel tessellation clips."""
    rng = np.random.default_rng(seed)
    h0 = scenes.sine_noise_heights(n, seed, 0.06)
    h1 = scenes.sine_noise_heights(n, seed + 1, 0.04)
    a0 = scenes.Asset(scenes.close_tile(h0, repeat=False).astype(np.float32))
    a1 = scenes.Asset(scenes.close_tile(h1, repeat=True).astype(np.float32), scale=1.0, offset=0.01, repeat=True)
    P = [np.array([0.0, 0.0, 0.0]), np.array([1.2, 0.1, 0.05]), np.array([0.2, 1.1, -0.1])]
    N = [v / np.linalg.norm(v) for v in (np.array([0.05, -0.1, 1.0]), np.array([0.1, 0.0, 1.0]),
                                          np.array([-0.08, 0.1, 1.0]))]

    def rec(t0, t1, t2, shift=np.zeros(3)):
        return np.concatenate([P[0] + shift, P[1] + shift, P[2] + shift, N[0], N[1], N[2], t0, t1, t2])

    tris = [rec([0.13, 0.21], [0.87, 0.30], [0.25, 0.91]),
            rec([0.13, 0.21], [0.25, 0.91], [0.87, 0.30], np.array([0.0, 0.0, 0.6])),   # mirrored chart
            rec([-0.31, 0.42], [1.27, -0.18], [0.52, 1.61], np.array([1.5, 0.0, 0.0]))]  # repeat, off the tile
    tris = np.stack(tris)
    tris[:, 18:24] += rng.random(6) * 1e-3  # off the dyadic lattice
    return scenes.Scene([a0, a1], tris, np.array([0, 0, 1], np.int32), name=f"charts{n}", extent=3.0)


def oracle_flat_loop_by_groups(oracle, scene, rays, group=16, threads=0):
    """The reference's flat loop over every triangle of `scene`, in index
    order, evaluated `group` assets at a time so that only one group's FP64
    pyramids are held at once: each group's flat loop runs with the t_max the
    earlier groups left (the hit's t, as the loop itself sets it), so the
    chained result is the whole loop's, record for record. Triangles must be
    grouped by asset in index order (tri_asset non-decreasing)."""
    import py_oracle
    ta = scene.tri_asset
    assert (np.diff(ta) >= 0).all(), "triangles must be in asset order"
    r = np.ascontiguousarray(rays, np.float64).copy()
    best = np.zeros((len(r), py_oracle.HIT))
    best[:, 0] = np.inf
    best[:, 10:12] = -1  # triangle, object
    for g0 in range(0, len(scene.assets), group):
        keep = (ta >= g0) & (ta < g0 + group)
        first = int(np.argmax(keep))
        sub = scenes.Scene(scene.assets[g0:g0 + group], scene.tris[keep], (ta[keep] - g0).astype(np.int32))
        cpu = py_oracle.CpuScene(oracle, sub)
        h, _ = cpu.intersect(r, order="index", threads=threads)
        del cpu
        found = h[:, 10] >= 0
        h[found, 10] += first
        h[found, 11] += g0  # objects are assets in order
        best[found] = h[found]
        r[found, 7] = h[found, 0]
    return best
