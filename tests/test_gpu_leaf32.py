"""The FP32 certified leaf (leaf_precision="f32"): the leaf's sub-square
search and Newton iteration in FP32 with outward-rounded bounds, FP64 Newton
polish of roots whose Jacobian's condition number exceeds polish_cond.

Its hits are judged the way the FP32 product path is judged against the FP64
oracle:
- the hit/miss set equals the oracle's, except rays in the grazing band
  (|cos| between the ray and the oracle's surface normal below 1e-3, where
  the reference's own FP64 Newton sits at its conditioning limit);
- no false miss on rays aimed at surface points (the bounds are conservative
  and Newton starts in every sub-square that holds a root);
- |t - t_oracle| <= 1e-5 of the scene extent and uv within 1e-4 on every
  hit both report (an unpolished root, cond(J) <= polish_cond, sits within
  the FP32 residual of the root, which its conditioning turns into about
  1e-8 cond(J) of uv); unit normals within 1e-4 except on texel edges, where
  the reference's own normal (Su x Sv with the gradient of the cell the
  point falls in) jumps, so a root a rounding away on the other side takes
  the neighbour texel's gradient; a different triangle is allowed only where
  the two hits are the same point (a shared edge).
"""
import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu

TOL_T = 1e-5   # of the scene extent
TOL_UV = 1e-4   # texture units: a root's uv moves with its conditioning
TOL_NG = 1e-4
GRAZING = 1e-3


@pytest.fixture(scope="module")
def ctx():
    return dm.Context(0)


def judge(h, ho, rays, extent):
    """FP32-leaf hits (HIT64) against oracle records; asserts the bar and
    returns the error summary."""
    g_hit, o_hit = h["tri"] >= 0, ho[:, 10] >= 0
    d = rays[:, 3:6].astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    cos = np.abs(np.sum(d * ho[:, 5:8], axis=1))
    grazing = o_hit & (cos < GRAZING)
    diff = g_hit != o_hit
    assert not (diff & ~grazing).any(), f"{int((diff & ~grazing).sum())} hit/miss differences outside the grazing band"
    both = g_hit & o_hit
    dt = np.abs(h["t"][both] - ho[both, 0])
    assert dt.max(initial=0.0) <= TOL_T * extent, f"max |dt| {dt.max()} over {TOL_T} x extent"
    other = both & (h["tri"] != ho[:, 10].astype(np.int32))
    same = both & ~other
    duv = np.abs(h["st"][same] - ho[same, 1:3]).max(initial=0.0)
    dng_each = np.abs(h["ng"][same] - ho[same, 5:8]).max(axis=1) if same.any() else np.zeros(1)
    dng = float(dng_each.max())
    assert duv <= TOL_UV, duv
    assert np.mean(dng_each <= TOL_NG) >= 0.999 and dng <= 0.05, dng
    return {"hits": int(o_hit.sum()), "grazing_diff": int(diff.sum()), "max_rel_dt": float(dt.max(initial=0.0) / extent),
            "max_duv": float(duv), "max_dng": float(dng), "triangle_diff": int(other.sum())}


PATHS = [dict(schedule="wavefront", rounds=3, blocks_per_sm=4), dict(schedule="wavefront", rounds=0, blocks_per_sm=2),
         dict(schedule="simple")]


@pytest.mark.parametrize("path", PATHS, ids=["wave", "inline", "simple"])
@pytest.mark.parametrize("name", ["quad", "sphere", "charts"])
def test_leaf32_within_tolerance_of_the_oracle(ctx, oracle, path, name):
    sc = {"quad": lambda: scenes.quad_scene(64), "sphere": lambda: helpers.small_sphere(32),
          "charts": lambda: helpers.chart_scene(32)}[name]()
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    aimed, t_s, miss_dist, _ = helpers.aimed_rays(cpu, 1500)
    rays = np.concatenate([helpers.near_surface_rays(cpu, 1500), aimed])
    for order in ("nearest", "index"):
        ho, _ = cpu.intersect(rays, order=order)
        h = dev.intersect(rays, dm.TraversalOptions(precision="f32", leaf_precision="f32", order=order, **path))
        s = judge(h, ho, rays, sc.extent)
        assert s["hits"] > 1000
        # never-miss (validate_traversal.cpp:392-461): a ray through a surface
        # point finds a hit
        ha = h[len(rays) - len(aimed):]
        assert (ha["tri"][miss_dist < 1e-6] >= 0).all(), "an aimed ray missed"


def test_leaf32_grazing_f16(ctx, oracle):
    sc = helpers.small_sphere(32)
    sc = scenes.Scene([scenes.Asset(a.nodes.astype(np.float16), a.scale, a.offset, a.repeat) for a in sc.assets],
                      sc.tris, sc.tri_asset, extent=sc.extent)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    p, m = scenes.base_points(sc, 4000, seed=17)
    rays = scenes.grazing_rays(p, m, seed=18)
    ho, _ = cpu.intersect(rays, order="index")
    h = dev.intersect(rays, dm.TraversalOptions(precision="f32", leaf_precision="f32", order="index"))
    s = judge(h, ho, rays, sc.extent)
    assert s["hits"] > 2000


def test_polish_flags(ctx, oracle):
    """polish_cond 0 refines every root in FP64 (flagged, and equal to the
    oracle's root to within its Newton tolerance); a huge polish_cond keeps
    every root FP32 (no flag)."""
    sc = helpers.small_sphere(32)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([helpers.near_surface_rays(cpu, 1000), helpers.aimed_rays(cpu, 1000)[0]])
    ho, _ = cpu.intersect(rays)
    hit = ho[:, 10] >= 0
    always = dev.intersect(rays, dm.TraversalOptions(precision="f32", leaf_precision="f32", polish_cond=0.0))
    never = dev.intersect(rays, dm.TraversalOptions(precision="f32", leaf_precision="f32", polish_cond=1e30))
    ga, gn = always["tri"] >= 0, never["tri"] >= 0
    both_flags = dm.HIT_POLISHED | dm.HIT_FP64_LEAF
    assert np.mean((always["flags"][ga] & both_flags) == both_flags) > 0.95
    assert not (never["flags"][gn] & both_flags).any()
    both = ga & hit & (always["tri"] == ho[:, 10].astype(np.int32)) & ((always["flags"] & both_flags) == both_flags)
    assert both.sum() > 500
    # a polished root is an FP64 Newton root: within 1e-9 of the oracle's
    assert np.abs(always["t"][both] - ho[both, 0]).max() <= 1e-9 * sc.extent
