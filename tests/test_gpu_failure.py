"""Failure paths of the query, made on the host: rays the query cannot
answer, and a walk cap the caller sets low enough to run out. Neither may
hang or fault; both come back as defined results.

- A ray with a non-finite origin or direction component, a zero direction
  or a NaN t_min / t_max is answered as a miss, on every path, and the
  other rays of the same batch get exactly the answers they get without it.
- A triangle walk that visits more cells than dmap_options.node_visit_cap
  gives up: the call returns DMAP_ERR_LIMIT, the rays it happened to are
  flagged DMAP_HIT_CAPPED, every other ray's record is the uncapped one, and
  the next call on the context is clean again.
"""
import ctypes as C

import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu

PATHS = [dict(precision="f64"), dict(precision="f32", schedule="simple"),
         dict(precision="f32", schedule="wavefront", rounds=3, blocks_per_sm=4),
         dict(precision="f32", schedule="wavefront", rounds=0, blocks_per_sm=2)]


@pytest.fixture(scope="module")
def world(oracle):
    ctx = dm.Context(0)
    sc = helpers.small_sphere(32)
    cpu = py_oracle.CpuScene(oracle, sc)
    dev = dm.Scene.from_synthetic(ctx, sc, keep_f64=True)
    rays = np.concatenate([helpers.near_surface_rays(cpu, 1500), helpers.aimed_rays(cpu, 1500)[0]])
    return ctx, cpu, dev, rays


def _unanswerable(rays):
    """Six broken copies of real rays, one per defect."""
    bad = np.repeat(rays[:6], 1, axis=0).copy()
    bad[0, 0] = np.nan          # origin NaN
    bad[1, 4] = np.inf          # direction component infinite
    bad[2, 3:6] = 0.0           # zero direction
    bad[3, 6] = np.nan          # t_min NaN
    bad[4, 7] = np.nan          # t_max NaN
    bad[5, 2] = -np.inf         # origin infinite
    return bad


@pytest.mark.parametrize("path", PATHS, ids=["f64", "f32-simple", "f32-wave", "f32-inline"])
@pytest.mark.parametrize("mode", ["closest", "occluded"])
def test_unanswerable_rays_are_misses(world, path, mode):
    ctx, cpu, dev, rays = world
    bad = _unanswerable(rays)
    mixed = np.empty((len(rays) + len(bad), 8), np.float32)
    # the broken rays spread through the batch, among the good ones
    slots = np.linspace(0, len(mixed) - 1, len(bad)).astype(int)
    good = np.setdiff1d(np.arange(len(mixed)), slots)
    mixed[slots] = bad
    mixed[good] = rays
    opt = dm.TraversalOptions(mode=mode, **path, leaf_precision="f64")
    h_mixed = dev.intersect(mixed, opt)
    h_alone = dev.intersect(rays, opt)
    assert (h_mixed["tri"][slots] == -1).all() and np.isinf(h_mixed["t"][slots]).all()
    assert (h_mixed["flags"][slots] == 0).all()
    assert np.array_equal(h_mixed[good].tobytes(), h_alone.tobytes())
    if mode == "closest":
        ho, _ = cpu.intersect(rays)
        hit = ho[:, 10] >= 0
        assert np.array_equal(h_alone["tri"], ho[:, 10].astype(np.int32))
        assert np.array_equal(h_alone["t"][hit], ho[hit, 0])


def test_degenerate_t_range_is_a_miss(world):
    ctx, cpu, dev, rays = world
    r = rays[:64].copy()
    r[:, 6], r[:, 7] = 2.0, 1.0   # t_min > t_max: nothing to find
    for path in PATHS:
        h = dev.intersect(r, dm.TraversalOptions(**path, leaf_precision="f64"))
        assert (h["tri"] == -1).all()


def _raw_intersect(dev, rays, opt):
    """dmap_intersect_host through the C ABI, returning the status with the
    records (the binding raises on a non-OK status)."""
    L = dm.lib()
    hits = np.empty(len(rays), dm.HIT64)
    o = opt.c()
    st = L.dmap_intersect_host(dev.h, rays.ctypes.data, dm.F32, len(rays), C.byref(o), hits.ctypes.data, dm.F64,
                               None)
    return st, hits


@pytest.mark.parametrize("schedule", ["simple", "wavefront"])
def test_walk_cap_runs_out_and_flags_its_rays(world, schedule):
    ctx, cpu, dev, rays = world
    # and rays that leave the sphere behind: no box, no walk, never capped
    away = np.zeros((16, 8), np.float32)
    away[:, 0], away[:, 3], away[:, 7] = 10.0, 1.0, np.inf
    rays = np.ascontiguousarray(np.concatenate([rays, away]), np.float32)
    base = dict(precision="f32", schedule=schedule, rounds=3, blocks_per_sm=4)
    st0, full = _raw_intersect(dev, rays, dm.TraversalOptions(**base, leaf_precision="f64"))
    assert st0 == 0
    assert not (full["flags"] & dm.HIT_CAPPED).any()
    st, capped = _raw_intersect(dev, rays, dm.TraversalOptions(node_visit_cap=6, **base, leaf_precision="f64"))
    assert st == 6  # DMAP_ERR_LIMIT
    flagged = (capped["flags"] & dm.HIT_CAPPED) != 0
    assert flagged.sum() > len(rays) // 2 and not flagged[-16:].any()
    # a ray no cap touched walked exactly as without the cap
    keep = ~flagged
    assert np.array_equal(capped[keep].tobytes(), full[keep].tobytes())
    # the context is usable again, and the status does not stick
    st2, again = _raw_intersect(dev, rays, dm.TraversalOptions(**base, leaf_precision="f64"))
    assert st2 == 0 and np.array_equal(again.tobytes(), full.tobytes())


def test_negative_cap_is_rejected(world):
    ctx, cpu, dev, rays = world
    st, _ = _raw_intersect(dev, np.ascontiguousarray(rays[:8], np.float32), dm.TraversalOptions(node_visit_cap=-1, leaf_precision="f64"))
    assert st == 1  # DMAP_ERR_INVALID
