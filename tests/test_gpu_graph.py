"""Graph-replayed host queries (dmap_options.graph): the query's launches
(3 x rounds + 1 kernels and their memsets) captured once per scene,
options and power-of-two batch capacity, the ray count read on the device
at each replay. Every record must equal the one-by-one launch's, for batch
sizes inside one capacity class and across classes, for both schedules,
both modes and both leaves, with scenes and options interleaved."""
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
    sph = helpers.small_sphere(32)
    cpu = py_oracle.CpuScene(oracle, sph)
    devs = [dm.Scene.from_synthetic(ctx, sph), dm.Scene.from_synthetic(ctx, scenes.quad_scene(64))]
    pools = [np.concatenate([helpers.near_surface_rays(cpu, 3000), helpers.aimed_rays(cpu, 3000)[0]]),
             np.concatenate([scenes.quad_camera_rays(64, 64)] * 2)]
    return ctx, devs, pools


@pytest.mark.parametrize("opts", [dict(), dict(mode="occluded"), dict(schedule="simple"),
                                  dict(leaf_precision="f32"), dict(rounds=0, blocks_per_sm=2)],
                         ids=["wave", "occluded", "simple", "leaf32", "inline"])
def test_graph_replay_equals_launches(world, opts):
    ctx, devs, pools = world
    rng = np.random.default_rng(5)
    for k, n in enumerate([1, 37, 1000, 1024, 1025, 3000, 700, 5999]):
        d = devs[k % 2]
        pool = pools[k % 2]
        lo = int(rng.integers(0, len(pool) - n + 1))
        rays = pool[lo:lo + n]
        a = d.intersect(rays, dm.TraversalOptions(graph=True, **opts))
        b = d.intersect(rays, dm.TraversalOptions(graph=False, **opts))
        assert np.array_equal(a.tobytes(), b.tobytes()), (n, opts)


def test_graph_counts_launches(world):
    ctx, devs, pools = world
    opt = dm.TraversalOptions(graph=True, rounds=3)
    devs[0].intersect(pools[0][:500], opt)  # captures
    before = ctx.kernel_launches
    devs[0].intersect(pools[0][:600], opt)  # replays
    assert ctx.kernel_launches - before == 3 * 3 + 1
