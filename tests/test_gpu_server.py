"""The serving loop (dmap_server_*): requests of mixed sizes, scenes and
kinds submitted together are packed into shared launches, and every result
equals the one the request gets alone through dmap_intersect_host /
dmap_render; admission keeps the held device bytes within the budget;
queued requests can be cancelled."""
import numpy as np
import pytest

import dmap_b200 as dm
from dmap_b200 import scenes
import py_oracle
import helpers

pytestmark = pytest.mark.gpu

VIEW = scenes.path_tracer_view(24, 16)


@pytest.fixture(scope="module")
def world(oracle):
    ctx = dm.Context(0)
    quad = scenes.quad_scene(64)
    sph = helpers.small_sphere(32)
    pt = scenes.path_tracer_scene(n_sphere=32, n_ground=64)
    devs = {"quad": dm.Scene.from_synthetic(ctx, quad), "sphere": dm.Scene.from_synthetic(ctx, sph),
            "pt": dm.Scene.from_synthetic(ctx, pt)}
    cpu = py_oracle.CpuScene(oracle, sph)
    pools = {"quad": np.concatenate([scenes.quad_camera_rays(64, 64)] * 4),
             "sphere": np.concatenate([helpers.near_surface_rays(cpu, 6000), helpers.aimed_rays(cpu, 6000)[0]]),
             "pt": scenes.pinhole_rays(np.array(VIEW["eye"]), np.array(VIEW["target"]), np.array(VIEW["up"]),
                                       VIEW["fov_deg"], 128, 96, jitter_seed=5)}
    return ctx, devs, pools, pt


def _mix(pools, rng, n_req):
    reqs = []
    for k in range(n_req):
        name = ["quad", "sphere", "pt"][k % 3]
        pool = pools[name]
        n = int(np.exp(rng.uniform(np.log(50), np.log(len(pool)))))
        lo = int(rng.integers(0, len(pool) - n + 1))
        mode = "occluded" if rng.random() < 0.2 else "closest"
        reqs.append((name, pool[lo:lo + n].copy(), mode))
    return reqs


def test_results_alone_equal_results_in_the_mix(world):
    ctx, devs, pools, pt = world
    rng = np.random.default_rng(11)
    reqs = _mix(pools, rng, 36)
    srv = dm.Server(ctx, max_batch_rays=8192, slots=2)
    sub = []
    for k, (name, rays, mode) in enumerate(reqs):
        sub.append(("rays", name, mode, rays) + srv.submit_rays(devs[name], rays, mode))
        if k % 9 == 4:
            kw = dict(spp=2, max_depth=3, rr_depth=2, seed=100 + k)
            sub.append(("render", "pt", kw, None) + srv.submit_render(devs["pt"], VIEW, pt.emitter, **kw))
    assert srv.drain(120.0) == 0
    st = srv.stats()
    assert st["completed"] == len(sub) and st["failed"] == 0
    total = sum(len(r[3]) for r in sub if r[0] == "rays")
    # small requests shared launches, large ones were split across launches
    assert st["launches"] < len(sub) + total // 8192 + 8
    assert 0 <= st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    for kind, name, arg, rays, rid, out in sub:
        assert srv.poll(rid) == 0
        assert srv.latency_ms(rid) >= 0.0
        if kind == "rays":
            alone = devs[name].intersect(rays, dm.TraversalOptions(mode=arg), np.float32)
            assert np.array_equal(out["tri"], alone["tri"])
            if arg == "closest":
                assert out.tobytes() == alone.tobytes()
        else:
            img, _, _ = devs["pt"].render(VIEW, pt.emitter, **arg)
            assert np.array_equal(out, img)
    srv.close()


def test_pinned_buffers_take_the_direct_path(world):
    torch = pytest.importorskip("torch")
    ctx, devs, pools, pt = world
    rays = pools["sphere"][:5000]
    rin = torch.from_numpy(rays.copy()).pin_memory()
    hout = torch.empty(len(rays) * dm.HIT32.itemsize, dtype=torch.uint8).pin_memory()
    hits = hout.numpy().view(dm.HIT32)
    srv = dm.Server(ctx, max_batch_rays=1024)
    rid, out = srv.submit_rays(devs["sphere"], rin.numpy(), hits=hits)
    assert srv.wait(rid, 60.0) == 0
    alone = devs["sphere"].intersect(rays, hit_dtype=np.float32)
    assert hits.tobytes() == alone.tobytes()
    srv.close()


def test_budget_admission_and_rejection(world):
    ctx, devs, pools, pt = world
    probe = dm.Server(ctx, max_batch_rays=4096, slots=1)
    slot_bytes = probe.stats()["held_bytes"]
    probe.close()
    assets = sum(a.device_bytes for a in devs["pt"].assets)
    big = scenes.path_tracer_view(160, 120)
    # room for the slot, the scene's assets and one small render job at a
    # time (a 24 x 16 x 2 spp job holds about 0.3 MB)
    budget = slot_bytes + assets + 450_000
    srv = dm.Server(ctx, hbm_budget_bytes=budget, max_batch_rays=4096, slots=1)
    with pytest.raises(dm.DmapError) as e:
        srv.submit_render(devs["pt"], big, pt.emitter, spp=8)
    assert e.value.status == 5  # DMAP_ERR_BUDGET
    ids = [srv.submit_render(devs["pt"], VIEW, pt.emitter, spp=2, max_depth=2, seed=s)[0] for s in range(4)]
    ids += [srv.submit_rays(devs["pt"], pools["pt"][:3000])[0]]
    assert srv.drain(120.0) == 0
    st = srv.stats()
    assert all(srv.poll(i) == 0 for i in ids)
    assert st["peak_bytes"] <= budget
    srv.close()


def test_cancel_queued_request(world):
    ctx, devs, pools, pt = world
    srv = dm.Server(ctx, max_batch_rays=2048, max_inflight=1, slots=1)
    srv.pause()  # admission held: every submitted request stays queued
    first = srv.submit_rays(devs["sphere"], pools["sphere"])[0]
    rest = [srv.submit_rays(devs["quad"], pools["quad"][:500])[0] for _ in range(6)]
    cancelled = rest[-1]
    assert srv.cancel(cancelled) == 9  # DMAP_ERR_CANCELLED: it was still queued
    assert srv.poll(cancelled) == 9
    assert srv.poll(first) == 7  # DMAP_ERR_NOT_READY: held
    srv.pause(False)
    assert srv.drain(120.0) == 0
    assert srv.poll(first) == 0
    assert all(srv.poll(i) == 0 for i in rest[:-1])
    assert srv.poll(cancelled) == 9
    assert srv.cancel(first) == 0  # done: cancel reports the request's own status
    st = srv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 6
    srv.close()


def test_filter_cannot_change_under_served_requests(world):
    """While a server holds a request on a scene, the scene's filter stays as
    it was when the request was admitted; once the request is done (here:
    cancelled) it can change."""
    ctx, devs, pools, pt = world
    scene = devs["quad"]
    srv = dm.Server(ctx, max_batch_rays=2048, slots=1)
    srv.pause()
    rid = srv.submit_rays(scene, pools["quad"][:256])[0]
    mask = np.ones((4, 4), np.uint8)
    with pytest.raises(dm.DmapError) as e:
        scene.set_opacity(mask)
    assert e.value.status == 7  # DMAP_ERR_NOT_READY
    assert srv.cancel(rid) == 9
    scene.set_opacity(mask)
    scene.set_opacity(None)
    srv.pause(False)
    srv.close()


@pytest.mark.parametrize("policy", ["oldest", "shortest"])
def test_policy_orders_the_slots(world, policy):
    """With one slot and admission held, a large closest-hit request
    submitted before a small occlusion request (different modes: never in
    one launch) finishes first under the arrival-order policy and last under
    the shortest-first one; both answer as they do alone."""
    ctx, devs, pools, pt = world
    srv = dm.Server(ctx, max_batch_rays=1024, slots=1, policy=policy)
    srv.pause()
    big_rays, small_rays = pools["sphere"][:12000], pools["sphere"][:300]
    big, big_out = srv.submit_rays(devs["sphere"], big_rays, "closest")
    small, small_out = srv.submit_rays(devs["sphere"], small_rays, "occluded")
    srv.pause(False)
    assert srv.drain(120.0) == 0
    t_big, t_small = srv.latency_ms(big), srv.latency_ms(small)
    if policy == "oldest":
        assert t_small > t_big
    else:
        assert t_small < t_big
    alone = devs["sphere"].intersect(big_rays, dm.TraversalOptions(), np.float32)
    assert big_out.tobytes() == alone.tobytes()
    occ = devs["sphere"].intersect(small_rays, dm.TraversalOptions(mode="occluded"), np.float32)
    assert np.array_equal(small_out["tri"], occ["tri"])
    srv.close()
