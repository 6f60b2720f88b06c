"""The batched path tracer (dmap_render), checked by ray replay: every
extension and shadow query the device render issues is recorded with the
device's answer and re-run through the oracle's intersector. The shading
model is the library's own (the reference renders through ks's SmallPT,
whose sources are not part of the reference), so parity is per query; the
image is checked for invariance to batching, graph capture and schedule."""
import numpy as np
import pytest

import dmap_b200 as dm
from dmap_b200 import scenes
import py_oracle

pytestmark = pytest.mark.gpu

F64_LEAF = dm.TraversalOptions(leaf_precision="f64")  # replayed hits equal the oracle's bit for bit

VIEW = scenes.path_tracer_view(48, 27)


@pytest.fixture(scope="module")
def pt(oracle):
    sc = scenes.path_tracer_scene(n_sphere=32, n_ground=64)
    ctx = dm.Context(0)
    dev = dm.Scene.from_synthetic(ctx, sc)
    cpu = py_oracle.CpuScene(oracle, sc)
    return sc, ctx, dev, cpu


def test_render_ray_replay(pt):
    sc, ctx, dev, cpu = pt
    img, st, rec = dev.render(VIEW, sc.emitter, spp=2, record=200_000, options=F64_LEAF)
    assert rec["count"] == st["extension_rays"] + st["shadow_rays"] == len(rec["kind"])
    assert st["paths"] == 2 * VIEW["width"] * VIEW["height"]
    rays = rec["rays"].astype(np.float64)
    h, _ = cpu.intersect(rays)
    ext = rec["kind"] == 0
    sh = ~ext
    assert ext.sum() == st["extension_rays"] and ext.sum() >= st["paths"]
    assert sh.sum() > 300
    # extension rays: the device's closest hit is the oracle's
    assert np.array_equal(rec["tri"][ext], h[ext, 10].astype(np.int32))
    hit = ext & (rec["tri"] >= 0)
    assert hit.sum() > 1000
    assert np.array_equal(rec["t"][hit], h[hit, 0].astype(np.float32))
    # shadow rays: occluded exactly when the oracle finds a hit before t_max
    assert np.array_equal(rec["tri"][sh] >= 0, h[sh, 10] >= 0)
    assert 0 < (rec["tri"][sh] >= 0).sum() < sh.sum()
    assert np.isfinite(img).all() and (img >= 0).all() and img.mean() > 0


def test_render_invariant_to_batching_graph_and_schedule(pt):
    sc, ctx, dev, cpu = pt
    wh = VIEW["width"] * VIEW["height"]
    a, sa, _ = dev.render(VIEW, sc.emitter, spp=4, use_graph=True, options=F64_LEAF)
    b, sb, _ = dev.render(VIEW, sc.emitter, spp=4, use_graph=False, paths_per_batch=wh, options=F64_LEAF)
    c, sc_, _ = dev.render(VIEW, sc.emitter, spp=4, use_graph=True, paths_per_batch=2 * wh, options=F64_LEAF)
    d, sd, _ = dev.render(VIEW, sc.emitter, spp=4, options=dm.TraversalOptions(schedule="simple", leaf_precision="f64"))
    assert sa["batches"] == 1 and sb["batches"] == 4 and sc_["batches"] == 2
    for img, st in ((b, sb), (c, sc_), (d, sd)):
        assert np.array_equal(a, img)
        assert st["extension_rays"] == sa["extension_rays"] and st["shadow_rays"] == sa["shadow_rays"]


def test_render_depth_and_roulette(pt):
    sc, ctx, dev, cpu = pt
    _, s1, _ = dev.render(VIEW, sc.emitter, spp=2, max_depth=1, options=F64_LEAF)
    _, s5, _ = dev.render(VIEW, sc.emitter, spp=2, max_depth=5, rr_depth=3, options=F64_LEAF)
    _, s5n, _ = dev.render(VIEW, sc.emitter, spp=2, max_depth=5, rr_depth=5, options=F64_LEAF)
    assert s1["extension_rays"] == s1["paths"]
    assert s1["extension_rays"] < s5["extension_rays"] <= s5n["extension_rays"] <= 5 * s5n["paths"]
    assert s5["shadow_rays"] <= s5["extension_rays"]
    # a different seed, a different image of the same scene
    a, _, _ = dev.render(VIEW, sc.emitter, spp=2, seed=1, options=F64_LEAF)
    b, _, _ = dev.render(VIEW, sc.emitter, spp=2, seed=2, options=F64_LEAF)
    assert not np.array_equal(a, b) and abs(a.mean() - b.mean()) < 0.5 * max(a.mean(), b.mean())
