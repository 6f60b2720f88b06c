"""The opacity filter on the device (dmap_scene_set_opacity) against the
oracle's restatement, which is pinned to the intersect callback's passes run
over the reference's own intersector (test_oracle_filter.py): the FP64 path,
the FP32 one-thread-per-ray walk and the FP32 wavefront (which hands the rays
that took a rejected crossing to the one-thread-per-ray walk), closest and
occlusion queries, both triangle orders; and the calls that refuse a
filtered scene."""
import numpy as np
import pytest

import dmap_b200 as dm
import helpers
from dmap_b200 import scenes
from test_oracle_filter import MAPS, checker, scene_and_rays

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return dm.Context(0)


@pytest.mark.parametrize("name,mapname", [("quad", "identity"), ("charts", "scaled"), ("sphere", "scaled")])
@pytest.mark.parametrize("precision,schedule", [("f64", "simple"), ("f32", "simple"), ("f32", "wavefront")])
@pytest.mark.parametrize("order", ["nearest", "index"])
def test_filtered_device_equals_oracle(ctx, oracle, name, mapname, precision, schedule, order):
    sc, so, rays = scene_and_rays(name, oracle)
    dev = dm.Scene.from_synthetic(ctx, sc, keep_f64=True)
    scale, off, flip = MAPS[mapname]
    flags = (np.arange(so.n_tri) % 3 != 1).astype(np.uint8)
    m = checker(5)
    so.set_opacity(m, scale, off, flip, flags)
    dev.set_opacity(m, scale, off, flip, flags)
    ho, _ = so.intersect(rays, order=order)
    opt = dm.TraversalOptions(precision=precision, schedule=schedule, order=order, leaf_precision="f64")
    hd = dev.intersect(rays, opt, np.float64)
    hit = ho[:, 10] >= 0
    assert hit.sum() > 100
    assert np.array_equal(hd["tri"], ho[:, 10].astype(np.int32))
    assert np.array_equal(hd["t"][hit], ho[hit, 0])
    assert np.array_equal(hd["st"][hit], ho[hit, 1:3])
    assert np.array_equal(hd["bary"][hit], ho[hit, 3:5])
    assert np.array_equal(hd["ng"][hit], ho[hit, 5:8])
    assert np.isinf(hd["t"][~hit]).all()
    # the filter culled hits here: the unfiltered query differs
    so.set_opacity(None)
    assert (so.intersect(rays, order=order)[0][:, 10] != ho[:, 10]).sum() > 20
    # occlusion through the filter: occluded exactly where the filtered closest query hits
    occ = dev.intersect(rays, dm.TraversalOptions(precision=precision, schedule=schedule, order=order,
                                                  mode="occluded", leaf_precision="f64"), np.float64)
    assert np.array_equal(occ["tri"] >= 0, hit)
    # the filter removed: the device query is the unfiltered one again
    dev.set_opacity(None)
    h0, _ = so.intersect(rays, order=order)
    assert np.array_equal(dev.intersect(rays, opt, np.float64)["tri"], h0[:, 10].astype(np.int32))


def test_filtered_scene_on_every_path(ctx):
    """A filtered scene runs its filter's passes on every path: a wavefront
    query (every round count, the rays that took a rejected crossing answered
    again by the one-thread-per-ray schedule), the server, the path tracer;
    each equals the explicit simple schedule's answer."""
    sc = scenes.quad_scene(16)
    dev = dm.Scene.from_synthetic(ctx, sc)
    rays = scenes.quad_camera_rays(24, 24)
    dev.set_opacity(checker(4))
    simple = dev.intersect(rays, dm.TraversalOptions(schedule="simple", leaf_precision="f64"), np.float32)
    for rounds in (0, 1, 3):
        wave = dev.intersect(rays, dm.TraversalOptions(leaf_precision="f64", rounds=rounds), np.float32)
        assert wave.tobytes() == simple.tobytes()
    unfiltered = dm.Scene.from_synthetic(ctx, sc).intersect(rays, dm.TraversalOptions(leaf_precision="f64"),
                                                             np.float32)
    assert (unfiltered["tri"] != simple["tri"]).sum() > 10  # the filter culled crossings
    srv = dm.Server(ctx, max_batch_rays=1024, slots=1, options=dm.TraversalOptions(leaf_precision="f64"))
    rid, out = srv.submit_rays(dev, rays)
    assert srv.wait(rid, 60.0) == 0
    assert out.tobytes() == simple.tobytes()
    srv.close()
    pt = scenes.with_ground_and_emitter(helpers.small_sphere(16, patches=(0,)), 16)
    dpt = dm.Scene.from_synthetic(ctx, pt)
    dpt.set_opacity(checker(4))
    view = scenes.path_tracer_view(16, 12)
    a, sa, _ = dpt.render(view, pt.emitter, options=dm.TraversalOptions(leaf_precision="f64"))
    b, sb, _ = dpt.render(view, pt.emitter, options=dm.TraversalOptions(schedule="simple", leaf_precision="f64"))
    assert np.array_equal(a, b) and sa["extension_rays"] == sb["extension_rays"]
    for bad in (dict(mask=np.zeros((0, 3), np.uint8)), dict(mask=checker(4), uv_scale=(0.0, 1.0)),
                dict(mask=checker(4), uv_scale=(np.inf, 1.0))):
        with pytest.raises((dm.DmapError, ValueError)):
            dev.set_opacity(**bad)
    dev.set_opacity(None)
    dev.intersect(rays, dm.TraversalOptions(leaf_precision="f64"), np.float64)
