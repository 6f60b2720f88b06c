"""The opacity filter behind embree's filter functions (displaced_geometry.cpp:
53-106, the intersect callback's passes): the oracle's restatement against
the same passes run over the reference's own DisplacedIntersector::intersect
and BaseTriangle::param (compiled here), bit for bit, and the properties the
reference's validate_displaced_geometry.cpp (4) checks with a checkerboard
opacity: no accepted hit on a transparent texel, hits behind a culled
crossing found, no filtered hit nearer than the unfiltered one."""
import numpy as np
import pytest

import py_oracle
from dmap_b200 import scenes
import helpers

MAPS = {"identity": ((1.0, 1.0), (0.0, 0.0), False), "scaled": ((0.5, 0.75), (0.25, -0.1), True)}


def checker(n=8):
    i, j = np.meshgrid(np.arange(n), np.arange(n))
    return ((i + j) % 2).astype(np.uint8)


def texel(scene, hits, mask, uv_scale, uv_offset, flip_v):
    """The mask texel under each hit, formed as compute_hit_texcoord forms
    the coordinate (float barycentrics, param, object uv, float)."""
    tri = hits[:, 10].astype(np.int64)
    u = hits[:, 3].astype(np.float32).astype(np.float64)[:, None]
    v = hits[:, 4].astype(np.float32).astype(np.float64)[:, None]
    T = scene.tris[tri]
    t0, t1, t2 = T[:, 18:20], T[:, 20:22], T[:, 22:24]
    st = (t0 + u * (t1 - t0)) + v * (t2 - t0)
    x = (st[:, 0] - uv_offset[0]) / uv_scale[0]
    y = (st[:, 1] - uv_offset[1]) / uv_scale[1]
    if flip_v:
        y = 1.0 - y
    h, w = mask.shape
    i = np.floor(x.astype(np.float32).astype(np.float64) * w).astype(np.int64) % w
    j = np.floor(y.astype(np.float32).astype(np.float64) * h).astype(np.int64) % h
    return mask[j, i]


def scene_and_rays(name, cpu_lib):
    sc = {"quad": lambda: scenes.quad_scene(32), "charts": lambda: helpers.chart_scene(32),
          "sphere": lambda: helpers.small_sphere(16)}[name]()
    assert np.all(np.diff(sc.tri_asset) >= 0)  # the checkers' triangle order is the scene's
    cpu = py_oracle.CpuScene(cpu_lib, sc)
    cam = scenes.quad_camera_rays(40, 40) if name == "quad" else scenes.sphere_camera_rays(48, 27)
    rays = np.concatenate([cam, helpers.near_surface_rays(cpu, 600), helpers.aimed_rays(cpu, 600)[0]])
    return sc, cpu, rays


@pytest.mark.parametrize("name", ["quad", "charts", "sphere"])
@pytest.mark.parametrize("mapname", ["identity", "scaled"])
def test_filtered_oracle_equals_reference(oracle, reference, name, mapname):
    sc, so, rays = scene_and_rays(name, oracle)
    sr = py_oracle.CpuScene(reference, sc)
    scale, off, flip = MAPS[mapname]
    flags = (np.arange(so.n_tri) % 3 != 1).astype(np.uint8)  # one triangle in three not covered
    for m, tf in ((checker(8), None), (checker(5), flags)):
        so.set_opacity(m, scale, off, flip, tf)
        sr.set_opacity(m, scale, off, flip, tf)
        ho, sto = so.intersect(rays, stats=True, order="index")
        hr, st_r = sr.intersect(rays, stats=True, order="index")
        assert np.array_equal(ho, hr)
        assert np.array_equal(sto[:, [0, 1, 2, 3]], st_r[:, [0, 1, 2, 3]])
        assert (ho[:, 10] >= 0).sum() > 100


@pytest.mark.parametrize("name", ["quad", "charts", "sphere"])
def test_filter_properties(oracle, name):
    sc, so, rays = scene_and_rays(name, oracle)
    h0, _ = so.intersect(rays, order="index")
    scale, off, flip = MAPS["scaled"]
    m = checker(6)
    so.set_opacity(m, scale, off, flip)
    hf, _ = so.intersect(rays, order="index")
    hit0, hitf = h0[:, 10] >= 0, hf[:, 10] >= 0
    # no accepted hit on a transparent texel; every hit the filter kept is the unfiltered one
    assert (texel(sc, hf[hitf], m, scale, off, flip) != 0).all()
    opaque0 = np.zeros(len(rays), bool)
    opaque0[hit0] = texel(sc, h0[hit0], m, scale, off, flip) != 0
    assert np.array_equal(hf[opaque0], h0[opaque0])
    # culled crossings: the filtered hit is never nearer, and often there is a surface behind
    culled = hit0 & ~opaque0
    assert culled.sum() > 50
    assert not (hitf & ~hit0).any()
    assert (hf[culled & hitf, 0] > h0[culled & hitf, 0]).all()
    assert (culled & hitf).sum() > 0
    # all-opaque mask: the unfiltered query exactly; the filter removed: the same
    so.set_opacity(np.ones((3, 7), np.uint8), scale, off, flip)
    assert np.array_equal(so.intersect(rays, order="index")[0], h0)
    so.set_opacity(None)
    assert np.array_equal(so.intersect(rays, order="index")[0], h0)


@pytest.mark.parametrize("name", ["quad", "sphere"])
def test_filtered_nearest_order_same_hits(oracle, name):
    """Nearest-first order under the filter: the flat loop's filtered hits."""
    sc, so, rays = scene_and_rays(name, oracle)
    so.set_opacity(checker(8))
    hi, _ = so.intersect(rays, order="index")
    hn, _ = so.intersect(rays, order="nearest")
    hit = hi[:, 10] >= 0
    assert np.array_equal(hit, hn[:, 10] >= 0)
    assert np.array_equal(hi[hit, 10], hn[hit, 10])
    tol = np.array([so.triangle_info(t)[2] for t in range(so.n_tri)])
    assert (np.abs(hi[hit, 0] - hn[hit, 0]) <= 4 * tol[hi[hit, 10].astype(int)]).all()


@pytest.mark.parametrize("lib", ["oracle", "reference"])
def test_filter_limits(request, lib):
    """A mask that is transparent everywhere leaves no hit; one that covers
    no triangle leaves the unfiltered query."""
    cpu_lib = request.getfixturevalue(lib)
    sc, cpu, rays = scene_and_rays("charts", cpu_lib)
    h0, _ = cpu.intersect(rays, order="index")
    assert (h0[:, 10] >= 0).sum() > 100
    cpu.set_opacity(np.zeros((4, 4), np.uint8))
    assert not (cpu.intersect(rays, order="index")[0][:, 10] >= 0).any()
    cpu.set_opacity(np.zeros((4, 4), np.uint8), tri_flags=np.zeros(cpu.n_tri, np.uint8))
    assert np.array_equal(cpu.intersect(rays, order="index")[0], h0)
