"""The oracle meshes (displaced_tessellation.cpp): the C restatement of the
uniform barycentric tessellation and the texel-aligned tessellation against
the reference's own append_displaced_triangle / append_texel_tessellation
compiled here, bit for bit, and the properties the meshes must have: the
texel faces partition each triangle's uv domain, the uniform faces have
equal parameter area, and with m = 1 the texel mesh is the two-triangle
leaf's surface (the reference's MeshOracle cross-check,
traversal_test_util.h:81-124)."""
import numpy as np
import pytest

import py_oracle
import helpers
from dmap_b200 import scenes


@pytest.fixture(scope="module", params=["quad", "charts", "sphere"])
def scene(request):
    return {"quad": lambda: scenes.quad_scene(16), "charts": lambda: helpers.chart_scene(32),
            "sphere": lambda: helpers.small_sphere(16, patches=(0, 40))}[request.param]()


def _domain_area(tri):
    t0, t1, t2 = tri[18:20], tri[20:22], tri[22:24]
    a, b = t1 - t0, t2 - t0
    return 0.5 * abs(a[0] * b[1] - a[1] * b[0])


def _st_areas(st):
    a, b = st[:, 1] - st[:, 0], st[:, 2] - st[:, 0]
    return 0.5 * np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0])


@pytest.mark.parametrize("n", [1, 2, 5])
def test_uniform_equals_reference(oracle, reference, scene, n):
    so, sr = py_oracle.CpuScene(oracle, scene), py_oracle.CpuScene(reference, scene)
    for t in range(so.n_tri):
        a, b = so.tessellate_uniform(t, n), sr.tessellate_uniform(t, n)
        for k in a:
            assert np.array_equal(a[k], b[k]), (t, k)


@pytest.mark.parametrize("m", [1, 2, 3])
def test_texel_equals_reference(oracle, reference, scene, m):
    so, sr = py_oracle.CpuScene(oracle, scene), py_oracle.CpuScene(reference, scene)
    for t in range(so.n_tri):
        a, b = so.tessellate_texel(t, m), sr.tessellate_texel(t, m)
        assert len(a["interior"]) > 0
        for k in a:
            assert np.array_equal(a[k], b[k]), (t, k)


@pytest.mark.parametrize("m", [1, 2])
def test_texel_faces_partition_domain(oracle, scene, m):
    so = py_oracle.CpuScene(oracle, scene)
    for t in range(so.n_tri):
        mesh = so.tessellate_texel(t, m)
        area = _st_areas(mesh["st"]).sum()
        assert abs(area - _domain_area(scene.tris[t])) <= 1e-12 * max(1.0, area)
        # interior faces are half sub-cells
        w = 1.0 / (scene.assets[scene.tri_asset[t]].n_leaf * m)
        inner = _st_areas(mesh["st"][mesh["interior"] == 1])
        assert np.allclose(inner, 0.5 * w * w, rtol=1e-12)
        # texcoords are the st rounded to float
        assert np.array_equal(mesh["texcoords"], mesh["st"].astype(np.float32))


def test_uniform_grid_layout(oracle):
    sc = helpers.chart_scene(32)
    so = py_oracle.CpuScene(oracle, sc)
    n = 6
    for t in range(so.n_tri):
        mesh = so.tessellate_uniform(t, n)
        V = (n + 1) * (n + 2) // 2
        assert mesh["indices"].shape == (n * n, 3) and mesh["indices"].max() == V - 1
        uv = mesh["texcoords"].astype(np.float64)[mesh["indices"]]
        a = _st_areas(uv)
        assert np.allclose(a, _domain_area(sc.tris[t]) / (n * n), rtol=1e-5)
        assert np.allclose(np.linalg.norm(mesh["normals"], axis=1), 1.0, atol=1e-6)


def _mesh_hits(rays, P):
    """Nearest hit of every ray on the float triangles P (F, 3, 3), in
    double (Moller-Trumbore, t in (t_min, t_max))."""
    P = P.astype(np.float64)
    o, d = rays[:, None, 0:3].astype(np.float64), rays[:, None, 3:6].astype(np.float64)
    e1, e2 = (P[:, 1] - P[:, 0])[None], (P[:, 2] - P[:, 0])[None]
    p = np.cross(d, e2)
    det = np.sum(e1 * p, axis=2)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / det
        s = o - P[None, :, 0]
        b1 = np.sum(s * p, axis=2) * inv
        q = np.cross(s, e1)
        b2 = np.sum(d * q, axis=2) * inv
        t = np.sum(e2 * q, axis=2) * inv
        ok = (det != 0) & (b1 >= 0) & (b2 >= 0) & (b1 + b2 <= 1) & (t > rays[:, 6:7]) & (t < rays[:, 7:8])
    t = np.where(ok, t, np.inf)
    return t.min(axis=1)


def test_texel_mesh_is_two_triangle_leaf(oracle):
    """m = 1 on the identity chart: the float mesh and the FP64
    two-triangle leaf give the same nearest hits."""
    sc = scenes.quad_scene(16)
    so = py_oracle.CpuScene(oracle, sc)
    P = np.concatenate([so.tessellate_texel(t, 1)["positions"] for t in range(so.n_tri)])
    rays = scenes.quad_camera_rays(40, 40)
    t_mesh = _mesh_hits(rays, P)
    t_leaf = so.intersect(rays, leaf="two_triangle")[0][:, 0]
    both = np.isfinite(t_mesh) & np.isfinite(t_leaf)
    assert both.sum() > 500
    assert (np.isfinite(t_mesh) == np.isfinite(t_leaf)).mean() > 0.995
    assert np.max(np.abs(t_mesh[both] - t_leaf[both]) / t_leaf[both]) < 1e-5
