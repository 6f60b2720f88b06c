"""Displaced-emitter sampling on the device (dmap_emitter_*) against the
oracle's restatement of DescentSampler, itself pinned bit for bit to the
reference's descent_sampler.cpp (test_oracle_emitter.py): footprints,
every sample (point, normal, sqrt det G, pdfs, draws used) from the same
uniforms, the pdf re-walk at sampled and arbitrary points, for the three
weight variants, with the clipped-polygon fallback exercised; the error
paths."""
import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu

SCENES = {
    "quad": lambda: scenes.quad_scene(32),
    "charts": lambda: helpers.chart_scene(32),
    "sphere": lambda: helpers.small_sphere(16, patches=(0, 1, 40, 95)),
}
RECV = np.array([0.3, 0.2, 1.5, 0.0, 0.0, -1.0])


@pytest.fixture(scope="module")
def ctx():
    return dm.Context(0)


def _texels(sc, seed):
    rng = np.random.default_rng(seed)
    return [rng.random((a.n_leaf, a.n_leaf)) * (rng.random((a.n_leaf, a.n_leaf)) > 0.3) for a in sc.assets]


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("variant", ["area", "product", "product_geometry"])
def test_emitter_equals_oracle(ctx, oracle, name, variant):
    sc = SCENES[name]()
    tex = _texels(sc, 5)
    dev = dm.Scene.from_synthetic(ctx, sc, keep_f64=True)
    em = dm.Emitter(dev, tex, variant, beta=0.05)
    cpu = py_oracle.CpuScene(oracle, sc)
    ems = [py_oracle.CpuEmitter(cpu, t, tex[sc.tri_asset[t]], variant, beta=0.05) for t in range(cpu.n_tri)]
    for t in range(cpu.n_tri):
        assert np.array_equal(em.triangle_info(t), ems[t].info())
    rng = np.random.default_rng(9)
    n = 80 * cpu.n_tri
    tri = np.repeat(np.arange(cpu.n_tri, dtype=np.int32), 80)
    u = rng.random((n, 96)).astype(np.float32)
    for k in range(n):  # every other sample: leaf draws at the far corner, so straddling leaves fall back
        if k % 2:
            u[k, int(ems[tri[k]].info()[0]) + 1:] = np.float32(0.999)
    recv = np.tile(RECV, (n, 1)) if variant == "product_geometry" else None
    got = em.sample(tri, u, recv)
    fallbacks = 0
    for k in range(n):
        want, draws = ems[tri[k]].sample(u[k], None if recv is None else recv[k])
        g = got[k]
        row = np.concatenate([[g["u"], g["v"]], g["p"], g["n"], [g["sqrt_det"], g["pdf_uv"], g["pdf_area"]]])
        assert g["tri"] == tri[k] and g["draws"] == draws, k
        assert np.array_equal(row, want), (k, row, want)
        fallbacks += draws > int(ems[tri[k]].info()[0]) + 3
    assert fallbacks > 0
    # the re-walk at the sampled points equals the sampled pdfs
    pu, pa = em.pdf(tri, np.stack([got["u"], got["v"]], 1), recv)
    assert np.array_equal(pu, got["pdf_uv"]) and np.array_equal(pa, got["pdf_area"])
    # and the oracle's at arbitrary points, in and out of the domains
    q = rng.random((n, 2)) * 1.4 - 0.2
    pu, pa = em.pdf(tri, q, recv)
    for k in range(0, n, 3):
        r = None if recv is None else recv[k]
        assert pu[k] == ems[tri[k]].pdf_uv(q[k, 0], q[k, 1], r)
        assert pa[k] == ems[tri[k]].pdf_area(q[k, 0], q[k, 1], r)


def test_emitter_errors(ctx):
    sc = scenes.quad_scene(16)
    dev = dm.Scene.from_synthetic(ctx, sc)  # FP32 pyramid only
    with pytest.raises(dm.DmapError) as e:
        dm.Emitter(dev)
    assert e.value.status == 8  # DMAP_ERR_UNSUPPORTED
    dev64 = dm.Scene.from_synthetic(ctx, sc, keep_f64=True)
    em = dm.Emitter(dev64, [np.zeros((16, 16))], "product")  # no mass anywhere
    out = em.sample(np.array([0, 1, 7], np.int32), np.full((3, 40), 0.5, np.float32))
    assert list(out["draws"]) == [-1, -1, -1]
    em_area = dm.Emitter(dev64, None, "area")  # uniform emission, area weights
    out = em_area.sample(np.zeros(4, np.int32), np.random.default_rng(1).random((4, 40)).astype(np.float32))
    assert (out["draws"] > 0).all() and (out["pdf_uv"] > 0).all()


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("variant", ["area", "product", "product_geometry"])
def test_light_wrapper_equals_oracle(ctx, oracle, name, variant):
    """The emitter as a light (DisplacedEmitterLight): device light samples,
    the solid-angle pdf from (u, v) and by the walk of the emitter's triangle
    (DisplacedAreaLight::pdf) equal the oracle's, which equal the
    reference's own classes (test_oracle_emitter.py)."""
    sc = SCENES[name]()
    tex = _texels(sc, 6)
    cos = variant != "product_geometry"
    dev = dm.Scene.from_synthetic(ctx, sc, keep_f64=True)
    em = dm.Emitter(dev, tex, variant, beta=0.05, emitter_cosine=cos)
    cpu = py_oracle.CpuScene(oracle, sc)
    ems = [py_oracle.CpuEmitter(cpu, t, tex[sc.tri_asset[t]], variant, beta=0.05, emitter_cosine=cos)
           for t in range(cpu.n_tri)]
    rng = np.random.default_rng(12)
    per = 40
    n = per * cpu.n_tri
    tri = np.repeat(np.arange(cpu.n_tri, dtype=np.int32), per)
    u = rng.random((n, 96)).astype(np.float32)
    centre = sc.tris[:, 0:3].mean(axis=0)
    p = centre + (rng.random((n, 3)) - 0.5) * 3.0
    nn = rng.normal(size=(n, 3))
    nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    shade = np.concatenate([p, nn], axis=1)
    pts = em.sample(tri, u, shade if variant == "product_geometry" else None)
    ls = em.light(pts, shade)
    fields = ("u", "v", "y", "n_y", "wi", "dist", "pdf_area", "pdf_omega", "Le")
    ok = 0
    for k in range(n):
        want = ems[tri[k]].light_sample(u[k], shade[k])
        got = np.concatenate([np.atleast_1d(ls[k][f]) for f in fields] + [[float(ls[k]["ok"])]])
        if want[15]:
            assert np.array_equal(got, want), k
            ok += 1
        else:
            assert ls[k]["ok"] == 0 and np.array_equal(got[:12], want[:12]), k
    assert ok > n // 2
    # the solid-angle pdf at the sampled (u, v) and at arbitrary points
    uv = np.stack([ls["u"], ls["v"]], axis=1)
    uv[1::2] = rng.random((n // 2, 2)) * 1.2 - 0.1
    pw, hit = em.light_pdf(tri, shade, uv=uv)
    want = np.array([ems[tri[k]].light_pdf_uv(shade[k], *uv[k]) for k in range(n)])
    assert np.array_equal(pw, want)
    # by the walk along the sampled directions, and along random ones
    wi = ls["wi"].copy()
    wi[1::2] = nn[1::2]
    pw, hit = em.light_pdf(tri, shade, wi=wi)
    for k in range(n):
        w_pdf, w_uv = ems[tri[k]].light_pdf_walk(shade[k], wi[k])
        assert pw[k] == w_pdf and np.array_equal(hit[k], w_uv, equal_nan=True), k
    assert (pw > 0).sum() > n // 4
