"""Displaced-emitter sampling: the oracle's restatement of DescentSampler
and EmissionTile (descent_sampler.cpp, emission_tile.cpp) against the
reference's own sampler compiled here, bit for bit, from the same streams of
uniforms (oracle/ref_shim/ks/rng.h replays them in order): footprints,
sample points, draw counts, pdf_uv / pdf_area / leaf probabilities, for
the three weight variants on identity, general, mirrored and off-tile
repeat charts; the clipped-polygon fallback after 32 rejections; and the
properties the sampler promises (leaf probabilities sum to one, the
re-walked pdf equals the sampled one, the footprint's area is the domain's)."""
import numpy as np
import pytest

import py_oracle
import helpers
from dmap_b200 import scenes

RECV = np.array([0.3, 0.2, 1.5, 0.0, 0.0, -1.0])


@pytest.fixture(scope="module", params=["quad", "charts", "sphere"])
def scene(request):
    return {"quad": lambda: scenes.quad_scene(32), "charts": lambda: helpers.chart_scene(32),
            "sphere": lambda: helpers.small_sphere(16, patches=(0, 40))}[request.param]()


def _texels(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random((n, n)) * (rng.random((n, n)) > 0.3)


@pytest.mark.parametrize("variant", ["area", "product", "product_geometry"])
def test_sampler_equals_reference(oracle, reference, scene, variant):
    so, sr = py_oracle.CpuScene(oracle, scene), py_oracle.CpuScene(reference, scene)
    rng = np.random.default_rng(11)
    recv = RECV if variant == "product_geometry" else None
    fallbacks = 0
    for t in range(so.n_tri):
        tex = _texels(scene.assets[scene.tri_asset[t]].n_leaf, 100 + t)
        eo = py_oracle.CpuEmitter(so, t, tex, variant, beta=0.05)
        er = py_oracle.CpuEmitter(sr, t, tex, variant, beta=0.05)
        assert np.array_equal(eo.info(), er.info())
        levels = int(eo.info()[0]) + 1
        for k in range(120):
            u = rng.random(96).astype(np.float32)
            if k % 2:  # leaf draws at the leaf's far corner: straddling leaves reject and fall back
                u[levels:] = np.float32(0.999)
            a, ka = eo.sample(u, recv)
            b, kb = er.sample(u, recv)
            assert ka == kb and np.array_equal(a, b), (t, k)
            fallbacks += ka > levels + 2
            assert eo.pdf_uv(a[0], a[1], recv) == er.pdf_uv(a[0], a[1], recv) == a[9]
            assert eo.pdf_area(a[0], a[1], recv) == er.pdf_area(a[0], a[1], recv) == a[10]
        for _ in range(50):  # arbitrary points and leaves, in and out of the domain
            uv = rng.random(2) * 1.4 - 0.2
            assert eo.pdf_uv(*uv, recv) == er.pdf_uv(*uv, recv)
            i, j = rng.integers(-2, 40, 2)
            assert eo.leaf_prob(int(i), int(j), recv) == er.leaf_prob(int(i), int(j), recv)
    assert fallbacks > 0


def test_sampler_properties(oracle):
    sc = helpers.chart_scene(32)
    so = py_oracle.CpuScene(oracle, sc)
    for t in range(so.n_tri):
        n = sc.assets[sc.tri_asset[t]].n_leaf
        e = py_oracle.CpuEmitter(so, t, _texels(n, 7), "product")
        root_level, i0, j0, area, mass, _ = e.info()
        t0, t1, t2 = sc.tris[t, 18:20], sc.tris[t, 20:22], sc.tris[t, 22:24]
        dom = 0.5 * abs((t1 - t0)[0] * (t2 - t0)[1] - (t1 - t0)[1] * (t2 - t0)[0])
        assert abs(area - dom) < 1e-12
        span = 2 << int(root_level)
        total = sum(e.leaf_prob(int(i0) * (1 << int(root_level)) + a, int(j0) * (1 << int(root_level)) + b)
                    for a in range(span) for b in range(span))
        assert abs(total - 1.0) < 1e-12


def test_sampler_without_emitter_cosine(oracle, reference):
    """ProductGeometry without the |emitter cosine| factor."""
    sc = helpers.chart_scene(32)
    so, sr = py_oracle.CpuScene(oracle, sc), py_oracle.CpuScene(reference, sc)
    rng = np.random.default_rng(4)
    for t in range(so.n_tri):
        tex = _texels(sc.assets[sc.tri_asset[t]].n_leaf, 50 + t)
        eo = py_oracle.CpuEmitter(so, t, tex, "product_geometry", beta=0.2, emitter_cosine=False)
        er = py_oracle.CpuEmitter(sr, t, tex, "product_geometry", beta=0.2, emitter_cosine=False)
        for _ in range(60):
            u = rng.random(64).astype(np.float32)
            a, ka = eo.sample(u, RECV)
            b, kb = er.sample(u, RECV)
            assert ka == kb and np.array_equal(a, b)


def _shade_points(rng, n, centre, spread=1.5):
    """Shading points around a scene with unit normals."""
    p = centre + (rng.random((n, 3)) - 0.5) * 2.0 * spread
    nn = rng.normal(size=(n, 3))
    nn /= np.linalg.norm(nn, axis=1, keepdims=True)
    return np.concatenate([p, nn], axis=1)


@pytest.mark.parametrize("variant", ["area", "product", "product_geometry"])
def test_light_wrapper_equals_reference(oracle, reference, scene, variant):
    """DisplacedEmitterLight (displaced_emitter_light.cpp:20-116): light
    samples seen from shading points, the solid-angle pdf from (u, v), and
    the pdf of a direction by the walk of the emitter's triangle
    (DisplacedAreaLight::pdf, displaced_area_light.cpp:174-186), the
    oracle's restatement against the reference's own classes."""
    so, sr = py_oracle.CpuScene(oracle, scene), py_oracle.CpuScene(reference, scene)
    rng = np.random.default_rng(21)
    cos = variant != "product_geometry"  # the light wrapper turns the receiver variant's emitter cosine off
    centre = scene.tris[:, 0:3].mean(axis=0)
    walked = 0
    for t in range(so.n_tri):
        tex = _texels(scene.assets[scene.tri_asset[t]].n_leaf, 300 + t)
        eo = py_oracle.CpuEmitter(so, t, tex, variant, beta=0.05, emitter_cosine=cos)
        er = py_oracle.CpuEmitter(sr, t, tex, variant, beta=0.05, emitter_cosine=cos)
        shades = _shade_points(rng, 40, centre)
        for k, sh in enumerate(shades):
            u = rng.random(96).astype(np.float32)
            a, b = eo.light_sample(u, sh), er.light_sample(u, sh)
            if b[15]:
                assert np.array_equal(a, b), (t, k)
                # the pdf of the sampled direction from its (u, v) is the sample's
                # (the two sides round differently: dist^2 against dist * dist)
                pu = eo.light_pdf_uv(sh, a[0], a[1])
                assert pu == er.light_pdf_uv(sh, a[0], a[1]) and abs(pu - a[13]) <= 1e-12 * a[13]
                pw_o, uv_o = eo.light_pdf_walk(sh, a[8:11])
                pw_r, uv_r = er.light_pdf_walk(sh, a[8:11])
                assert pw_o == pw_r and np.array_equal(uv_o, uv_r, equal_nan=True)
                walked += pw_o > 0.0
            else:
                assert a[15] == 0.0 and np.array_equal(a[:12], b[:12])
            uv = rng.random(2) * 1.2 - 0.1
            assert eo.light_pdf_uv(sh, *uv) == er.light_pdf_uv(sh, *uv)
    assert walked > 10
