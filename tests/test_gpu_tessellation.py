"""Oracle meshes on the device (dmap_tessellate_uniform / _texel) against
the C oracle's restatement of displaced_tessellation.cpp, itself pinned bit
for bit to the reference's code (test_oracle_tessellation.py): positions,
texture coordinates, normals, indices and TexelFace records equal for every
triangle, on identity charts, general and mirrored charts, a repeat-wrapped
chart off the unit tile, and FP16 maps; the full 512 x 512 quad compared
face by face; the error paths."""
import ctypes as C

import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu

SCENES = {
    "quad": lambda: scenes.quad_scene(16),
    "quad_f16": lambda: scenes.quad_scene(32, dtype=np.float16),
    "charts": lambda: helpers.chart_scene(32),
    "sphere": lambda: helpers.small_sphere(16),
}


@pytest.fixture(scope="module")
def ctx():
    return dm.Context(0)


def _pair(ctx, oracle, name):
    sc = SCENES[name]()
    return py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("n", [1, 3, 8])
def test_uniform_equals_oracle(ctx, oracle, name, n):
    cpu, dev = _pair(ctx, oracle, name)
    got = dev.tessellate_uniform(n)
    V, F = (n + 1) * (n + 2) // 2, n * n
    assert len(got["positions"]) == V * cpu.n_tri and len(got["indices"]) == F * cpu.n_tri
    for t in range(cpu.n_tri):
        want = cpu.tessellate_uniform(t, n)
        for k in ("positions", "texcoords", "normals"):
            assert np.array_equal(got[k][t * V:(t + 1) * V], want[k]), (t, k)
        assert np.array_equal(got["indices"][t * F:(t + 1) * F], want["indices"] + t * V), t


@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("m", [1, 2, 3])
def test_texel_equals_oracle(ctx, oracle, name, m):
    cpu, dev = _pair(ctx, oracle, name)
    got = dev.tessellate_texel(m)
    f = 0
    for t in range(cpu.n_tri):
        want = cpu.tessellate_texel(t, m)
        n = len(want["interior"])
        for k in ("positions", "texcoords", "normals"):
            assert np.array_equal(got[k][f:f + n], want[k]), (t, k)
        faces = got["faces"][f:f + n]
        assert (faces["triangle"] == t).all()
        assert np.array_equal(faces["interior"], want["interior"])
        assert np.array_equal(faces["st"], want["st"])
        f += n
    assert f == len(got["faces"])


def test_texel_full_quad_512(ctx, oracle):
    """Every face of the 512 x 512 quad (about 526k faces) equal to the
    oracle's, and the faces partition the unit square in uv."""
    sc = scenes.quad_scene(512)
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    got = dev.tessellate_texel(1)
    want = [cpu.tessellate_texel(t, 1) for t in range(cpu.n_tri)]
    for k in ("positions", "texcoords", "normals"):
        assert np.array_equal(got[k], np.concatenate([w[k] for w in want])), k
    assert np.array_equal(got["faces"]["st"], np.concatenate([w["st"] for w in want]))
    st = got["faces"]["st"]
    a, b = st[:, 1] - st[:, 0], st[:, 2] - st[:, 0]
    area = 0.5 * np.abs(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]).sum()
    assert abs(area - 1.0) < 1e-12
    assert (got["faces"]["interior"] == 1).sum() == 2 * 512 * 511


def test_uniform_full_sphere(ctx, oracle):
    """The 96-triangle cube sphere at n = 64: every vertex and index."""
    sc = helpers.small_sphere(64, patches=tuple(range(96)))
    cpu, dev = py_oracle.CpuScene(oracle, sc), dm.Scene.from_synthetic(ctx, sc)
    n = 64
    got = dev.tessellate_uniform(n)
    V = (n + 1) * (n + 2) // 2
    want = [cpu.tessellate_uniform(t, n) for t in range(cpu.n_tri)]
    for k in ("positions", "texcoords", "normals"):
        assert np.array_equal(got[k], np.concatenate([w[k] for w in want])), k
    assert np.array_equal(got["indices"], np.concatenate([w["indices"] + t * V for t, w in enumerate(want)]))
    # radius-1 sphere displaced by at most the amplitude
    r = np.linalg.norm(got["positions"].astype(np.float64), axis=1)
    assert (np.abs(r - 1.0) < 0.2).all()


def test_errors(ctx):
    dev = dm.Scene.from_synthetic(ctx, scenes.quad_scene(16))
    L = dm.lib()
    n = C.c_int64()
    assert L.dmap_tessellate_texel_host(dev.h, 1, 0, None, None, None, None, C.byref(n)) == 0
    F = n.value
    assert F > 0
    small = F - 1
    pos, uv = np.empty((small, 9), np.float32), np.empty((small, 6), np.float32)
    nrm, faces = np.empty((small, 9), np.float32), np.empty(small, dm.TEXEL_FACE)
    s = L.dmap_tessellate_texel_host(dev.h, 1, small, pos.ctypes.data, uv.ctypes.data, nrm.ctypes.data,
                                     faces.ctypes.data, C.byref(n))
    assert s == dm.ERR_INVALID and n.value == F
    assert L.dmap_tessellate_texel_host(dev.h, 0, 0, None, None, None, None, C.byref(n)) == dm.ERR_INVALID
    # more vertices than uint32 indices can address: refused before any work
    one = np.empty(1, np.float32)
    idx = np.empty(1, np.uint32)
    s = L.dmap_tessellate_uniform_host(dev.h, 70000, one.ctypes.data, one.ctypes.data, one.ctypes.data,
                                       idx.ctypes.data)
    assert s == dm.ERR_INVALID
    with pytest.raises(dm.DmapError):
        dev.tessellate_uniform(0)
