"""ctypes bindings of the CPU checkers. TEST INFRASTRUCTURE ONLY.

`Oracle` wraps liboracle.so (the C restatement, dmap_oracle.c); `Reference`
wraps _ref/libdmap_ref.so (the reference's own sources built in place). Both
expose the same methods, so a test can run one scene through either and
compare. Only tests/, the smoke check and bench.py's CPU-baseline leg use it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
HIT = 12          # doubles per hit record
ST = 8            # int64 per-ray statistics
ST_NAMES = ("triangle_tests", "node_tests", "leaf_tests", "sub_squares", "newton_iters",
            "node_tests_after_hit", "leaf_tests_after_hit")

BOUND = {"box": 0, "slab": 1, "both": 2}
LEAF = {"newton": 0, "two_triangle": 1}
ORDER = {"index": 0, "nearest": 1}

_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_int64)


def build(ref: bool = False) -> None:
    """Builds liboracle.so (and _ref/ when ref and the reference sources exist)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


class _Lib:
    prefix = "o_"
    path = HERE / "liboracle.so"

    def __init__(self):
        if not self.path.exists():
            build(ref=self.prefix == "r_")
        self.lib = C.CDLL(str(self.path))
        p = self.prefix
        L = self.lib

        def f(name, res, *args):
            fn = getattr(L, p + name)
            fn.restype = res
            fn.argtypes = list(args)
            return fn

        self._pyr_build = f("pyramid_build", C.c_void_p, _dp, C.c_int, C.c_double, C.c_double, C.c_int)
        self._pyr_free = f("pyramid_free", None, C.c_void_p)
        self._pyr_levels = f("pyramid_levels", C.c_int, C.c_void_p)
        self._pyr_level = f("pyramid_level", None, C.c_void_p, C.c_int, _dp)
        self._pyr_node = f("pyramid_node", None, C.c_void_p, C.c_int, C.c_int64, C.c_int64, _dp)
        self._sc_create = f("scene_create", C.c_void_p)
        self._sc_free = f("scene_free", None, C.c_void_p)
        self._sc_add = f("scene_add_object", C.c_int, C.c_void_p, _dp, C.c_int, C.c_double, C.c_double, C.c_int,
                         C.c_int, _dp, C.c_int)
        self._sc_ntri = f("scene_triangle_count", C.c_int, C.c_void_p)
        _u8 = C.POINTER(C.c_uint8)
        self._sc_opacity = f("scene_set_opacity", None, C.c_void_p, _u8, C.c_int, C.c_int, _dp, _u8)
        self._sc_info = f("scene_triangle_info", None, C.c_void_p, C.c_int, _dp)
        self._sc_frame = f("scene_triangle_frame", None, C.c_void_p, C.c_int, _dp)
        self._tri_isect = f("triangle_intersect", C.c_int, C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, C.c_int,
                            _dp, _lp)
        self._node_bound = f("node_bound", None, C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_int64, _dp, C.c_int,
                             C.c_int, _dp)
        self._disp = f("displaced_position", None, C.c_void_p, C.c_int, C.c_double, C.c_double, _dp)
        _fp = C.POINTER(C.c_float)
        self._tess_uniform = f("tessellate_uniform", None, C.c_void_p, C.c_int, C.c_int, _fp, _fp, _fp,
                               C.POINTER(C.c_uint32))
        self._tess_texel = f("tessellate_texel", C.c_int64, C.c_void_p, C.c_int, C.c_int, C.c_int64, _fp, _fp, _fp,
                             _dp, C.POINTER(C.c_int))
        self._em_create = f("emitter_create", C.c_void_p, C.c_void_p, C.c_int, _dp, C.c_int, C.c_int, C.c_double,
                            C.c_int)
        self._em_free = f("emitter_free", None, C.c_void_p)
        self._em_info = f("emitter_info", None, C.c_void_p, _dp)
        self._em_sample = f("emitter_sample", C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_int, _dp, _dp)
        self._em_pdf_uv = f("emitter_pdf_uv", C.c_double, C.c_void_p, C.c_double, C.c_double, _dp)
        self._em_pdf_area = f("emitter_pdf_area", C.c_double, C.c_void_p, C.c_double, C.c_double, _dp)
        self._em_leaf_prob = f("emitter_leaf_prob", C.c_double, C.c_void_p, C.c_int64, C.c_int64, _dp)
        self._em_light_sample = f("emitter_light_sample", C.c_int, C.c_void_p, C.POINTER(C.c_float), C.c_int, _dp,
                                  _dp)
        self._em_light_pdf_uv = f("emitter_light_pdf_uv", C.c_double, C.c_void_p, _dp, C.c_double, C.c_double)
        self._em_light_pdf_walk = f("emitter_light_pdf_walk", C.c_double, C.c_void_p, _dp, _dp, _dp)
        if self.prefix == "o_":
            self._sc_isect = f("scene_intersect", C.c_int64, C.c_void_p, _dp, C.c_int64, C.c_int, C.c_int, C.c_int,
                               _dp, _lp, _lp, C.c_int, C.c_int)
            self._param = f("triangle_param", None, C.c_void_p, C.c_int, C.c_double, C.c_double, _dp)
            self._surf = f("surface_point", None, C.c_void_p, C.c_int, C.c_double, C.c_double, _dp, _dp, C.c_int,
                           _dp)
        else:
            self._sc_isect = f("scene_intersect", C.c_int64, C.c_void_p, _dp, C.c_int64, C.c_int, C.c_int, C.c_int,
                               _dp, _lp, C.c_int)

    # -- pyramid --------------------------------------------------------
    def pyramid(self, values, scale=1.0, offset=0.0, build="fold"):
        """Levels of TaylorPyramid(values, scale, build, offset): a list of
        dicts of (m, m) channel arrays."""
        v = np.ascontiguousarray(values, np.float64)
        p = self._pyr_build(_ptr(v), v.shape[0], scale, offset, 0 if build == "fold" else 1)
        if not p:
            raise ValueError("pyramid needs a (2^L + 1) x (2^L + 1) node grid")
        try:
            out = []
            n = v.shape[0] - 1
            for lvl in range(self._pyr_levels(p)):
                m = n >> lvl
                buf = np.empty(8 * m * m)
                self._pyr_level(p, lvl, _ptr(buf))
                buf = buf.reshape(8, m, m)
                out.append({k: buf[c].copy() for c, k in enumerate(
                    ("h0", "gu", "gv", "r", "ru", "rv", "h_min", "h_max"))})
            return out
        finally:
            self._pyr_free(p)


class Oracle(_Lib):
    prefix = "o_"
    path = HERE / "liboracle.so"


class Reference(_Lib):
    prefix = "r_"
    path = HERE / "_ref" / "libdmap_ref.so"

    @classmethod
    def available(cls) -> bool:
        return cls.path.exists()


class CpuScene:
    """A scene on one of the CPU checkers: objects in asset order, each the
    reference's ObjectIntersector over its triangles."""

    def __init__(self, lib: _Lib, scene, build="fold"):
        self.lib = lib
        self.h = lib._sc_create()
        self.scene = scene
        for asset, tris in scene.objects():
            if len(tris) == 0:
                continue
            v = np.ascontiguousarray(asset.nodes, np.float64)
            t = np.ascontiguousarray(tris, np.float64)
            k = lib._sc_add(self.h, _ptr(v), v.shape[0], float(asset.scale), float(asset.offset),
                            int(asset.repeat), 0 if build == "fold" else 1, _ptr(t), len(t))
            if k < 0:
                raise ValueError("degenerate base triangle or bad node grid")
        self.n_tri = lib._sc_ntri(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib._sc_free(self.h)
            self.h = None

    def intersect(self, rays, bound="both", slab_max_level=1, leaf="newton", stats=False, threads=0,
                  order="nearest"):
        """rays: (n, 8) o, d, t_min, t_max. Returns (hits (n, 12), stats (n, 8) or None).
        order: "index" (the reference's flat loop) or "nearest" (box entry
        first, the library's default); the reference build has the flat loop only."""
        r = np.ascontiguousarray(rays, np.float64)
        n = len(r)
        hits = np.empty((n, HIT))
        st = np.zeros((n, ST), np.int64) if stats else None
        if isinstance(self.lib, Oracle):
            self.lib._sc_isect(self.h, _ptr(r), n, BOUND[bound], slab_max_level, LEAF[leaf], _ptr(hits),
                               _ptr(st, _lp), None, threads, ORDER[order])
        else:
            if order != "index":
                raise ValueError("the reference build runs the flat loop (order='index') only")
            self.lib._sc_isect(self.h, _ptr(r), n, BOUND[bound], slab_max_level, LEAF[leaf], _ptr(hits),
                               _ptr(st, _lp), threads)
        return hits, st

    def set_opacity(self, mask=None, uv_scale=(1.0, 1.0), uv_offset=(0.0, 0.0), flip_v=False, tri_flags=None):
        """The opacity filter of dmap_scene_set_opacity: mask (h, w) uint8,
        0 transparent; tri_flags (n_tri,) marks the triangles it covers
        (None: all). mask None removes it."""
        u8 = C.POINTER(C.c_uint8)
        if mask is None:
            self.lib._sc_opacity(self.h, None, 0, 0, None, None)
            return
        m = np.ascontiguousarray(mask, np.uint8)
        mp = np.array([uv_scale[0], uv_scale[1], uv_offset[0], uv_offset[1], 1.0 if flip_v else 0.0])
        tf = None if tri_flags is None else np.ascontiguousarray(tri_flags, np.uint8)
        self.lib._sc_opacity(self.h, m.ctypes.data_as(u8), m.shape[1], m.shape[0], _ptr(mp),
                             None if tf is None else tf.ctypes.data_as(u8))

    def triangle_info(self, tri):
        out = np.empty(11)
        self.lib._sc_info(self.h, tri, _ptr(out))
        return out

    def triangle_frame(self, tri):
        out = np.empty(12)
        self.lib._sc_frame(self.h, tri, _ptr(out))
        return out

    def node_bound(self, tri, level, i, j, ray, bound="both", slab_max_level=1):
        out = np.empty(16)
        r = np.ascontiguousarray(ray, np.float64)
        self.lib._node_bound(self.h, tri, level, i, j, _ptr(r), BOUND[bound], slab_max_level, _ptr(out))
        return out

    def displaced_position(self, tri, s, t):
        out = np.empty(3)
        self.lib._disp(self.h, tri, s, t, _ptr(out))
        return out

    def surface_point(self, tri, u, v, uv_scale=(1.0, 1.0), uv_offset=(0.0, 0.0), flip_v=False):
        """DisplacedGeometry::surface_point at barycentrics (u, v): 14 values
        p, ng, dpdu, dpdv, uv (C oracle only)."""
        out = np.empty(14)
        sc = np.array(uv_scale, np.float64)
        of = np.array(uv_offset, np.float64)
        self.lib._surf(self.h, tri, u, v, _ptr(sc), _ptr(of), int(flip_v), _ptr(out))
        return out

    def tessellate_uniform(self, tri, n):
        """append_displaced_triangle at subdivision n: dict of positions
        (V, 3), texcoords (V, 2), normals (V, 3) float32 and indices (n*n, 3)
        uint32 relative to the triangle's first vertex."""
        V = (n + 1) * (n + 2) // 2
        out = {"positions": np.empty((V, 3), np.float32), "texcoords": np.empty((V, 2), np.float32),
               "normals": np.empty((V, 3), np.float32), "indices": np.empty((n * n, 3), np.uint32)}
        fp = C.POINTER(C.c_float)
        self.lib._tess_uniform(self.h, tri, n, _ptr(out["positions"], fp), _ptr(out["texcoords"], fp),
                               _ptr(out["normals"], fp), _ptr(out["indices"], C.POINTER(C.c_uint32)))
        return out

    def tessellate_texel(self, tri, m):
        """append_texel_tessellation with m x m sub-cells: dict of per-face
        positions (F, 3, 3), texcoords (F, 3, 2), normals (F, 3, 3) float32,
        st (F, 3, 2) double and interior (F,) int32."""
        fp = C.POINTER(C.c_float)
        n = self.lib._tess_texel(self.h, tri, m, 0, None, None, None, None, None)
        out = {"positions": np.empty((n, 3, 3), np.float32), "texcoords": np.empty((n, 3, 2), np.float32),
               "normals": np.empty((n, 3, 3), np.float32), "st": np.empty((n, 3, 2)),
               "interior": np.empty(n, np.int32)}
        got = self.lib._tess_texel(self.h, tri, m, n, _ptr(out["positions"], fp), _ptr(out["texcoords"], fp),
                                   _ptr(out["normals"], fp), _ptr(out["st"]),
                                   _ptr(out["interior"], C.POINTER(C.c_int)))
        assert got == n
        return out


VARIANT = {"area": 0, "product": 1, "product_geometry": 2}


class CpuEmitter:
    """DescentSampler of one scene triangle (descent_sampler.h:105-160) on
    one of the CPU checkers, with an n_leaf x n_leaf emission texel grid."""

    def __init__(self, cpu: CpuScene, tri: int, texels, variant="product", beta=0.05, emitter_cosine=True):
        self.lib = cpu.lib
        self.cpu = cpu  # keeps the scene alive
        t = np.ascontiguousarray(texels, np.float64)
        self.h = self.lib._em_create(cpu.h, tri, _ptr(t), t.shape[0], VARIANT[variant], beta, int(emitter_cosine))
        if not self.h:
            raise ValueError("emission grid does not match the pyramid's leaf count")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib._em_free(self.h)
            self.h = None

    def info(self):
        out = np.empty(6)
        self.lib._em_info(self.h, _ptr(out))
        return out

    @staticmethod
    def _recv(receiver):
        return None if receiver is None else np.ascontiguousarray(receiver, np.float64)

    def sample(self, u, receiver=None):
        """u: float32 uniforms; returns (11 values u, v, p, n, sqrt_det,
        pdf_uv, pdf_area, draws used)."""
        uu = np.ascontiguousarray(u, np.float32)
        out = np.empty(11)
        r = self._recv(receiver)
        k = self.lib._em_sample(self.h, _ptr(uu, C.POINTER(C.c_float)), len(uu), _ptr(r), _ptr(out))
        return out, k

    def pdf_uv(self, u, v, receiver=None):
        return self.lib._em_pdf_uv(self.h, u, v, _ptr(self._recv(receiver)))

    def pdf_area(self, u, v, receiver=None):
        return self.lib._em_pdf_area(self.h, u, v, _ptr(self._recv(receiver)))

    def leaf_prob(self, i, j, receiver=None):
        return self.lib._em_leaf_prob(self.h, i, j, _ptr(self._recv(receiver)))

    # DisplacedEmitterLight (displaced_emitter_light.cpp:20-116) seen from
    # shade = (p, n), 6 doubles
    def light_sample(self, u, shade):
        """(16 values u, v, y, n_y, wi, dist, pdf_area, pdf_omega, Le, ok)."""
        uu = np.ascontiguousarray(u, np.float32)
        out = np.empty(16)
        self.lib._em_light_sample(self.h, _ptr(uu, C.POINTER(C.c_float)), len(uu),
                                  _ptr(np.ascontiguousarray(shade, np.float64)), _ptr(out))
        return out

    def light_pdf_uv(self, shade, u, v):
        return self.lib._em_light_pdf_uv(self.h, _ptr(np.ascontiguousarray(shade, np.float64)), u, v)

    def light_pdf_walk(self, shade, wi):
        """(pdf_omega, uv of the walk's crossing, NaN on a miss)."""
        uv = np.empty(2)
        pdf = self.lib._em_light_pdf_walk(self.h, _ptr(np.ascontiguousarray(shade, np.float64)),
                                          _ptr(np.ascontiguousarray(wi, np.float64)), _ptr(uv))
        return pdf, uv
