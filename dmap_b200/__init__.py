"""dmap_b200: the ray vs displaced-surface query of MangoSister/dmap on B200.

Python mirror of the reference's C++ interface for this path, over the C ABI
of include/dmap_b200.h (libdmap_b200.so, built in place by
``python -m dmap_b200.build``):

- ``Asset``: a displacement map's HeightGrid and its TaylorPyramid, built on
  the device (taylor_pyramid.h:89-92, displacement_asset.cpp:16-35).
- ``Scene``: ObjectIntersector over base triangles of one or more assets
  (displaced_intersector.h:176-198); ``intersect`` answers closest-hit
  queries (ObjectIntersector::intersect, embree intersect_callback) and
  occlusion queries (occluded_callback) for a batch of rays.
- ``TraversalOptions``: the reference's bound / slab_max_level / leaf
  (traversal_options.h:30-38) plus precision, mode and the schedule.
- ``Scene.render``: the batched path tracer (emitter-sampled shadow rays
  through the occlusion query); ``Server``: continuous batching of many
  callers' requests over resident scenes; ``Scene.autotune``: the schedule
  autotuner.

There is no CPU fallback: without the built library or a CUDA device every
entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

_PKG = Path(__file__).resolve().parent
# DMAP_B200_LIB names another build of the library (tuning variants)
LIB_PATH = Path(os.environ.get("DMAP_B200_LIB") or _PKG / "libdmap_b200.so")

F32, F16, F64, BF16 = 0, 1, 2, 3
BOUND = {"box": 0, "slab": 1, "both": 2}
LEAF = {"newton": 0, "two_triangle": 1}
PRECISION = {"f64": 0, "f32": 1}
MODE = {"closest": 0, "occluded": 1}
SCHEDULE = {"wavefront": 0, "simple": 1}
ORDER = {"index": 0, "nearest": 1}
KEEP_F64, BUILD_DIRECT = 1, 2
OK, ERR_INVALID, ERR_CUDA, ERR_OOM = 0, 1, 2, 3  # dmap_status
ERR_UNSUPPORTED = 8

HIT32 = np.dtype([("t", "<f4"), ("st", "<f4", 2), ("bary", "<f4", 2), ("ng", "<f4", 3), ("tri", "<i4"),
                  ("i", "<i4"), ("j", "<i4"), ("flags", "<i4")])
HIT64 = np.dtype([("t", "<f8"), ("st", "<f8", 2), ("bary", "<f8", 2), ("ng", "<f8", 3), ("tri", "<i4"),
                  ("i", "<i4"), ("j", "<i4"), ("flags", "<i4")])
STATS = ("triangle_tests", "node_tests", "leaf_tests", "sub_squares", "newton_iters", "node_tests_after_hit",
         "leaf_tests_after_hit", "reserved")
HIT_FP64_LEAF, HIT_CAPPED, HIT_POLISHED = 1, 2, 4


class DmapError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"dmap status {status}: {msg}")
        self.status = status


class _Options(C.Structure):
    _fields_ = [("bound", C.c_int), ("slab_max_level", C.c_int), ("leaf", C.c_int), ("precision", C.c_int),
                ("mode", C.c_int), ("polish_cond", C.c_double), ("schedule", C.c_int), ("rounds", C.c_int),
                ("blocks_per_sm", C.c_int), ("order", C.c_int), ("node_visit_cap", C.c_int),
                ("leaf_precision", C.c_int), ("graph", C.c_int)]


class _Camera(C.Structure):
    _fields_ = [("eye", C.c_double * 3), ("target", C.c_double * 3), ("up", C.c_double * 3), ("fov_deg", C.c_double),
                ("width", C.c_int), ("height", C.c_int)]


class _RenderDesc(C.Structure):
    _fields_ = [("camera", _Camera), ("emitter_p0", C.c_double * 3), ("emitter_e1", C.c_double * 3),
                ("emitter_e2", C.c_double * 3), ("radiance", C.c_double * 3), ("albedo", C.c_double * 3),
                ("spp", C.c_int), ("max_depth", C.c_int), ("rr_depth", C.c_int), ("seed", C.c_uint64),
                ("paths_per_batch", C.c_int64), ("use_graph", C.c_int)]


class _RenderStats(C.Structure):
    _fields_ = [("paths", C.c_int64), ("extension_rays", C.c_int64), ("shadow_rays", C.c_int64),
                ("batches", C.c_int64), ("kernel_launches", C.c_int64), ("device_ms", C.c_double)]


class _RayRecord(C.Structure):
    _fields_ = [("capacity", C.c_int64), ("rays", C.c_void_p), ("kind", C.c_void_p), ("tri", C.c_void_p),
                ("t", C.c_void_p), ("count", C.c_int64)]


class _UvMap(C.Structure):
    _fields_ = [("uv_scale", C.c_double * 2), ("uv_offset", C.c_double * 2), ("flip_v", C.c_int)]


# dmap_emitter_point
EMITTER_POINT = np.dtype([("u", "<f8"), ("v", "<f8"), ("p", "<f8", 3), ("n", "<f8", 3), ("sqrt_det", "<f8"),
                          ("pdf_uv", "<f8"), ("pdf_area", "<f8"), ("tri", "<i4"), ("draws", "<i4")])
DESCENT = {"area": 0, "product": 1, "product_geometry": 2}
EMITTER_LIGHT = np.dtype([("u", "<f8"), ("v", "<f8"), ("y", "<f8", 3), ("n_y", "<f8", 3), ("wi", "<f8", 3),
                          ("dist", "<f8"), ("pdf_area", "<f8"), ("pdf_omega", "<f8"), ("Le", "<f8"),
                          ("tri", "<i4"), ("ok", "<i4")])

# dmap_texel_face: triangle, interior, st[3][2]
TEXEL_FACE = np.dtype([("triangle", np.int32), ("interior", np.int32), ("st", np.float64, (3, 2))])


class _ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_batch_rays", C.c_int64), ("max_inflight", C.c_int),
                ("slots", C.c_int), ("options", _Options), ("policy", C.c_int)]


class _ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("cancelled", C.c_int64),
                ("queued", C.c_int64), ("active", C.c_int64), ("rays", C.c_int64), ("launches", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
                ("held_bytes", C.c_size_t), ("peak_bytes", C.c_size_t), ("busy_s", C.c_double),
                ("wall_s", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """The loaded C library; raises when it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise DmapError(-1, f"{LIB_PATH} is not built (python -m dmap_b200.build)")
        L = C.CDLL(str(LIB_PATH))
        vp, i32, i64, dbl, u32 = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_uint
        sigs = {
            "dmap_create": (i32, [i32, C.POINTER(vp)]),
            "dmap_destroy": (None, [vp]),
            "dmap_status_string": (C.c_char_p, [i32]),
            "dmap_last_error": (C.c_char_p, [vp]),
            "dmap_kernel_launches": (i64, [vp]),
            "dmap_options_default": (None, [C.POINTER(_Options)]),
            "dmap_asset_create": (i32, [vp, vp, i32, i32, dbl, dbl, i32, u32, C.POINTER(vp)]),
            "dmap_asset_destroy": (None, [vp]),
            "dmap_asset_levels": (i32, [vp]),
            "dmap_asset_bytes": (C.c_size_t, [vp]),
            "dmap_asset_build_ms": (dbl, [vp]),
            "dmap_asset_pyramid_level": (i32, [vp, i32, i32, vp]),
            "dmap_scene_create": (i32, [vp, vp, i32, vp, vp, i32, C.POINTER(vp)]),
            "dmap_scene_create_charts": (i32, [vp, vp, i32, vp, vp, i32, C.POINTER(vp)]),
            "dmap_scene_create_instanced": (i32, [vp, vp, i32, vp, vp, vp, i32, vp, vp, i32, C.POINTER(vp)]),
            "dmap_scene_destroy": (None, [vp]),
            "dmap_scene_triangle_count": (i32, [vp]),
            "dmap_scene_triangle_info": (i32, [vp, i32, vp]),
            "dmap_intersect": (i32, [vp, vp, i32, i64, C.POINTER(_Options), vp, i32, vp, vp]),
            "dmap_intersect_host": (i32, [vp, vp, i32, i64, C.POINTER(_Options), vp, i32, vp]),
            "dmap_render": (i32, [vp, C.POINTER(_RenderDesc), C.POINTER(_Options), vp, C.POINTER(_RenderStats),
                                  C.POINTER(_RayRecord)]),
            "dmap_autotune": (i32, [vp, vp, i32, i64, C.POINTER(_Options), C.c_char_p, C.POINTER(_Options),
                                    C.POINTER(dbl)]),
            "dmap_surface_points": (i32, [vp, vp, i32, i64, C.POINTER(_UvMap), vp, vp]),
            "dmap_surface_points_host": (i32, [vp, vp, i32, i64, C.POINTER(_UvMap), vp]),
            "dmap_scene_set_opacity": (i32, [vp, vp, i32, i32, C.POINTER(_UvMap), vp]),
            "dmap_tessellate_uniform": (i32, [vp, i32, vp, vp, vp, vp, vp]),
            "dmap_tessellate_uniform_host": (i32, [vp, i32, vp, vp, vp, vp]),
            "dmap_tessellate_texel": (i32, [vp, i32, i64, vp, vp, vp, vp, C.POINTER(i64), vp]),
            "dmap_tessellate_texel_host": (i32, [vp, i32, i64, vp, vp, vp, vp, C.POINTER(i64)]),
            "dmap_emitter_create": (i32, [vp, vp, i32, dbl, i32, C.POINTER(vp)]),
            "dmap_emitter_destroy": (None, [vp]),
            "dmap_emitter_triangle_info": (i32, [vp, i32, vp]),
            "dmap_emitter_sample": (i32, [vp, vp, vp, i32, vp, i64, vp, vp]),
            "dmap_emitter_pdf": (i32, [vp, vp, vp, vp, i64, vp, vp, vp]),
            "dmap_emitter_sample_host": (i32, [vp, vp, vp, i32, vp, i64, vp]),
            "dmap_emitter_pdf_host": (i32, [vp, vp, vp, vp, i64, vp, vp]),
            "dmap_emitter_light": (i32, [vp, vp, vp, i64, vp, vp]),
            "dmap_emitter_light_pdf": (i32, [vp, vp, vp, vp, vp, i64, vp, vp, vp]),
            "dmap_emitter_light_host": (i32, [vp, vp, vp, i64, vp]),
            "dmap_emitter_light_pdf_host": (i32, [vp, vp, vp, vp, vp, i64, vp, vp]),
            "dmap_server_create": (i32, [vp, C.POINTER(_ServerConfig), C.POINTER(vp)]),
            "dmap_server_destroy": (None, [vp]),
            "dmap_server_submit_rays": (i32, [vp, vp, vp, i64, i32, vp, C.POINTER(C.c_uint64)]),
            "dmap_server_submit_render": (i32, [vp, vp, C.POINTER(_RenderDesc), vp, C.POINTER(C.c_uint64)]),
            "dmap_server_poll": (i32, [vp, C.c_uint64]),
            "dmap_server_wait": (i32, [vp, C.c_uint64, dbl]),
            "dmap_server_cancel": (i32, [vp, C.c_uint64]),
            "dmap_server_pause": (i32, [vp, C.c_int]),
            "dmap_server_latency": (i32, [vp, C.c_uint64, C.POINTER(dbl)]),
            "dmap_server_drain": (i32, [vp, dbl]),
            "dmap_server_get_stats": (i32, [vp, C.POINTER(_ServerStats)]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> Sequence[str]:
    """Every function include/dmap_b200.h declares."""
    import re
    text = (_PKG.parent / "include" / "dmap_b200.h").read_text()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(dmap_\w+)\(", text, re.M)))


@dataclass
class TraversalOptions:
    bound: str = "both"
    slab_max_level: int = 1
    leaf: str = "newton"
    precision: str = "f32"
    mode: str = "closest"
    polish_cond: float = 1e4
    schedule: str = "wavefront"
    rounds: int = 2
    blocks_per_sm: int = 0
    order: str = "nearest"
    node_visit_cap: int = 0
    leaf_precision: str = "f32"
    graph: bool = False

    def c(self) -> _Options:
        return _Options(BOUND[self.bound], self.slab_max_level, LEAF[self.leaf], PRECISION[self.precision],
                        MODE[self.mode], self.polish_cond, SCHEDULE[self.schedule], self.rounds,
                        self.blocks_per_sm, ORDER[self.order], self.node_visit_cap,
                        PRECISION[self.leaf_precision], int(self.graph))


class Context:
    """One device: streams, staging and the device status word."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        s = lib().dmap_create(device, C.byref(h))
        if s:
            raise DmapError(s, f"dmap_create({device}): {lib().dmap_status_string(s).decode()}")
        self.h = h

    def check(self, s: int, what: str):
        if s:
            raise DmapError(s, f"{what}: {lib().dmap_status_string(s).decode()}: "
                               f"{lib().dmap_last_error(self.h).decode()}")

    @property
    def kernel_launches(self) -> int:
        return lib().dmap_kernel_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().dmap_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DT = {np.dtype(np.float32): F32, np.dtype(np.float16): F16, np.dtype(np.float64): F64}
CHANNELS = ("h0", "gu", "gv", "r", "ru", "rv", "h_min", "h_max")


def to_bf16(values: np.ndarray) -> np.ndarray:
    """Rounds values to bfloat16 (to nearest, ties to even) and returns the
    16-bit patterns (uint16), the texel layout of a DMAP_BF16 asset."""
    f = np.ascontiguousarray(values, np.float32)
    if not np.isfinite(f).all():
        raise ValueError("bfloat16 texels must be finite")
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16(bits: np.ndarray) -> np.ndarray:
    """The values of bfloat16 patterns, exactly, as float64."""
    return (np.ascontiguousarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


class Asset:
    """HeightGrid + TaylorPyramid of one node grid on the device. texel
    "bf16" stores the grid as bfloat16 (the values rounded by to_bf16);
    otherwise the array's own float32 / float16 / float64 type is kept."""

    def __init__(self, ctx: Context, nodes: np.ndarray, scale: float = 1.0, offset: float = 0.0,
                 repeat: bool = False, keep_f64: bool = False, build: str = "fold", texel: Optional[str] = None):
        if texel not in (None, "bf16"):
            raise ValueError("texel is None or 'bf16'")
        v = np.ascontiguousarray(nodes)
        if texel == "bf16":
            v = to_bf16(v)
        elif v.dtype not in _DT:
            v = v.astype(np.float64)
        if v.ndim != 2 or v.shape[0] != v.shape[1]:
            raise ValueError("the node grid must be square")
        if build not in ("fold", "direct"):
            raise ValueError("build is 'fold' or 'direct'")
        self.ctx = ctx
        h = C.c_void_p()
        flags = (KEEP_F64 if keep_f64 else 0) | (BUILD_DIRECT if build == "direct" else 0)
        dt = BF16 if texel == "bf16" else _DT[v.dtype]
        ctx.check(lib().dmap_asset_create(ctx.h, v.ctypes.data, dt, v.shape[0], scale, offset, int(repeat), flags,
                                          C.byref(h)), "dmap_asset_create")
        self.h = h
        self.nodes = v.shape[0]
        self.n_leaf = v.shape[0] - 1

    @property
    def n_levels(self) -> int:
        return lib().dmap_asset_levels(self.h)

    @property
    def device_bytes(self) -> int:
        return lib().dmap_asset_bytes(self.h)

    @property
    def build_ms(self) -> float:
        """CUDA-event time of the pyramid build kernels."""
        return lib().dmap_asset_build_ms(self.h)

    def level(self, level: int, precision: str = "f64") -> dict:
        m = self.n_leaf >> level
        out = np.empty(8 * m * m)
        self.ctx.check(lib().dmap_asset_pyramid_level(self.h, level, PRECISION[precision], out.ctypes.data),
                       "dmap_asset_pyramid_level")
        out = out.reshape(8, m, m)
        return {k: out[c].copy() for c, k in enumerate(CHANNELS)}

    def levels(self, precision: str = "f64"):
        return [self.level(l, precision) for l in range(self.n_levels)]

    def close(self):
        # after its context (finalizers at interpreter exit run in any
        # order) the handle is only forgotten: the process frees the device
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib().dmap_asset_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """ObjectIntersector over base triangles (n x 24 doubles: p0, p1, p2,
    m0, m1, m2, t0, t1, t2), triangle k displaced by assets[tri_asset[k]]."""

    def __init__(self, ctx: Context, assets: Sequence[Asset], tris: np.ndarray, tri_asset: np.ndarray):
        self.ctx = ctx
        self.assets = list(assets)
        t = np.ascontiguousarray(tris, np.float64).reshape(-1, 24)
        ta = np.ascontiguousarray(tri_asset, np.int32)
        arr = (C.c_void_p * len(self.assets))(*[a.h.value for a in self.assets])
        h = C.c_void_p()
        ctx.check(lib().dmap_scene_create(ctx.h, arr, len(self.assets), ta.ctypes.data, t.ctypes.data, len(t),
                                          C.byref(h)), "dmap_scene_create")
        self.h = h
        self.n_tri = len(t)

    @classmethod
    def instanced(cls, ctx: Context, assets: Sequence[Asset], tris: np.ndarray, tri_asset: np.ndarray,
                  object_first: Sequence[int], instance_object: Sequence[int], to_world: np.ndarray):
        """dmap_scene_create_instanced: objects are triangle ranges
        (object_first, n_objects + 1 offsets), instances (object, 3x4 rigid
        to_world) expanded in order."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.assets = list(assets)
        t = np.ascontiguousarray(tris, np.float64).reshape(-1, 24)
        ta = np.ascontiguousarray(tri_asset, np.int32)
        of = np.ascontiguousarray(object_first, np.int32)
        io = np.ascontiguousarray(instance_object, np.int32)
        M = np.ascontiguousarray(to_world, np.float64).reshape(-1, 12)
        arr = (C.c_void_p * len(self.assets))(*[a.h.value for a in self.assets])
        h = C.c_void_p()
        ctx.check(lib().dmap_scene_create_instanced(ctx.h, arr, len(self.assets), ta.ctypes.data, t.ctypes.data,
                                                    of.ctypes.data, len(of) - 1, io.ctypes.data, M.ctypes.data,
                                                    len(io), C.byref(h)), "dmap_scene_create_instanced")
        self.h = h
        self.n_tri = lib().dmap_scene_triangle_count(h)
        return self

    @classmethod
    def from_synthetic(cls, ctx: Context, scene, keep_f64: bool = False, build: str = "fold",
                       texel: Optional[str] = None):
        """A dmap_b200.scenes.Scene on the device (texel as Asset's)."""
        assets = [Asset(ctx, a.nodes, a.scale, a.offset, a.repeat, keep_f64, build, texel) for a in scene.assets]
        return cls(ctx, assets, scene.tris, scene.tri_asset)

    def triangle_info(self, tri: int) -> np.ndarray:
        out = np.empty(11)
        self.ctx.check(lib().dmap_scene_triangle_info(self.h, tri, out.ctypes.data), "dmap_scene_triangle_info")
        return out

    def intersect(self, rays: np.ndarray, options: Optional[TraversalOptions] = None, hit_dtype=np.float64,
                  stats: bool = False):
        """Host batch query: rays (n, 8) float32/float64 -> structured hits
        (HIT32 or HIT64) and, when asked, (n, 8) int64 counters."""
        opt = (options or TraversalOptions()).c()
        r = np.ascontiguousarray(rays)
        if r.dtype not in (np.float32, np.float64):
            r = r.astype(np.float64)
        n = len(r)
        hd = HIT64 if np.dtype(hit_dtype) == np.float64 else HIT32
        hits = np.empty(n, hd)
        st = np.zeros((n, 8), np.int64) if stats else None
        self.ctx.check(lib().dmap_intersect_host(self.h, r.ctypes.data, _DT[r.dtype], n, C.byref(opt),
                                                 hits.ctypes.data, F64 if hd is HIT64 else F32,
                                                 st.ctypes.data if stats else None), "dmap_intersect_host")
        return (hits, st) if stats else hits

    def intersect_device(self, rays_ptr: int, ray_dtype: int, n: int, hits_ptr: int, hit_dtype: int,
                         options: Optional[TraversalOptions] = None, stats_ptr: int = 0, stream: int = 0):
        """Device batch query on raw device pointers (asynchronous)."""
        opt = (options or TraversalOptions()).c()
        self.ctx.check(lib().dmap_intersect(self.h, rays_ptr, ray_dtype, n, C.byref(opt), hits_ptr, hit_dtype,
                                            stats_ptr or None, stream or None), "dmap_intersect")

    def surface_points(self, hits: np.ndarray, uv_scale=(1.0, 1.0), uv_offset=(0.0, 0.0), flip_v: bool = False):
        """DisplacedGeometry::surface_point for every hit record (HIT32 or
        HIT64 array): (n, 14) doubles p, ng, dpdu, dpdv, uv; zeros for misses."""
        h = np.ascontiguousarray(hits)
        dt = F64 if h.dtype == HIT64 else F32
        out = np.empty((len(h), 14))
        m = _UvMap((C.c_double * 2)(*uv_scale), (C.c_double * 2)(*uv_offset), int(flip_v))
        self.ctx.check(lib().dmap_surface_points_host(self.h, h.ctypes.data, dt, len(h), C.byref(m),
                                                      out.ctypes.data), "dmap_surface_points_host")
        return out

    def set_opacity(self, mask: Optional[np.ndarray] = None, uv_scale=(1.0, 1.0), uv_offset=(0.0, 0.0),
                    flip_v: bool = False, tri_flags: Optional[np.ndarray] = None):
        """dmap_scene_set_opacity: ks's opacity map as the scene's hit filter
        (embree's filter functions in DisplacedGeometry's callbacks), a (h, w)
        uint8 mask over the object's texture coordinates, 0 transparent;
        tri_flags (n_tri,) marks the triangles it covers (None: all). mask
        None removes it. Filtered scenes run precision "f64" or schedule
        "simple"."""
        if mask is None:
            self.ctx.check(lib().dmap_scene_set_opacity(self.h, None, 0, 0, None, None), "dmap_scene_set_opacity")
            return
        m = np.ascontiguousarray(mask, np.uint8)
        if m.ndim != 2:
            raise ValueError("the opacity mask is (h, w)")
        tf = None if tri_flags is None else np.ascontiguousarray(tri_flags, np.uint8)
        if tf is not None and tf.shape != (self.n_tri,):
            raise ValueError("tri_flags needs one byte per triangle")
        uvm = _UvMap((C.c_double * 2)(*uv_scale), (C.c_double * 2)(*uv_offset), int(flip_v))
        self.ctx.check(lib().dmap_scene_set_opacity(self.h, m.ctypes.data, m.shape[1], m.shape[0], C.byref(uvm),
                                                    None if tf is None else tf.ctypes.data), "dmap_scene_set_opacity")

    def tessellate_uniform(self, n: int) -> dict:
        """dmap_tessellate_uniform_host (append_displaced_triangle over the
        scene's triangles at subdivision n): positions (V, 3), texcoords
        (V, 2), normals (V, 3) float32, indices (F, 3) uint32 (global)."""
        nt = self.n_tri
        V, F = (n + 1) * (n + 2) // 2 * nt, n * n * nt
        out = {"positions": np.empty((V, 3), np.float32), "texcoords": np.empty((V, 2), np.float32),
               "normals": np.empty((V, 3), np.float32), "indices": np.empty((F, 3), np.uint32)}
        self.ctx.check(lib().dmap_tessellate_uniform_host(self.h, n, out["positions"].ctypes.data,
                                                          out["texcoords"].ctypes.data, out["normals"].ctypes.data,
                                                          out["indices"].ctypes.data), "dmap_tessellate_uniform_host")
        return out

    def tessellate_texel(self, m: int = 1) -> dict:
        """dmap_tessellate_texel_host (append_texel_tessellation over the
        scene's triangles, m x m sub-cells per leaf cell): per face positions
        (F, 3, 3), texcoords (F, 3, 2), normals (F, 3, 3) float32 and the
        TexelFace records (F,) of TEXEL_FACE."""
        n = C.c_int64()
        self.ctx.check(lib().dmap_tessellate_texel_host(self.h, m, 0, None, None, None, None, C.byref(n)),
                       "dmap_tessellate_texel_host")
        F = n.value
        out = {"positions": np.empty((F, 3, 3), np.float32), "texcoords": np.empty((F, 3, 2), np.float32),
               "normals": np.empty((F, 3, 3), np.float32), "faces": np.empty(F, TEXEL_FACE)}
        if F:
            self.ctx.check(lib().dmap_tessellate_texel_host(self.h, m, F, out["positions"].ctypes.data,
                                                            out["texcoords"].ctypes.data,
                                                            out["normals"].ctypes.data, out["faces"].ctypes.data,
                                                            C.byref(n)), "dmap_tessellate_texel_host")
        return out

    def autotune(self, rays_ptr: int, ray_dtype: int, n: int, base: Optional[TraversalOptions] = None,
                 cache_path: Optional[str] = None):
        """dmap_autotune on device rays: (TraversalOptions with the fastest
        rounds / blocks_per_sm, its time in ms on the sample)."""
        b = base or TraversalOptions()
        out = _Options()
        ms = C.c_double()
        self.ctx.check(lib().dmap_autotune(self.h, rays_ptr, ray_dtype, n, C.byref(b.c()),
                                           cache_path.encode() if cache_path else None, C.byref(out), C.byref(ms)),
                       "dmap_autotune")
        t = TraversalOptions(**{**b.__dict__, "schedule": "wavefront", "rounds": out.rounds,
                                "blocks_per_sm": out.blocks_per_sm})
        return t, ms.value

    def render(self, view: dict, emitter: np.ndarray, spp: int = 1, max_depth: int = 5, rr_depth: int = 3,
               radiance=(10.0, 10.0, 10.0), albedo=(0.7, 0.7, 0.7), seed: int = 2027, paths_per_batch: int = 0,
               use_graph: bool = True, options: Optional[TraversalOptions] = None, record: int = 0):
        """The batched path tracer (dmap_render): view as scenes.path_tracer_view,
        emitter as the (4, 3) corners p00, p10, p01, p11 of the light rectangle.
        Returns (image (h, w, 3) float32, stats dict, record dict or None)."""
        d = render_desc(view, emitter, spp, max_depth, rr_depth, radiance, albedo, seed, paths_per_batch, use_graph)
        img = np.empty((view["height"], view["width"], 3), np.float32)
        st = _RenderStats()
        rec = None
        rp = None
        if record > 0:
            rec = {"rays": np.zeros((record, 8), np.float32), "kind": np.zeros(record, np.int32),
                   "tri": np.zeros(record, np.int32), "t": np.zeros(record, np.float32)}
            rp = _RayRecord(record, rec["rays"].ctypes.data, rec["kind"].ctypes.data, rec["tri"].ctypes.data,
                            rec["t"].ctypes.data, 0)
        opt = (options or TraversalOptions()).c()
        self.ctx.check(lib().dmap_render(self.h, C.byref(d), C.byref(opt), img.ctypes.data, C.byref(st),
                                         C.byref(rp) if rp is not None else None), "dmap_render")
        if rec is not None:
            m = min(rp.count, record)
            rec = {k: v[:m] for k, v in rec.items()}
            rec["count"] = rp.count
        stats = {k: getattr(st, k) for k, _ in _RenderStats._fields_}
        return img, stats, rec

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib().dmap_scene_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_desc(view: dict, emitter: np.ndarray, spp: int = 1, max_depth: int = 5, rr_depth: int = 3,
                radiance=(10.0, 10.0, 10.0), albedo=(0.7, 0.7, 0.7), seed: int = 2027, paths_per_batch: int = 0,
                use_graph: bool = True) -> _RenderDesc:
    """dmap_render_desc of a view (scenes.path_tracer_view) and the (4, 3)
    corners p00, p10, p01, p11 of the emitter rectangle."""
    cam = _Camera((C.c_double * 3)(*view["eye"]), (C.c_double * 3)(*view["target"]),
                  (C.c_double * 3)(*view["up"]), view["fov_deg"], view["width"], view["height"])
    e = np.asarray(emitter, np.float64)
    return _RenderDesc(cam, (C.c_double * 3)(*e[0]), (C.c_double * 3)(*(e[1] - e[0])),
                       (C.c_double * 3)(*(e[2] - e[0])), (C.c_double * 3)(*radiance), (C.c_double * 3)(*albedo),
                       spp, max_depth, rr_depth, seed, paths_per_batch, int(use_graph))


class Server:
    """Continuous-batching server over resident scenes (dmap_server_*).
    Submitted buffers are kept alive here until their request completes."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int = 0, max_batch_rays: int = 0, max_inflight: int = 0,
                 slots: int = 0, options: Optional[TraversalOptions] = None, policy: str = "oldest"):
        """policy: "oldest" (arrival order) or "shortest" (fewest queries left first)."""
        self.ctx = ctx
        cfg = _ServerConfig(hbm_budget_bytes, max_batch_rays, max_inflight, slots, (options or TraversalOptions()).c(),
                            {"oldest": 0, "shortest": 1}[policy])
        h = C.c_void_p()
        ctx.check(lib().dmap_server_create(ctx.h, C.byref(cfg), C.byref(h)), "dmap_server_create")
        self.h = h
        self._bufs = {}

    def submit_rays(self, scene: Scene, rays: np.ndarray, mode: str = "closest", hits: Optional[np.ndarray] = None):
        """rays (n, 8) float32 (pinned or not) -> (request id, HIT32 array filled on completion)."""
        r = np.ascontiguousarray(rays, np.float32)
        out = np.empty(len(r), HIT32) if hits is None else hits
        rid = C.c_uint64()
        s = lib().dmap_server_submit_rays(self.h, scene.h, r.ctypes.data, len(r), MODE[mode], out.ctypes.data,
                                          C.byref(rid))
        if s:
            raise DmapError(s, f"dmap_server_submit_rays: {lib().dmap_status_string(s).decode()}")
        self._bufs[rid.value] = (r, out)
        return rid.value, out

    def submit_render(self, scene: Scene, view: dict, emitter: np.ndarray, **kw):
        """A render request (render_desc's keywords) -> (request id, image filled on completion)."""
        d = render_desc(view, emitter, **kw)
        img = np.empty((view["height"], view["width"], 3), np.float32)
        rid = C.c_uint64()
        s = lib().dmap_server_submit_render(self.h, scene.h, C.byref(d), img.ctypes.data, C.byref(rid))
        if s:
            raise DmapError(s, f"dmap_server_submit_render: {lib().dmap_status_string(s).decode()}")
        self._bufs[rid.value] = (img,)
        if len(self._bufs) % 256 == 0:
            self.reap()
        return rid.value, img

    def poll(self, rid: int) -> int:
        return lib().dmap_server_poll(self.h, rid)

    def wait(self, rid: int, timeout_s: float = -1.0) -> int:
        return lib().dmap_server_wait(self.h, rid, timeout_s)

    def cancel(self, rid: int) -> int:
        return lib().dmap_server_cancel(self.h, rid)

    def pause(self, paused: bool = True):
        """Holds (or resumes) admission: submitted requests stay queued."""
        self.ctx.check(lib().dmap_server_pause(self.h, int(paused)), "dmap_server_pause")

    def latency_ms(self, rid: int) -> float:
        ms = C.c_double()
        s = lib().dmap_server_latency(self.h, rid, C.byref(ms))
        if s:
            raise DmapError(s, f"dmap_server_latency: {lib().dmap_status_string(s).decode()}")
        return ms.value

    def drain(self, timeout_s: float = -1.0) -> int:
        s = lib().dmap_server_drain(self.h, timeout_s)
        if s == 0:
            self._bufs.clear()   # every request is done with its buffers
        return s

    def reap(self):
        """Drops the references to the buffers of finished requests."""
        for rid in [r for r in self._bufs if lib().dmap_server_poll(self.h, r) != 7]:
            del self._bufs[rid]

    def stats(self) -> dict:
        st = _ServerStats()
        lib().dmap_server_get_stats(self.h, C.byref(st))
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib().dmap_server_destroy(self.h)
        self.h = None
        self._bufs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Emitter:
    """DescentSampler for every triangle of a scene (dmap_emitter_*):
    texels is one n_leaf x n_leaf emission grid per scene asset (None: a
    uniform emission of 1 everywhere, or None entries per asset)."""

    def __init__(self, scene: Scene, texels=None, variant: str = "product", beta: float = 0.05,
                 emitter_cosine: bool = True):
        self.scene = scene
        self.ctx = scene.ctx
        keep = []
        arr = None
        if texels is not None:
            if len(texels) != len(scene.assets):
                raise ValueError(f"one emission grid per scene asset: {len(texels)} for {len(scene.assets)}")
            ptrs = []
            for a_, t in zip(scene.assets, texels):
                if t is not None and np.shape(t) != (a_.n_leaf, a_.n_leaf):
                    raise ValueError(f"emission grid {np.shape(t)} does not match {a_.n_leaf}^2 leaf cells")
                if t is None:
                    ptrs.append(None)
                else:
                    a = np.ascontiguousarray(t, np.float64)
                    keep.append(a)
                    ptrs.append(a.ctypes.data)
            arr = (C.c_void_p * len(ptrs))(*ptrs)
        h = C.c_void_p()
        self.ctx.check(lib().dmap_emitter_create(scene.h, arr, DESCENT[variant], beta, int(emitter_cosine),
                                                 C.byref(h)), "dmap_emitter_create")
        self.h = h

    def triangle_info(self, tri: int) -> np.ndarray:
        out = np.empty(6)
        self.ctx.check(lib().dmap_emitter_triangle_info(self.h, tri, out.ctypes.data), "dmap_emitter_triangle_info")
        return out

    def sample(self, tri, uniforms, receivers=None) -> np.ndarray:
        """Samples on triangles tri (n,) from float32 uniforms (n, K):
        EMITTER_POINT records."""
        t = np.ascontiguousarray(tri, np.int32)
        u = np.ascontiguousarray(uniforms, np.float32).reshape(len(t), -1)
        r = None if receivers is None else np.ascontiguousarray(receivers, np.float64).reshape(len(t), 6)
        out = np.empty(len(t), EMITTER_POINT)
        self.ctx.check(lib().dmap_emitter_sample_host(self.h, t.ctypes.data, u.ctypes.data, u.shape[1],
                                                      None if r is None else r.ctypes.data, len(t),
                                                      out.ctypes.data), "dmap_emitter_sample_host")
        return out

    def pdf(self, tri, uv, receivers=None):
        """(pdf_uv, pdf_area) at points uv (n, 2) of triangles tri (n,)."""
        t = np.ascontiguousarray(tri, np.int32)
        q = np.ascontiguousarray(uv, np.float64).reshape(len(t), 2)
        r = None if receivers is None else np.ascontiguousarray(receivers, np.float64).reshape(len(t), 6)
        pu, pa = np.empty(len(t)), np.empty(len(t))
        self.ctx.check(lib().dmap_emitter_pdf_host(self.h, t.ctypes.data, q.ctypes.data,
                                                   None if r is None else r.ctypes.data, len(t), pu.ctypes.data,
                                                   pa.ctypes.data), "dmap_emitter_pdf_host")
        return pu, pa

    def light(self, points, shade) -> np.ndarray:
        """DisplacedEmitterLight::sample's conversion of sampled points
        (EMITTER_POINT records, drawn with receivers = shade) seen from
        shade (n, 6): EMITTER_LIGHT records."""
        pts = np.ascontiguousarray(points, EMITTER_POINT)
        sh = np.ascontiguousarray(shade, np.float64).reshape(len(pts), 6)
        out = np.empty(len(pts), EMITTER_LIGHT)
        self.ctx.check(lib().dmap_emitter_light_host(self.h, pts.ctypes.data, sh.ctypes.data, len(pts),
                                                     out.ctypes.data), "dmap_emitter_light_host")
        return out

    def light_pdf(self, tri, shade, uv=None, wi=None):
        """Solid-angle pdfs seen from shade (n, 6): at uv (n, 2), or with uv
        None by the walk of triangle tri along wi (n, 3). Returns (pdf_omega
        (n,), the (u, v) used (n, 2), NaN on a miss)."""
        t = np.ascontiguousarray(tri, np.int32)
        sh = np.ascontiguousarray(shade, np.float64).reshape(len(t), 6)
        q = None if uv is None else np.ascontiguousarray(uv, np.float64).reshape(len(t), 2)
        w = None if wi is None else np.ascontiguousarray(wi, np.float64).reshape(len(t), 3)
        pw, hit = np.empty(len(t)), np.empty((len(t), 2))
        self.ctx.check(lib().dmap_emitter_light_pdf_host(self.h, t.ctypes.data, sh.ctypes.data,
                                                         None if q is None else q.ctypes.data,
                                                         None if w is None else w.ctypes.data, len(t),
                                                         pw.ctypes.data, hit.ctypes.data),
                       "dmap_emitter_light_pdf_host")
        return pw, hit

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib().dmap_emitter_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
