"""Synthetic displaced scenes and ray sets for the benchmark workloads.

The reference's scene files and height textures are not available, so seeded
synthetic inputs with the benchmark shapes stand in for them:

- ``quad_scene``: one unit quad at z = 0, normal +z, split into two base
  triangles on the (1,0)-(0,1) diagonal (the texel split of
  displaced_intersector.h:29-31), displaced by an N x N height map of 8
  seeded sines plus value noise scaled to max |h| = amplitude.
- ``cube_sphere_scene``: a radius-1 cube sphere of 6 x k x k patches, each a
  quad split the same way with radial vertex normals and its own map.
- ``ground_plane``: a displaced ridged-multifractal plane (path-tracer scene).

Heights are texel maps (N x N); ``close_tile`` adds the closing row and
column the way texture_grid.cpp:118-132 does, giving the (N+1)^2 node grid.
All arrays are numpy; nothing here touches the GPU.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

SEED = 2027


# --------------------------------------------------------------------------
# Height maps
# --------------------------------------------------------------------------

def _interp_weights(n_samples: int, n_lattice: int, period: bool) -> np.ndarray:
    """(n_samples x n_lattice) weights of smoothstep interpolation between
    lattice values at sample positions x = s / (n_samples - 1) in [0, 1]."""
    x = np.linspace(0.0, 1.0, n_samples) * (n_lattice - 1)
    i0 = np.minimum(np.floor(x).astype(np.int64), n_lattice - 2)
    f = x - i0
    f = f * f * (3.0 - 2.0 * f)
    W = np.zeros((n_samples, n_lattice))
    rows = np.arange(n_samples)
    W[rows, i0] += 1.0 - f
    W[rows, i0 + 1] += f
    return W


def value_noise(n: int, cells: int, rng: np.random.Generator) -> np.ndarray:
    """n x n samples of smoothstep-interpolated random lattice values on a
    (cells+1)^2 lattice, values uniform in [-1, 1]."""
    L = rng.uniform(-1.0, 1.0, size=(cells + 1, cells + 1))
    W = _interp_weights(n, cells + 1, False)
    return W @ L @ W.T


def sine_noise_heights(n: int, seed: int, amplitude: float, n_sines: int = 8, octaves: int = 2,
                       noise_weight: float = 0.35) -> np.ndarray:
    """The benchmark height generator: sum of n_sines seeded plane waves
    (frequencies log-uniform in [1, 32] cycles per tile, amplitude 1/f,
    random direction and phase) plus octaves of value noise, normalized to
    max |h| = amplitude. Returns an n x n float64 texel map, [j, i] with the
    i axis along u. Each wave is separable: sin(a + b) = sin a cos b + cos a sin b."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = (np.arange(n) + 0.5) / n
    h = np.zeros((n, n))
    freqs = np.exp(rng.uniform(math.log(1.0), math.log(32.0), size=n_sines))
    thetas = rng.uniform(0.0, 2.0 * math.pi, size=n_sines)
    phis = rng.uniform(0.0, 2.0 * math.pi, size=n_sines)
    for f, th, ph in zip(freqs, thetas, phis):
        a = 2.0 * math.pi * f * math.cos(th) * u           # along i (u)
        b = 2.0 * math.pi * f * math.sin(th) * u + ph      # along j (v)
        h += (np.outer(np.cos(b), np.sin(a)) + np.outer(np.sin(b), np.cos(a))) / f
    h /= np.abs(h).max()
    noise = np.zeros((n, n))
    cells = 8
    for o in range(octaves):
        noise += value_noise(n, min(cells, max(n - 1, 1)), rng) * 0.5 ** o
        cells *= 2
    noise /= max(np.abs(noise).max(), 1e-30)
    h = h + noise_weight * noise
    return h * (amplitude / np.abs(h).max())


def ridged_heights(n: int, seed: int, amplitude: float, octaves: int = 6) -> np.ndarray:
    """Ridged multifractal of value noise: sum over octaves of
    (1 - |noise|)^2 * gain^o, normalized to [0, amplitude]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h = np.zeros((n, n))
    cells = 4
    for o in range(octaves):
        r = 1.0 - np.abs(value_noise(n, min(cells, max(n - 1, 1)), rng))
        h += (r * r) * 0.5 ** o
        cells *= 2
    h -= h.min()
    return h * (amplitude / max(h.max(), 1e-30))


def close_tile(texels: np.ndarray, repeat: bool) -> np.ndarray:
    """N x N texels -> (N+1) x (N+1) node grid; the closing row and column
    wrap (repeat) or duplicate the last (clamp), texture_grid.cpp:118-132."""
    n = texels.shape[0]
    idx = np.arange(n + 1)
    idx = idx % n if repeat else np.minimum(idx, n - 1)
    return texels[np.ix_(idx, idx)]


# --------------------------------------------------------------------------
# Scenes
# --------------------------------------------------------------------------

@dataclass
class Asset:
    """One displacement map: the node grid (values), h = scale * v + offset."""
    nodes: np.ndarray            # (N+1, N+1), float32 or float16
    scale: float = 1.0
    offset: float = 0.0
    repeat: bool = False

    @property
    def n_leaf(self) -> int:
        return self.nodes.shape[0] - 1


@dataclass
class Scene:
    assets: List[Asset]
    tris: np.ndarray             # (T, 24) float64: p0,p1,p2,m0,m1,m2,t0,t1,t2
    tri_asset: np.ndarray        # (T,) int32
    name: str = ""
    emitter: Optional[np.ndarray] = None   # (4, 3) corners of a flat rectangle light
    extent: float = 1.0          # length of the scene's bounding-box diagonal

    def objects(self):
        """Triangles grouped by asset, in asset order: [(asset, tris)]."""
        out = []
        for a, asset in enumerate(self.assets):
            out.append((asset, self.tris[self.tri_asset == a]))
        return out


def quad_triangles(P00, P10, P01, P11, N00, N10, N01, N11) -> np.ndarray:
    """Two base triangles of a quad sharing the (1,0)-(0,1) diagonal, the
    chart putting the quad's (u, v) at its corners."""
    a = np.concatenate([P00, P10, P01, N00, N10, N01, [0.0, 0.0, 1.0, 0.0, 0.0, 1.0]])
    b = np.concatenate([P11, P01, P10, N11, N01, N10, [1.0, 1.0, 0.0, 1.0, 1.0, 0.0]])
    return np.stack([a, b])


def quad_scene(n: int = 512, seed: int = SEED, amplitude: float = 0.05, dtype=np.float32) -> Scene:
    """One unit quad [0,1]^2 at z = 0 with normal +z, clamp wrap."""
    h = sine_noise_heights(n, seed, amplitude)
    nodes = close_tile(h, repeat=False).astype(dtype)
    z = np.array([0.0, 0.0, 1.0])
    tris = quad_triangles(np.array([0.0, 0, 0]), np.array([1.0, 0, 0]), np.array([0.0, 1, 0]),
                          np.array([1.0, 1, 0]), z, z, z, z)
    return Scene([Asset(nodes)], tris, np.zeros(2, np.int32), name=f"quad{n}",
                 extent=math.sqrt(2.0 + (2 * amplitude) ** 2))


_FACES = [  # (normal axis, sign): the face's (u, v) axes chosen right-handed around the outward normal
    (np.array([1.0, 0, 0]), np.array([0.0, 1, 0]), np.array([0.0, 0, 1])),
    (np.array([-1.0, 0, 0]), np.array([0.0, 0, 1]), np.array([0.0, 1, 0])),
    (np.array([0.0, 1, 0]), np.array([0.0, 0, 1]), np.array([1.0, 0, 0])),
    (np.array([0.0, -1, 0]), np.array([1.0, 0, 0]), np.array([0.0, 0, 1])),
    (np.array([0.0, 0, 1]), np.array([1.0, 0, 0]), np.array([0.0, 1, 0])),
    (np.array([0.0, 0, -1]), np.array([0.0, 1, 0]), np.array([1.0, 0, 0])),
]


def cube_sphere_scene(n: int = 2048, k: int = 4, seed: int = SEED, amplitude: float = 0.08,
                      dtype=np.float32, faces: Optional[List[int]] = None,
                      patches: Optional[List[int]] = None) -> Scene:
    """Radius-1 cube sphere: 6 faces x k x k patches, each two base triangles
    with radial vertex normals and its own n x n map (seed + patch id,
    clamp wrap). `patches` selects a subset of patch ids (tests)."""
    assets, tris, tri_asset = [], [], []
    pid = 0
    for f, (nrm, ax_u, ax_v) in enumerate(_FACES):
        for b in range(k):
            for a in range(k):
                this = pid
                pid += 1
                if faces is not None and f not in faces:
                    continue
                if patches is not None and this not in patches:
                    continue

                def corner(ia, ib):
                    c = nrm + ax_u * (2.0 * ia / k - 1.0) + ax_v * (2.0 * ib / k - 1.0)
                    return c / np.linalg.norm(c)

                P00, P10, P01, P11 = corner(a, b), corner(a + 1, b), corner(a, b + 1), corner(a + 1, b + 1)
                h = sine_noise_heights(n, seed + this, amplitude, octaves=4)
                assets.append(Asset(close_tile(h, repeat=False).astype(dtype)))
                tris.append(quad_triangles(P00, P10, P01, P11, P00, P10, P01, P11))
                tri_asset += [len(assets) - 1] * 2
    return Scene(assets, np.concatenate(tris), np.array(tri_asset, np.int32),
                 name=f"cube_sphere{k}x{k}x6_{n}", extent=2.0 * math.sqrt(3.0) * (1.0 + amplitude))


def sphere_benchmark_scene(n: int = 2048, texel=np.float32, threads: int = 16) -> Scene:
    """The GPU-scale plain-method scene: the radius-1 cube sphere of 96
    patches, each its own n x n map of seeded sines + 4 octaves of value
    noise (amplitude 0.08, seed + patch id), stored as `texel` (float32, or
    float16 for the precision variant). The 96 maps are generated on
    `threads` threads."""
    import concurrent.futures as cf
    k = 4

    def one(pid):
        return close_tile(sine_noise_heights(n, SEED + pid, 0.08, octaves=4), repeat=False).astype(texel)

    with cf.ThreadPoolExecutor(max(1, threads)) as ex:
        maps = list(ex.map(one, range(6 * k * k)))
    sc = cube_sphere_scene(1, k)  # the geometry; its 1 x 1 maps are replaced
    for pid, a in enumerate(sc.assets):
        a.nodes = maps[pid]
    sc.name = f"cube_sphere{k}x{k}x6_{n}"
    return sc


def ground_plane_asset(n: int = 4096, seed: int = SEED + 1000, amplitude: float = 0.2,
                       dtype=np.float32) -> Asset:
    return Asset(close_tile(ridged_heights(n, seed, amplitude), repeat=False).astype(dtype))


def path_tracer_scene(n_sphere: int = 2048, n_ground: int = 4096, k: int = 4, seed: int = SEED,
                      dtype=np.float32) -> Scene:
    """The cube sphere plus a displaced ground plane (4 x 4 units at
    y = -1.3, normal +y, 2 triangles) and a 0.5 x 0.5 emitter rectangle
    above the sphere."""
    return with_ground_and_emitter(cube_sphere_scene(n_sphere, k, seed, dtype=dtype), n_ground, seed, dtype)


def with_ground_and_emitter(sc: Scene, n_ground: int = 4096, seed: int = SEED, dtype=np.float32) -> Scene:
    """A scene plus the path tracer's ground plane and emitter."""
    g = ground_plane_asset(n_ground, seed + 1000, dtype=dtype)
    y = -1.3
    up = np.array([0.0, 1.0, 0.0])
    P00, P10 = np.array([-2.0, y, 2.0]), np.array([2.0, y, 2.0])
    P01, P11 = np.array([-2.0, y, -2.0]), np.array([2.0, y, -2.0])
    gt = quad_triangles(P00, P10, P01, P11, up, up, up, up)
    assets = sc.assets + [g]
    tris = np.concatenate([sc.tris, gt])
    tri_asset = np.concatenate([sc.tri_asset, np.full(2, len(assets) - 1, np.int32)])
    emitter = np.array([[-0.25, 2.0, -0.25], [0.25, 2.0, -0.25], [-0.25, 2.0, 0.25], [0.25, 2.0, 0.25]])
    return Scene(assets, tris, tri_asset, name="path_tracer", emitter=emitter, extent=float(np.linalg.norm([4, 3.5, 4])))


def path_tracer_view(width: int = 1280, height: int = 720) -> dict:
    """The path tracer's camera: in front of the sphere, slightly above it,
    the ground plane and the emitter's light pool in view."""
    return dict(eye=(0.0, 1.0, 4.6), target=(0.0, -0.3, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0,
                width=width, height=height)


# --------------------------------------------------------------------------
# Rays. Every ray set is (n, 8) float32: o(3), d(3), t_min, t_max.
# --------------------------------------------------------------------------

def pinhole_rays(eye, target, up, fov_deg: float, width: int, height: int, jitter_seed: Optional[int] = None
                 ) -> np.ndarray:
    """One ray per pixel (pixel centre, or jittered within the pixel with a
    seeded generator), row-major from the top-left pixel."""
    eye, target, up = (np.asarray(x, np.float64) for x in (eye, target, up))
    w = target - eye
    w /= np.linalg.norm(w)
    u = np.cross(w, up)
    u /= np.linalg.norm(u)
    v = np.cross(u, w)
    th = math.tan(math.radians(fov_deg) * 0.5)
    aspect = width / height
    jj, ii = np.mgrid[0:height, 0:width]
    if jitter_seed is None:
        ox = oy = 0.5
    else:
        rng = np.random.Generator(np.random.PCG64(jitter_seed))
        ox = rng.random((height, width))
        oy = rng.random((height, width))
    px = ((ii + ox) / width * 2.0 - 1.0) * th * aspect
    py = (1.0 - (jj + oy) / height * 2.0) * th
    d = w[None, None, :] + px[..., None] * u[None, None, :] + py[..., None] * v[None, None, :]
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    rays = np.zeros((height * width, 8), np.float32)
    rays[:, 0:3] = eye.astype(np.float32)
    rays[:, 3:6] = d.reshape(-1, 3).astype(np.float32)
    rays[:, 6] = 0.0
    rays[:, 7] = np.inf
    return rays


def quad_camera_rays(width: int = 256, height: int = 256) -> np.ndarray:
    """Pinhole at distance 2 along +z over the quad's centre, 45 deg FOV."""
    return pinhole_rays([0.5, 0.5, 2.0], [0.5, 0.5, 0.0], [0.0, 1.0, 0.0], 45.0, width, height)


def sphere_camera_rays(width: int = 1920, height: int = 1080, seed: int = SEED) -> np.ndarray:
    """Pinhole at distance 3 from the sphere's centre, 45 deg FOV, jittered."""
    return pinhole_rays([0.9, 1.1, 2.6], [0.0, 0.0, 0.0], [0.0, 1.0, 0.0], 45.0, width, height,
                        jitter_seed=seed)


def bounce_rays(rays: np.ndarray, t: np.ndarray, ng: np.ndarray, seed: int = SEED, eps: float = 1e-4
                ) -> np.ndarray:
    """One cosine-weighted diffuse bounce per hit (finite t): origin at the
    hit point offset by eps along the normal facing the incoming ray."""
    hit = np.isfinite(t)
    o = rays[hit, 0:3].astype(np.float64) + t[hit, None] * rays[hit, 3:6].astype(np.float64)
    n = ng[hit].astype(np.float64)
    flip = np.sum(n * rays[hit, 3:6], axis=1) > 0.0
    n[flip] = -n[flip]
    rng = np.random.Generator(np.random.PCG64(seed))
    u1, u2 = rng.random(len(n)), rng.random(len(n))
    r, phi = np.sqrt(u1), 2.0 * math.pi * u2
    a = np.where(np.abs(n[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0.0, 1, 0]]))
    t1 = np.cross(a, n)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(n, t1)
    d = (r * np.cos(phi))[:, None] * t1 + (r * np.sin(phi))[:, None] * t2 + np.sqrt(1.0 - u1)[:, None] * n
    out = np.zeros((len(n), 8), np.float32)
    out[:, 0:3] = o + eps * n
    out[:, 3:6] = d
    out[:, 6] = 0.0
    out[:, 7] = np.inf
    return out


def uniform_direction(rng, n):
    z = 1.0 - 2.0 * rng.random(n)
    phi = 2.0 * math.pi * rng.random(n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def base_points(scene: Scene, n: int, seed: int = SEED):
    """n random points on the scene's base triangles (uniform triangle,
    uniform barycentrics) and their interpolated vertex normals."""
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.integers(0, len(scene.tris), n)
    a, b = rng.random(n), rng.random(n)
    flip = a + b > 1.0
    a, b = np.where(flip, 1.0 - a, a), np.where(flip, 1.0 - b, b)
    t = scene.tris[k]
    w = np.stack([1.0 - a - b, a, b], 1)
    p = w[:, 0:1] * t[:, 0:3] + w[:, 1:2] * t[:, 3:6] + w[:, 2:3] * t[:, 6:9]
    m = w[:, 0:1] * t[:, 9:12] + w[:, 1:2] * t[:, 12:15] + w[:, 2:3] * t[:, 15:18]
    return p, m / np.linalg.norm(m, axis=1, keepdims=True)


def grazing_rays(points: np.ndarray, normals: np.ndarray, seed: int = SEED) -> np.ndarray:
    """Rays aimed at surface points from a tangent direction tilted
    0.1-5 deg (log-uniform) toward the surface, origin backed off 0.05-1."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = normals / np.linalg.norm(normals, axis=1, keepdims=True)
    a = np.where(np.abs(n[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0.0, 1, 0]]))
    t1 = np.cross(a, n)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(n, t1)
    phi = 2.0 * math.pi * rng.random(len(n))
    tang = np.cos(phi)[:, None] * t1 + np.sin(phi)[:, None] * t2
    ang = np.radians(np.exp(rng.uniform(math.log(0.1), math.log(5.0), len(n))))
    d = np.cos(ang)[:, None] * tang - np.sin(ang)[:, None] * n
    back = rng.uniform(0.05, 1.0, len(n))
    out = np.zeros((len(n), 8), np.float32)
    out[:, 0:3] = points - back[:, None] * d
    out[:, 3:6] = d
    out[:, 7] = np.inf
    return out
