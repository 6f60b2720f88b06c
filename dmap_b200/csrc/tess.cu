// Oracle meshes on the device (include/dmap_b200.h, dmap_tessellate_*):
// the uniform barycentric tessellation and the texel-aligned tessellation of
// displaced_tessellation.cpp, every vertex evaluated in double with the
// reference's operation order (compiled with -fmad=false) and rounded to
// float, so that both meshes match the reference's MeshData bit for bit.
//
// Uniform grid: one thread per vertex and one per face over the whole scene
// (the grid's row of a node or face is found from its index in closed form
// and corrected exactly in integers). Texel grid: one thread per leaf cell
// of each triangle's uv bounding box, in two passes over the same cells —
// a count of the cell's faces, an exclusive scan of the counts (CUB), and an
// emit pass that writes each cell's faces at its scanned offset — so the
// faces come out in the reference's loop order (triangle, j, i, sub-cell
// row b, column a, fan index).
#include "api_internal.h"
#include "f64_math.cuh"

#include <cub/device/device_scan.cuh>

#include <algorithm>

using namespace dmapi;

namespace
{
using namespace d64;

// Eigen's normalized(): a zero vector stays as it is.
__device__ __forceinline__ v3 eigen_normalized(v3 a)
{
    double z = dot3(a, a);
    return z > 0.0 ? div3(a, sqrt(z)) : a;
}

// displaced_position (displaced_surface.cpp:162-166) and the unit normal of
// pointwise_fields(...).n (:110-158), both from one frame and one grid
// lookup; the values equal those of the reference's separate calls.
__device__ __forceinline__ void surface_vertex(const TriDev &T, const AssetDev &g, double s, double t, v3 &S, v3 &n)
{
    nframe f = normal_frame_at(T, s, t);
    double h;
    v2 gh;
    grid_h_grad(g, s, t, h, gh);
    S = add3(tri_P(T, s, t), mul3(h, f.N));
    v3 Su = add3(add3(L3(T.e1), mul3(gh.x, f.N)), mul3(h, f.Nu));
    v3 Sv = add3(add3(L3(T.e2), mul3(gh.y, f.N)), mul3(h, f.Nv));
    n = eigen_normalized(cross3(Su, Sv));
}

__device__ __forceinline__ void put3(float *p, v3 a)
{
    p[0] = (float)a.x;
    p[1] = (float)a.y;
    p[2] = (float)a.z;
}

// ---- uniform barycentric grid (displaced_tessellation.cpp:11-56) --------

// First node of row j: index(0, j) = j (n + 1) - j (j - 1) / 2.
__device__ __forceinline__ int64_t row_node(int64_t n, int64_t j) { return j * (n + 1) - j * (j - 1) / 2; }
// First face of row j: rows j' < j hold 2 (n - j') - 1 faces each.
__device__ __forceinline__ int64_t row_face(int64_t n, int64_t j) { return j * (2 * n - j); }

__global__ void uniform_vertices_kernel(const TriDev *__restrict__ tris, const AssetDev *__restrict__ assets, int n,
                                        int64_t total, float *pos, float *uv, float *nrm)
{
    const int64_t V = (int64_t)(n + 1) * (n + 2) / 2;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t tri = k / V, r = k - tri * V;
        // row_node(n, j) <= r: j ~ ((2n + 3) - sqrt((2n + 3)^2 - 8 r)) / 2, then exact correction
        double b = 2.0 * n + 3.0;
        int64_t j = (int64_t)floor(0.5 * (b - sqrt(fmax(b * b - 8.0 * (double)r, 0.0))));
        j = j < 0 ? 0 : (j > n ? n : j);
        while (j > 0 && row_node(n, j) > r)
            --j;
        while (j < n && row_node(n, j + 1) <= r)
            ++j;
        int64_t i = r - row_node(n, j);
        const TriDev &T = tris[tri];
        const AssetDev &g = assets[T.asset];
        // BaseTriangle::param (displaced_surface.h:87) at the barycentric node (i/n, j/n)
        double u = (double)i / n, v = (double)j / n;
        v2 t0 = L2(T.t0), t1 = L2(T.t1), t2 = L2(T.t2);
        v2 st = add2(add2(t0, mul2(u, sub2(t1, t0))), mul2(v, sub2(t2, t0)));
        v3 S, nn;
        surface_vertex(T, g, st.x, st.y, S, nn);
        put3(pos + 3 * k, S);
        uv[2 * k] = (float)st.x;
        uv[2 * k + 1] = (float)st.y;
        put3(nrm + 3 * k, nn);
    }
}

__global__ void uniform_faces_kernel(int n, int64_t total, uint32_t *idx)
{
    const int64_t V = (int64_t)(n + 1) * (n + 2) / 2, F = (int64_t)n * n;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t tri = k / F, r = k - tri * F;
        // row_face(n, j) <= r: j ~ n - sqrt(n^2 - r), then exact correction
        int64_t j = (int64_t)floor((double)n - sqrt(fmax((double)n * n - (double)r, 0.0)));
        j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
        while (j > 0 && row_face(n, j) > r)
            --j;
        while (j < n - 1 && row_face(n, j + 1) <= r)
            ++j;
        int64_t q = r - row_face(n, j), i = q >> 1;
        uint32_t base = (uint32_t)(tri * V);
        uint32_t *o = idx + 3 * k;
        if ((q & 1) == 0) { // (index(i, j), index(i + 1, j), index(i, j + 1))
            o[0] = base + (uint32_t)(row_node(n, j) + i);
            o[1] = base + (uint32_t)(row_node(n, j) + i + 1);
            o[2] = base + (uint32_t)(row_node(n, j + 1) + i);
        } else { // (index(i + 1, j), index(i + 1, j + 1), index(i, j + 1)), i + j < n - 1
            o[0] = base + (uint32_t)(row_node(n, j) + i + 1);
            o[1] = base + (uint32_t)(row_node(n, j + 1) + i + 1);
            o[2] = base + (uint32_t)(row_node(n, j + 1) + i);
        }
    }
}

// ---- texel-aligned tessellation (displaced_tessellation.cpp:58-137) -----

// The cell range of one triangle: cells (i, j) with i in [i_lo, i_lo + ni),
// j in [j_lo, ...), numbered from `first` in row-major (j, i) order.
struct TexelRange
{
    int64_t first, i_lo, j_lo, ni, nj;
    int64_t tile_first, tiles_x; // tiles of the m = 1 emit pass, row-major over the range
};

__device__ __forceinline__ int find_triangle(const TexelRange *__restrict__ ranges, int n_tri, int64_t cell)
{
    int lo = 0, hi = n_tri - 1; // last range with first <= cell
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ranges[mid].first <= cell)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

struct TexelSink
{
    float *pos, *uv, *nrm;
    dmap_texel_face *faces;
};

// One vertex of append_vertex (:62-76): its tile coordinates, position and
// unit normal, the normal flipped under a mirrored chart.
struct vtx
{
    v2 st;
    v3 S, N;
};

__device__ __forceinline__ vtx make_vtx(const TriDev &T, const AssetDev &g, v2 st, bool mirrored)
{
    vtx r;
    r.st = st;
    surface_vertex(T, g, st.x, st.y, r.S, r.N);
    if (mirrored)
        r.N = V3(-r.N.x, -r.N.y, -r.N.z);
    return r;
}

// append_face (:78-95): b and c swapped under a mirrored chart. Each
// vertex is a pure function of its tile coordinates, so a vertex shared by
// several faces is evaluated once.
__device__ __forceinline__ void put_vertex(const vtx &v, int64_t k, const TexelSink &o)
{
    put3(o.pos + 3 * k, v.S);
    o.uv[2 * k] = (float)v.st.x;
    o.uv[2 * k + 1] = (float)v.st.y;
    put3(o.nrm + 3 * k, v.N);
}

__device__ inline void emit_face(int tri, bool mirrored, const vtx &a, const vtx &b, const vtx &c, int interior,
                                 int64_t f, const TexelSink &o)
{
    // selects, not a pointer table: the vertices stay in registers
    const vtx b2 = mirrored ? c : b, c2 = mirrored ? b : c;
    put_vertex(a, 3 * f, o);
    put_vertex(b2, 3 * f + 1, o);
    put_vertex(c2, 3 * f + 2, o);
    dmap_texel_face rec;
    rec.triangle = tri;
    rec.interior = interior;
    rec.st[0][0] = a.st.x;
    rec.st[0][1] = a.st.y;
    rec.st[1][0] = b2.st.x;
    rec.st[1][1] = b2.st.y;
    rec.st[2][0] = c2.st.x;
    rec.st[2][1] = c2.st.y;
    o.faces[f] = rec;
}

// One leaf cell of append_texel_tessellation's loop: counts its faces
// (EMIT false) or writes them from face index `f` on (EMIT true).
template <bool EMIT>
__device__ inline int texel_cell(const TriDev &T, const AssetDev &g, int tri, bool mirrored, int64_t i, int64_t j,
                                 int m, int64_t f, const TexelSink &o, int &overlap)
{
    double w = 1.0 / g.n_leaf;
    v2 c = V2((i + 0.5) * w, (j + 0.5) * w);
    overlap = classify_square(T, c, 0.5 * w);
    if (overlap == OUTSIDE)
        return 0;
    double ws = w / m;
    int count = 0;
    for (int b = 0; b < m; ++b)
        for (int a = 0; a < m; ++a) {
            v2 p00 = V2(i * w + a * ws, j * w + b * ws);
            v2 p10 = add2(p00, V2(ws, 0.0)), p01 = add2(p00, V2(0.0, ws)), p11 = add2(p00, V2(ws, ws));
            v2 sc = add2(p00, V2(0.5 * ws, 0.5 * ws));
            int sub = overlap == INSIDE ? INSIDE : classify_square(T, sc, 0.5 * ws);
            if (sub == OUTSIDE)
                continue;
            if (sub == STRADDLE) {
                ClipPoly poly = clip_square(T, sc, 0.5 * ws);
                for (int k = 1; k + 1 < poly.n; ++k) {
                    if (EMIT)
                        emit_face(tri, mirrored, make_vtx(T, g, poly.p[0], mirrored),
                                  make_vtx(T, g, poly.p[k], mirrored), make_vtx(T, g, poly.p[k + 1], mirrored), 0,
                                  f + count, o);
                    ++count;
                }
                continue;
            }
            if (EMIT) {
                vtx v00 = make_vtx(T, g, p00, mirrored), v10 = make_vtx(T, g, p10, mirrored);
                vtx v01 = make_vtx(T, g, p01, mirrored), v11 = make_vtx(T, g, p11, mirrored);
                emit_face(tri, mirrored, v00, v10, v01, 1, f + count, o);
                emit_face(tri, mirrored, v10, v11, v01, 1, f + count + 1, o);
            }
            count += 2;
        }
    return count;
}

// chart_mirrored (displaced_surface.cpp:160)
__device__ __forceinline__ bool chart_mirrored(const TriDev &T)
{
    return dot3(cross3(L3(T.e1), L3(T.e2)), L3(T.wn)) < 0.0;
}

// The count pass (EMIT false) and the general emit pass (EMIT true), one
// thread per leaf cell. With a list, the count pass also records the cells
// that straddle the domain's boundary and have faces (for m = 1, whose
// inside cells the tiled pass writes).
template <bool EMIT>
__global__ void texel_kernel(const TriDev *__restrict__ tris, const AssetDev *__restrict__ assets,
                             const TexelRange *__restrict__ ranges, int n_tri, int64_t cells, int m,
                             int64_t *__restrict__ counts, const int64_t *__restrict__ offsets, TexelSink o,
                             int *__restrict__ straddle, unsigned long long *__restrict__ n_straddle)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cells; k += (int64_t)gridDim.x * blockDim.x) {
        if (EMIT && counts[k] == 0)
            continue;
        int tri = find_triangle(ranges, n_tri, k);
        TexelRange R = ranges[tri];
        int64_t r = k - R.first, jj = r / R.ni, ii = r - jj * R.ni;
        const TriDev &T = tris[tri];
        int overlap;
        int c = texel_cell<EMIT>(T, assets[T.asset], tri, chart_mirrored(T), R.i_lo + ii, R.j_lo + jj, m,
                                 EMIT ? offsets[k] : 0, o, overlap);
        if (!EMIT) {
            counts[k] = c;
            if (straddle && overlap == STRADDLE && c > 0)
                straddle[atomicAdd(n_straddle, 1ull)] = (int)k;
        }
    }
}

// The straddling cells of the m = 1 pass, from the count pass's list.
__global__ void texel_emit_list(const TriDev *__restrict__ tris, const AssetDev *__restrict__ assets,
                                const TexelRange *__restrict__ ranges, int n_tri, const int *__restrict__ straddle,
                                const unsigned long long *__restrict__ n_straddle,
                                const int64_t *__restrict__ offsets, TexelSink o)
{
    const int64_t n = (int64_t)*n_straddle;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = straddle[q];
        const int tri = find_triangle(ranges, n_tri, k);
        const TexelRange R = ranges[tri];
        const int64_t r = k - R.first, jj = r / R.ni, ii = r - jj * R.ni;
        const TriDev &T = tris[tri];
        int overlap;
        texel_cell<true>(T, assets[T.asset], tri, chart_mirrored(T), R.i_lo + ii, R.j_lo + jj, 1, offsets[k], o,
                         overlap);
    }
}

// The emit pass for m = 1 over the cells inside the domain (two faces each,
// over the cell's four corners), in tiles of 32 x 8 cells, one warp per
// tile row. With the power-of-two cell width w, corner (I, J) of every
// cell around it is the same point (I w, J w) bit for bit (the reference's
// i w + a ws and its sums with ws are exact), so the tile evaluates its
// 33 x 9 lattice nodes once into shared memory, about 1.2 evaluations per
// cell instead of 4. A tile row's inside cells are consecutive (the domain
// is convex) and so are their faces in the output, so the warp stages the
// row's faces in shared memory in output order, one output array at a
// time, and writes each out as whole lines. Straddling cells are left to
// texel_emit_list.
#ifndef DMAP_TESS_MIN_BLOCKS
#define DMAP_TESS_MIN_BLOCKS 2 // resident blocks per SM the tiled pass is compiled for
#endif
constexpr int kTileX = 32, kTileY = 8, kTileThreads = kTileX * kTileY;
constexpr int kNodesX = kTileX + 1, kNodes = kNodesX * (kTileY + 1);

__device__ __forceinline__ int find_tile_triangle(const TexelRange *__restrict__ ranges, int n_tri, int64_t tile)
{
    int lo = 0, hi = n_tri - 1; // last range with tile_first <= tile
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ranges[mid].tile_first <= tile)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Corner (dx, dy) of vertex q of the cell's face 0 (p00, p10, p01) or face 1
// (p10, p11, p01); a mirrored chart swaps vertices 1 and 2 (append_face).
__device__ __forceinline__ void face_corner(int face, int q, bool mirrored, int &dx, int &dy)
{
    const int qq = mirrored && q > 0 ? 3 - q : q;
    if (face == 0) {
        dx = qq == 1;
        dy = qq == 2;
    } else {
        dx = qq != 2;
        dy = qq >= 1;
    }
}

__global__ void __launch_bounds__(kTileThreads, DMAP_TESS_MIN_BLOCKS)
texel_emit_tiles(const TriDev *__restrict__ tris, const AssetDev *__restrict__ assets,
                 const TexelRange *__restrict__ ranges, int n_tri, int64_t tiles,
                 const int64_t *__restrict__ offsets, TexelSink o)
{
    __shared__ float sS[kNodes * 3], sN[kNodes * 3];
    __shared__ unsigned long long s_stage[kTileY][2 * kTileX * 7]; // one row's faces, 7 words each at most
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) { // uniform per block
        const int tri = find_tile_triangle(ranges, n_tri, tile);
        const TexelRange R = ranges[tri];
        const int64_t lt = tile - R.tile_first, tyi = lt / R.tiles_x, txi = lt - tyi * R.tiles_x;
        const int64_t ci = txi * kTileX + tx, cj = tyi * kTileY + ty; // cell within the range
        const int64_t i0 = R.i_lo + txi * kTileX, j0 = R.j_lo + tyi * kTileY;
        const TriDev &T = tris[tri];
        const AssetDev &g = assets[T.asset];
        const double w = 1.0 / g.n_leaf;
        bool inside = false;
        if (ci < R.ni && cj < R.nj)
            inside = classify_square(T, V2((R.i_lo + ci + 0.5) * w, (R.j_lo + cj + 0.5) * w), 0.5 * w) == INSIDE;
        if (!__syncthreads_or(inside))
            continue;
        const bool mirrored = chart_mirrored(T);
        for (int n = threadIdx.x; n < kNodes; n += kTileThreads) {
            const int nx = n % kNodesX, ny = n / kNodesX;
            v3 S, N;
            surface_vertex(T, g, (double)(i0 + nx) * w, (double)(j0 + ny) * w, S, N);
            if (mirrored)
                N = V3(-N.x, -N.y, -N.z);
            put3(sS + 3 * n, S);
            put3(sN + 3 * n, N);
        }
        __syncthreads();
        const unsigned mask = __ballot_sync(0xffffffffu, inside);
        if (mask) {
            // Each output array in turn: every inside lane writes its two
            // faces into the warp's stage in output order, then the warp
            // copies the row's run out with whole-line stores.
            const int a = __ffs(mask) - 1, nf = 2 * __popc(mask), slot = tx - a;
            const int64_t F = offsets[R.first + cj * R.ni + (txi * kTileX + a)];
            float *sf = reinterpret_cast<float *>(s_stage[ty]);
            unsigned long long *sw = s_stage[ty];
            int node[2][3];
            if (inside)
                for (int f = 0; f < 2; ++f)
                    for (int q = 0; q < 3; ++q) {
                        int dx, dy;
                        face_corner(f, q, mirrored, dx, dy);
                        node[f][q] = (ty + dy) * kNodesX + tx + dx;
                    }
            const float *src[2] = {sS, sN};
            float *dst[2] = {o.pos + 9 * F, o.nrm + 9 * F};
            for (int arr = 0; arr < 2; ++arr) {
                if (inside)
                    for (int f = 0; f < 2; ++f)
                        for (int q = 0; q < 3; ++q)
                            for (int c = 0; c < 3; ++c)
                                sf[(2 * slot + f) * 9 + 3 * q + c] = src[arr][3 * node[f][q] + c];
                __syncwarp();
                for (int e = tx; e < 9 * nf; e += 32)
                    dst[arr][e] = sf[e];
                __syncwarp();
            }
            if (inside)
                for (int f = 0; f < 2; ++f)
                    for (int q = 0; q < 3; ++q) {
                        const int n = node[f][q], nx = n % kNodesX, ny = n / kNodesX;
                        sf[(2 * slot + f) * 6 + 2 * q] = (float)((double)(i0 + nx) * w);
                        sf[(2 * slot + f) * 6 + 2 * q + 1] = (float)((double)(j0 + ny) * w);
                    }
            __syncwarp();
            for (int e = tx; e < 6 * nf; e += 32)
                o.uv[6 * F + e] = sf[e];
            __syncwarp();
            // dmap_texel_face as 7 words: (triangle, interior = 1), then st[3][2]
            if (inside)
                for (int f = 0; f < 2; ++f) {
                    unsigned long long *r = sw + (2 * slot + f) * 7;
                    r[0] = (unsigned long long)(unsigned)tri | (1ull << 32);
                    for (int q = 0; q < 3; ++q) {
                        const int n = node[f][q], nx = n % kNodesX, ny = n / kNodesX;
                        r[1 + 2 * q] = (unsigned long long)__double_as_longlong((double)(i0 + nx) * w);
                        r[2 + 2 * q] = (unsigned long long)__double_as_longlong((double)(j0 + ny) * w);
                    }
                }
            __syncwarp();
            unsigned long long *df = reinterpret_cast<unsigned long long *>(o.faces + F);
            for (int e = tx; e < 7 * nf; e += 32)
                df[e] = sw[e];
            __syncwarp();
        }
        __syncthreads(); // the next tile overwrites the nodes
    }
}

unsigned grid_for(int64_t n, int threads)
{
    int64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 64));
}

} // namespace

extern "C" {

dmap_status dmap_tessellate_uniform(dmap_scene *s, int n, float *vertices_dev, float *texcoords_dev,
                                    float *normals_dev, uint32_t *indices_dev, void *stream)
{
    if (!s || n < 1 || !vertices_dev || !texcoords_dev || !normals_dev || !indices_dev)
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_tessellate_uniform: bad argument");
    if (s->n_inst)
        return fail(s->ctx, DMAP_ERR_UNSUPPORTED, "dmap_tessellate_uniform: scenes with non-rigid instances");
    dmap_context *ctx = s->ctx;
    const int64_t V = (int64_t)(n + 1) * (n + 2) / 2, F = (int64_t)n * n;
    const int64_t nv = V * s->n_tri, nf = F * s->n_tri;
    if (nv > (int64_t)UINT32_MAX)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_tessellate_uniform: vertex count exceeds the uint32 index range");
    if (s->n_tri == 0)
        return DMAP_OK;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    uniform_vertices_kernel<<<grid_for(nv, 128), 128, 0, st>>>(s->tris_dev, s->assets_dev, n, nv, vertices_dev,
                                                                 texcoords_dev, normals_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    uniform_faces_kernel<<<grid_for(nf, 256), 256, 0, st>>>(n, nf, indices_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    ctx->launches += 2;
    return DMAP_OK;
}

dmap_status dmap_tessellate_uniform_host(dmap_scene *s, int n, float *vertices, float *texcoords, float *normals,
                                         uint32_t *indices)
{
    if (!s || n < 1 || !vertices || !texcoords || !normals || !indices)
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_tessellate_uniform_host: bad argument");
    dmap_context *ctx = s->ctx;
    const int64_t nv = (int64_t)(n + 1) * (n + 2) / 2 * s->n_tri, nf = (int64_t)n * n * s->n_tri;
    if (nv > (int64_t)UINT32_MAX)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_tessellate_uniform_host: vertex count exceeds the uint32 index range");
    if (s->n_tri == 0)
        return DMAP_OK;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t b_pos = (size_t)nv * 3 * sizeof(float), b_uv = (size_t)nv * 2 * sizeof(float);
    const size_t b_idx = (size_t)nf * 3 * sizeof(uint32_t);
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, 2 * b_pos + b_uv + b_idx, st));
    float *d_pos = (float *)buf, *d_nrm = (float *)(buf + b_pos), *d_uv = (float *)(buf + 2 * b_pos);
    uint32_t *d_idx = (uint32_t *)(buf + 2 * b_pos + b_uv);
    dmap_status r = dmap_tessellate_uniform(s, n, d_pos, d_uv, d_nrm, d_idx, st);
    if (r == DMAP_OK) {
        cudaError_t e = cudaMemcpyAsync(vertices, d_pos, b_pos, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(normals, d_nrm, b_pos, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(texcoords, d_uv, b_uv, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(indices, d_idx, b_idx, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            r = cuda_fail(ctx, e, "dmap_tessellate_uniform_host: copy");
    }
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    return sync_and_check(ctx, "dmap_tessellate_uniform_host");
}

dmap_status dmap_tessellate_texel(dmap_scene *s, int m, int64_t capacity, float *vertices_dev, float *texcoords_dev,
                                  float *normals_dev, dmap_texel_face *faces_dev, int64_t *n_faces, void *stream)
{
    if (!s || m < 1 || !n_faces || capacity < 0 ||
        (vertices_dev && (!texcoords_dev || !normals_dev || !faces_dev)))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_tessellate_texel: bad argument");
    if (s->n_inst)
        return fail(s->ctx, DMAP_ERR_UNSUPPORTED, "dmap_tessellate_texel: scenes with non-rigid instances");
    dmap_context *ctx = s->ctx;
    *n_faces = 0;
    if (s->n_tri == 0)
        return DMAP_OK;
    // Each triangle's cell range from its uv bounding box, as the
    // reference's loop bounds (floor(lo / w) .. ceil(hi / w) - 1); w is a
    // power of two, so the divisions are exact.
    std::vector<TexelRange> ranges(s->n_tri);
    int64_t cells = 0, tiles = 0;
    for (int t = 0; t < s->n_tri; ++t) {
        const TriDev &T = s->tris_host[t];
        double w = 1.0 / s->assets[T.asset]->dev.n_leaf;
        int64_t i_lo = (int64_t)std::floor(T.lo[0] / w), i_hi = (int64_t)std::ceil(T.hi[0] / w) - 1;
        int64_t j_lo = (int64_t)std::floor(T.lo[1] / w), j_hi = (int64_t)std::ceil(T.hi[1] / w) - 1;
        int64_t ni = std::max<int64_t>(0, i_hi - i_lo + 1), nj = std::max<int64_t>(0, j_hi - j_lo + 1);
        const int64_t tx = (ni + kTileX - 1) / kTileX, ty = (nj + kTileY - 1) / kTileY;
        ranges[t] = {cells, i_lo, j_lo, ni > 0 ? ni : 1, nj, tiles, tx > 0 ? tx : 1};
        cells += ni * nj;
        tiles += tx * ty;
    }
    if (cells >= (int64_t)INT32_MAX)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_tessellate_texel: more than 2^31 leaf cells");
    if (cells == 0)
        return DMAP_OK;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;

    size_t scan_bytes = 0;
    DMAP_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const int64_t *)nullptr, (int64_t *)nullptr,
                                                 (int)cells, st));
    const size_t b_ranges = ((sizeof(TexelRange) * s->n_tri + 255) / 256) * 256;
    const size_t b_counts = ((sizeof(int64_t) * (size_t)cells + 255) / 256) * 256;
    const size_t b_offs = ((sizeof(int64_t) * (size_t)cells + 255) / 256) * 256;
    // m = 1: the straddling cells' list (at most every cell) and its length
    const size_t b_list = m == 1 ? ((sizeof(int) * (size_t)cells + 255) / 256) * 256 + 256 : 0;
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, b_ranges + b_counts + b_offs + b_list + scan_bytes, st));
    TexelRange *d_ranges = (TexelRange *)buf;
    int64_t *d_counts = (int64_t *)(buf + b_ranges);
    int64_t *d_offs = (int64_t *)(buf + b_ranges + b_counts);
    unsigned long long *d_nlist = m == 1 ? (unsigned long long *)(buf + b_ranges + b_counts + b_offs) : nullptr;
    int *d_list = m == 1 ? (int *)(buf + b_ranges + b_counts + b_offs + 256) : nullptr;
    void *d_scan = buf + b_ranges + b_counts + b_offs + b_list;

    dmap_status r = DMAP_OK;
    int64_t last[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(d_ranges, ranges.data(), sizeof(TexelRange) * s->n_tri, cudaMemcpyHostToDevice, st);
    TexelSink sink{vertices_dev, texcoords_dev, normals_dev, faces_dev};
    if (e == cudaSuccess && d_nlist)
        e = cudaMemsetAsync(d_nlist, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) {
        texel_kernel<false><<<grid_for(cells, 128), 128, 0, st>>>(s->tris_dev, s->assets_dev, d_ranges, s->n_tri,
                                                                   cells, m, d_counts, nullptr, sink, d_list, d_nlist);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cub::DeviceScan::ExclusiveSum(d_scan, scan_bytes, d_counts, d_offs, (int)cells, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&last[0], d_offs + cells - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&last[1], d_counts + cells - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        r = cuda_fail(ctx, e, "dmap_tessellate_texel: count");
    int64_t total = last[0] + last[1];
    int launches = 1; // the scan's kernels are CUB's
    if (r == DMAP_OK) {
        *n_faces = total;
        if (vertices_dev && total > capacity)
            r = fail(ctx, DMAP_ERR_INVALID, "dmap_tessellate_texel: capacity below the face count");
        else if (vertices_dev && total > 0) {
            if (m == 1) {
                texel_emit_tiles<<<(unsigned)std::min<int64_t>(tiles, 148 * 16), kTileThreads, 0, st>>>(
                    s->tris_dev, s->assets_dev, d_ranges, s->n_tri, tiles, d_offs, sink);
                e = cudaGetLastError();
                if (e == cudaSuccess) {
                    texel_emit_list<<<148 * 4, 128, 0, st>>>(s->tris_dev, s->assets_dev, d_ranges, s->n_tri, d_list,
                                                             d_nlist, d_offs, sink);
                    e = cudaGetLastError();
                }
                launches += 2;
            } else {
                texel_kernel<true><<<grid_for(cells, 128), 128, 0, st>>>(s->tris_dev, s->assets_dev, d_ranges,
                                                                          s->n_tri, cells, m, d_counts, d_offs, sink,
                                                                          nullptr, nullptr);
                e = cudaGetLastError();
                launches += 1;
            }
            if (e != cudaSuccess)
                r = cuda_fail(ctx, e, "dmap_tessellate_texel: emit");
        }
    }
    ctx->launches += launches;
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "dmap_tessellate_texel");
    return DMAP_OK;
}

dmap_status dmap_tessellate_texel_host(dmap_scene *s, int m, int64_t capacity, float *vertices, float *texcoords,
                                       float *normals, dmap_texel_face *faces, int64_t *n_faces)
{
    if (!s || m < 1 || !n_faces || capacity < 0 || (vertices && (!texcoords || !normals || !faces)))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_tessellate_texel_host: bad argument");
    dmap_context *ctx = s->ctx;
    dmap_status r = dmap_tessellate_texel(s, m, 0, nullptr, nullptr, nullptr, nullptr, n_faces, ctx->stream);
    if (r != DMAP_OK || !vertices)
        return r;
    const int64_t nf = *n_faces;
    if (nf > capacity)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_tessellate_texel_host: capacity below the face count");
    if (nf == 0)
        return DMAP_OK;
    cudaStream_t st = ctx->stream;
    const size_t b_pos = (size_t)nf * 9 * sizeof(float), b_uv = (size_t)nf * 6 * sizeof(float);
    const size_t b_faces = (size_t)nf * sizeof(dmap_texel_face);
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, b_faces + 2 * b_pos + b_uv, st));
    dmap_texel_face *d_faces = (dmap_texel_face *)buf;
    float *d_pos = (float *)(buf + b_faces), *d_nrm = (float *)(buf + b_faces + b_pos);
    float *d_uv = (float *)(buf + b_faces + 2 * b_pos);
    int64_t got = 0;
    r = dmap_tessellate_texel(s, m, nf, d_pos, d_uv, d_nrm, d_faces, &got, st);
    if (r == DMAP_OK) {
        cudaError_t e = cudaMemcpyAsync(vertices, d_pos, b_pos, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(normals, d_nrm, b_pos, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(texcoords, d_uv, b_uv, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(faces, d_faces, b_faces, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess)
            r = cuda_fail(ctx, e, "dmap_tessellate_texel_host: copy");
    }
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    return sync_and_check(ctx, "dmap_tessellate_texel_host");
}

} // extern "C"
