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
    int64_t first, i_lo, j_lo, ni;
};

struct ClipPoly
{
    int n;
    v2 p[8];
};

// clip_square (uv_clip.cpp:61-90): Sutherland-Hodgman of the square (c, s)
// against the domain's three inward half-planes.
__device__ inline ClipPoly clip_square(const TriDev &T, v2 c, double s)
{
    ClipPoly in;
    in.n = 4;
    in.p[0] = add2(c, V2(-s, -s));
    in.p[1] = add2(c, V2(s, -s));
    in.p[2] = add2(c, V2(s, s));
    in.p[3] = add2(c, V2(-s, s));
    for (int k = 0; k < 3; ++k) {
        ClipPoly out;
        out.n = 0;
        v2 nk = L2(T.un[k]);
        double dk = T.ud[k];
        for (int a = 0; a < in.n; ++a) {
            v2 pa = in.p[a], pb = in.p[a + 1 == in.n ? 0 : a + 1];
            double fa = dot2(nk, pa) - dk, fb = dot2(nk, pb) - dk;
            if (fa >= 0.0)
                out.p[out.n++] = pa;
            if ((fa >= 0.0) != (fb >= 0.0)) {
                double t = fa / (fa - fb);
                out.p[out.n++] = add2(pa, mul2(t, sub2(pb, pa)));
            }
        }
        in = out;
        if (in.n == 0)
            break;
    }
    return in;
}

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

// append_face / append_vertex (:60-95): b and c swapped under a mirrored
// chart, the normal flipped with it.
__device__ inline void emit_face(const TriDev &T, const AssetDev &g, int tri, bool mirrored, v2 a, v2 b, v2 c,
                                 int interior, int64_t f, const TexelSink &o)
{
    if (mirrored) {
        v2 x = b;
        b = c;
        c = x;
    }
    v2 v[3] = {a, b, c};
    dmap_texel_face rec;
    rec.triangle = tri;
    rec.interior = interior;
    for (int q = 0; q < 3; ++q) {
        v3 S, nn;
        surface_vertex(T, g, v[q].x, v[q].y, S, nn);
        if (mirrored)
            nn = V3(-nn.x, -nn.y, -nn.z);
        int64_t k = 3 * f + q;
        put3(o.pos + 3 * k, S);
        o.uv[2 * k] = (float)v[q].x;
        o.uv[2 * k + 1] = (float)v[q].y;
        put3(o.nrm + 3 * k, nn);
        rec.st[q][0] = v[q].x;
        rec.st[q][1] = v[q].y;
    }
    o.faces[f] = rec;
}

// One leaf cell of append_texel_tessellation's loop: counts its faces
// (EMIT false) or writes them from face index `f` on (EMIT true).
template <bool EMIT>
__device__ inline int texel_cell(const TriDev &T, const AssetDev &g, int tri, bool mirrored, int64_t i, int64_t j,
                                 int m, int64_t f, const TexelSink &o)
{
    double w = 1.0 / g.n_leaf;
    v2 c = V2((i + 0.5) * w, (j + 0.5) * w);
    int overlap = classify_square(T, c, 0.5 * w);
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
                        emit_face(T, g, tri, mirrored, poly.p[0], poly.p[k], poly.p[k + 1], 0, f + count, o);
                    ++count;
                }
                continue;
            }
            if (EMIT) {
                emit_face(T, g, tri, mirrored, p00, p10, p01, 1, f + count, o);
                emit_face(T, g, tri, mirrored, p10, p11, p01, 1, f + count + 1, o);
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

template <bool EMIT>
__global__ void texel_kernel(const TriDev *__restrict__ tris, const AssetDev *__restrict__ assets,
                             const TexelRange *__restrict__ ranges, int n_tri, int64_t cells, int m,
                             int64_t *__restrict__ counts, const int64_t *__restrict__ offsets, TexelSink o)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cells; k += (int64_t)gridDim.x * blockDim.x) {
        if (EMIT && counts[k] == 0)
            continue;
        int tri = find_triangle(ranges, n_tri, k);
        TexelRange R = ranges[tri];
        int64_t r = k - R.first, jj = r / R.ni, ii = r - jj * R.ni;
        const TriDev &T = tris[tri];
        int c = texel_cell<EMIT>(T, assets[T.asset], tri, chart_mirrored(T), R.i_lo + ii, R.j_lo + jj, m,
                                 EMIT ? offsets[k] : 0, o);
        if (!EMIT)
            counts[k] = c;
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
    dmap_context *ctx = s->ctx;
    *n_faces = 0;
    if (s->n_tri == 0)
        return DMAP_OK;
    // Each triangle's cell range from its uv bounding box, as the
    // reference's loop bounds (floor(lo / w) .. ceil(hi / w) - 1); w is a
    // power of two, so the divisions are exact.
    std::vector<TexelRange> ranges(s->n_tri);
    int64_t cells = 0;
    for (int t = 0; t < s->n_tri; ++t) {
        const TriDev &T = s->tris_host[t];
        double w = 1.0 / s->assets[T.asset]->dev.n_leaf;
        int64_t i_lo = (int64_t)std::floor(T.lo[0] / w), i_hi = (int64_t)std::ceil(T.hi[0] / w) - 1;
        int64_t j_lo = (int64_t)std::floor(T.lo[1] / w), j_hi = (int64_t)std::ceil(T.hi[1] / w) - 1;
        int64_t ni = std::max<int64_t>(0, i_hi - i_lo + 1), nj = std::max<int64_t>(0, j_hi - j_lo + 1);
        ranges[t] = {cells, i_lo, j_lo, ni > 0 ? ni : 1};
        cells += ni * nj;
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
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, b_ranges + b_counts + b_offs + scan_bytes, st));
    TexelRange *d_ranges = (TexelRange *)buf;
    int64_t *d_counts = (int64_t *)(buf + b_ranges);
    int64_t *d_offs = (int64_t *)(buf + b_ranges + b_counts);
    void *d_scan = buf + b_ranges + b_counts + b_offs;

    dmap_status r = DMAP_OK;
    int64_t last[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(d_ranges, ranges.data(), sizeof(TexelRange) * s->n_tri, cudaMemcpyHostToDevice, st);
    TexelSink sink{vertices_dev, texcoords_dev, normals_dev, faces_dev};
    if (e == cudaSuccess) {
        texel_kernel<false><<<grid_for(cells, 128), 128, 0, st>>>(s->tris_dev, s->assets_dev, d_ranges, s->n_tri,
                                                                   cells, m, d_counts, nullptr, sink);
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
    int launches = 2;
    if (r == DMAP_OK) {
        *n_faces = total;
        if (vertices_dev && total > capacity)
            r = fail(ctx, DMAP_ERR_INVALID, "dmap_tessellate_texel: capacity below the face count");
        else if (vertices_dev && total > 0) {
            texel_kernel<true><<<grid_for(cells, 128), 128, 0, st>>>(s->tris_dev, s->assets_dev, d_ranges, s->n_tri,
                                                                      cells, m, d_counts, d_offs, sink);
            e = cudaGetLastError();
            if (e != cudaSuccess)
                r = cuda_fail(ctx, e, "dmap_tessellate_texel: emit");
            launches += 1;
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
