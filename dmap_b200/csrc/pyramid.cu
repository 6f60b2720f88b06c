// K1: the Taylor bound pyramid on the device (taylor_pyramid.cpp:45-138,
// leaf_level and fold, the reference's default Fold build).
//
// One CTA per tile of T x T leaf cells (T = min(16, 2^L)), one thread per
// cell in Morton order, so that the four children of every parent are four
// consecutive threads. The (T+1)^2 node tile is staged in shared memory by
// one TMA 2-D tiled load (cp.async.bulk.tensor, no multicast); each thread
// builds its leaf node in double, then the CTA folds 4 -> 1 with warp
// shuffles (max/min/hull reductions over the four children) until its tile
// is one cell, writing every level as it goes. Upper levels above the tile
// are folded by further launches of the fold kernel over the stored FP64
// level. Compiled with -fmad=false: every double operation is the
// reference's, so the FP64 levels equal the reference bit for bit.
//
// Outputs per cell: 8 doubles (no offset; added on read) and 8 floats
// (offset added, rounded outward: h0, gu, gv to nearest with r, ru, rv
// widened by the rounding error, h_min down, h_max up).
#include "dmap_b200.h"
#include "device_types.cuh"
#include "launch.h"
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <mutex>

namespace
{
using dmapdev::AssetDev;

constexpr int64_t kDirectPartials = 32768; // partial hulls after the cells' slope hulls in the Direct scratch
constexpr int kMaxTile = 16;  // 256 threads per CTA: the FP64 fold keeps its registers
constexpr int kTilePitch = 24; // staged row pitch bound in elements (>= 17, TMA box inner extent rounded to 16 B)

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }

// Morton decode of a tile-local cell index: even bits -> x (u, i), odd -> y (v, j).
__device__ __forceinline__ unsigned compact1by1(unsigned x)
{
    x &= 0x55555555u;
    x = (x ^ (x >> 1)) & 0x33333333u;
    x = (x ^ (x >> 2)) & 0x0f0f0f0fu;
    x = (x ^ (x >> 4)) & 0x00ff00ffu;
    x = (x ^ (x >> 8)) & 0x0000ffffu;
    return x;
}

struct Node8 { double h0, gu, gv, r, ru, rv, mn, mx; };

__device__ __forceinline__ double shfl(double v, int lane_mask)
{
    return __shfl_xor_sync(0xffffffffu, v, lane_mask);
}

// Fold four children held by lanes {L, L^1, L^2, L^3} of one warp into
// their parent (taylor_pyramid.cpp:77-138). `b` is the lane's child u bit,
// `a` its v bit; s is the parent half-extent. Every lane returns the parent.
__device__ __forceinline__ Node8 fold4(const Node8 &c, int a, int b, double s)
{
    double gu_hi = c.gu + c.ru, gu_lo = c.gu - c.ru, gv_hi = c.gv + c.rv, gv_lo = c.gv - c.rv;
    double mn = c.mn, mx = c.mx;
#pragma unroll
    for (int m = 1; m <= 2; m <<= 1) {
        gu_hi = dmax(gu_hi, shfl(gu_hi, m));
        gu_lo = dmin(gu_lo, shfl(gu_lo, m));
        gv_hi = dmax(gv_hi, shfl(gv_hi, m));
        gv_lo = dmin(gv_lo, shfl(gv_lo, m));
        mn = dmin(mn, shfl(mn, m));
        mx = dmax(mx, shfl(mx, m));
    }
    Node8 p;
    double gu_p = 0.5 * (gu_hi + gu_lo);
    double gv_p = 0.5 * (gv_hi + gv_lo);
    p.gu = gu_p;
    p.ru = 0.5 * (gu_hi - gu_lo);
    p.gv = gv_p;
    p.rv = 0.5 * (gv_hi - gv_lo);
    p.mn = mn;
    p.mx = mx;
    const double off0 = -0.5 * s, off1 = 0.5 * s;
    double dx = b ? off1 : off0, dy = a ? off1 : off0;
    double du_g = c.gu - gu_p;
    double dv_g = c.gv - gv_p;
    double base = (c.h0 - c.gu * dx) - c.gv * dy;
    double upper = -INFINITY, lower = INFINITY;
#pragma unroll
    for (int cu = 0; cu < 2; ++cu) {
#pragma unroll
        for (int cv = 0; cv < 2; ++cv) {
            double corner = (base + du_g * (dx + (cu ? off1 : off0))) + dv_g * (dy + (cv ? off1 : off0));
            upper = dmax(upper, corner + c.r);
            lower = dmin(lower, corner - c.r);
        }
    }
#pragma unroll
    for (int m = 1; m <= 2; m <<= 1) {
        upper = dmax(upper, shfl(upper, m));
        lower = dmin(lower, shfl(lower, m));
    }
    p.h0 = 0.5 * (upper + lower);
    p.r = 0.5 * (upper - lower);
    return p;
}

// store64: write the FP64 cell too (every level when the FP64 pyramid is
// kept; otherwise only the levels a later fold launch reads).
__device__ __forceinline__ void store_node(const Node8 &n, double offset, size_t k, double *pyr64, float *pyr32,
                                           bool store64)
{
    if (store64) {
        double2 *p = reinterpret_cast<double2 *>(pyr64 + 8 * k);
        p[0] = make_double2(n.h0, n.gu);
        p[1] = make_double2(n.gv, n.r);
        p[2] = make_double2(n.ru, n.rv);
        p[3] = make_double2(n.mn, n.mx);
    }
    double h0 = n.h0, mn = n.mn, mx = n.mx;
    if (offset != 0.0) {
        h0 += offset;
        mn += offset;
        mx += offset;
    }
    float h0f = __double2float_rn(h0), guf = __double2float_rn(n.gu), gvf = __double2float_rn(n.gv);
    float rf = __double2float_ru(__dadd_ru(n.r, fabs(h0 - (double)h0f)));
    float ruf = __double2float_ru(__dadd_ru(n.ru, fabs(n.gu - (double)guf)));
    float rvf = __double2float_ru(__dadd_ru(n.rv, fabs(n.gv - (double)gvf)));
    float4 *q = reinterpret_cast<float4 *>(pyr32 + 8 * k);
    q[0] = make_float4(h0f, guf, gvf, rf);
    q[1] = make_float4(ruf, rvf, __double2float_rd(mn), __double2float_ru(mx));
}

// Folds the CTA's cells (count = T*T held one per thread, Morton order) up
// to one cell, storing each level. `level0` is the level of the held cells,
// (tx, ty) the tile's position in units of T cells at level0.
__device__ void fold_tile(Node8 v, int T, int level0, int tx, int ty, const AssetDev &a, double *pyr64,
                          float *pyr32, Node8 *smem, bool all64)
{
    int t = threadIdx.x;
    int count = T * T;
    int level = level0;
    int side = T;
    while (count > 1) {
        int lvl = level + 1;
        int m = a.n_leaf >> lvl;       // cells per side at the parent level
        double s = 0.5 / m;            // parent half-extent
        Node8 p;
        if (t < ((count + 31) & ~31)) { // whole warps only, inactive lanes hold copies
            p = fold4(v, (t >> 1) & 1, t & 1, s);
        }
        if (t < count && (t & 3) == 0) {
            int pc = t >> 2;
            smem[pc] = p;
            int x = (int)compact1by1((unsigned)pc), y = (int)compact1by1((unsigned)pc >> 1);
            int ps = side >> 1;
            size_t k = (size_t)a.level_off[lvl] + (size_t)(ty * ps + y) * m + (tx * ps + x);
            store_node(p, a.offset, k, pyr64, pyr32, all64 || count == 4); // the tile's top: the next launch reads it
        }
        __syncthreads();
        count >>= 2;
        side >>= 1;
        level = lvl;
        if (t < count)
            v = smem[t];
        else if (count > 0)
            v = smem[0];
        __syncthreads();
    }
}

template <typename In>
__device__ __forceinline__ double to_d(In x);
template <>
__device__ __forceinline__ double to_d<float>(float x) { return (double)x; }
template <>
__device__ __forceinline__ double to_d<__half>(__half x) { return (double)__half2float(x); }
template <>
__device__ __forceinline__ double to_d<__nv_bfloat16>(__nv_bfloat16 x) { return (double)__bfloat162float(x); }
template <>
__device__ __forceinline__ double to_d<double>(double x) { return x; }

__device__ __forceinline__ bool mbar_wait(unsigned bar_addr, unsigned phase)
{
    // Bounded wait on the TMA transaction barrier.
    for (int it = 0; it < (1 << 24); ++it) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar_addr), "r"(phase)
                     : "memory");
        if (done)
            return true;
        __nanosleep(32);
    }
    return false;
}

// Leaf level + in-tile folds. Block: T*T threads. Grid: (n_leaf/T)^2 tiles.
template <typename In>
__global__ void __launch_bounds__(256) pyramid_leaf_kernel(const __grid_constant__ CUtensorMap tmap, AssetDev a,
                                                            int T, double *pyr64, float *pyr32, unsigned *status,
                                                            bool all64)
{
    __shared__ alignas(128) In tile[(kMaxTile + 1) * kTilePitch];
    __shared__ alignas(8) unsigned long long bar;
    __shared__ Node8 smem[kMaxTile * kMaxTile / 4];
    int tiles_x = a.n_leaf / T;
    int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    unsigned bar_addr = (unsigned)__cvta_generic_to_shared(&bar);
    unsigned tile_addr = (unsigned)__cvta_generic_to_shared(tile);
    const int box_w = ((T + 1) * (int)sizeof(In) + 15) / 16 * 16 / (int)sizeof(In);
    const unsigned bytes = (unsigned)(box_w * (T + 1) * sizeof(In));
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_addr) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int x0 = tx * T, y0 = ty * T; // x0 * sizeof(In) is a multiple of 16 for T = 16 and 0 otherwise
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_addr), "r"(bytes)
                     : "memory");
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3}], [%4];" ::"r"(tile_addr),
                     "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(x0), "r"(y0), "r"(bar_addr)
                     : "memory");
    }
    bool ok = mbar_wait(bar_addr, 0);
    if (!ok) {
        if (threadIdx.x == 0)
            atomicOr(status, dmapdev::kStatusCapped);
        return;
    }
    int t = threadIdx.x;
    bool active = t < T * T; // a 1-, 2- or 4-cell tile still runs one full warp
    int x = active ? (int)compact1by1((unsigned)t) : 0, y = active ? (int)compact1by1((unsigned)t >> 1) : 0;
    // leaf_level (taylor_pyramid.cpp:45-67) on V = values * scale
    double v00 = to_d(tile[y * box_w + x]) * a.scale, v10 = to_d(tile[y * box_w + x + 1]) * a.scale;
    double v01 = to_d(tile[(y + 1) * box_w + x]) * a.scale, v11 = to_d(tile[(y + 1) * box_w + x + 1]) * a.scale;
    double w = 1.0 / a.n_leaf;
    double s = 0.5 * w;
    Node8 n;
    n.h0 = 0.25 * (((v00 + v10) + v01) + v11);
    n.gu = 0.5 * ((v10 - v00) + (v11 - v01)) / w;
    n.gv = 0.5 * ((v01 - v00) + (v11 - v10)) / w;
    double c3 = (((v00 - v10) - v01) + v11) / (w * w);
    n.r = fabs(c3) * s * s;
    n.ru = fabs(c3) * s;
    n.rv = fabs(c3) * s;
    n.mn = dmin(dmin(v00, v10), dmin(v01, v11));
    n.mx = dmax(dmax(v00, v10), dmax(v01, v11));
    size_t k = (size_t)(ty * T + y) * a.n_leaf + (tx * T + x);
    if (active)
        store_node(n, a.offset, k, pyr64, pyr32, all64 || T == 1);
    fold_tile(n, T, 0, tx, ty, a, pyr64, pyr32, smem, all64);
}

// Folds level `level0` (m0 x m0 cells, FP64 without offset) upward.
// Block: T*T threads, grid: (m0/T)^2.
__global__ void __launch_bounds__(256) pyramid_fold_kernel(AssetDev a, int level0, int T, double *pyr64,
                                                            float *pyr32, bool all64)
{
    __shared__ Node8 smem[kMaxTile * kMaxTile / 4];
    int m0 = a.n_leaf >> level0;
    int tiles_x = m0 / T;
    int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    int t = threadIdx.x;
    bool active = t < T * T;
    int x = active ? (int)compact1by1((unsigned)t) : 0, y = active ? (int)compact1by1((unsigned)t >> 1) : 0;
    size_t k = (size_t)a.level_off[level0] + (size_t)(ty * T + y) * m0 + (tx * T + x);
    const double2 *p = reinterpret_cast<const double2 *>(pyr64 + 8 * k);
    double2 q0 = p[0], q1 = p[1], q2 = p[2], q3 = p[3];
    Node8 n = {q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y};
    fold_tile(n, T, level0, tx, ty, a, pyr64, pyr32, smem, all64);
}

// ---- the Direct build (taylor_pyramid.cpp:151-202) -------------------------
// Every level from the node grid instead of by folding: a cell's gradient
// plane is the middle of the hull of its texels' bilinear slopes widened by
// their twist, and h0, r the middle and half-width of the node residuals
// against that plane over the cell's (k+1)^2 nodes. Max and min are exact in
// any order, so the hierarchical and team reductions below give the
// reference's serial loops' values bit for bit.

__device__ __forceinline__ double direct_value(const AssetDev &a, int j, int i) // V = values * scale
{
    size_t k = (size_t)j * a.pitch + i;
    double v = a.dtype == 0   ? (double)static_cast<const float *>(a.nodes)[k]
               : a.dtype == 1 ? (double)__half2float(static_cast<const __half *>(a.nodes)[k])
               : a.dtype == 3 ? (double)__bfloat162float(static_cast<const __nv_bfloat16 *>(a.nodes)[k])
                              : static_cast<const double *>(a.nodes)[k];
    return v * a.scale;
}

// Level 0 of the slope hull: {gu_hi, gu_lo, gv_hi, gv_lo} per texel.
__global__ void direct_hull_leaf(AssetDev a, double4 *hull)
{
    const int n = a.n_leaf;
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n)
        return;
    int i = (int)(t % n), j = (int)(t / n);
    double v00 = direct_value(a, j, i), v10 = direct_value(a, j, i + 1);
    double v01 = direct_value(a, j + 1, i), v11 = direct_value(a, j + 1, i + 1);
    double w = 1.0 / n;
    double s_texel = 0.5 / n;
    double c1 = 0.5 * ((v10 - v00) + (v11 - v01)) / w;
    double c2 = 0.5 * ((v01 - v00) + (v11 - v10)) / w;
    double c3 = (((v00 - v10) - v01) + v11) / (w * w);
    double spread = fabs(c3) * s_texel;
    hull[t] = make_double4(c1 + spread, c1 - spread, c2 + spread, c2 - spread);
}

// The slope hull one level up (m x m parent cells).
__global__ void direct_hull_fold(int m, const double4 *child, double4 *parent)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)m * m)
        return;
    int I = (int)(t % m), J = (int)(t / m);
    double4 h = child[(int64_t)(2 * J) * (2 * m) + 2 * I];
    for (int q = 1; q < 4; ++q) {
        double4 c = child[(int64_t)(2 * J + (q >> 1)) * (2 * m) + 2 * I + (q & 1)];
        h.x = dmax(h.x, c.x);
        h.y = dmin(h.y, c.y);
        h.z = dmax(h.z, c.z);
        h.w = dmin(h.w, c.w);
    }
    parent[t] = h;
}

// One level's cells: TEAM threads per cell (1, a warp, or the block).
template <int TEAM>
__global__ void __launch_bounds__(256) direct_cells(AssetDev a, int level, const double4 *hull, double *pyr64,
                                                   float *pyr32, bool all64)
{
    const int n = a.n_leaf, k = 1 << level, m = n >> level;
    int64_t c;
    int lane;
    if (TEAM == 1) {
        c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
        lane = 0;
    } else if (TEAM == 32) {
        c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        lane = threadIdx.x & 31;
    } else {
        c = blockIdx.x;
        lane = threadIdx.x;
    }
    const bool live = c < (int64_t)m * m; // whole teams are live or not
    double upper = -INFINITY, lower = INFINITY, h_min = INFINITY, h_max = -INFINITY;
    double gu = 0.0, gv = 0.0, ru = 0.0, rv = 0.0;
    int I = 0, J = 0;
    if (live) {
        I = (int)(c % m);
        J = (int)(c / m);
        double4 h = hull[c];
        gu = 0.5 * (h.x + h.y);
        ru = 0.5 * (h.x - h.y);
        gv = 0.5 * (h.z + h.w);
        rv = 0.5 * (h.z - h.w);
        const int side = k + 1;
        for (int idx = lane; idx < side * side; idx += TEAM) {
            int b = idx / side, aa = idx % side;
            double dv = (b - 0.5 * k) / n;
            double du = (aa - 0.5 * k) / n;
            double value = direct_value(a, J * k + b, I * k + aa);
            double residual = (value - gu * du) - gv * dv;
            upper = dmax(upper, residual);
            lower = dmin(lower, residual);
            h_min = dmin(h_min, value);
            h_max = dmax(h_max, value);
        }
    }
    if (TEAM >= 32) {
        for (int o = 16; o > 0; o >>= 1) {
            upper = dmax(upper, __shfl_xor_sync(0xffffffffu, upper, o));
            lower = dmin(lower, __shfl_xor_sync(0xffffffffu, lower, o));
            h_min = dmin(h_min, __shfl_xor_sync(0xffffffffu, h_min, o));
            h_max = dmax(h_max, __shfl_xor_sync(0xffffffffu, h_max, o));
        }
    }
    if (TEAM > 32) {
        __shared__ double red[4][TEAM > 32 ? TEAM / 32 : 1];
        int wid = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
            red[0][wid] = upper;
            red[1][wid] = lower;
            red[2][wid] = h_min;
            red[3][wid] = h_max;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int q = 1; q < TEAM / 32; ++q) {
                upper = dmax(upper, red[0][q]);
                lower = dmin(lower, red[1][q]);
                h_min = dmin(h_min, red[2][q]);
                h_max = dmax(h_max, red[3][q]);
            }
    }
    if (live && lane == 0) {
        Node8 nd;
        nd.h0 = 0.5 * (upper + lower);
        nd.gu = gu;
        nd.gv = gv;
        nd.r = 0.5 * (upper - lower);
        nd.ru = ru;
        nd.rv = rv;
        nd.mn = h_min;
        nd.mx = h_max;
        store_node(nd, a.offset, (size_t)a.level_off[level] + (size_t)c, pyr64, pyr32, all64);
    }
}

// Coarse levels have few cells of many nodes: each cell's node rows are cut
// into `chunks` pieces, one block each, whose partial hulls (upper, lower,
// h_min, h_max) a second kernel reduces and stores.
__global__ void __launch_bounds__(256) direct_cells_partial(AssetDev a, int level, const double4 *hull, int chunks,
                                                            double4 *partial)
{
    const int n = a.n_leaf, k = 1 << level, m = n >> level, side = k + 1;
    const int64_t c = blockIdx.x / chunks;
    const int piece = blockIdx.x % chunks;
    const int I = (int)(c % m), J = (int)(c / m);
    double4 h = hull[c];
    double gu = 0.5 * (h.x + h.y), gv = 0.5 * (h.z + h.w);
    int r0 = (int)((int64_t)side * piece / chunks), r1 = (int)((int64_t)side * (piece + 1) / chunks);
    double upper = -INFINITY, lower = INFINITY, h_min = INFINITY, h_max = -INFINITY;
    for (int b = r0; b < r1; ++b) {
        double dv = (b - 0.5 * k) / n;
        for (int aa = threadIdx.x; aa < side; aa += blockDim.x) {
            double du = (aa - 0.5 * k) / n;
            double value = direct_value(a, J * k + b, I * k + aa);
            double residual = (value - gu * du) - gv * dv;
            upper = dmax(upper, residual);
            lower = dmin(lower, residual);
            h_min = dmin(h_min, value);
            h_max = dmax(h_max, value);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        upper = dmax(upper, __shfl_xor_sync(0xffffffffu, upper, o));
        lower = dmin(lower, __shfl_xor_sync(0xffffffffu, lower, o));
        h_min = dmin(h_min, __shfl_xor_sync(0xffffffffu, h_min, o));
        h_max = dmax(h_max, __shfl_xor_sync(0xffffffffu, h_max, o));
    }
    __shared__ double4 red[8];
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = make_double4(upper, lower, h_min, h_max);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
            upper = dmax(upper, red[q].x);
            lower = dmin(lower, red[q].y);
            h_min = dmin(h_min, red[q].z);
            h_max = dmax(h_max, red[q].w);
        }
        partial[blockIdx.x] = make_double4(upper, lower, h_min, h_max);
    }
}

__global__ void direct_cells_final(AssetDev a, int level, const double4 *hull, int chunks, const double4 *partial,
                                   double *pyr64, float *pyr32, bool all64)
{
    const int m = a.n_leaf >> level;
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (int64_t)m * m)
        return;
    double4 p = partial[c * chunks];
    for (int q = 1; q < chunks; ++q) {
        double4 x = partial[c * chunks + q];
        p.x = dmax(p.x, x.x);
        p.y = dmin(p.y, x.y);
        p.z = dmin(p.z, x.z);
        p.w = dmax(p.w, x.w);
    }
    double4 h = hull[c];
    Node8 nd;
    nd.h0 = 0.5 * (p.x + p.y);
    nd.gu = 0.5 * (h.x + h.y);
    nd.gv = 0.5 * (h.z + h.w);
    nd.r = 0.5 * (p.x - p.y);
    nd.ru = 0.5 * (h.x - h.y);
    nd.rv = 0.5 * (h.z - h.w);
    nd.mn = p.z;
    nd.mx = p.w;
    store_node(nd, a.offset, (size_t)a.level_off[level] + (size_t)c, pyr64, pyr32, all64);
}

template <typename In>
cudaError_t launch_leaf(const void *tmap, const AssetDev &a, int T, double *pyr64, float *pyr32, unsigned *status,
                        bool all64, cudaStream_t stream)
{
    int tiles = (a.n_leaf / T) * (a.n_leaf / T);
    int threads = T * T < 32 ? 32 : T * T;
    pyramid_leaf_kernel<In><<<tiles, threads, 0, stream>>>(*reinterpret_cast<const CUtensorMap *>(tmap), a, T,
                                                           pyr64, pyr32, status, all64);
    return cudaGetLastError();
}

} // namespace

namespace dmapk
{
cudaError_t launch_pyramid(const void *tmap, const dmapdev::AssetDev &a, int tile, double *pyr64, float *pyr32,
                           unsigned *status, cudaStream_t stream, bool all64)
{
    cudaError_t e;
    if (a.dtype == 0)
        e = launch_leaf<float>(tmap, a, tile, pyr64, pyr32, status, all64, stream);
    else if (a.dtype == 1)
        e = launch_leaf<__half>(tmap, a, tile, pyr64, pyr32, status, all64, stream);
    else if (a.dtype == 3)
        e = launch_leaf<__nv_bfloat16>(tmap, a, tile, pyr64, pyr32, status, all64, stream);
    else
        e = launch_leaf<double>(tmap, a, tile, pyr64, pyr32, status, all64, stream);
    if (e != cudaSuccess)
        return e;
    // levels above the first tile fold
    int level = 0, T = tile;
    while ((1 << level) * T < a.n_leaf) {
        level += __builtin_ctz((unsigned)T); // the tile fold produced levels up to level + log2(T)
        int m = a.n_leaf >> level;
        T = m < kMaxTile ? m : kMaxTile;
        int threads = T * T < 32 ? 32 : T * T;
        pyramid_fold_kernel<<<(m / T) * (m / T), threads, 0, stream>>>(a, level, T, pyr64, pyr32, all64);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

int direct_launches(int n_leaf)
{
    int c = 0;
    for (int l = 0; (1 << l) <= n_leaf; ++l)
        c += ((1 << l) <= 64 || (int64_t)(n_leaf >> l) * (n_leaf >> l) >= 2048) ? 2 : 3;
    return c;
}

cudaError_t launch_pyramid_direct(const dmapdev::AssetDev &a, double *pyr64, float *pyr32, void *hull_scratch,
                                  cudaStream_t stream, bool all64)
{
    double4 *hull = static_cast<double4 *>(hull_scratch);
    const int n = a.n_leaf;
    int64_t total_cells = 0;
    for (int l = 0; l < a.n_levels; ++l)
        total_cells += (int64_t)(n >> l) * (n >> l);
    cudaError_t e;
    for (int l = 0; l < a.n_levels; ++l) {
        int m = n >> l;
        int64_t cells = (int64_t)m * m;
        double4 *h = hull + a.level_off[l];
        if (l == 0)
            direct_hull_leaf<<<(unsigned)((cells + 255) / 256), 256, 0, stream>>>(a, h);
        else
            direct_hull_fold<<<(unsigned)((cells + 255) / 256), 256, 0, stream>>>(m, hull + a.level_off[l - 1], h);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return e;
        int k = 1 << l;
        if (k <= 4) {
            direct_cells<1><<<(unsigned)((cells + 255) / 256), 256, 0, stream>>>(a, l, h, pyr64, pyr32, all64);
        } else if (k <= 64) {
            direct_cells<32><<<(unsigned)((cells * 32 + 255) / 256), 256, 0, stream>>>(a, l, h, pyr64, pyr32, all64);
        } else if (cells >= 2048) {
            direct_cells<256><<<(unsigned)cells, 256, 0, stream>>>(a, l, h, pyr64, pyr32, all64);
        } else {
            // about 2048 blocks per level, at least one node row each
            int64_t chunks = std::min<int64_t>((2048 + cells - 1) / cells, k + 1);
            chunks = std::min<int64_t>(chunks, kDirectPartials / cells);
            double4 *partial = hull + total_cells;
            direct_cells_partial<<<(unsigned)(cells * chunks), 256, 0, stream>>>(a, l, h, (int)chunks, partial);
            if ((e = cudaGetLastError()) != cudaSuccess)
                return e;
            direct_cells_final<<<(unsigned)((cells + 255) / 256), 256, 0, stream>>>(a, l, h, (int)chunks, partial,
                                                                                  pyr64, pyr32, all64);
        }
        if ((e = cudaGetLastError()) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}
} // namespace dmapk

// ---------------------------------------------------------------------------
// dmap_pyramid_build_noalloc: the pyramid build for callers that cannot
// allocate device memory.
//
// The regular build (dmap_asset_create) allocates its FP64 working levels,
// and its node grid and output, with cudaMalloc. Callers that own every byte
// of device memory through their own pool, or that must not allocate while
// a frame is in flight, cannot let the library do that. For them this entry
// point takes the node grid and the FP32 output pyramid as device buffers
// they already hold, and keeps the FP64 working levels in the fixed array
// below instead of allocating. The array is file-scope device memory: every
// GPU that loads the library holds it (22.4 MB) until the process exits, and
// it bounds the map size this entry point accepts to 512 x 512 texels.
// Every call reuses the same array, so calls whose kernels overlap on the
// GPU (two streams, or two host threads) race on it: serialize them.
// ---------------------------------------------------------------------------

namespace
{
constexpr int kNoallocMaxLeaf = 512;                    // texels per side
constexpr size_t kNoallocCells = (size_t)349525;        // cells of a 512^2 pyramid: (4^10 - 1) / 3
constexpr size_t kNoallocHead = 32;                     // doubles ahead of the levels: the status word
static __device__ __align__(256) double g_noalloc_scratch[kNoallocHead + 8 * kNoallocCells];

typedef CUresult (*NoallocEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                    const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                    CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                    CUtensorMapFloatOOBfill);

typedef CUresult (*NoallocCtxCurrentFn)(CUcontext *);
typedef CUresult (*NoallocCtxIdFn)(CUcontext, unsigned long long *);

// The unique id of the calling thread's current context (cuCtxGetId ids are
// never reused within a process), or false when none is current yet.
bool noalloc_context_id(unsigned long long &id)
{
    static NoallocCtxCurrentFn get_current = nullptr;
    static NoallocCtxIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<NoallocCtxCurrentFn>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<NoallocCtxIdFn>(fn);
    });
    CUcontext ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx)
        return false;
    return get_id(ctx, &id) == CUDA_SUCCESS;
}

// The device address of the scratch array in the calling thread's current
// context (the host-side symbol is only a stand-in and must never reach a
// kernel). The address is looked up with cudaGetSymbolAddress the first time
// a device is used and again whenever that device's context is new (after a
// cudaDeviceReset, or a primary context released and retained again), so a
// cached address never outlives its context; a mutex orders the look-ups of
// concurrent first calls.
double *noalloc_scratch(int device, cudaError_t &err)
{
    struct Slot
    {
        unsigned long long ctx_id;
        double *addr;
    };
    static std::mutex mu;
    static Slot slots[64] = {};
    err = cudaSuccess;
    if (device < 0 || device >= 64)
        return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    unsigned long long id = 0;
    if (noalloc_context_id(id) && slots[device].addr && slots[device].ctx_id == id)
        return slots[device].addr;
    double *p = nullptr;
    err = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (err != cudaSuccess)
        return nullptr;
    // the look-up made the device's primary context current if none was
    if (noalloc_context_id(id))
        slots[device] = Slot{id, p};
    return p;
}
} // namespace

extern "C" dmap_status dmap_pyramid_build_noalloc(const void *nodes_dev, dmap_dtype dtype, int nodes, int pitch,
                                                  double scale, double offset, int repeat, float *pyr32_dev,
                                                  void *stream)
{
    int n = nodes - 1;
    if (!nodes_dev || !pyr32_dev)
        return DMAP_ERR_INVALID;
    if (nodes < 2 || (n & (n - 1)) != 0)
        return DMAP_ERR_INVALID;
    if (n > kNoallocMaxLeaf)
        return DMAP_ERR_INVALID; // beyond the fixed scratch: use dmap_asset_create
    if (dtype != DMAP_F32 && dtype != DMAP_F16 && dtype != DMAP_BF16 && dtype != DMAP_F64)
        return DMAP_ERR_INVALID;
    size_t es = dtype == DMAP_F64 ? 8 : (dtype == DMAP_F16 || dtype == DMAP_BF16) ? 2 : 4;
    if (pitch < nodes || ((size_t)pitch * es) % 16 != 0 || ((uintptr_t)nodes_dev & 15) != 0 ||
        ((uintptr_t)pyr32_dev & 15) != 0 || !std::isfinite(scale) || !std::isfinite(offset))
        return DMAP_ERR_INVALID;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess)
        return DMAP_ERR_CUDA;
    cudaError_t err;
    double *scratch = noalloc_scratch(device, err);
    if (!scratch)
        return DMAP_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;

    AssetDev a{};
    a.nodes = nodes_dev;
    a.dtype = dtype == DMAP_F32 ? 0 : dtype == DMAP_F16 ? 1 : dtype == DMAP_BF16 ? 3 : 2;
    a.W = nodes;
    a.pitch = pitch;
    a.n_leaf = n;
    a.n_levels = 1;
    while ((1 << a.n_levels) <= n)
        ++a.n_levels;
    a.repeat = repeat ? 1 : 0;
    a.scale = scale;
    a.offset = offset;
    int64_t cells = 0;
    for (int l = 0; l < a.n_levels; ++l) {
        a.level_off[l] = cells;
        int64_t m = n >> l;
        cells += m * m;
    }
    double *levels = scratch + kNoallocHead;
    unsigned *status = reinterpret_cast<unsigned *>(scratch);
    a.pyr64 = levels;
    a.pyr32 = pyr32_dev;

    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
        return DMAP_ERR_CUDA;
    int T = n < kMaxTile ? n : kMaxTile;
    cuuint32_t box_w = (cuuint32_t)(((T + 1) * es + 15) / 16 * 16 / es);
    CUtensorMap tmap;
    cuuint64_t dims[2] = {(cuuint64_t)nodes, (cuuint64_t)nodes};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * es};
    cuuint32_t box[2] = {box_w, (cuuint32_t)(T + 1)};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMapDataType tdt = dtype == DMAP_F32    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                              : dtype == DMAP_F16  ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                              : dtype == DMAP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if (reinterpret_cast<NoallocEncodeFn>(fn)(&tmap, tdt, 2, const_cast<void *>(nodes_dev), dims, strides, box, estr,
                                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return DMAP_ERR_CUDA;
    // the status word must start at zero; the levels are overwritten whole
    if (cudaMemsetAsync(status, 0, sizeof(unsigned), s) != cudaSuccess)
        return DMAP_ERR_CUDA;
    if (dmapk::launch_pyramid(&tmap, a, T, levels, pyr32_dev, status, s) != cudaSuccess)
        return DMAP_ERR_CUDA;
    unsigned st = 0;
    if (cudaMemcpyAsync(&st, status, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return DMAP_ERR_CUDA;
    return st ? DMAP_ERR_LIMIT : DMAP_OK;
}
