// The FP32 query path: the reference's walk (displaced_intersector.cpp:175-237)
// with every node test evaluated in FP32 and widened outward (f32_node.cuh),
// so that a cell the double-precision test admits is admitted here too;
// leaves run the reference's certified Newton leaf in double (f64_leaf.cuh),
// which makes every reported hit the reference's own FP64 root.
//
// Conservative FP32 arithmetic. A form is c + a eu + b ev + rho with
// |rho| <= k; c, a, b are rounded to nearest and k is an upper bound kept
// with round-up operations. Every operation adds to k a bound on the
// rounding of the coefficients it produced: G * (sum of the magnitudes of
// the terms that entered them), G = 2^-20 (16 units in the last place, more
// than the few roundings of each step), and every input rounded from double
// (the triangle's frame, normals, pyramid nodes) carries its own rounding
// into k the same way. The reciprocal norm is bounded with directed rounding
// around rsqrtf's documented 2-ulp error. The box of a cell is the outward
// interval hull; the tangent-space ray (transformed in double, then rounded)
// is covered by widening every box by the ray's own rounding error over the
// triangle's t range. Slab tests use directed-rounding interval arithmetic.
//
// Two schedules:
//  - simple: one thread per ray, one launch (the plain per-request kernel).
//    Its lanes serialize on divergence: each lane walks its own triangles
//    while the others wait (measured 1.6 active threads per warp
//    instruction on the cube-sphere workload).
//  - wavefront (default): rounds of two persistent kernels. The walk kernel
//    keeps every lane on a node test each step: a lane whose ray reaches a
//    leaf writes a leaf job, parks the ray's walk state and takes the next
//    ray; the leaf kernel runs the parked leaves, one job per lane, each
//    lane taking the next job when its own is done, and queues their rays
//    to resume. After `rounds` rounds a last walk runs the few
//    remaining rays with their leaves inline. Every ray still visits its
//    cells in the reference's order with the reference's t_max, so its hit
//    is the one the simple schedule finds.
//
// The kernels live in this header and are instantiated by two translation
// units (walk32_launch.h lists which launches each one owns):
//  - walk32.cu, compiled with FMA contraction: the walk rounds, whose
//    arithmetic is conservative by its error bounds, so a fused multiply-add
//    (one rounding instead of two) stays inside them, and whose rounding
//    never reaches a result (every leaf cell is re-tested in FP64);
//  - walk32_exact.cu, compiled with -fmad=false: everything that must round
//    like the reference or the same way wherever it runs: the simple
//    schedule, the last walk with leaves inline, the leaf rounds of both
//    leaves and the FP64 re-test of parked cells.
// FP32 code asks for fused multiply-adds explicitly (fmaf) where its bounds
// are written for one.
#pragma once
#include "walk32_launch.h"
#include "f32_node.cuh"
#include "bvh.cuh"
#include "leaf32.cuh"
#include "order.cuh"
#include "filter.cuh"
#include "instance.cuh"

namespace
{
using namespace d32;
using dmapdev::AssetDev;
using dmapdev::TriDev;
using dmapdev::TriDev32;

// Resident 128-thread CTAs per SM the walk and leaf kernels are compiled for
// (register budget: 65536 / (128 x blocks) per thread). The walk rounds over
// the per-ray candidate mask (scenes of up to 256 triangles) take 4 (119
// registers, no spills: faster than 5 at 96 registers with spills); over the
// triangle tree, whose candidate buffer lives in local memory either way, 5.
#ifndef DMAP_WALK_MIN_BLOCKS
#define DMAP_WALK_MIN_BLOCKS 4
#endif
#ifndef DMAP_WALK_TREE_MIN_BLOCKS
#define DMAP_WALK_TREE_MIN_BLOCKS 5
#endif
#ifndef DMAP_LEAF_MIN_BLOCKS
#define DMAP_LEAF_MIN_BLOCKS 1
#endif
// Node tests a ray may run past its first collected leaf before it parks.
#ifndef DMAP_STALE_CAP
#define DMAP_STALE_CAP 32
#endif

constexpr int kMaskWords = 8; // scenes of up to 256 triangles take the object-box candidate mask
constexpr unsigned FULL = 0xffffffffu;

// The tangent-space ray of a triangle: transformed in double, rounded to
// float, and E covering, for t in [0, t_far], the distance between the float
// ray and the reference's double ray (A (o - q0), A d in its own operation
// order): the rounding to float, at most 2^-24 of each coordinate (2^-22
// taken), plus the difference of two double evaluations of the transform,
// a few units of 2^-53 of the sums of the terms' magnitudes (2^-40 taken).
__device__ __forceinline__ void tangent_ray(const TriDev32 &T, const double *o, const double *d, float t_far,
                                            Ray32 &r)
{
    float ro[3], rd[3], e[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double u0 = o[0] - T.q0[0], u1 = o[1] - T.q0[1], u2 = o[2] - T.q0[2];
        double x = u0 * T.A[a][0];
        x = __fma_rn(T.A[a][1], u1, x);
        x = __fma_rn(T.A[a][2], u2, x);
        double y = __fma_rn(T.A[a][2], d[2], __fma_rn(T.A[a][1], d[1], T.A[a][0] * d[0]));
        double mx = fabs(T.A[a][0] * u0) + fabs(T.A[a][1] * u1) + fabs(T.A[a][2] * u2);
        double my = fabs(T.A[a][0] * d[0]) + fabs(T.A[a][1] * d[1]) + fabs(T.A[a][2] * d[2]);
        ro[a] = (float)x;
        rd[a] = (float)y;
        float sum = ru_add(__double2float_ru(mx), ru_mul(t_far, __double2float_ru(my)));
        e[a] = ru_add(ru_mul(0x1p-22f, ru_add(fabsf(ro[a]), ru_mul(t_far, fabsf(rd[a])))), ru_mul(0x1p-40f, sum));
    }
    r.ox = ro[0], r.oy = ro[1], r.oz = ro[2];
    r.dx = rd[0], r.dy = rd[1], r.dz = rd[2];
    r.ix = r.dx != 0.0f ? __frcp_rn(r.dx) : 0.0f;
    r.iy = r.dy != 0.0f ? __frcp_rn(r.dy) : 0.0f;
    r.iz = r.dz != 0.0f ? __frcp_rn(r.dz) : 0.0f;
    r.ex = e[0], r.ey = e[1], r.ez = e[2];
}

__device__ __forceinline__ float far_bound(float t1) { return ru_add(ru_mul(t1, 1.0f + 4.0f * G), G); }

// ---- simple schedule: one thread per ray ----------------------------------

// A leaf cell the FP32 walk reached, in the simple schedule and the
// inline-leaf walk: the cell's FP64 node test, then the certified leaf in the
// query's leaf precision (FP64: the reference's leaf; FP32: leaf32.cuh).
// flags: DMAP_HIT_* of the root.
__device__ __noinline__ bool leaf_cell(const TriDev32 &T32, const TriDev &T, const AssetDev &g, const double *o,
                                       const double *d, double t_min, double t_max, int i, int j, d64::hit64 &h,
                                       int &flags, int64_t *st, const dmapk::QueryOpts &opt)
{
    // an instanced triangle meets the ray in its object space (instance.cuh)
    double oo[3], od[3];
    if (T.inst) {
        dmapdev::object_ray(opt.inst_xf + dmapdev::kInstDoubles * (T.inst - 1), o, d, oo, od);
        o = oo;
        d = od;
    }
    bool ok;
    if (opt.leaf_precision != 1) {
        flags = DMAP_HIT_FP64_LEAF;
        ok = leaf64(T, g, o, d, t_min, t_max, i, j, h, st, opt);
    } else {
        d64::v3 O = d64::V3(o[0], o[1], o[2]), D = d64::V3(d[0], d[1], d[2]);
        ok = d64::leaf_cell_admitted(T, g, O, D, t_min, t_max, i, j, opt) &&
             l32::intersect_newton32(T, T32, g, O, D, t_min, t_max, i, j, opt.polish_cond, h, flags, st);
    }
    if (ok && T.inst)
        dmapdev::world_normal(opt.inst_xf + dmapdev::kInstDoubles * (T.inst - 1), h.ng);
    return ok;
}

// DisplacedIntersector::intersect with the FP32 node test.
__device__ bool triangle_walk32(const TriDev32 &T, const TriDev &T64, const AssetDev &g, const double *o,
                                const double *d, double t_min, double &t_max, const dmapk::QueryOpts &opt,
                                d64::hit64 &hit, int &hflags, int64_t *st, float t_far, unsigned *status,
                                bool &capped)
{
    Ray32 r;
    tangent_ray(T, o, d, t_far, r);
    int si = r.dx < 0.0f, sj = r.dy < 0.0f;
    float tmin_f = __double2float_rd(t_min);
    bool found = false;
    int64_t nah = 0, lah = 0;
    const int log2n = __ffs(g.n_leaf) - 1;
    for (int q = 0; q < T.n_roots; ++q) {
        Cell32 cur = {T.root_level, T.roots_i[q], T.roots_j[q]}, end = cur;
        cell_next(end, si, sj, T.root_level);
        int guard = 0;
        while (!(cur.level == end.level && cur.i == end.i && cur.j == end.j)) {
            if (++guard > opt.guard_cap) { // a finite tree: the cap guards corrupt records
                atomicOr(status, dmapdev::kStatusCapped);
                capped = true;
                break;
            }
            float w = pow2f(cur.level - log2n);
            if (!square_meets_domain(T, ((float)cur.i + 0.5f) * w, ((float)cur.j + 0.5f) * w, 0.5f * w)) {
                cell_next(cur, si, sj, T.root_level);
                continue;
            }
            if (st) {
                ++st[DMAP_ST_NODE];
                ++nah;
            }
            float tmax_f = __double2float_ru(t_max);
            if (!node_test32(T, g, r, cur.level, cur.i, cur.j, tmin_f, tmax_f, opt.bound, opt.slab_max_level)) {
                cell_next(cur, si, sj, T.root_level);
                continue;
            }
            if (cur.level > 0) {
                --cur.level;
                cur.i = 2 * cur.i + si;
                cur.j = 2 * cur.j + sj;
                continue;
            }
            if (st) {
                ++st[DMAP_ST_LEAF];
                ++lah;
            }
            d64::hit64 lh;
            int lf = 0;
            if (leaf_cell(T, T64, g, o, d, t_min, t_max, cur.i, cur.j, lh, lf, st, opt) && lh.t < t_max) {
                hit = lh;
                hflags = lf;
                t_max = lh.t;
                found = true;
                nah = lah = 0;
                if (opt.mode == 1 && !opt.op_mask) // a filter judges the nearest crossing
                    return true;
            }
            cell_next(cur, si, sj, T.root_level);
        }
    }
    if (st && found) {
        st[DMAP_ST_NAH] += nah;
        st[DMAP_ST_LAH] += lah;
    }
    return found;
}

template <typename R, typename H, typename Fp>
__global__ void __launch_bounds__(128) walk32_simple(const TriDev32 *__restrict__ tris32,
                                                     const TriDev *__restrict__ tris64, int n_tri,
                                                     const AssetDev *__restrict__ assets, const R *__restrict__ rays,
                                                     int64_t n, dmapk::QueryOpts opt, H *__restrict__ hits,
                                                     int64_t *__restrict__ stats, unsigned *status,
                                                     const int *__restrict__ ray_list = nullptr,
                                                     const unsigned long long *list_n = nullptr)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ray_list) {
        // the rays a filtered wavefront query hands back (check_crossing)
        if ((unsigned long long)k >= *list_n)
            return;
        k = ray_list[k];
    } else if (k >= n || (opt.n_dev && k >= *opt.n_dev)) {
        return;
    }
    double o[3], d[3], t_min, t_max;
    load_ray(rays, k, o, d, t_min, t_max);
    float of[3], df[3], invf[3];
    for (int a = 0; a < 3; ++a) {
        of[a] = (float)o[a];
        df[a] = (float)d[a];
        invf[a] = df[a] != 0.0f ? __frcp_rn(df[a]) : 0.0f;
    }
    int64_t st[DMAP_ST_N] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t *sp = stats ? st : nullptr;
    d64::hit64 best;
    int best_tri = -1, best_flags = 0;
    bool found = false, capped = false;
    // the next triangle: the smallest (key, index) past the cursor among the
    // candidates the ray still reaches, the key being the index (index
    // order) or the box entry (nearest)
    double inv[3], ckey = -INFINITY;
    int cidx = -1;
    d64::ray_inverse(d, inv);
    // scenes of more than 256 triangles: the triangle tree (bvh.cuh)
    const d32::BvhView bvh = {opt.bvh_nodes, opt.bvh_tri, opt.bvh_range, opt.bvh_n_nodes};
    d32::NearBuf nbuf;
    nbuf.n = -1;
    nbuf.pos = 0;
    for (int step = 0; step < n_tri; ++step) {
        int t = step;
        float t1 = __double2float_ru(t_max);
        if (bvh.nodes) {
            bool err = false;
            const float tmin_f = __double2float_rd(t_min);
            t = opt.order == 1 ? d32::near_next<true>(nbuf, bvh, tris32, tris64, o, d, inv, t_min, of, df, invf,
                                                      tmin_f, t1, ckey, cidx, t1, err)
                               : d32::near_next<false>(nbuf, bvh, tris32, tris64, o, d, inv, t_min, of, df, invf,
                                                       tmin_f, t1, ckey, cidx, t1, err);
            if (err)
                atomicOr(status, dmapdev::kStatusCapped);
            if (t < 0)
                break;
        } else if (opt.order == 1) {
            const float tmf = t1;
            double bk = 0.0;
            int bt = -1;
            for (int q = 0; q < n_tri; ++q) {
                const double key = d64::entry_key(tris64[q], o, d, inv, t_min);
                if (!d64::after_cursor(key, q, ckey, cidx) || !d64::before_best(key, q, bk, bt))
                    continue;
                float tt = tmf;
                if (!object_box(tris32[q], of, df, invf, __double2float_rd(t_min), tt))
                    continue;
                bk = key;
                bt = q;
                t1 = tt;
            }
            if (bt < 0)
                break;
            t = bt;
            ckey = bk;
            cidx = bt;
        } else if (!object_box(tris32[t], of, df, invf, __double2float_rd(t_min), t1)) {
            continue;
        }
        const TriDev32 &T = tris32[t];
        if (sp)
            ++st[DMAP_ST_TRI];
        d64::hit64 h;
        int hf = 0;
        bool got = false;
        // the callbacks' filter passes (displaced_geometry.cpp:53-106); no filter: one walk
        double t_lo = t_min;
        for (int pass = 0; pass < (opt.op_mask ? dmapdev::kFilterPasses : 1); ++pass) {
            double tm = t_max;
            if (!triangle_walk32(T, tris64[t], assets[T.asset], o, d, t_lo, tm, opt, h, hf, sp, far_bound(t1), status,
                                 capped))
                break;
            if (dmapdev::crossing_opaque(opt, tris64[t], t, h.bary.x, h.bary.y)) {
                got = true;
                break;
            }
            t_lo = h.t;
        }
        if (got) {
            best = h;
            best_flags = hf;
            best_tri = t;
            t_max = h.t;
            found = true;
            if (opt.mode == 1)
                break;
        }
    }
    store_hit<H, Fp>(hits, k, found, best, best_tri, (found ? best_flags : 0) | (capped ? DMAP_HIT_CAPPED : 0));
    if (stats)
        for (int q = 0; q < DMAP_ST_N; ++q)
            stats[DMAP_ST_N * k + q] = st[q];
}

// ---- wavefront schedule ---------------------------------------------------------

// A parked walk: the ray's position in ObjectIntersector's triangle loop and
// in DisplacedIntersector's walk, its current t_max and result, its
// candidate mask and the counters of the triangle in progress.
struct RayState
{
    double t_max;
    double ckey; // nearest-first order: the cursor (key, index) of the last triangle taken
    int cidx;
    int tri, root, best_tri, flags;
    int cl, ci, cj, el, ei, ej;
    int nah, lah;
    unsigned mask[kMaskWords];
    // scenes of more than 256 triangles: the buffered candidates, kept
    // across parks so a resumed ray does not walk the tree again
    d32::NearBuf buf;
};
// Up to kCollect consecutive leaves of one triangle's walk, in walk order.
// The walk goes on past a leaf with the t_max it has (it cannot know the
// leaf's result yet), so it may also reach leaves the reference prunes with
// the smaller t_max of a hit; the leaf kernel runs them with that smaller
// t_max, where they cannot report a nearer root than the one found, so the
// ray's hit is unchanged.
constexpr int kCollect = 4; // leaf slots of a job
// Leaves a ray collects before it parks (at most kCollect).
#ifndef DMAP_COLLECT
#define DMAP_COLLECT 4
#endif
static_assert(DMAP_COLLECT >= 1 && DMAP_COLLECT <= kCollect, "leaf slots");
struct LeafJob
{
    int ray, tri, n, pad;
    int i[kCollect], j[kCollect];
};
// RayState.flags
constexpr int kFoundInTri = 1; // a hit was taken in the triangle in progress
constexpr int kResumeHere = 2; // parked before visiting cell `cur` (or at the walk's end): resume without cell_next
constexpr int kCapped = 4;     // a triangle walk of this ray ran out of its cell-visit cap (DMAP_HIT_CAPPED)
constexpr int kRerun = 8;      // listed for the filter's schedule (it took a crossing the filter rejects)

// A filtered scene's wavefront query commits crossings as it finds them,
// without the filter's passes. A ray whose every committed crossing the
// filter accepts has the answer the passes give (each triangle's first pass
// finds the crossing it committed, with the same t_max); a ray that took a
// crossing the filter rejects is listed once, and the filter's own schedule
// (walk32_simple) answers it again after the query.
__device__ __forceinline__ void check_crossing(const dmapk::QueryOpts &opt, const TriDev &T, int tri,
                                               const d64::hit64 &h, int ray, int &flags, unsigned long long *ctr,
                                               int *rerun)
{
    if (!opt.op_mask || (flags & kRerun) || dmapdev::crossing_opaque(opt, T, tri, h.bary.x, h.bary.y))
        return;
    flags |= kRerun;
    rerun[atomicAdd(ctr + 4 * (dmapk::kMaxRounds + 1), 1ull)] = ray;
}

// Counter slots of one round: the walk's fetch counter, the leaf queue's
// length, the leaf kernel's fetch counter, the resume queue's length.
__device__ __forceinline__ unsigned long long *round_ctr(unsigned long long *c, int round, int k)
{
    return c + 4 * round + k;
}

// One lane's walk from its parked or fresh state to the next leaf (parked,
// job written) or to the end of the ray. Every lane of the warp executes one
// node test per step; lanes that finish take another ray.
// The walk rounds are compiled for DMAP_WALK_MIN_BLOCKS (mask) or
// DMAP_WALK_TREE_MIN_BLOCKS (tree) CTAs per SM; the last walk (INLINE_LEAF),
// which runs the few rays left with their leaves inline, for
// DMAP_DRAIN_MIN_BLOCKS, so that the leaf it calls is not squeezed into the
// rounds' register budget.
#ifndef DMAP_DRAIN_MIN_BLOCKS
#define DMAP_DRAIN_MIN_BLOCKS 2
#endif
template <bool ST, bool INLINE_LEAF, bool TREE, bool NEAR, typename R, typename H, typename Fp>
__global__ void __launch_bounds__(128, INLINE_LEAF ? DMAP_DRAIN_MIN_BLOCKS
                                                  : (TREE ? DMAP_WALK_TREE_MIN_BLOCKS : DMAP_WALK_MIN_BLOCKS))
    wave_walk(const TriDev32 *__restrict__ tris32, const TriDev *__restrict__ tris64, int n_tri,
              const AssetDev *__restrict__ assets, const R *__restrict__ rays, int64_t n, dmapk::QueryOpts opt,
              H *__restrict__ hits, int64_t *__restrict__ stats, RayState *__restrict__ states,
              const int *__restrict__ q_in, int round, LeafJob *__restrict__ q_leaf, unsigned long long *ctr,
              unsigned *status, int *__restrict__ rerun)
{
    enum : int { NEED = 0, TOP = 1, WALK = 2, DONE = 3 };
    const int lane = threadIdx.x & 31;
    // the candidates: scenes of up to 256 triangles take a mask of one bit
    // per triangle whose box the ray meets (built by the warp at the ray's
    // start), larger scenes (TREE) the triangle tree (bvh.cuh), in either
    // order; the launcher takes the mask only for up to 256 triangles, so its
    // loops are never compiled into the kernels of larger scenes
    constexpr bool use_mask = !TREE;
    const d32::BvhView bvh = {opt.bvh_nodes, opt.bvh_tri, opt.bvh_range, opt.bvh_n_nodes};
    // scenes of up to 256 triangles: their object boxes in shared memory
    // (outward FP32 for the box tests, FP64 for the nearest order's keys),
    // which every candidate test of the CTA reads
    constexpr int kStaged = TREE ? 1 : 32 * kMaskWords;
    __shared__ float s_box32[6 * kStaged];
    __shared__ double s_box64[6 * kStaged];
    if (!TREE) {
        for (int k = threadIdx.x; k < 6 * n_tri; k += blockDim.x) {
            const int t = k / 6, c = k - 6 * t;
            s_box32[k] = c < 3 ? tris32[t].box_lo[c] : tris32[t].box_hi[c - 3];
            s_box64[k] = c < 3 ? tris64[t].box_lo[c] : tris64[t].box_hi[c - 3];
        }
        __syncthreads();
    }
    // items of this round: every ray in round 0, else the resume queue
    unsigned long long count = round == 0 ? (unsigned long long)n : *round_ctr(ctr, round - 1, 3);
    if (round == 0 && opt.n_dev && (unsigned long long)*opt.n_dev < count)
        count = *opt.n_dev < 0 ? 0ull : (unsigned long long)*opt.n_dev;
    unsigned long long *fetch = round_ctr(ctr, round, 0);
    int phase = NEED;
    int ray = 0;
    double o[3], d[3], t_min = 0.0, t_max = 0.0;
    float of[3], df[3], invf[3], tmin_f = 0.0f;
    int tri = 0, best_tri = -1, root = 0, si = 0, sj = 0, nah = 0, lah = 0, flags = 0, guard = 0;
    double ckey = -INFINITY;
    int cidx = -1;
    // the triangle tree (TREE): the lane's buffered candidates, refilled
    // from the ray's cursor for a fresh ray, kept in the ray's state across
    // parks
    d32::NearBuf nbuf;
    nbuf.n = -1;
    nbuf.pos = 0;
    Ray32 r;
    Cell32 cur = {0, 0, 0}, end = {0, 0, 0};
    unsigned mask[kMaskWords];
#pragma unroll
    for (int w = 0; w < kMaskWords; ++w)
        mask[w] = 0u;
    int64_t stl[DMAP_ST_N];
    int nl = 0, li0 = 0, lj0 = 0, li1 = 0, lj1 = 0, li2 = 0, lj2 = 0, li3 = 0, lj3 = 0; // collected leaves
    int since = 0; // node tests since the first collected leaf

    auto flush_stats = [&]() {
        if (ST)
            for (int q = 0; q < DMAP_ST_N; ++q)
                stats[DMAP_ST_N * (int64_t)ray + q] += stl[q];
    };
    // Park the ray: its collected leaves become one job, its walk state
    // waits for the next round (here: resume at `cur` itself, which is the
    // next cell to visit or the end of the triangle's walk; otherwise `cur`
    // is the last collected leaf and the walk resumes past it).
    auto park = [&](bool here) {
        RayState &s = states[ray];
        s.t_max = t_max;
        s.ckey = ckey;
        s.cidx = cidx;
        s.tri = tri;
        s.root = root;
        s.best_tri = best_tri;
        s.flags = here ? (flags | kResumeHere) : (flags & ~kResumeHere);
        s.cl = cur.level, s.ci = cur.i, s.cj = cur.j;
        s.el = end.level, s.ei = end.i, s.ej = end.j;
        s.nah = nah;
        s.lah = lah;
#pragma unroll
        for (int w = 0; w < kMaskWords; ++w)
            s.mask[w] = mask[w];
        if (TREE)
            s.buf = nbuf;
        unsigned long long slot = atomicAdd(round_ctr(ctr, round, 1), 1ull);
        LeafJob job;
        job.ray = ray;
        job.tri = tri;
        job.n = nl;
        job.pad = 0;
        job.i[0] = li0, job.j[0] = lj0, job.i[1] = li1, job.j[1] = lj1;
        job.i[2] = li2, job.j[2] = lj2, job.i[3] = li3, job.j[3] = lj3;
        q_leaf[slot] = job;
        nl = 0;
        since = 0;
        flush_stats();
        phase = NEED;
    };

    for (;;) {
        // 1. lanes without work take the next items, one atomic per warp
        unsigned need = __ballot_sync(FULL, phase == NEED);
        bool fresh = false;
        if (need) {
            int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader)
                base = atomicAdd(fetch, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (phase == NEED) {
                unsigned long long item = base + (unsigned long long)__popc(need & ((1u << lane) - 1u));
                if (item >= count) {
                    phase = DONE;
                } else {
                    ray = round == 0 ? (int)item : q_in[item];
                    load_ray(rays, ray, o, d, t_min, t_max);
                    nbuf.n = -1;
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        of[a] = (float)o[a];
                        df[a] = (float)d[a];
                        invf[a] = df[a] != 0.0f ? __frcp_rn(df[a]) : 0.0f;
                    }
                    tmin_f = __double2float_rd(t_min);
                    if (ST)
                        for (int q = 0; q < DMAP_ST_N; ++q)
                            stl[q] = 0;
                    if (round == 0) {
                        tri = 0;
                        ckey = -INFINITY;
                        cidx = -1;
                        best_tri = -1;
                        flags = 0;
                        nah = lah = 0;
                        fresh = true;
                        phase = TOP;
                    } else {
                        const RayState &s = states[ray];
                        t_max = s.t_max;
                        ckey = s.ckey;
                        cidx = s.cidx;
                        tri = s.tri;
                        root = s.root;
                        best_tri = s.best_tri;
                        flags = s.flags;
                        nah = s.nah;
                        lah = s.lah;
#pragma unroll
                        for (int w = 0; w < kMaskWords; ++w)
                            mask[w] = s.mask[w];
                        if (TREE)
                            nbuf = s.buf;
                        // back into the walk just after the leaf (displaced_intersector.cpp:229)
                        const TriDev32 &T = tris32[tri];
                        float t1 = __double2float_ru(t_max);
                        object_box(T, of, df, invf, tmin_f, t1);
                        tangent_ray(T, o, d, far_bound(fmaxf(t1, tmin_f)), r);
                        si = r.dx < 0.0f;
                        sj = r.dy < 0.0f;
                        cur = {s.cl, s.ci, s.cj};
                        end = {s.el, s.ei, s.ej};
                        if (!(flags & kResumeHere))
                            cell_next(cur, si, sj, T.root_level); // past the last leaf (displaced_intersector.cpp:229)
                        flags &= ~kResumeHere;
                        guard = 0;
                        nl = 0;
                        phase = WALK;
                    }
                }
            }
        }
        // round 0: the warp finds the fresh rays' candidate triangles together, 32 boxes per ballot
        if (use_mask) {
            unsigned todo = __ballot_sync(FULL, fresh);
            while (todo) {
                int src = __ffs(todo) - 1;
                todo &= todo - 1;
                float so[3], sd[3], sv[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    so[a] = __shfl_sync(FULL, of[a], src);
                    sd[a] = __shfl_sync(FULL, df[a], src);
                    sv[a] = __shfl_sync(FULL, invf[a], src);
                }
                float s_tmin = __shfl_sync(FULL, tmin_f, src);
                float s_tmax = __shfl_sync(FULL, __double2float_ru(t_max), src);
#pragma unroll 1
                for (int w = 0; w < ((n_tri + 31) >> 5); ++w) {
                    int t = 32 * w + lane;
                    float t1 = s_tmax;
                    bool pass = t < n_tri && box_pass(s_box32 + 6 * t, s_box32 + 6 * t + 3, so, sd, sv, s_tmin, t1);
                    unsigned bits = __ballot_sync(FULL, pass);
                    if (lane == src) {
#pragma unroll
                        for (int q = 0; q < kMaskWords; ++q)
                            mask[q] = q == w ? bits : mask[q];
                    }
                }
            }
        }
        if (__all_sync(FULL, phase == DONE))
            break;

        // 2. the next triangle whose object box the ray meets (intersect_flat's loop)
        if (phase == TOP) {
            float t1 = 0.0f;
            bool hit_box = false;
            if (NEAR) {
                // nearest box entry first: the smallest (key, index) past the
                // cursor among the candidates the ray still reaches
                double inv[3];
                d64::ray_inverse(d, inv);
                double bk = 0.0;
                int bt = -1;
                const float tmf = __double2float_ru(t_max);
                if (TREE) {
                    bool err = false;
                    bt = d32::near_next<true>(nbuf, bvh, tris32, tris64, o, d, inv, t_min, of, df, invf, tmin_f, tmf,
                                        ckey, cidx, t1, err);
                    bk = ckey;
                    if (err)
                        atomicOr(status, dmapdev::kStatusCapped);
                } else {
                    // the best (key, index) past the cursor among the bits
                    // of the ray's mask (boxes met at the ray's start), each
                    // box re-tested with the current t_max first; a bit whose
                    // box no longer passes, or whose key is not past the
                    // cursor, is cleared for good (t_max only shrinks, the
                    // cursor only advances), so later picks scan fewer
                    const int words = (n_tri + 31) >> 5;
#pragma unroll 1
                    for (int w = 0; w < words; ++w) {
                        unsigned bits = mask[0];
#pragma unroll
                        for (int q = 1; q < kMaskWords; ++q)
                            bits = w == q ? mask[q] : bits;
                        unsigned drop = 0u;
                        while (bits) {
                            const int b = __ffs(bits) - 1;
                            bits &= bits - 1;
                            const int t = 32 * w + b;
                            float e = tmin_f, tt = tmf;
                            if (!box_range(s_box32 + 6 * t, s_box32 + 6 * t + 3, of, df, invf, e, tt)) {
                                drop |= 1u << b;
                                continue;
                            }
                            if (bt >= 0 && (double)e > bk)
                                continue; // its key (at least e) is past the best
                            const double key = d64::entry_key(s_box64 + 6 * t, s_box64 + 6 * t + 3, o, d, inv, t_min);
                            if (!d64::after_cursor(key, t, ckey, cidx)) {
                                drop |= 1u << b;
                                continue;
                            }
                            if (!d64::before_best(key, t, bk, bt))
                                continue;
                            bk = key;
                            bt = t;
                            t1 = tt;
                        }
                        if (drop) {
#pragma unroll
                            for (int q = 0; q < kMaskWords; ++q)
                                mask[q] = w == q ? (mask[q] & ~drop) : mask[q];
                        }
                    }
                }
                if (bt >= 0) {
                    tri = bt;
                    ckey = bk;
                    cidx = bt;
                    hit_box = true;
                } else {
                    tri = n_tri;
                }
            } else if (TREE) {
                // index order: the smallest index from tri on whose box the
                // ray still meets
                bool err = false;
                double ck = tri - 1;
                int ci = tri - 1;
                const int t = d32::near_next<false>(nbuf, bvh, tris32, tris64, o, d, nullptr, t_min, of, df, invf,
                                                    tmin_f, __double2float_ru(t_max), ck, ci, t1, err);
                if (err)
                    atomicOr(status, dmapdev::kStatusCapped);
                if (t >= 0) {
                    tri = t;
                    hit_box = true;
                } else {
                    tri = n_tri;
                }
            } else {
                while (tri < n_tri) {
                    int w = tri >> 5;
                    unsigned bits = mask[0];
#pragma unroll
                    for (int q = 1; q < kMaskWords; ++q)
                        bits = w == q ? mask[q] : bits;
                    bits &= ~0u << (tri & 31);
                    if (!bits) {
                        tri = (w + 1) << 5;
                        continue;
                    }
                    tri = (w << 5) + __ffs(bits) - 1;
                    t1 = __double2float_ru(t_max); // the candidate again, with the current t_max
                    if (tri < n_tri && box_pass(s_box32 + 6 * tri, s_box32 + 6 * tri + 3, of, df, invf, tmin_f, t1)) {
                        hit_box = true;
                        break;
                    }
                    ++tri;
                }
            }
            if (!hit_box) {
                if (best_tri < 0) {
                    d64::hit64 none;
                    store_hit<H, Fp>(hits, ray, false, none, -1, (flags & kCapped) ? DMAP_HIT_CAPPED : 0);
                } else if (flags & kCapped) {
                    hits[ray].flags |= DMAP_HIT_CAPPED; // the stored hit is final: this lane owns the ray
                }
                flush_stats();
                phase = NEED;
            } else {
                const TriDev32 &T = tris32[tri];
                tangent_ray(T, o, d, far_bound(t1), r);
                si = r.dx < 0.0f;
                sj = r.dy < 0.0f;
                root = 0;
                cur = {T.root_level, T.roots_i[0], T.roots_j[0]};
                end = cur;
                cell_next(end, si, sj, T.root_level);
                guard = 0;
                flags &= ~kFoundInTri;
                nah = lah = 0;
                if (ST)
                    ++stl[DMAP_ST_TRI];
                phase = WALK;
            }
        }

        // 3a. advance to the next cell inside the domain (cheap, divergent)
        bool cand = false;
        if (phase == WALK) {
            const TriDev32 &T = tris32[tri];
            const int log2n = __ffs(assets[T.asset].n_leaf) - 1;
            for (;;) {
                if (cur.level == end.level && cur.i == end.i && cur.j == end.j) {
                    if (root + 1 < T.n_roots) {
                        ++root;
                        cur = {T.root_level, T.roots_i[root], T.roots_j[root]};
                        end = cur;
                        cell_next(end, si, sj, T.root_level);
                        continue;
                    }
                    if (!INLINE_LEAF && nl > 0) {
                        // the collected leaves decide this triangle's t_max before the next one
                        park(true);
                        break;
                    }
                    if (ST && (flags & kFoundInTri)) {
                        stl[DMAP_ST_NAH] += nah;
                        stl[DMAP_ST_LAH] += lah;
                    }
                    ++tri;
                    phase = TOP;
                    break;
                }
                if (++guard > opt.guard_cap) { // a finite tree: the cap guards corrupt records
                    atomicOr(status, dmapdev::kStatusCapped);
                    flags |= kCapped;
                    ++tri;
                    phase = TOP;
                    break;
                }
                float w = pow2f(cur.level - log2n);
                if (!square_meets_domain(T, ((float)cur.i + 0.5f) * w, ((float)cur.j + 0.5f) * w, 0.5f * w)) {
                    cell_next(cur, si, sj, T.root_level);
                    continue;
                }
                cand = true;
                break;
            }
        }
        __syncwarp();

        // 3b. one node test for every lane with a candidate, all together
        if (cand) {
            const TriDev32 &T = tris32[tri];
            if (ST) {
                ++stl[DMAP_ST_NODE];
                ++nah;
            }
            if (!node_test32(T, assets[T.asset], r, cur.level, cur.i, cur.j, tmin_f, __double2float_ru(t_max),
                             opt.bound, opt.slab_max_level)) {
                cell_next(cur, si, sj, T.root_level);
            } else if (cur.level > 0) {
                --cur.level;
                cur.i = 2 * cur.i + si;
                cur.j = 2 * cur.j + sj;
            } else {
                if (ST) {
                    ++stl[DMAP_ST_LEAF];
                    ++lah;
                }
                if (INLINE_LEAF) {
                    // the last round: the few remaining rays finish here
                    d64::hit64 lh;
                    int lf = 0;
                    if (leaf_cell(T, tris64[tri], assets[T.asset], o, d, t_min, t_max, cur.i, cur.j, lh, lf,
                                  ST ? stl : nullptr, opt) &&
                        lh.t < t_max) {
                        t_max = lh.t;
                        best_tri = tri;
                        flags |= kFoundInTri;
                        nah = lah = 0;
                        store_hit<H, Fp>(hits, ray, true, lh, tri, lf | ((flags & kCapped) ? DMAP_HIT_CAPPED : 0));
                        check_crossing(opt, tris64[tri], tri, lh, ray, flags, ctr, rerun);
                        if (opt.mode == 1) {
                            flush_stats();
                            phase = NEED;
                        }
                    }
                    if (phase == WALK)
                        cell_next(cur, si, sj, T.root_level);
                } else {
                    // collect the leaf; park once kCollect are held
                    li0 = nl == 0 ? cur.i : li0;
                    lj0 = nl == 0 ? cur.j : lj0;
                    li1 = nl == 1 ? cur.i : li1;
                    lj1 = nl == 1 ? cur.j : lj1;
                    li2 = nl == 2 ? cur.i : li2;
                    lj2 = nl == 2 ? cur.j : lj2;
                    li3 = nl == 3 ? cur.i : li3;
                    lj3 = nl == 3 ? cur.j : lj3;
                    if (++nl == DMAP_COLLECT)
                        park(false);
                    else
                        cell_next(cur, si, sj, T.root_level);
                }
            }
        }
        // a ray holding collected leaves walks on with the t_max it had
        // before them; after DMAP_STALE_CAP such node tests it parks (at the
        // next cell to visit) so that the leaves can shrink t_max first
        if (!INLINE_LEAF && phase == WALK && nl > 0 && ++since > DMAP_STALE_CAP)
            park(true);
        __syncwarp();
    }
}

// The leaf cells of a round's jobs through the reference's own node test in
// double (node_bounds.cpp:83-211 at level 0, the node computed from the
// grid): the FP32 walk, widened by its roundings, reaches more leaf cells
// than the FP64 walk, and a cell the FP64 walk rejects has no leaf there.
// The ray's t_max is the one it parked with; earlier leaves of the same job
// can only shrink it, so a cell kept here may still be rejected by the FP64
// walk at that point, and its search then finds nothing the reference
// would not. Cells are compacted in walk order; a job may end up empty.
// Kept apart from the leaf kernel so that kernel's code stays small.
template <typename R>
__global__ void __launch_bounds__(128)
    wave_filter(const TriDev *__restrict__ tris64, const AssetDev *__restrict__ assets, const R *__restrict__ rays,
                dmapk::QueryOpts opt, const RayState *__restrict__ states, LeafJob *__restrict__ q_leaf, int round,
                const unsigned long long *ctr)
{
    const unsigned long long count = *round_ctr(const_cast<unsigned long long *>(ctr), round, 1);
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < count;
         k += (unsigned long long)gridDim.x * blockDim.x) {
        LeafJob job = q_leaf[k];
        double o[3], d[3], t_min, t_max;
        load_ray(rays, job.ray, o, d, t_min, t_max);
        t_max = states[job.ray].t_max;
        const TriDev &T = tris64[job.tri];
        const AssetDev &g = assets[T.asset];
        if (T.inst) {
            double oo[3], od[3];
            dmapdev::object_ray(opt.inst_xf + dmapdev::kInstDoubles * (T.inst - 1), o, d, oo, od);
            for (int a = 0; a < 3; ++a) {
                o[a] = oo[a];
                d[a] = od[a];
            }
        }
        d64::tray r = d64::tangent_ray64(T, d64::V3(o[0], o[1], o[2]), d64::V3(d[0], d[1], d[2]), t_min, t_max);
        int m = 0;
#pragma unroll 1
        for (int q = 0; q < job.n; ++q) {
            if (d64::leaf_cell_admitted(T, g, r, job.i[q], job.j[q], opt)) {
                job.i[m] = job.i[q];
                job.j[m] = job.j[q];
                ++m;
            }
        }
        if (m != job.n) {
            job.n = m;
            q_leaf[k] = job;
        }
    }
}

// The parked leaves of a round (the certified leaf, d64::intersect_newton,
// displaced_intersector.cpp:239-323). Each lane holds one job at a time and
// takes the next one as soon as its own is done, so a warp's lanes stay busy
// however long their leaves run. A step of the loop runs, for the lanes that
// need it: the leaf setup, one sub-square expansion (four bounds, the sort,
// the push) or one Newton run, with the warp reconverged between blocks.
// Each lane's search is intersect_newton's, in the same order with the same
// arithmetic, so each ray's result equals it bit for bit. A ray whose walk
// has cells left goes back to the resume queue.
template <bool ST, typename R, typename H, typename Fp>
__global__ void __launch_bounds__(128, DMAP_LEAF_MIN_BLOCKS)
    wave_leaf(const TriDev *__restrict__ tris64, const AssetDev *__restrict__ assets, const R *__restrict__ rays,
              dmapk::QueryOpts opt, H *__restrict__ hits, int64_t *__restrict__ stats, RayState *__restrict__ states,
              const LeafJob *__restrict__ q_leaf, int round, int *__restrict__ q_out, unsigned long long *ctr,
              int *__restrict__ rerun)
{
    using namespace d64;
    constexpr int kDepth = 5; // subdivision_depth
    enum : int { NEED = 0, SETUP = 1, SEARCH = 2, DONE = 3 };
    const int lane = threadIdx.x & 31;
    const unsigned long long count = *round_ctr(ctr, round, 1);
    unsigned long long *fetch = round_ctr(ctr, round, 2);
    int phase = NEED;
    unsigned long long item = 0;
    int ray = 0, tri = 0, n_leaves = 0, q = 0, li = 0, lj = 0, sp = 0;
    bool first = false, answered = false;
    double t_min = 0.0, t_max = 0.0;
    v3 O = V3(0.0, 0.0, 0.0), D = O;
    leafbound L;
    leafent stack[4 * kDepth + 4];
    int64_t subs = 0, iters = 0;

    for (;;) {
        // lanes without a job take the next ones, one atomic per warp
        unsigned need = __ballot_sync(FULL, phase == NEED);
        if (need) {
            int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader)
                base = atomicAdd(fetch, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (phase == NEED) {
                item = base + (unsigned long long)__popc(need & ((1u << lane) - 1u));
                if (item >= count) {
                    phase = DONE;
                } else {
                    const LeafJob &J = q_leaf[item];
                    ray = J.ray;
                    tri = J.tri;
                    n_leaves = J.n;
                    q = 0;
                    if (n_leaves == 0) {
                        // the filter rejected every cell of the job: the walk goes on
                        unsigned long long slot = atomicAdd(round_ctr(ctr, round, 3), 1ull);
                        q_out[slot] = ray;
                    } else {
                        double o[3], d[3];
                        load_ray(rays, ray, o, d, t_min, t_max);
                        if (tris64[tri].inst) {
                            double oo[3], od[3];
                            dmapdev::object_ray(opt.inst_xf + dmapdev::kInstDoubles * (tris64[tri].inst - 1), o, d,
                                                oo, od);
                            for (int a = 0; a < 3; ++a) {
                                o[a] = oo[a];
                                d[a] = od[a];
                            }
                        }
                        O = V3(o[0], o[1], o[2]);
                        D = V3(d[0], d[1], d[2]);
                        t_max = states[ray].t_max;
                        answered = false;
                        subs = iters = 0;
                        phase = SETUP;
                    }
                }
            }
        }
        if (__all_sync(FULL, phase == DONE))
            break;
        const TriDev &T = tris64[tri];
        const AssetDev &g = assets[T.asset];
        // leaf q of the job (a cell wave_filter kept): the texel's corners,
        // its normal form and the ray's plane basis (:239-264)
        if (phase == SETUP) {
            li = q_leaf[item].i[q];
            lj = q_leaf[item].j[q];
            sp = 0;
            phase = SEARCH;
            L.w = cell_width(g, 0);
            L.lo = {li * L.w, lj * L.w};
            L.h00 = grid_h(g, L.lo.x, L.lo.y);
            L.h10 = grid_h(g, L.lo.x + L.w, L.lo.y);
            L.h01 = grid_h(g, L.lo.x, L.lo.y + L.w);
            L.h11 = grid_h(g, L.lo.x + L.w, L.lo.y + L.w);
            v2 c = add2(L.lo, V2(0.5 * L.w, 0.5 * L.w));
            double hw = 0.5 * L.w;
            L.N_hat = AF3(add3(add3(L3(T.m0), mul3(c.x, L3(T.Mu))), mul3(c.y, L3(T.Mv))), mul3(hw, L3(T.Mu)),
                          mul3(hw, L3(T.Mv)));
            normalize(L.N_hat);
            L.o = O;
            L.d_len = norm3(D);
            L.dn = div3(D, L.d_len);
            plane_basis(L.dn, L.d1, L.d2);
            stack[sp++] = {0.5, 0.5, -INFINITY, 0};
            first = true;
        }
        // the next live entry of the search (a pop is a call of search_leaf;
        // an entry at or beyond t_max is the sorted loop's break)
        bool expand = false, newton = false;
        leafent e = {0.0, 0.0, 0.0, 0};
        if (phase == SEARCH) {
            while (sp > 0) {
                e = stack[--sp];
                if (first || e.t_lo < t_max) {
                    first = false;
                    newton = e.depth == kDepth;
                    expand = !newton;
                    break;
                }
            }
            if (!expand && !newton) {
                // the leaf is done; the next of the job, or the job is done
                if (++q < n_leaves && !answered) {
                    phase = SETUP;
                } else {
                    if (ST) {
                        stats[DMAP_ST_N * (int64_t)ray + DMAP_ST_SUB] += subs;
                        stats[DMAP_ST_N * (int64_t)ray + DMAP_ST_NEWTON] += iters;
                    }
                    if (!answered) {
                        unsigned long long slot = atomicAdd(round_ctr(ctr, round, 3), 1ull);
                        q_out[slot] = ray;
                    }
                    phase = NEED;
                }
            }
        }
        __syncwarp();
        if (expand) {
            double r = 0.5 * ldexp(0.5, -e.depth);
            leafent ch[4];
            int n = 0;
#pragma unroll 1
            for (int k = 0; k < 4; ++k) {
                double ca = e.a + ((k & 1) ? r : -r), cb = e.b + ((k & 2) ? r : -r), t_lo;
                ++subs;
                if (sub_square_bound(T, L, ca, cb, r, t_min, t_max, t_lo))
                    ch[n++] = {ca, cb, t_lo, e.depth + 1};
            }
            for (int p = 1; p < n; ++p)
                for (int k = p; k > 0 && ch[k].t_lo < ch[k - 1].t_lo; --k) {
                    leafent x = ch[k];
                    ch[k] = ch[k - 1];
                    ch[k - 1] = x;
                }
            for (int k = n - 1; k >= 0; --k)
                stack[sp++] = ch[k];
        }
        __syncwarp();
        if (newton) {
            hit64 h;
            if (newton_from(T, g, O, D, t_min, t_max, li, lj, add2(L.lo, mul2(L.w, V2(e.a, e.b))), h, iters)) {
                // a nearer root of this leaf (each later one is nearer still)
                t_max = h.t;
                RayState &s = states[ray];
                s.t_max = h.t;
                s.best_tri = tri;
                s.flags |= kFoundInTri;
                s.nah = s.lah = 0;
                if (tris64[tri].inst)
                    dmapdev::world_normal(opt.inst_xf + dmapdev::kInstDoubles * (tris64[tri].inst - 1), h.ng);
                store_hit<H, Fp>(hits, ray, true, h, tri,
                                 DMAP_HIT_FP64_LEAF | ((s.flags & kCapped) ? DMAP_HIT_CAPPED : 0));
                check_crossing(opt, tris64[tri], tri, h, ray, s.flags, ctr, rerun);
                if (opt.mode == 1) { // occlusion: any hit answers the query
                    answered = true;
                    sp = 0;
                }
            }
        }
        __syncwarp();
    }
}

// The parked leaves of a round with the FP32 certified leaf (leaf32.cuh):
// wave_leaf's schedule (one job per lane, a lane takes the next job when its
// own is done, one search step per loop iteration) over the FP32 leaf state.
#ifndef DMAP_LEAF32_MIN_BLOCKS
#define DMAP_LEAF32_MIN_BLOCKS 1
#endif
template <bool ST, typename R, typename H, typename Fp>
__global__ void __launch_bounds__(128, DMAP_LEAF32_MIN_BLOCKS)
    wave_leaf32(const TriDev32 *__restrict__ tris32, const TriDev *__restrict__ tris64,
                const AssetDev *__restrict__ assets, const R *__restrict__ rays, dmapk::QueryOpts opt,
                H *__restrict__ hits, int64_t *__restrict__ stats, RayState *__restrict__ states,
                const LeafJob *__restrict__ q_leaf, int round, int *__restrict__ q_out, unsigned long long *ctr,
                int *__restrict__ rerun)
{
    using namespace d64;
    constexpr int kDepth = 5; // subdivision_depth
    enum : int { NEED = 0, SETUP = 1, SEARCH = 2, DONE = 3 };
    const int lane = threadIdx.x & 31;
    const unsigned long long count = *round_ctr(ctr, round, 1);
    unsigned long long *fetch = round_ctr(ctr, round, 2);
    int phase = NEED;
    unsigned long long item = 0;
    int ray = 0, tri = 0, n_leaves = 0, q = 0, li = 0, lj = 0, sp = 0;
    bool first = false, answered = false;
    double t_min = 0.0, t_max = 0.0;
    v3 O = V3(0.0, 0.0, 0.0), D = O;
    l32::Leaf32 L;
    l32::Ent32 stack[4 * kDepth + 4];
    int64_t subs = 0, iters = 0;

    for (;;) {
        unsigned need = __ballot_sync(FULL, phase == NEED);
        if (need) {
            int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader)
                base = atomicAdd(fetch, (unsigned long long)__popc(need));
            base = __shfl_sync(FULL, base, leader);
            if (phase == NEED) {
                item = base + (unsigned long long)__popc(need & ((1u << lane) - 1u));
                if (item >= count) {
                    phase = DONE;
                } else {
                    const LeafJob &J = q_leaf[item];
                    ray = J.ray;
                    tri = J.tri;
                    n_leaves = J.n;
                    q = 0;
                    if (n_leaves == 0) {
                        unsigned long long slot = atomicAdd(round_ctr(ctr, round, 3), 1ull);
                        q_out[slot] = ray;
                    } else {
                        double o[3], d[3];
                        load_ray(rays, ray, o, d, t_min, t_max);
                        if (tris64[tri].inst) {
                            double oo[3], od[3];
                            dmapdev::object_ray(opt.inst_xf + dmapdev::kInstDoubles * (tris64[tri].inst - 1), o, d,
                                                oo, od);
                            for (int a = 0; a < 3; ++a) {
                                o[a] = oo[a];
                                d[a] = od[a];
                            }
                        }
                        O = V3(o[0], o[1], o[2]);
                        D = V3(d[0], d[1], d[2]);
                        t_max = states[ray].t_max;
                        answered = false;
                        subs = iters = 0;
                        phase = SETUP;
                    }
                }
            }
        }
        if (__all_sync(FULL, phase == DONE))
            break;
        const TriDev &T = tris64[tri];
        const AssetDev &g = assets[T.asset];
        if (phase == SETUP) {
            li = q_leaf[item].i[q];
            lj = q_leaf[item].j[q];
            l32::leaf_setup32(T, g, O, D, li, lj, L);
            sp = 0;
            stack[sp++] = {0.5f, 0.5f, -INFINITY, 0};
            first = true;
            phase = SEARCH;
        }
        bool expand = false, newton = false;
        l32::Ent32 e = {0.0f, 0.0f, 0.0f, 0};
        if (phase == SEARCH) {
            while (sp > 0) {
                e = stack[--sp];
                if (first || (double)e.t_lo < t_max) {
                    first = false;
                    newton = e.depth == kDepth;
                    expand = !newton;
                    break;
                }
            }
            if (!expand && !newton) {
                if (++q < n_leaves && !answered) {
                    phase = SETUP;
                } else {
                    if (ST) {
                        stats[DMAP_ST_N * (int64_t)ray + DMAP_ST_SUB] += subs;
                        stats[DMAP_ST_N * (int64_t)ray + DMAP_ST_NEWTON] += iters;
                    }
                    if (!answered) {
                        unsigned long long slot = atomicAdd(round_ctr(ctr, round, 3), 1ull);
                        q_out[slot] = ray;
                    }
                    phase = NEED;
                }
            }
        }
        __syncwarp();
        if (expand) {
            const TriDev32 &T32 = tris32[tri];
            float r = __int_as_float((125 - e.depth) << 23); // half of the entry's rho = 0.5 * 2^-depth
            l32::Ent32 ch[4];
            int n = 0;
#pragma unroll 1
            for (int k = 0; k < 4; ++k) {
                float ca = e.a + ((k & 1) ? r : -r), cb = e.b + ((k & 2) ? r : -r), tl;
                ++subs;
                if (l32::sub_square_bound32(T32, L, ca, cb, r, t_min, t_max, tl))
                    ch[n++] = {ca, cb, tl, e.depth + 1};
            }
            for (int p = 1; p < n; ++p)
                for (int k = p; k > 0 && ch[k].t_lo < ch[k - 1].t_lo; --k) {
                    l32::Ent32 x = ch[k];
                    ch[k] = ch[k - 1];
                    ch[k - 1] = x;
                }
            for (int k = n - 1; k >= 0; --k)
                stack[sp++] = ch[k];
        }
        __syncwarp();
        if (newton) {
            l32::Root32 root;
            hit64 h;
            int fl = 0;
            if (l32::newton32(T, L, e.a, e.b, root, iters) &&
                l32::accept_root(T, g, L.lo_s, L.lo_t, L.w, L.Q3, L.inv_dlen, O, D, t_min, t_max, li, lj, root,
                                 opt.polish_cond, h, fl, iters)) {
                t_max = h.t;
                RayState &s = states[ray];
                s.t_max = h.t;
                s.best_tri = tri;
                s.flags |= kFoundInTri;
                s.nah = s.lah = 0;
                if (tris64[tri].inst)
                    dmapdev::world_normal(opt.inst_xf + dmapdev::kInstDoubles * (tris64[tri].inst - 1), h.ng);
                store_hit<H, Fp>(hits, ray, true, h, tri, fl | ((s.flags & kCapped) ? DMAP_HIT_CAPPED : 0));
                check_crossing(opt, tris64[tri], tri, h, ray, s.flags, ctr, rerun);
                if (opt.mode == 1) {
                    answered = true;
                    sp = 0;
                }
            }
        }
        __syncwarp();
    }
}

int sm_count()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return sms;
}

} // namespace
