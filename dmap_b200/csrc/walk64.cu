// The FP64 query path: one thread per ray, every triangle of the scene in
// order behind its AABB (ObjectIntersector::intersect_flat,
// displaced_intersector.cpp:778-799), each walked with TFDM's stackless
// quadtree walk and the certified Newton leaf
// (displaced_intersector.cpp:175-388, node_bounds.cpp:83-211), in double
// with the reference's operation order (compiled with -fmad=false). This is
// the device oracle and the plain one-launch-per-request comparator; its
// results equal the reference's CPU build bit for bit.
#include "device_types.cuh"
#include "f64_math.cuh"
#include "f64_leaf.cuh"
#include "launch.h"

namespace
{
using namespace d64;
using dmapdev::AssetDev;
using dmapdev::TriDev;

struct nodebound { int level; node n; v2 centre; af3 m; box3 box; };

__device__ void node_bound(nodebound &nb, const TriDev &T, const AssetDev &a, int level, int64_t i, int64_t j)
{
    // node_bounds.cpp:83-109
    nb.level = level;
    nb.n = pyramid_node(a, level, i, j);
    double w = cell_width(a, level);
    nb.centre = {(i + 0.5) * w, (j + 0.5) * w};
    v2 tri_lo = L2(T.lo), tri_hi = L2(T.hi);
    v2 rect_lo = max2(V2(i * w, j * w), tri_lo);
    v2 rect_hi = min2(V2((i + 1) * w, (j + 1) * w), tri_hi);
    v2 c = mul2(0.5, add2(rect_lo, rect_hi));
    v2 hh = mul2(0.5, sub2(rect_hi, rect_lo));
    v2 half = {dmax(hh.x, 0.0), dmax(hh.y, 0.0)};
    af3 N = AF3(add3(add3(L3(T.m0), mul3(c.x, L3(T.Mu))), mul3(c.y, L3(T.Mv))), mul3(half.x, L3(T.Mu)),
                mul3(half.y, L3(T.Mv)));
    normalize(N);
    nb.m = matmul(T.A, N);
    af h = AF(0.5 * (nb.n.h_min + nb.n.h_max), 0.0, 0.0, 0.5 * (nb.n.h_max - nb.n.h_min));
    af3 p = AF3(V3(c.x, c.y, 0.0), V3(half.x, 0.0, 0.0), V3(0.0, half.y, 0.0));
    nb.box = hull(add(p, scale_form(h, nb.m)));
}

__device__ __forceinline__ ivl IV(double lo, double hi) { return {lo, hi}; }
__device__ __forceinline__ ivl iv_add(ivl a, ivl b) { return {a.lo + b.lo, a.hi + b.hi}; }
__device__ __forceinline__ ivl iv_scale(double s, ivl a) { return s >= 0.0 ? IV(s * a.lo, s * a.hi) : IV(s * a.hi, s * a.lo); }

struct tray { v3 o, d; double t_min, t_max; };

__device__ __forceinline__ bool box_interval(const nodebound &nb, const tray &r, double &t0, double &t1)
{
    t0 = r.t_min;
    t1 = r.t_max;
    return box_clip(nb.box, r.o, r.d, t0, t1);
}

__device__ bool slab_interval(const nodebound &nb, const tray &r, double &t0, double &t1) // node_bounds.cpp:137-179
{
    box3 column = nb.box;
    column.lo.z = -INFINITY;
    column.hi.z = INFINITY;
    t0 = r.t_min;
    t1 = r.t_max;
    if (!box_clip(column, r.o, r.d, t0, t1))
        return false;
    v3 anchor = add3(r.o, mul3(t0, r.d));
    double span = t1 - t0;
    // slab_form, node_bounds.cpp:111-122
    const node &n = nb.n;
    ivl mx = interval(nb.m.x), my = interval(nb.m.y), mz = interval(nb.m.z);
    ivl A = iv_add(iv_add(IV(1.0, 1.0), iv_scale(n.gu, mx)), iv_scale(n.gv, my));
    ivl B = iv_scale(-n.gu, mz);
    ivl C = iv_scale(-n.gv, mz);
    ivl D = iv_scale(-((n.h0 - n.gu * nb.centre.x) - n.gv * nb.centre.y), mz);
    double R = n.r * dmax(fabs(mz.lo), fabs(mz.hi));
    ivl F0 = iv_add(iv_add(iv_add(iv_scale(anchor.z, A), iv_scale(anchor.x, B)), iv_scale(anchor.y, C)), D);
    ivl F1 = iv_add(iv_add(iv_scale(r.d.z, A), iv_scale(r.d.x, B)), iv_scale(r.d.y, C));
    double s0 = 0.0, s1 = span;
    if (F1.lo > 0.0)
        s1 = dmin(s1, (R - F0.lo) / F1.lo);
    else if (F1.lo < 0.0)
        s0 = dmax(s0, (R - F0.lo) / F1.lo);
    else if (F0.lo > R)
        return false;
    if (F1.hi > 0.0)
        s0 = dmax(s0, (-R - F0.hi) / F1.hi);
    else if (F1.hi < 0.0)
        s1 = dmin(s1, (-R - F0.hi) / F1.hi);
    else if (F0.hi < -R)
        return false;
    if (s0 > s1 + interval_tolerance(fabs(t0) + span))
        return false;
    if (s0 > s1) {
        double x = s0;
        s0 = s1;
        s1 = x;
    }
    t1 = t0 + s1;
    t0 = t0 + s0;
    return true;
}

__device__ bool node_interval(const nodebound &nb, const tray &r, const dmapk::QueryOpts &opt, double &t0,
                              double &t1) // node_bounds.cpp:181-211
{
    bool read_slab = nb.level <= opt.slab_max_level;
    if (opt.bound == 0 || !read_slab)
        return box_interval(nb, r, t0, t1);
    if (opt.bound == 1)
        return slab_interval(nb, r, t0, t1);
    double b0, b1, s0, s1;
    if (!box_interval(nb, r, b0, b1) || !slab_interval(nb, r, s0, s1))
        return false;
    t0 = dmax(b0, s0);
    t1 = dmin(b1, s1);
    double tol = interval_tolerance(dmax(fabs(t0), fabs(t1)));
    if (t0 > t1 + tol)
        return false;
    if (t0 > t1) {
        double x = t0;
        t0 = t1;
        t1 = x;
    }
    return true;
}

// ---- cells (displaced_intersector.cpp:18-19, 85-121) ------------------
struct cell { int level; int64_t i, j; };
__device__ __forceinline__ int64_t floor_div2(int64_t x) { return x >= 0 ? x / 2 : -((-x + 1) / 2); }
__device__ __forceinline__ int floor_mod2(int64_t x) { return (int)(x - 2 * floor_div2(x)); }
__device__ __forceinline__ void cell_next(cell &c, bool si, bool sj, int root_level)
{
    for (;;) {
        int code = 2 * floor_mod2(c.i + (si ? 1 : 0)) + floor_mod2(c.j + (sj ? 1 : 0));
        if (code == 1) {
            c.j += sj ? 1 : -1;
            c.i += si ? -1 : 1;
            return;
        }
        if (code == 3) {
            ++c.level;
            c.i = floor_div2(c.i);
            c.j = floor_div2(c.j);
            if (c.level > root_level)
                return;
            continue;
        }
        c.j += sj ? -1 : 1;
        return;
    }
}

// DisplacedIntersector::intersect (:175-237)
__device__ bool triangle_intersect(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max,
                                   const dmapk::QueryOpts &opt, hit64 &hit, int64_t *st)
{
    tray ray = {mat3mul(T.A, sub3(o, L3(T.q0))), mat3mul(T.A, d), t_min, t_max};
    bool si = ray.d.x < 0.0, sj = ray.d.y < 0.0;
    bool found = false;
    int64_t nah = 0, lah = 0;
    for (int r = 0; r < T.n_roots; ++r) {
        cell cur = {T.root_level, T.roots_i[r], T.roots_j[r]}, end = cur;
        cell_next(end, si, sj, T.root_level);
        while (!(cur.level == end.level && cur.i == end.i && cur.j == end.j)) {
            double w = cell_width(g, cur.level);
            v2 c = {(cur.i + 0.5) * w, (cur.j + 0.5) * w};
            if (classify_square(T, c, 0.5 * w) == OUTSIDE) {
                cell_next(cur, si, sj, T.root_level);
                continue;
            }
            if (st) {
                ++st[DMAP_ST_NODE];
                ++nah;
            }
            nodebound nb;
            node_bound(nb, T, g, cur.level, cur.i, cur.j);
            ray.t_max = t_max;
            double t0, t1;
            if (!node_interval(nb, ray, opt, t0, t1)) {
                cell_next(cur, si, sj, T.root_level);
                continue;
            }
            if (cur.level > 0) {
                --cur.level;
                cur.i = 2 * cur.i + (si ? 1 : 0);
                cur.j = 2 * cur.j + (sj ? 1 : 0);
                continue;
            }
            if (st) {
                ++st[DMAP_ST_LEAF];
                ++lah;
            }
            hit64 lh;
            bool lf = opt.leaf == 0 ? intersect_newton(T, g, o, d, t_min, t_max, cur.i, cur.j, lh, st)
                                    : intersect_two_triangle(T, g, o, d, t_min, t_max, cur.i, cur.j, lh);
            if (lf && lh.t < t_max) {
                hit = lh;
                t_max = lh.t;
                found = true;
                nah = lah = 0;
                if (opt.mode == 1)
                    return true; // occlusion: any hit answers the query
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

template <typename R>
__device__ __forceinline__ void load_ray(const R *rays, int64_t k, v3 &o, v3 &d, double &t_min, double &t_max)
{
    const R *r = rays + 8 * k;
    o = {(double)r[0], (double)r[1], (double)r[2]};
    d = {(double)r[3], (double)r[4], (double)r[5]};
    t_min = (double)r[6];
    t_max = (double)r[7];
}

template <typename H, typename F>
__device__ __forceinline__ void store_hit(H *hits, int64_t k, bool found, const hit64 &h, int tri)
{
    H out;
    if (found) {
        out.t = (F)h.t;
        out.st[0] = (F)h.st.x;
        out.st[1] = (F)h.st.y;
        out.bary[0] = (F)h.bary.x;
        out.bary[1] = (F)h.bary.y;
        out.ng[0] = (F)h.ng.x;
        out.ng[1] = (F)h.ng.y;
        out.ng[2] = (F)h.ng.z;
        out.tri = tri;
        out.i = (int32_t)h.i;
        out.j = (int32_t)h.j;
    } else {
        out.t = (F)INFINITY;
        out.st[0] = out.st[1] = out.bary[0] = out.bary[1] = (F)0;
        out.ng[0] = out.ng[1] = out.ng[2] = (F)0;
        out.tri = -1;
        out.i = out.j = 0;
    }
    out.flags = 0;
    hits[k] = out;
}

template <typename R, typename H, typename F>
__global__ void __launch_bounds__(128) walk64_kernel(const TriDev *__restrict__ tris, int n_tri,
                                                     const AssetDev *__restrict__ assets, const R *__restrict__ rays,
                                                     int64_t n, dmapk::QueryOpts opt, H *__restrict__ hits,
                                                     int64_t *__restrict__ stats)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    v3 o, d;
    double t_min, t_max;
    load_ray(rays, k, o, d, t_min, t_max);
    int64_t st[DMAP_ST_N] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t *sp = stats ? st : nullptr;
    hit64 best;
    int best_tri = -1;
    bool found = false;
    for (int t = 0; t < n_tri; ++t) {
        const TriDev &T = tris[t];
        box3 box = {L3(T.box_lo), L3(T.box_hi)};
        double t0 = t_min, t1 = t_max;
        if (T.status != 0 || !box_clip(box, o, d, t0, t1))
            continue;
        if (sp)
            ++st[DMAP_ST_TRI];
        hit64 h;
        if (triangle_intersect(T, assets[T.asset], o, d, t_min, t_max, opt, h, sp)) {
            best = h;
            best_tri = t;
            t_max = h.t;
            found = true;
            if (opt.mode == 1)
                break;
        }
    }
    store_hit<H, F>(hits, k, found, best, best_tri);
    if (stats)
        for (int q = 0; q < DMAP_ST_N; ++q)
            stats[DMAP_ST_N * k + q] = st[q];
}

template <typename R, typename H, typename F>
cudaError_t launch(const TriDev *tris, int n_tri, const AssetDev *assets, const void *rays, int64_t n,
                   const dmapk::QueryOpts &opt, void *hits, int64_t *stats, cudaStream_t stream)
{
    int threads = 128;
    int64_t blocks = (n + threads - 1) / threads;
    walk64_kernel<R, H, F><<<(unsigned)blocks, threads, 0, stream>>>(
        tris, n_tri, assets, static_cast<const R *>(rays), n, opt, static_cast<H *>(hits), stats);
    return cudaGetLastError();
}

} // namespace

namespace dmapk
{
cudaError_t launch_walk64(const dmapdev::TriDev *tris, int n_tri, const dmapdev::AssetDev *assets, const void *rays,
                          int64_t n, const QueryOpts &opt, void *hits, int64_t *stats, unsigned *, cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    bool r64 = opt.ray_dtype == 2, h64 = opt.hit_dtype == 2;
    if (r64 && h64)
        return launch<double, dmapdev::Hit64, double>(tris, n_tri, assets, rays, n, opt, hits, stats, stream);
    if (r64)
        return launch<double, dmapdev::Hit32, float>(tris, n_tri, assets, rays, n, opt, hits, stats, stream);
    if (h64)
        return launch<float, dmapdev::Hit64, double>(tris, n_tri, assets, rays, n, opt, hits, stats, stream);
    return launch<float, dmapdev::Hit32, float>(tris, n_tri, assets, rays, n, opt, hits, stats, stream);
}
} // namespace dmapk
