// The FP64 query path: one thread per ray, every triangle of the scene in
// order behind its AABB (ObjectIntersector::intersect_flat,
// displaced_intersector.cpp:578-599), each walked with TFDM's stackless
// quadtree walk and the certified Newton leaf
// (displaced_intersector.cpp:175-388, node_bounds.cpp:83-211), in double
// with the reference's operation order (compiled with -fmad=false). This is
// the device oracle and the plain one-launch-per-request comparator; its
// results equal the reference's CPU build bit for bit.
#include "device_types.cuh"
#include "f64_math.cuh"
#include "f64_leaf.cuh"
#include "f64_node.cuh"
#include "f64_walk.cuh"
#include "order.cuh"
#include "filter.cuh"
#include "instance.cuh"
#include "launch.h"

namespace
{
using namespace d64;
using dmapdev::AssetDev;
using dmapdev::TriDev;

// The intersect / occluded callback's passes over DisplacedIntersector::intersect
// (displaced_geometry.cpp:53-106): a crossing the scene's filter rejects
// raises t_min to its t and the triangle is walked again. No filter: one walk.
__device__ bool triangle_filtered_obj(const TriDev &T, int tri, const AssetDev &g, v3 o, v3 d, double t_min,
                                      double t_max, const dmapk::QueryOpts &opt, hit64 &hit, int64_t *st)
{
    if (!opt.op_mask)
        return triangle_intersect(T, g, o, d, t_min, t_max, opt, hit, st);
    double t_lo = t_min;
    for (int pass = 0; pass < dmapdev::kFilterPasses; ++pass) {
        if (!triangle_intersect(T, g, o, d, t_lo, t_max, opt, hit, st))
            return false;
        if (dmapdev::crossing_opaque(opt, T, tri, hit.bary.x, hit.bary.y))
            return true;
        t_lo = hit.t; // the walk accepts t > t_min only
    }
    return false;
}

// The same for a triangle of a non-rigid instance: the ray moved to the
// object's space first, the hit's normal moved back (instance.cuh).
__device__ bool triangle_filtered(const TriDev &T, int tri, const AssetDev &g, v3 o, v3 d, double t_min,
                                  double t_max, const dmapk::QueryOpts &opt, hit64 &hit, int64_t *st)
{
    if (!T.inst)
        return triangle_filtered_obj(T, tri, g, o, d, t_min, t_max, opt, hit, st);
    const double *xf = opt.inst_xf + dmapdev::kInstDoubles * (T.inst - 1);
    const double ow[3] = {o.x, o.y, o.z}, dw[3] = {d.x, d.y, d.z};
    double oo[3], od[3];
    dmapdev::object_ray(xf, ow, dw, oo, od);
    if (!triangle_filtered_obj(T, tri, g, V3(oo[0], oo[1], oo[2]), V3(od[0], od[1], od[2]), t_min, t_max, opt, hit,
                               st))
        return false;
    dmapdev::world_normal(xf, hit.ng);
    return true;
}

template <typename R>
__device__ __forceinline__ void load_ray(const R *rays, int64_t k, v3 &o, v3 &d, double &t_min, double &t_max)
{
    const R *r = rays + 8 * k;
    double oo[3] = {(double)r[0], (double)r[1], (double)r[2]}, dd[3] = {(double)r[3], (double)r[4], (double)r[5]};
    t_min = (double)r[6];
    t_max = (double)r[7];
    dmapdev::sanitize_ray(oo, dd, t_min, t_max);
    o = {oo[0], oo[1], oo[2]};
    d = {dd[0], dd[1], dd[2]};
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
    // the next triangle: index order (the flat loop), or (nearest) the
    // smallest (key, index) past the cursor whose box the ray still meets
    const double od[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    double inv[3], ckey = -INFINITY;
    int cidx = -1;
    ray_inverse(dd, inv);
    for (int step = 0; step < n_tri; ++step) {
        int t = step;
        if (opt.order == 1) {
            double bk = 0.0;
            int bt = -1;
            for (int q = 0; q < n_tri; ++q) {
                const TriDev &Q = tris[q];
                if (Q.status != 0)
                    continue;
                const double key = entry_key(Q, od, dd, inv, t_min);
                if (!after_cursor(key, q, ckey, cidx) || !before_best(key, q, bk, bt))
                    continue;
                box3 box = {L3(Q.box_lo), L3(Q.box_hi)};
                double t0 = t_min, t1 = t_max;
                if (!box_clip(box, o, d, t0, t1))
                    continue;
                bk = key;
                bt = q;
            }
            if (bt < 0)
                break;
            t = bt;
            ckey = bk;
            cidx = bt;
        }
        const TriDev &T = tris[t];
        box3 box = {L3(T.box_lo), L3(T.box_hi)};
        double t0 = t_min, t1 = t_max;
        if (T.status != 0 || !box_clip(box, o, d, t0, t1))
            continue;
        if (sp)
            ++st[DMAP_ST_TRI];
        hit64 h;
        if (triangle_filtered(T, t, assets[T.asset], o, d, t_min, t_max, opt, h, sp)) {
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
