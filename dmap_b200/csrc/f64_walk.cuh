// DisplacedIntersector::intersect (displaced_intersector.cpp:175-237) in
// double with the reference's operation order: TFDM's stackless quadtree
// walk over one triangle's footprint and the certified leaf. Shared by the
// FP64 query (walk64.cu) and the displaced emitter's re-walk (emitter.cu);
// included by translation units compiled with -fmad=false.
#pragma once
#include "device_types.cuh"
#include "f64_math.cuh"
#include "f64_leaf.cuh"
#include "f64_node.cuh"
#include "launch.h"

namespace d64
{
using dmapdev::AssetDev;
using dmapdev::TriDev;

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
__device__ inline bool triangle_intersect(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max,
                                   const dmapk::QueryOpts &opt, hit64 &hit, int64_t *st)
{
    tray ray = tangent_ray64(T, o, d, t_min, t_max);
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
                if (opt.mode == 1 && !opt.op_mask)
                    return true; // occlusion: any hit answers the query (a filter judges the nearest)
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

} // namespace d64
