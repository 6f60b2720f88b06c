// The node test in double with the reference's operation order
// (node_bounds.cpp:83-211: node_bound, box_interval, slab_interval,
// node_interval) and the level-0 pyramid node computed straight from the
// node grid (leaf_level, taylor_pyramid.cpp:45-67), for translation units
// compiled with -fmad=false: the FP64 walk, and the FP32 path's check of a
// leaf cell before its leaf runs.
#pragma once
#include "device_types.cuh"
#include "f64_math.cuh"
#include "launch.h"

namespace d64
{

struct nodebound { int level; node n; v2 centre; af3 m; box3 box; };

// TaylorPyramid::node at level 0, from the node grid instead of the stored
// FP64 level (which the FP32 path frees): the arithmetic of the device
// pyramid build's leaf cell, so the result equals the stored node bit for
// bit, offset added as pyramid_node adds it.
__device__ __forceinline__ node leaf_node(const AssetDev &a, int64_t i, int64_t j)
{
    int64_t m = a.n_leaf;
    int64_t ri = i % m, rj = j % m;
    if (ri < 0)
        ri += m;
    if (rj < 0)
        rj += m;
    int x = (int)ri, y = (int)rj;
    double v00 = grid_value(a, y, x) * a.scale, v10 = grid_value(a, y, x + 1) * a.scale;
    double v01 = grid_value(a, y + 1, x) * a.scale, v11 = grid_value(a, y + 1, x + 1) * a.scale;
    double w = 1.0 / a.n_leaf;
    double s = 0.5 * w;
    node n;
    n.h0 = 0.25 * (((v00 + v10) + v01) + v11);
    n.gu = 0.5 * ((v10 - v00) + (v11 - v01)) / w;
    n.gv = 0.5 * ((v01 - v00) + (v11 - v10)) / w;
    double c3 = (((v00 - v10) - v01) + v11) / (w * w);
    n.r = fabs(c3) * s * s;
    n.ru = fabs(c3) * s;
    n.rv = fabs(c3) * s;
    n.h_min = dmin(dmin(v00, v10), dmin(v01, v11));
    n.h_max = dmax(dmax(v00, v10), dmax(v01, v11));
    if (a.offset != 0.0) {
        n.h0 += a.offset;
        n.h_min += a.offset;
        n.h_max += a.offset;
    }
    return n;
}

// node_bounds.cpp:83-109 for a given pyramid node
__device__ __forceinline__ void node_bound_of(nodebound &nb, const TriDev &T, const AssetDev &a, int level,
                                              int64_t i, int64_t j, const node &pn)
{
    nb.level = level;
    nb.n = pn;
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

__device__ __forceinline__ void node_bound(nodebound &nb, const TriDev &T, const AssetDev &a, int level, int64_t i,
                                           int64_t j)
{
    node_bound_of(nb, T, a, level, i, j, pyramid_node(a, level, i, j));
}

__device__ __forceinline__ ivl IV(double lo, double hi) { return {lo, hi}; }
__device__ __forceinline__ ivl iv_add(ivl a, ivl b) { return {a.lo + b.lo, a.hi + b.hi}; }
__device__ __forceinline__ ivl iv_scale(double s, ivl a) { return s >= 0.0 ? IV(s * a.lo, s * a.hi) : IV(s * a.hi, s * a.lo); }

// The ray in the triangle's tangent frame (displaced_intersector.cpp:178).
struct tray { v3 o, d; double t_min, t_max; };

__device__ __forceinline__ tray tangent_ray64(const TriDev &T, v3 o, v3 d, double t_min, double t_max)
{
    return {mat3mul(T.A, sub3(o, L3(T.q0))), mat3mul(T.A, d), t_min, t_max};
}

__device__ __forceinline__ bool box_interval(const nodebound &nb, const tray &r, double &t0, double &t1)
{
    t0 = r.t_min;
    t1 = r.t_max;
    return box_clip(nb.box, r.o, r.d, t0, t1);
}

__device__ inline bool slab_interval(const nodebound &nb, const tray &r, double &t0, double &t1) // node_bounds.cpp:137-179
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

__device__ inline bool node_interval(const nodebound &nb, const tray &r, const dmapk::QueryOpts &opt, double &t0,
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

// The reference's own node test of leaf cell (i, j) for the tangent-space
// ray r: false exactly when the FP64 walk would reject the cell at r.t_max.
__device__ inline bool leaf_cell_admitted(const TriDev &T, const AssetDev &a, const tray &r, int64_t i, int64_t j,
                                          const dmapk::QueryOpts &opt)
{
    nodebound nb;
    node_bound_of(nb, T, a, 0, i, j, leaf_node(a, i, j));
    double t0, t1;
    return node_interval(nb, r, opt, t0, t1);
}

__device__ inline bool leaf_cell_admitted(const TriDev &T, const AssetDev &a, v3 o, v3 d, double t_min,
                                          double t_max, int64_t i, int64_t j, const dmapk::QueryOpts &opt)
{
    return leaf_cell_admitted(T, a, tangent_ray64(T, o, d, t_min, t_max), i, j, opt);
}

} // namespace d64
