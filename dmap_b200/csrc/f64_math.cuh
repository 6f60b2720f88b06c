// The reference's double-precision arithmetic on the device, operation for
// operation (MangoSister/dmap code/cpp/src: affine_form.cpp, taylor_pyramid.cpp,
// displaced_surface.cpp, uv_clip.cpp, node_bounds.cpp,
// displaced_intersector.cpp). Every translation unit that includes this file
// is compiled with -fmad=false, so each double operation rounds on its own
// and results agree bit for bit with the reference's CPU build.
//
// Operation order: dot(a, b) = (a0*b0 + a1*b1) + a2*b2; M*v row by row in
// the same order; std::min(a, b) = b < a ? b : a; std::max(a, b) = a < b ? b : a.
#pragma once
#include "device_types.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace d64
{
using dmapdev::AssetDev;
using dmapdev::TriDev;

struct v2 { double x, y; };
struct v3 { double x, y, z; };

__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ v2 V2(double x, double y) { return {x, y}; }
__device__ __forceinline__ v3 V3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ v3 L3(const double *p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ v2 L2(const double *p) { return {p[0], p[1]}; }
__device__ __forceinline__ v2 sub2(v2 a, v2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ v2 add2(v2 a, v2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ v2 mul2(double s, v2 a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ v2 min2(v2 a, v2 b) { return {dmin(a.x, b.x), dmin(a.y, b.y)}; }
__device__ __forceinline__ v2 max2(v2 a, v2 b) { return {dmax(a.x, b.x), dmax(a.y, b.y)}; }
__device__ __forceinline__ double dot2(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ v3 add3(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 sub3(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 mul3(double s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ v3 div3(v3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ v3 cross3(v3 a, v3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double norm3(v3 a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ v3 normalized3(v3 a)
{
    double z = dot3(a, a);
    if (z > 0.0)
        return div3(a, sqrt(z));
    return a;
}
__device__ __forceinline__ double comp(v3 a, int k) { return k == 0 ? a.x : k == 1 ? a.y : a.z; }
__device__ __forceinline__ v3 mat3mul(const double (*A)[3], v3 v)
{
    return {(A[0][0] * v.x + A[0][1] * v.y) + A[0][2] * v.z, (A[1][0] * v.x + A[1][1] * v.y) + A[1][2] * v.z,
            (A[2][0] * v.x + A[2][1] * v.y) + A[2][2] * v.z};
}

// ---- affine forms (affine_form.cpp) ------------------------------------
struct af { double c, a, b, k; };
struct af3 { af x, y, z; };
struct ivl { double lo, hi; };

__device__ __forceinline__ af AF(double c, double a, double b, double k) { return {c, a, b, k}; }
__device__ __forceinline__ ivl interval(af f) // affine_form.h:50-54
{
    double e = (fabs(f.a) + fabs(f.b)) + f.k;
    return {f.c - e, f.c + e};
}
__device__ __forceinline__ af add(af x, af y) { return {x.c + y.c, x.a + y.a, x.b + y.b, x.k + y.k}; } // affine_form.cpp:17-24
__device__ __forceinline__ af scale(double s, af x) { return {x.c * s, x.a * s, x.b * s, x.k * fabs(s)}; } // affine_form.cpp:49-56
__device__ __forceinline__ af mul(af x, af r) // affine_form.cpp:35-47
{
    double u = (fabs(x.a) + fabs(x.b)) + x.k;
    double v = (fabs(r.a) + fabs(r.b)) + r.k;
    double c0 = x.c;
    af o;
    o.c = c0 * r.c;
    o.a = c0 * r.a + r.c * x.a;
    o.b = c0 * r.b + r.c * x.b;
    o.k = (fabs(r.c) * x.k + fabs(c0) * r.k) + u * v;
    return o;
}
__device__ __forceinline__ double grs(double x) { return 1.0 / sqrt(x); }
__device__ __forceinline__ af rsqrt_form(af f) // affine_form.cpp:64-76, Min-Range
{
    ivl range = interval(f);
    double lo = range.lo, hi = range.hi;
    double alpha = -0.5 * grs(hi) * grs(hi) * grs(hi);
    double beta = 0.5 * (grs(lo) + grs(hi) - alpha * (lo + hi));
    double delta = 0.5 * fabs(grs(lo) - grs(hi) - alpha * (lo - hi));
    return {alpha * f.c + beta, alpha * f.a, alpha * f.b, fabs(alpha) * f.k + delta};
}
__device__ __forceinline__ af3 AF3(v3 c, v3 a, v3 b)
{
    return {{c.x, a.x, b.x, 0.0}, {c.y, a.y, b.y, 0.0}, {c.z, a.z, b.z, 0.0}};
}
__device__ __forceinline__ af sq_length(const af3 &v) // affine_form.cpp:78-85
{
    v3 xc = {v.x.c, v.y.c, v.z.c}, xu = {v.x.a, v.y.a, v.z.a}, xv = {v.x.b, v.y.b, v.z.b};
    v3 xk = {v.x.k, v.y.k, v.z.k};
    v3 dev = {(fabs(xu.x) + fabs(xv.x)) + xk.x, (fabs(xu.y) + fabs(xv.y)) + xk.y, (fabs(xu.z) + fabs(xv.z)) + xk.z};
    double offset = 0.5 * dot3(dev, dev);
    return {dot3(xc, xc) + offset, 2.0 * dot3(xc, xu), 2.0 * dot3(xc, xv), 2.0 * fabs(dot3(xc, xk)) + offset};
}
__device__ __forceinline__ void normalize(af3 &v) // affine_form.cpp:87-95
{
    af l = sq_length(v);
    if (interval(l).lo <= 0.0) {
        v.x = v.y = v.z = AF(0.0, 0.0, 0.0, 1.0);
        return;
    }
    af r = rsqrt_form(l);
    v.x = mul(r, v.x);
    v.y = mul(r, v.y);
    v.z = mul(r, v.z);
}
__device__ __forceinline__ af3 add(const af3 &a, const af3 &b) { return {add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
__device__ __forceinline__ af dot(v3 a, const af3 &b) // affine_form.cpp:101
{
    return add(add(scale(a.x, b.x), scale(a.y, b.y)), scale(a.z, b.z));
}
__device__ __forceinline__ af3 matmul(const double (*A)[3], const af3 &v) // affine_form.cpp:103-106
{
    return {dot(V3(A[0][0], A[0][1], A[0][2]), v), dot(V3(A[1][0], A[1][1], A[1][2]), v),
            dot(V3(A[2][0], A[2][1], A[2][2]), v)};
}
__device__ __forceinline__ af3 scale_form(af s, const af3 &v) { return {mul(s, v.x), mul(s, v.y), mul(s, v.z)}; }

// ---- pyramid and height grid -------------------------------------------
struct node { double h0, gu, gv, r, ru, rv, h_min, h_max; };

__device__ __forceinline__ double cell_width(const AssetDev &a, int level) // taylor_pyramid.h:94
{
    return ldexp(1.0, level) / a.n_leaf;
}

__device__ __forceinline__ node pyramid_node(const AssetDev &a, int level, int64_t i, int64_t j) // taylor_pyramid.cpp:259-274
{
    node n;
    // pyr64 holds the levels before the offset; the reference adds it once
    // after the build (taylor_pyramid.cpp:239-250), here on read.
    if (level >= a.n_levels) {
        const double *root = a.pyr64 + 8 * a.level_off[a.n_levels - 1];
        double lo = root[6], hi = root[7];
        if (a.offset != 0.0) {
            lo += a.offset;
            hi += a.offset;
        }
        n.h0 = 0.5 * (lo + hi);
        n.gu = 0.0;
        n.gv = 0.0;
        n.r = 0.5 * (hi - lo);
        n.ru = root[4];
        n.rv = root[5];
        n.h_min = lo;
        n.h_max = hi;
        return n;
    }
    int64_t m = a.n_leaf >> level;
    int64_t ri = i % m, rj = j % m;
    if (ri < 0)
        ri += m;
    if (rj < 0)
        rj += m;
    const double2 *p = reinterpret_cast<const double2 *>(a.pyr64 + 8 * (a.level_off[level] + rj * m + ri));
    double2 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3);
    n.h0 = q0.x;
    n.gu = q0.y;
    n.gv = q1.x;
    n.r = q1.y;
    n.ru = q2.x;
    n.rv = q2.y;
    n.h_min = q3.x;
    n.h_max = q3.y;
    if (a.offset != 0.0) {
        n.h0 += a.offset;
        n.h_min += a.offset;
        n.h_max += a.offset;
    }
    return n;
}

__device__ __forceinline__ double grid_value(const AssetDev &a, int j, int i)
{
    size_t k = (size_t)j * a.pitch + i;
    if (a.dtype == 0)
        return (double)__ldg(static_cast<const float *>(a.nodes) + k);
    if (a.dtype == 1)
        return (double)__half2float(static_cast<const __half *>(a.nodes)[k]);
    if (a.dtype == 3)
        return (double)__bfloat162float(static_cast<const __nv_bfloat16 *>(a.nodes)[k]);
    return __ldg(static_cast<const double *>(a.nodes) + k);
}

__device__ __forceinline__ void grid_cell(const AssetDev &g, double x, double y, int &i, int &j, double &s, double &t)
{
    // displaced_surface.cpp:12-27
    if (g.repeat) {
        x -= floor(x);
        y -= floor(y);
    } else {
        x = x < 0.0 ? 0.0 : (1.0 < x ? 1.0 : x);
        y = y < 0.0 ? 0.0 : (1.0 < y ? 1.0 : y);
    }
    double fx = x * (g.W - 1);
    double fy = y * (g.W - 1);
    int ii = (int)fx, jj = (int)fy;
    i = g.W - 2 < ii ? g.W - 2 : ii;
    j = g.W - 2 < jj ? g.W - 2 : jj;
    s = fx - i;
    t = fy - j;
}

__device__ __forceinline__ double grid_h(const AssetDev &g, double x, double y) // displaced_surface.cpp:29-37
{
    int i, j;
    double s, t;
    grid_cell(g, x, y, i, j, s, t);
    return g.scale * (((((1.0 - s) * (1.0 - t)) * grid_value(g, j, i) + (s * (1.0 - t)) * grid_value(g, j, i + 1)) +
                       ((1.0 - s) * t) * grid_value(g, j + 1, i)) +
                      (s * t) * grid_value(g, j + 1, i + 1)) +
           g.offset;
}

__device__ __forceinline__ void grid_h_grad(const AssetDev &g, double x, double y, double &h, v2 &gr)
{
    // displaced_surface.cpp:29-47, h and grad from one cell lookup
    int i, j;
    double s, t;
    grid_cell(g, x, y, i, j, s, t);
    double v00 = grid_value(g, j, i), v10 = grid_value(g, j, i + 1);
    double v01 = grid_value(g, j + 1, i), v11 = grid_value(g, j + 1, i + 1);
    h = g.scale * (((((1.0 - s) * (1.0 - t)) * v00 + (s * (1.0 - t)) * v10) + ((1.0 - s) * t) * v01) + (s * t) * v11) +
        g.offset;
    double dh_ds = (1.0 - t) * (v10 - v00) + t * (v11 - v01);
    double dh_dt = (1.0 - s) * (v01 - v00) + s * (v11 - v10);
    gr = {g.scale * (dh_ds * (g.W - 1)), g.scale * (dh_dt * (g.W - 1))};
}

// ---- base triangle (displaced_surface.h:83-87, .cpp:99-108) -----------
__device__ __forceinline__ v3 tri_P(const TriDev &T, double s, double t)
{
    return add3(add3(L3(T.q0), mul3(s, L3(T.e1))), mul3(t, L3(T.e2)));
}
__device__ __forceinline__ v3 tri_M(const TriDev &T, double s, double t)
{
    return add3(add3(L3(T.m0), mul3(s, L3(T.Mu))), mul3(t, L3(T.Mv)));
}
__device__ __forceinline__ v2 tri_bary(const TriDev &T, double s, double t)
{
    double x = s - T.t0[0], y = t - T.t0[1];
    return {T.J[0][0] * x + T.J[0][1] * y, T.J[1][0] * x + T.J[1][1] * y};
}
struct nframe { v3 N, Nu, Nv; };
__device__ __forceinline__ nframe normal_frame_at(const TriDev &T, double s, double t)
{
    v3 M = tri_M(T, s, t);
    double Mlen = norm3(M);
    nframe f;
    f.N = div3(M, Mlen);
    f.Nu = div3(sub3(L3(T.Mu), mul3(dot3(f.N, L3(T.Mu)), f.N)), Mlen);
    f.Nv = div3(sub3(L3(T.Mv), mul3(dot3(f.N, L3(T.Mv)), f.N)), Mlen);
    return f;
}
__device__ __forceinline__ v3 displaced_position(const TriDev &T, const AssetDev &g, double s, double t)
{
    nframe f = normal_frame_at(T, s, t);
    return add3(tri_P(T, s, t), mul3(grid_h(g, s, t), f.N));
}

// ---- uv domain (uv_clip.cpp:27-44) ---------------------------------------
enum { OUTSIDE = 0, INSIDE = 1, STRADDLE = 2 };
__device__ __forceinline__ bool uv_inside(const TriDev &T, v2 p)
{
    for (int k = 0; k < 3; ++k)
        if (T.un[k][0] * p.x + T.un[k][1] * p.y < T.ud[k])
            return false;
    return true;
}
__device__ __forceinline__ int classify_square(const TriDev &T, v2 c, double s)
{
    if (c.x + s <= T.lo[0] || c.x - s >= T.hi[0] || c.y + s <= T.lo[1] || c.y - s >= T.hi[1])
        return OUTSIDE;
    bool all_inside = true;
    for (int k = 0; k < 3; ++k) {
        double proj = T.un[k][0] * c.x + T.un[k][1] * c.y;
        double ext = (fabs(T.un[k][0]) + fabs(T.un[k][1])) * s;
        if (proj + ext <= T.ud[k])
            return OUTSIDE;
        if (proj - ext < T.ud[k])
            all_inside = false;
    }
    return all_inside ? INSIDE : STRADDLE;
}

struct ClipPoly
{
    int n;
    v2 p[8];
};

// clip_square (uv_clip.cpp:56-83): Sutherland-Hodgman of the square (c, s)
// against the domain's three inward half-planes (at most 7 vertices).
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

// ---- boxes and node tests (node_bounds.cpp) ----------------------------
__device__ __forceinline__ double interval_tolerance(double t_scale) { return 1e-9 * dmax(1.0, t_scale); }

struct box3 { v3 lo, hi; };

__device__ __forceinline__ bool box_clip(const box3 &B, v3 o, v3 d, double &t0, double &t1) // node_bounds.cpp:25-44
{
    for (int a = 0; a < 3; ++a) {
        double da = comp(d, a), oa = comp(o, a);
        double lo = comp(B.lo, a), hi = comp(B.hi, a);
        if (da != 0.0) {
            double ta = (lo - oa) / da, tb = (hi - oa) / da;
            if (ta > tb) {
                double x = ta;
                ta = tb;
                tb = x;
            }
            t0 = dmax(t0, ta);
            t1 = dmin(t1, tb);
        } else if (oa < lo || oa > hi) {
            return false;
        }
    }
    if (t0 > t1 + interval_tolerance(dmax(fabs(t0), fabs(t1))))
        return false;
    if (t0 > t1) {
        double x = t0;
        t0 = t1;
        t1 = x;
    }
    return true;
}

__device__ __forceinline__ box3 hull(const af3 &S)
{
    ivl x = interval(S.x), y = interval(S.y), z = interval(S.z);
    return {{x.lo, y.lo, z.lo}, {x.hi, y.hi, z.hi}};
}

} // namespace d64
