// Outward-rounded FP32 node tests of the displaced-surface walk, shared by
// the FP32 kernels (walk32.cu describes the scheme). Every quantity lives in
// named scalars: no array is indexed by a run-time value, so nothing spills
// to the stack frame.
#pragma once
#include "device_types.cuh"
#include "f64_math.cuh"
#include "f64_leaf.cuh"
#include "f64_node.cuh"
#include "launch.h"

namespace d32
{
using dmapdev::AssetDev;
using dmapdev::TriDev;
using dmapdev::TriDev32;

constexpr float G = 9.5367431640625e-07f;     // 2^-20: bound factor for the roundings of one step
constexpr float U2 = 1.1920928955078125e-07f; // 2^-23

__device__ __forceinline__ float ru_add(float x, float y) { return __fadd_ru(x, y); }
__device__ __forceinline__ float rd_add(float x, float y) { return __fadd_rd(x, y); }
__device__ __forceinline__ float ru_mul(float x, float y) { return __fmul_ru(x, y); }
__device__ __forceinline__ float rd_mul(float x, float y) { return __fmul_rd(x, y); }
__device__ __forceinline__ float ru_fma(float x, float y, float z) { return __fmaf_ru(x, y, z); }
__device__ __forceinline__ float mag3(float x, float y, float z) { return ru_add(ru_add(fabsf(x), fabsf(y)), fabsf(z)); }
// 2^e exactly, -126 <= e <= 127
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((e + 127) << 23); }

struct Node32 { float h0, gu, gv, r, mn, mx; };

// TaylorPyramid::node (taylor_pyramid.cpp:259-274) on the FP32 pyramid:
// wrapped indices (the level's width is a power of two), above the root the
// root's height range as a min-max node.
__device__ __forceinline__ Node32 fetch_node(const AssetDev &a, int level, int i, int j)
{
    Node32 n;
    if (level >= a.n_levels) {
        const float4 *p = reinterpret_cast<const float4 *>(a.pyr32 + 8 * a.level_off[a.n_levels - 1]);
        float4 q1 = __ldg(p + 1);
        n.mn = q1.z;
        n.mx = q1.w;
        n.h0 = 0.5f * (n.mn + n.mx);
        n.r = fmaxf(__fsub_ru(n.mx, n.h0), __fsub_ru(n.h0, n.mn));
        n.gu = n.gv = 0.0f;
        return n;
    }
    int m = a.n_leaf >> level;
    int ri = i & (m - 1), rj = j & (m - 1);
    const float4 *p = reinterpret_cast<const float4 *>(a.pyr32 + 8 * (a.level_off[level] + (int64_t)rj * m + ri));
    float4 q0 = __ldg(p), q1 = __ldg(p + 1);
    n.h0 = q0.x;
    n.gu = q0.y;
    n.gv = q0.z;
    n.r = q0.w;
    n.mn = q1.z;
    n.mx = q1.w;
    return n;
}

// The tangent-space ray (o, d), its reciprocal directions and the widening
// E that covers its rounding from the double ray.
struct Ray32 { float ox, oy, oz, dx, dy, dz, ix, iy, iz, ex, ey, ez; };

struct Cell32 { int level, i, j; };

__device__ __forceinline__ int fdiv2(int x) { return x >> 1; } // arithmetic shift: floor division by 2
__device__ __forceinline__ void cell_next(Cell32 &c, int si, int sj, int root_level)
{
    // displaced_intersector.cpp:99-121
    for (;;) {
        int code = 2 * ((c.i + si) & 1) + ((c.j + sj) & 1);
        if (code == 1) {
            c.j += sj ? 1 : -1;
            c.i += si ? -1 : 1;
            return;
        }
        if (code == 3) {
            ++c.level;
            c.i = fdiv2(c.i);
            c.j = fdiv2(c.j);
            if (c.level > root_level)
                return;
            continue;
        }
        c.j += sj ? -1 : 1;
        return;
    }
}

// classify_square (uv_clip.cpp:27-44) reporting Outside only when the
// separation exceeds the rounding of the test.
__device__ __forceinline__ bool square_meets_domain(const TriDev32 &T, float cx, float cy, float s)
{
    if (cx + s <= T.lo[0] || cx - s >= T.hi[0] || cy + s <= T.lo[1] || cy - s >= T.hi[1])
        return false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float proj = __fmaf_rn(T.un[k][1], cy, T.un[k][0] * cx);
        float ext = (fabsf(T.un[k][0]) + fabsf(T.un[k][1])) * s;
        float slack = G * (fabsf(T.un[k][0] * cx) + fabsf(T.un[k][1] * cy) + fabsf(T.ud[k]) + ext);
        if (proj + ext + slack <= T.ud[k])
            return false;
    }
    return true;
}

struct Iv { float lo, hi; };
__device__ __forceinline__ Iv iv_scale(float s, Iv a)
{
    return s >= 0.0f ? Iv{rd_mul(s, a.lo), ru_mul(s, a.hi)} : Iv{rd_mul(s, a.hi), ru_mul(s, a.lo)};
}
__device__ __forceinline__ Iv iv_add(Iv a, Iv b) { return {rd_add(a.lo, b.lo), ru_add(a.hi, b.hi)}; }
__device__ __forceinline__ Iv iv_mul(Iv a, Iv b)
{
    float p0 = rd_mul(a.lo, b.lo), p1 = rd_mul(a.lo, b.hi), p2 = rd_mul(a.hi, b.lo), p3 = rd_mul(a.hi, b.hi);
    float q0 = ru_mul(a.lo, b.lo), q1 = ru_mul(a.lo, b.hi), q2 = ru_mul(a.hi, b.lo), q3 = ru_mul(a.hi, b.hi);
    return {fminf(fminf(p0, p1), fminf(p2, p3)), fmaxf(fmaxf(q0, q1), fmaxf(q2, q3))};
}
__device__ __forceinline__ float iv_mag(Iv a) { return fmaxf(fabsf(a.lo), fabsf(a.hi)); }

__device__ __forceinline__ float tol32(float t) { return G * fmaxf(1.0f, fabsf(t)); }

// One axis of Aabb3::clip (node_bounds.cpp:25-44).
__device__ __forceinline__ void clip_axis(float o, float d, float inv, float lo, float hi, float &t0, float &t1,
                                          bool &ok)
{
    if (d != 0.0f) {
        float ta = (lo - o) * inv, tb = (hi - o) * inv;
        t0 = fmaxf(t0, fminf(ta, tb));
        t1 = fminf(t1, fmaxf(ta, tb));
    } else if (o < lo || o > hi) {
        ok = false;
    }
}

// The range of 1/|N| over the rectangle [cx +- hx] x [cy +- hy], with
// |N(s,t)|^2 = qc + 2 s q1 + 2 t q2 + s^2 q11 + 2 s t q12 + t^2 q22, as
// midpoint rm and radius rr; false when |N| may vanish there.
__device__ __forceinline__ bool inv_norm_range(const TriDev32 &T, float cx, float cy, float hx, float hy, float &rm,
                                               float &rr)
{
    float gs = 2.0f * hx * __fmaf_rn(cy, T.q12, __fmaf_rn(cx, T.q11, T.q1));
    float gt = 2.0f * hy * __fmaf_rn(cy, T.q22, __fmaf_rn(cx, T.q12, T.q2));
    float sx = cx * cx, sy = cy * cy, sxy = cx * cy;
    float qv = __fmaf_rn(2.0f * cy, T.q2, __fmaf_rn(2.0f * cx, T.q1, T.qc));
    qv = __fmaf_rn(sy, T.q22, __fmaf_rn(2.0f * sxy, T.q12, __fmaf_rn(sx, T.q11, qv)));
    float mag = ru_add(ru_add(fabsf(T.qc), ru_mul(2.0f, ru_add(fabsf(cx * T.q1), fabsf(cy * T.q2)))),
                       ru_add(ru_add(sx * fabsf(T.q11), sy * fabsf(T.q22)), 2.0f * fabsf(sxy * T.q12)));
    float quad = ru_add(ru_mul(hx * hx, fabsf(T.q11)), ru_mul(hy * hy, fabsf(T.q22)));
    float spread = ru_add(ru_add(fabsf(gs), fabsf(gt)), ru_mul(2.0f, ru_mul(ru_mul(hx, hy), fabsf(T.q12))));
    float err = ru_mul(G, ru_add(ru_add(mag, spread), quad));
    float q_lo = __fsub_rd(__fsub_rd(qv, spread), err);
    float q_hi = ru_add(ru_add(ru_add(qv, spread), err), quad);
    if (!(q_lo > 0.0f) || !(q_hi < INFINITY))
        return false;
    const float up = 1.0f + 9.5367431640625e-07f, dn = 1.0f - 9.5367431640625e-07f;
    float r_lo = rd_mul(rsqrtf(q_hi), dn), r_hi = ru_mul(rsqrtf(q_lo), up);
    rm = 0.5f * (r_lo + r_hi);
    rr = fmaxf(__fsub_ru(r_hi, rm), __fsub_ru(rm, r_lo));
    return true;
}

// One component of the tangent normal's enclosure m_k = (A N)_k / |N|: the
// affine form of (A N)_k = a0 + s au + t av over the rectangle (its
// coefficients rounded from double, their rounding in k0) times the interval
// rm +- rr. Then the box coordinate p_k + h m_k with h = mid +- hh and the
// base point's form (pc, pa, pb), hulled outward and widened by the ray's E.
__device__ __forceinline__ void box_axis(float a0, float au, float av, float cx, float cy, float hx, float hy,
                                         bool ok, float rm, float rr, float rowsum, float mid, float hh, float pc,
                                         float pa, float pb, float E, float &lo, float &hi, float &m_lo, float &m_hi)
{
    float c, a, b, k;
    if (ok) {
        float tu = cx * au, tv = cy * av;
        float nc = __fmaf_rn(cy, av, __fmaf_rn(cx, au, a0));
        float na = hx * au, nb = hy * av;
        float k0 = ru_mul(G, ru_add(mag3(a0, tu, tv), ru_add(fabsf(na), fabsf(nb))));
        c = rm * nc;
        a = rm * na;
        b = rm * nb;
        k = ru_fma(G, mag3(c, a, b), ru_fma(rr, ru_add(mag3(nc, na, nb), k0), ru_mul(rm, k0)));
    } else {
        // |N| can vanish over the rectangle: a unit normal maps into |m_k| <= sum_j |A_kj|
        c = a = b = 0.0f;
        k = rowsum;
    }
    float half = ru_add(ru_add(fabsf(a), fabsf(b)), k);
    m_lo = __fsub_rd(c, half);
    m_hi = __fadd_ru(c, half);
    // h m (affine_form.cpp:35-47 with h = mid +- hh), then + p
    float sc = mid * c, sa = mid * a, sb = mid * b;
    float sk = ru_fma(G, mag3(sc, sa, sb), ru_fma(hh, ru_add(mag3(c, a, b), k), ru_mul(fabsf(mid), k)));
    float tc = sc + pc, ta = sa + pa, tb = sb + pb;
    sk = ru_fma(G, mag3(tc, ta, tb), sk);
    float e = ru_add(ru_add(ru_add(fabsf(ta), fabsf(tb)), sk), E);
    lo = __fsub_rd(tc, e);
    hi = __fadd_ru(tc, e);
    float gw = ru_mul(G, fmaxf(fabsf(lo), fabsf(hi))); // the clip's own rounding
    lo = __fsub_rd(lo, gw);
    hi = __fadd_ru(hi, gw);
}

// The node test of one cell (node_bounds.cpp:83-211): the box, and at levels
// <= slab_max_level the slab, both enclosing their double counterparts.
__device__ __forceinline__ bool node_test32(const TriDev32 &T, const AssetDev &a, const Ray32 &r, int level, int i,
                                            int j, float t_min, float t_max, int bound, int slab_max_level)
{
    Node32 n = fetch_node(a, level, i, j);
    float w = pow2f(level - (__ffs(a.n_leaf) - 1));
    float u0 = ((float)i + 0.5f) * w, v0 = ((float)j + 0.5f) * w;
    float rlx = fmaxf((float)i * w, T.lo[0]), rly = fmaxf((float)j * w, T.lo[1]);
    float rhx = fminf((float)(i + 1) * w, T.hi[0]), rhy = fminf((float)(j + 1) * w, T.hi[1]);
    float cx = 0.5f * (rlx + rhx), cy = 0.5f * (rly + rhy);
    float hx = fmaxf(fmaxf(__fsub_ru(rhx, cx), __fsub_ru(cx, rlx)), 0.0f);
    float hy = fmaxf(fmaxf(__fsub_ru(rhy, cy), __fsub_ru(cy, rly)), 0.0f);
    float rm = 0.0f, rr = 0.0f;
    bool ok = inv_norm_range(T, cx, cy, hx, hy, rm, rr);
    float mid = 0.5f * (n.mn + n.mx);
    float hh = fmaxf(__fsub_ru(n.mx, mid), __fsub_ru(mid, n.mn));
    float lx, hx_, ly, hy_, lz, hz, mxl, mxh, myl, myh, mzl, mzh;
    box_axis(T.a0[0], T.au[0], T.av[0], cx, cy, hx, hy, ok, rm, rr, T.rowsum[0], mid, hh, cx, hx, 0.0f, r.ex, lx,
             hx_, mxl, mxh);
    box_axis(T.a0[1], T.au[1], T.av[1], cx, cy, hx, hy, ok, rm, rr, T.rowsum[1], mid, hh, cy, 0.0f, hy, r.ey, ly,
             hy_, myl, myh);
    box_axis(T.a0[2], T.au[2], T.av[2], cx, cy, hx, hy, ok, rm, rr, T.rowsum[2], mid, hh, 0.0f, 0.0f, 0.0f, r.ez,
             lz, hz, mzl, mzh);
    bool read_slab = level <= slab_max_level;
    float b0 = t_min, b1 = t_max;
    if (bound != 1 || !read_slab) {
        bool okc = true;
        clip_axis(r.ox, r.dx, r.ix, lx, hx_, b0, b1, okc);
        clip_axis(r.oy, r.dy, r.iy, ly, hy_, b0, b1, okc);
        clip_axis(r.oz, r.dz, r.iz, lz, hz, b0, b1, okc);
        if (!okc || b0 > b1 + tol32(fmaxf(fabsf(b0), fabsf(b1))))
            return false;
        if (bound == 0 || !read_slab)
            return true;
    }
    // slab (node_bounds.cpp:111-122, 137-179) in outward interval arithmetic
    float c0 = t_min, c1 = t_max;
    bool okc = true;
    clip_axis(r.ox, r.dx, r.ix, lx, hx_, c0, c1, okc);
    clip_axis(r.oy, r.dy, r.iy, ly, hy_, c0, c1, okc);
    if (!okc || c0 > c1 + tol32(fmaxf(fabsf(c0), fabsf(c1))))
        return false;
    Iv mx = {mxl, mxh}, my = {myl, myh}, mz = {mzl, mzh};
    Iv A = iv_add(iv_add(Iv{1.0f, 1.0f}, iv_scale(n.gu, mx)), iv_scale(n.gv, my));
    Iv B = iv_scale(-n.gu, mz), C = iv_scale(-n.gv, mz);
    float p1lo = rd_mul(n.gu, u0), p1hi = ru_mul(n.gu, u0), p2lo = rd_mul(n.gv, v0), p2hi = ru_mul(n.gv, v0);
    Iv P0 = {__fsub_rd(__fsub_rd(n.h0, p1hi), p2hi), __fsub_ru(__fsub_ru(n.h0, p1lo), p2lo)};
    Iv D = iv_mul(Iv{-P0.hi, -P0.lo}, mz);
    // the FP32 plane's gradient rounding, |dgu| s + |dgv| s, joins the remainder
    float reff = ru_fma(U2 * (0.5f * w), ru_add(fabsf(n.gu), fabsf(n.gv)), n.r);
    float R = ru_mul(reff, iv_mag(mz));
    R = ru_fma(iv_mag(A), 2.0f * r.ez, ru_fma(iv_mag(B), 2.0f * r.ex, ru_fma(iv_mag(C), 2.0f * r.ey, R)));
    float ax = __fmaf_rn(c0, r.dx, r.ox), ay = __fmaf_rn(c0, r.dy, r.oy), az = __fmaf_rn(c0, r.dz, r.oz);
    float span = c1 - c0;
    Iv F0 = iv_add(iv_add(iv_add(iv_scale(az, A), iv_scale(ax, B)), iv_scale(ay, C)), D);
    Iv F1 = iv_add(iv_add(iv_scale(r.dz, A), iv_scale(r.dx, B)), iv_scale(r.dy, C));
    float s0 = 0.0f, s1 = span;
    if (F1.lo > 0.0f)
        s1 = fminf(s1, __fdiv_ru(__fsub_ru(R, F0.lo), F1.lo));
    else if (F1.lo < 0.0f)
        s0 = fmaxf(s0, __fdiv_rd(__fsub_ru(R, F0.lo), F1.lo));
    else if (F0.lo > R)
        return false;
    if (F1.hi > 0.0f)
        s0 = fmaxf(s0, __fdiv_rd(__fsub_rd(-R, F0.hi), F1.hi));
    else if (F1.hi < 0.0f)
        s1 = fminf(s1, __fdiv_ru(__fsub_rd(-R, F0.hi), F1.hi));
    else if (F0.hi < -R)
        return false;
    if (s0 > s1 + tol32(fabsf(c0) + span))
        return false;
    if (bound == 1)
        return true;
    float t0 = fmaxf(b0, c0 + s0), t1 = fminf(b1, c0 + s1);
    return !(t0 > t1 + tol32(fmaxf(fabsf(t0), fabsf(t1))));
}

template <typename R>
__device__ __forceinline__ void load_ray(const R *rays, int64_t k, double *o, double *d, double &t_min, double &t_max)
{
    const R *r = rays + 8 * k;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o[a] = (double)r[a];
        d[a] = (double)r[3 + a];
    }
    t_min = (double)r[6];
    t_max = (double)r[7];
    dmapdev::sanitize_ray(o, d, t_min, t_max);
}

template <typename H, typename Fp>
__device__ __forceinline__ void store_hit(H *hits, int64_t k, bool found, const d64::hit64 &h, int tri, int flags)
{
    H out;
    if (found) {
        out.t = (Fp)h.t;
        out.st[0] = (Fp)h.st.x;
        out.st[1] = (Fp)h.st.y;
        out.bary[0] = (Fp)h.bary.x;
        out.bary[1] = (Fp)h.bary.y;
        out.ng[0] = (Fp)h.ng.x;
        out.ng[1] = (Fp)h.ng.y;
        out.ng[2] = (Fp)h.ng.z;
        out.tri = tri;
        out.i = (int32_t)h.i;
        out.j = (int32_t)h.j;
        out.flags = flags;
    } else {
        out.t = (Fp)INFINITY;
        out.st[0] = out.st[1] = out.bary[0] = out.bary[1] = (Fp)0;
        out.ng[0] = out.ng[1] = out.ng[2] = (Fp)0;
        out.tri = -1;
        out.i = out.j = 0;
        out.flags = flags;
    }
    hits[k] = out;
}

// A leaf cell the FP32 walk reached: first the reference's own node test of
// the cell in double (the FP32 tests, widened by the ray's rounding, admit
// more leaf cells than the FP64 walk; a cell the FP64 walk rejects has no
// leaf there), then the certified Newton leaf.
__device__ __noinline__ inline bool leaf64(const TriDev &T, const AssetDev &g, const double *o, const double *d,
                                           double t_min, double t_max, int i, int j, d64::hit64 &h, int64_t *st,
                                           const dmapk::QueryOpts &opt)
{
    d64::v3 O = d64::V3(o[0], o[1], o[2]), D = d64::V3(d[0], d[1], d[2]);
    if (!d64::leaf_cell_admitted(T, g, O, D, t_min, t_max, i, j, opt))
        return false;
    return d64::intersect_newton(T, g, O, D, t_min, t_max, i, j, h, st);
}

} // namespace d32
