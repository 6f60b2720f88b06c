// The FP32 query path: the reference's walk (displaced_intersector.cpp:175-237)
// with every node test evaluated in FP32 and widened outward, so that a cell
// the double-precision test admits is admitted here too; leaves run the
// reference's certified Newton leaf in double (f64_leaf.cuh), which makes
// every reported hit the reference's own FP64 root.
//
// Conservative FP32 affine arithmetic. A form is c + a eu + b ev + rho with
// |rho| <= k; c, a, b are rounded to nearest and k is an upper bound kept
// with round-up operations. Every operation adds to k a bound on the
// rounding of the coefficients it produced: G * (sum of the magnitudes of
// the terms that entered them), G = 2^-20 (16 units in the last place, more
// than the few roundings of each step), and every input rounded from double
// (the triangle's frame, normals, pyramid nodes) carries its own rounding
// into k the same way. The Min-Range reciprocal square root is bounded with
// directed rounding around rsqrtf's documented 2-ulp error. The box of a cell
// is the outward interval hull; the tangent-space ray (transformed in double,
// then rounded) is covered by widening every box by the ray's own rounding
// error over the triangle's t range. Slab tests use directed-rounding
// interval arithmetic throughout.
//
// This translation unit is compiled with -fmad=false (the FP64 leaf must
// round like the reference); FP32 code uses explicit fmaf where it wants one.
#include "device_types.cuh"
#include "f64_math.cuh"
#include "f64_leaf.cuh"
#include "launch.h"

namespace
{
using dmapdev::AssetDev;
using dmapdev::TriDev;
using dmapdev::TriDev32;

constexpr float G = 9.5367431640625e-07f;  // 2^-20
constexpr float U2 = 1.1920928955078125e-07f; // 2^-23

struct F { float c, a, b, k; };

__device__ __forceinline__ float ru_add(float x, float y) { return __fadd_ru(x, y); }
__device__ __forceinline__ float rd_add(float x, float y) { return __fadd_rd(x, y); }
__device__ __forceinline__ float ru_mul(float x, float y) { return __fmul_ru(x, y); }
__device__ __forceinline__ float rd_mul(float x, float y) { return __fmul_rd(x, y); }
__device__ __forceinline__ float ru_fma(float x, float y, float z) { return __fmaf_ru(x, y, z); }
__device__ __forceinline__ float mag3(float x, float y, float z) { return ru_add(ru_add(fabsf(x), fabsf(y)), fabsf(z)); }

__device__ __forceinline__ F f_add(const F &x, const F &y)
{
    F r;
    r.c = x.c + y.c;
    r.a = x.a + y.a;
    r.b = x.b + y.b;
    r.k = ru_fma(G, mag3(r.c, r.a, r.b), ru_add(x.k, y.k));
    return r;
}

// x * y, both forms (affine_form.cpp:146-156 plus the rounding of c, a, b).
__device__ __forceinline__ F f_mul(const F &x, const F &y)
{
    F r;
    float ta = y.c * x.a, tb = y.c * x.b;
    r.c = x.c * y.c;
    r.a = __fmaf_rn(x.c, y.a, ta);
    r.b = __fmaf_rn(x.c, y.b, tb);
    float u = ru_add(ru_add(fabsf(x.a), fabsf(x.b)), x.k);
    float v = ru_add(ru_add(fabsf(y.a), fabsf(y.b)), y.k);
    float k = ru_fma(fabsf(y.c), x.k, ru_mul(fabsf(x.c), y.k));
    k = ru_fma(u, v, k);
    float e = ru_add(mag3(r.c, r.a, r.b), ru_add(fabsf(ta), fabsf(tb)));
    r.k = ru_fma(G, e, k);
    return r;
}

__device__ __forceinline__ float f_half(const F &x) { return ru_add(ru_add(fabsf(x.a), fabsf(x.b)), x.k); }
__device__ __forceinline__ float f_lo(const F &x) { return __fsub_rd(x.c, f_half(x)); }
__device__ __forceinline__ float f_hi(const F &x) { return __fadd_ru(x.c, f_half(x)); }

struct F3 { F x, y, z; };

// GfxExp's normalization (affine_form.cpp:187-204) with a remainder term
// that holds for any remainders: the linear-times-remainder part is bounded
// by 2 sum_i |c_i| k_i.
__device__ __forceinline__ void f_normalize(F3 &v)
{
    const F *q[3] = {&v.x, &v.y, &v.z};
    float dev2 = 0.0f, cc = 0.0f, ca = 0.0f, cb = 0.0f, ck = 0.0f, sa = 0.0f, sb = 0.0f, sc = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const F &f = *q[i];
        float dev = ru_add(ru_add(fabsf(f.a), fabsf(f.b)), f.k);
        dev2 = ru_fma(dev, dev, dev2);
        cc = __fmaf_rn(f.c, f.c, cc);
        ca = __fmaf_rn(f.c, f.a, ca);
        cb = __fmaf_rn(f.c, f.b, cb);
        ck = ru_fma(fabsf(f.c), f.k, ck);
        sc = ru_fma(fabsf(f.c), fabsf(f.c), sc);
        sa = ru_fma(fabsf(f.c), fabsf(f.a), sa);
        sb = ru_fma(fabsf(f.c), fabsf(f.b), sb);
    }
    float offset = ru_mul(0.5f, dev2);
    F l;
    l.c = cc + offset;
    l.a = 2.0f * ca;
    l.b = 2.0f * cb;
    float err = ru_add(ru_add(sc, offset), ru_mul(2.0f, ru_add(sa, sb)));
    l.k = ru_fma(G, err, ru_fma(2.0f, ck, offset));
    float lo = f_lo(l), hi = f_hi(l);
    if (!(lo > 0.0f) || !(hi < INFINITY)) {
        v.x = v.y = v.z = F{0.0f, 0.0f, 0.0f, 1.0f};
        return;
    }
    // Min-Range 1/sqrt on [lo, hi] (affine_form.cpp:173-185): any alpha >=
    // g'(hi) keeps g(t) - alpha t non-increasing, so its range is bounded by
    // its values at the two ends, taken with outward margins around rsqrtf.
    const float up = 1.0f + 9.5367431640625e-07f, dn = 1.0f - 9.5367431640625e-07f;
    float yl = rsqrtf(lo), yh = rsqrtf(hi);
    float glo_hi = ru_mul(yl, up), ghi_lo = rd_mul(yh, dn);
    float alpha = -0.5f * rd_mul(rd_mul(ghi_lo, ghi_lo), ghi_lo);
    float upper = ru_add(glo_hi, ru_mul(-alpha, lo));
    float lower = rd_add(ghi_lo, rd_mul(-alpha, hi));
    float beta = 0.5f * (upper + lower);
    float delta = fmaxf(__fsub_ru(upper, beta), __fsub_ru(beta, lower));
    F r;
    r.c = __fmaf_rn(alpha, l.c, beta);
    r.a = alpha * l.a;
    r.b = alpha * l.b;
    r.k = ru_fma(G, ru_add(mag3(r.c, r.a, r.b), fabsf(alpha * l.c)), ru_fma(-alpha, l.k, delta));
    v.x = f_mul(r, v.x);
    v.y = f_mul(r, v.y);
    v.z = f_mul(r, v.z);
}

// A * v with A the FP32 rounding of the double to_tangent: G covers the dot
// products' roundings and A's own (affine_form.cpp:210-215).
__device__ __forceinline__ F f_row(const float *A, const F3 &v)
{
    F r;
    r.c = __fmaf_rn(A[2], v.z.c, __fmaf_rn(A[1], v.y.c, A[0] * v.x.c));
    r.a = __fmaf_rn(A[2], v.z.a, __fmaf_rn(A[1], v.y.a, A[0] * v.x.a));
    r.b = __fmaf_rn(A[2], v.z.b, __fmaf_rn(A[1], v.y.b, A[0] * v.x.b));
    float kx = ru_fma(G, ru_add(mag3(v.x.c, v.x.a, v.x.b), v.x.k), v.x.k);
    float ky = ru_fma(G, ru_add(mag3(v.y.c, v.y.a, v.y.b), v.y.k), v.y.k);
    float kz = ru_fma(G, ru_add(mag3(v.z.c, v.z.a, v.z.b), v.z.k), v.z.k);
    r.k = ru_fma(fabsf(A[2]), kz, ru_fma(fabsf(A[1]), ky, ru_mul(fabsf(A[0]), kx)));
    return r;
}

struct Node32 { float h0, gu, gv, r, mn, mx; };

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
    int ri = i % m, rj = j % m;
    ri += ri < 0 ? m : 0;
    rj += rj < 0 ? m : 0;
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

struct Ray32 { float o[3], d[3], inv[3], E[3]; };

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
// separation exceeds the rounding of the test; returns 0 outside, else 1.
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

// Clip of the ray to [lo, hi] within [t0, t1] (node_bounds.cpp:25-44).
__device__ __forceinline__ bool clip32(const Ray32 &r, const float *lo, const float *hi, int axes, float &t0,
                                       float &t1)
{
    for (int a = 0; a < axes; ++a) {
        if (r.d[a] != 0.0f) {
            float ta = (lo[a] - r.o[a]) * r.inv[a], tb = (hi[a] - r.o[a]) * r.inv[a];
            float x = fminf(ta, tb), y = fmaxf(ta, tb);
            t0 = fmaxf(t0, x);
            t1 = fminf(t1, y);
        } else if (r.o[a] < lo[a] || r.o[a] > hi[a]) {
            return false;
        }
    }
    return !(t0 > t1 + tol32(fmaxf(fabsf(t0), fabsf(t1))));
}

// The node test of one cell: box, and the slab at levels <= slab_max_level.
__device__ bool node_test32(const TriDev32 &T, const AssetDev &a, const Ray32 &r, int level, int i, int j,
                            float t_min, float t_max, int bound, int slab_max_level)
{
    Node32 n = fetch_node(a, level, i, j);
    float w = ldexpf(1.0f, level) / (float)a.n_leaf;
    float u0 = ((float)i + 0.5f) * w, v0 = ((float)j + 0.5f) * w;
    float rlx = fmaxf((float)i * w, T.lo[0]), rly = fmaxf((float)j * w, T.lo[1]);
    float rhx = fminf((float)(i + 1) * w, T.hi[0]), rhy = fminf((float)(j + 1) * w, T.hi[1]);
    float cx = 0.5f * (rlx + rhx), cy = 0.5f * (rly + rhy);
    float hx = fmaxf(fmaxf(__fsub_ru(rhx, cx), __fsub_ru(cx, rlx)), 0.0f);
    float hy = fmaxf(fmaxf(__fsub_ru(rhy, cy), __fsub_ru(cy, rly)), 0.0f);
    // normal form over the rectangle (node_bounds.cpp:66-69), rounded inputs in k
    F3 N;
    F *q[3] = {&N.x, &N.y, &N.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        F &f = *q[k];
        float tu = cx * T.Mu[k], tv = cy * T.Mv[k];
        f.c = __fmaf_rn(cy, T.Mv[k], __fmaf_rn(cx, T.Mu[k], T.m0[k]));
        f.a = hx * T.Mu[k];
        f.b = hy * T.Mv[k];
        f.k = ru_mul(G, ru_add(mag3(T.m0[k], tu, tv), ru_add(fabsf(f.a), fabsf(f.b))));
    }
    f_normalize(N);
    F3 m = {f_row(T.Af[0], N), f_row(T.Af[1], N), f_row(T.Af[2], N)};
    // p + h m, hull (node_bounds.cpp:101-108)
    float mid = 0.5f * (n.mn + n.mx);
    float hh = fmaxf(__fsub_ru(n.mx, mid), __fsub_ru(mid, n.mn));
    float lo[3], hi[3];
    const F *mq[3] = {&m.x, &m.y, &m.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const F &f = *mq[k];
        F s;
        s.c = mid * f.c;
        s.a = mid * f.a;
        s.b = mid * f.b;
        float v = ru_add(ru_add(ru_add(fabsf(f.c), fabsf(f.a)), fabsf(f.b)), f.k);
        s.k = ru_fma(G, mag3(s.c, s.a, s.b), ru_fma(hh, v, ru_mul(fabsf(mid), f.k)));
        if (k == 0) {
            float c0 = s.c;
            s.c = s.c + cx;
            s.a = s.a + hx;
            s.k = ru_fma(G, ru_add(fabsf(s.c), fabsf(s.a)), ru_add(s.k, G * fabsf(c0)));
        } else if (k == 1) {
            s.c = s.c + cy;
            s.b = s.b + hy;
            s.k = ru_fma(G, ru_add(fabsf(s.c), fabsf(s.b)), s.k);
        }
        float e = ru_add(f_half(s), r.E[k]);
        lo[k] = __fsub_rd(s.c, e);
        hi[k] = __fadd_ru(s.c, e);
        float gw = ru_mul(G, fmaxf(fabsf(lo[k]), fabsf(hi[k])));
        lo[k] = __fsub_rd(lo[k], gw);
        hi[k] = __fadd_ru(hi[k], gw);
    }
    float b0 = t_min, b1 = t_max;
    bool read_slab = level <= slab_max_level;
    if (bound != 1 || !read_slab) {
        if (!clip32(r, lo, hi, 3, b0, b1))
            return false;
        if (bound == 0 || !read_slab)
            return true;
    }
    // slab (node_bounds.cpp:111-122, 137-179) in outward interval arithmetic
    float c0 = t_min, c1 = t_max;
    if (!clip32(r, lo, hi, 2, c0, c1))
        return false;
    Iv mx = {f_lo(m.x), f_hi(m.x)}, my = {f_lo(m.y), f_hi(m.y)}, mz = {f_lo(m.z), f_hi(m.z)};
    Iv A = iv_add(iv_add(Iv{1.0f, 1.0f}, iv_scale(n.gu, mx)), iv_scale(n.gv, my));
    Iv B = iv_scale(-n.gu, mz), C = iv_scale(-n.gv, mz);
    float p1lo = rd_mul(n.gu, u0), p1hi = ru_mul(n.gu, u0), p2lo = rd_mul(n.gv, v0), p2hi = ru_mul(n.gv, v0);
    Iv P0 = {__fsub_rd(__fsub_rd(n.h0, p1hi), p2hi), __fsub_ru(__fsub_ru(n.h0, p1lo), p2lo)};
    Iv D = iv_mul(Iv{-P0.hi, -P0.lo}, mz);
    float s_half = 0.5f * w;
    float reff = ru_fma(U2 * s_half, ru_add(fabsf(n.gu), fabsf(n.gv)), n.r);
    float R = ru_mul(reff, iv_mag(mz));
    R = ru_fma(iv_mag(A), 2.0f * r.E[2], ru_fma(iv_mag(B), 2.0f * r.E[0], ru_fma(iv_mag(C), 2.0f * r.E[1], R)));
    float ax = __fmaf_rn(c0, r.d[0], r.o[0]), ay = __fmaf_rn(c0, r.d[1], r.o[1]), az = __fmaf_rn(c0, r.d[2], r.o[2]);
    float span = c1 - c0;
    Iv F0 = iv_add(iv_add(iv_add(iv_scale(az, A), iv_scale(ax, B)), iv_scale(ay, C)), D);
    Iv F1 = iv_add(iv_add(iv_scale(r.d[2], A), iv_scale(r.d[0], B)), iv_scale(r.d[1], C));
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
    for (int a = 0; a < 3; ++a) {
        o[a] = (double)r[a];
        d[a] = (double)r[3 + a];
    }
    t_min = (double)r[6];
    t_max = (double)r[7];
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

__device__ __noinline__ bool leaf64(const TriDev &T, const AssetDev &g, const double *o, const double *d,
                                    double t_min, double t_max, int i, int j, d64::hit64 &h, int64_t *st)
{
    return d64::intersect_newton(T, g, d64::V3(o[0], o[1], o[2]), d64::V3(d[0], d[1], d[2]), t_min, t_max, i, j,
                                 h, st);
}

// DisplacedIntersector::intersect with the FP32 node test.
__device__ bool triangle_walk32(const TriDev32 &T, const TriDev &T64, const AssetDev &g, const double *o,
                                const double *d, double t_min, double &t_max, const dmapk::QueryOpts &opt,
                                d64::hit64 &hit, int64_t *st, float t_far)
{
    // tangent-space ray in double (the reference's), then rounded; E covers
    // that rounding over t in [0, t_far]
    Ray32 r;
    double ot[3], dt[3];
    for (int a = 0; a < 3; ++a) {
        double x = (o[0] - T.q0[0]) * T.A[a][0];
        x = __fma_rn(T.A[a][1], o[1] - T.q0[1], x);
        x = __fma_rn(T.A[a][2], o[2] - T.q0[2], x);
        double y = __fma_rn(T.A[a][2], d[2], __fma_rn(T.A[a][1], d[1], T.A[a][0] * d[0]));
        ot[a] = x;
        dt[a] = y;
        r.o[a] = (float)x;
        r.d[a] = (float)y;
        r.inv[a] = r.d[a] != 0.0f ? __frcp_rn(r.d[a]) : 0.0f;
        r.E[a] = ru_mul(2.0f * G, ru_add(ru_add(fabsf(r.o[a]), ru_mul(t_far, fabsf(r.d[a]))), 1.0f));
    }
    int si = r.d[0] < 0.0f, sj = r.d[1] < 0.0f;
    float tmin_f = __double2float_rd(t_min);
    bool found = false;
    int64_t nah = 0, lah = 0;
    const float inv_n = 1.0f / (float)g.n_leaf;
    for (int q = 0; q < T.n_roots; ++q) {
        Cell32 cur = {T.root_level, T.roots_i[q], T.roots_j[q]}, end = cur;
        cell_next(end, si, sj, T.root_level);
        int guard = 0;
        while (!(cur.level == end.level && cur.i == end.i && cur.j == end.j)) {
            if (++guard > (1 << 24))
                break; // a finite tree; the cap only protects against corrupt records
            float w = ldexpf(inv_n, cur.level);
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
            if (leaf64(T64, g, o, d, t_min, t_max, cur.i, cur.j, lh, st) && lh.t < t_max) {
                hit = lh;
                t_max = lh.t;
                found = true;
                nah = lah = 0;
                if (opt.mode == 1)
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
__global__ void __launch_bounds__(128) walk32_kernel(const TriDev32 *__restrict__ tris32,
                                                     const TriDev *__restrict__ tris64, int n_tri,
                                                     const AssetDev *__restrict__ assets, const R *__restrict__ rays,
                                                     int64_t n, dmapk::QueryOpts opt, H *__restrict__ hits,
                                                     int64_t *__restrict__ stats)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    double o[3], d[3], t_min, t_max;
    load_ray(rays, k, o, d, t_min, t_max);
    float of[3] = {(float)o[0], (float)o[1], (float)o[2]};
    float df[3] = {(float)d[0], (float)d[1], (float)d[2]};
    float invf[3];
    for (int a = 0; a < 3; ++a)
        invf[a] = df[a] != 0.0f ? __frcp_rn(df[a]) : 0.0f;
    int64_t st[DMAP_ST_N] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t *sp = stats ? st : nullptr;
    d64::hit64 best;
    int best_tri = -1;
    bool found = false;
    for (int t = 0; t < n_tri; ++t) {
        const TriDev32 &T = tris32[t];
        // the triangle's object box, widened; a float ray (rounded from the
        // caller's) meets it wherever the exact ray meets the exact box
        float t0 = __double2float_rd(t_min), t1 = __double2float_ru(t_max);
        bool ok = true;
        for (int a = 0; a < 3; ++a) {
            // where the exact ray is inside the box, |t d| <= |o| + |box|, so
            // the float ray is within u (2|o| + |box|) of it
            float bmag = fmaxf(fabsf(T.box_lo[a]), fabsf(T.box_hi[a]));
            float pad = ru_mul(2.0f * G, ru_add(ru_fma(2.0f, fabsf(of[a]), bmag), 1.0f));
            float lo = __fsub_rd(T.box_lo[a], pad), hi = __fadd_ru(T.box_hi[a], pad);
            if (df[a] != 0.0f) {
                float ta = (lo - of[a]) * invf[a], tb = (hi - of[a]) * invf[a];
                t0 = fmaxf(t0, fminf(ta, tb));
                t1 = fminf(t1, fmaxf(ta, tb));
            } else if (of[a] < lo || of[a] > hi) {
                ok = false;
            }
        }
        if (!ok || t0 > t1 + tol32(fmaxf(fabsf(t0), fabsf(t1))))
            continue;
        if (sp)
            ++st[DMAP_ST_TRI];
        float t_far = ru_add(ru_mul(t1, 1.0f + 4.0f * G), G);
        double tm = t_max;
        d64::hit64 h;
        if (triangle_walk32(T, tris64[t], assets[T.asset], o, d, t_min, tm, opt, h, sp, t_far)) {
            best = h;
            best_tri = t;
            t_max = h.t;
            found = true;
            if (opt.mode == 1)
                break;
        }
    }
    store_hit<H, Fp>(hits, k, found, best, best_tri, found ? DMAP_HIT_FP64_LEAF : 0);
    if (stats)
        for (int q = 0; q < DMAP_ST_N; ++q)
            stats[DMAP_ST_N * k + q] = st[q];
}

template <typename R, typename H, typename Fp>
cudaError_t launch(const TriDev32 *t32, const TriDev *t64, int n_tri, const AssetDev *assets, const void *rays,
                   int64_t n, const dmapk::QueryOpts &opt, void *hits, int64_t *stats, cudaStream_t stream)
{
    int threads = 128;
    int64_t blocks = (n + threads - 1) / threads;
    walk32_kernel<R, H, Fp><<<(unsigned)blocks, threads, 0, stream>>>(t32, t64, n_tri, assets,
                                                                       static_cast<const R *>(rays), n, opt,
                                                                       static_cast<H *>(hits), stats);
    return cudaGetLastError();
}

} // namespace

namespace dmapk
{
cudaError_t launch_walk32(const dmapdev::TriDev32 *t32, const dmapdev::TriDev *t64, int n_tri,
                          const dmapdev::AssetDev *assets, const void *rays, int64_t n, const QueryOpts &opt,
                          void *hits, int64_t *stats, unsigned *, cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    bool r64 = opt.ray_dtype == 2, h64 = opt.hit_dtype == 2;
    if (r64 && h64)
        return launch<double, dmapdev::Hit64, double>(t32, t64, n_tri, assets, rays, n, opt, hits, stats, stream);
    if (r64)
        return launch<double, dmapdev::Hit32, float>(t32, t64, n_tri, assets, rays, n, opt, hits, stats, stream);
    if (h64)
        return launch<float, dmapdev::Hit64, double>(t32, t64, n_tri, assets, rays, n, opt, hits, stats, stream);
    return launch<float, dmapdev::Hit32, float>(t32, t64, n_tri, assets, rays, n, opt, hits, stats, stream);
}
} // namespace dmapk
