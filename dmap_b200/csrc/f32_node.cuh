// Outward-rounded FP32 node tests of the displaced-surface walk (see
// walk32.cu for the scheme), shared by the FP32 kernels.
#pragma once
#include "device_types.cuh"
#include "f64_math.cuh"
#include "f64_leaf.cuh"
#include "launch.h"


namespace d32
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

// An outward affine enclosure of m = A N(s,t) / |N(s,t)| over the rectangle
// [cx +- hx] x [cy +- hy]: the tangent-space normal A N = a0 + s au + t av
// is affine in the cell symbols, |N|^2 is a quadratic whose range over the
// rectangle bounds 1/|N| to [r_lo, r_hi], and the product of an affine form
// with an interval adds half the interval's width times the form's magnitude
// to the remainder. The reference normalizes with the Min-Range affine
// reciprocal square root and maps through A afterwards
// (node_bounds.cpp:101-103); both enclose the same set.
__device__ __forceinline__ void tangent_normal_bound(const TriDev32 &T, float cx, float cy, float hx, float hy, F3 &m)
{
    float gs = 2.0f * hx * __fmaf_rn(cy, T.q12, __fmaf_rn(cx, T.q11, T.q1));
    float gt = 2.0f * hy * __fmaf_rn(cy, T.q22, __fmaf_rn(cx, T.q12, T.q2));
    float sx = cx * cx, sy = cy * cy, sxy = cx * cy;
    float qv = __fmaf_rn(2.0f * cy, T.q2, __fmaf_rn(2.0f * cx, T.q1, T.qc));
    qv = __fmaf_rn(sy, T.q22, __fmaf_rn(2.0f * sxy, T.q12, __fmaf_rn(sx, T.q11, qv)));
    float mag = ru_add(ru_add(fabsf(T.qc), ru_mul(2.0f, ru_add(fabsf(cx * T.q1), fabsf(cy * T.q2)))),
                       ru_add(ru_add(sx * fabsf(T.q11), sy * fabsf(T.q22)), 2.0f * fabsf(sxy * T.q12)));
    float cross = ru_mul(2.0f, ru_mul(ru_mul(hx, hy), fabsf(T.q12)));
    float spread = ru_add(ru_add(fabsf(gs), fabsf(gt)), cross);
    float err = ru_mul(G, ru_add(ru_add(mag, spread), ru_add(hx * hx * fabsf(T.q11), hy * hy * fabsf(T.q22))));
    float q_lo = __fsub_rd(__fsub_rd(qv, spread), err);
    float q_hi = ru_add(ru_add(ru_add(qv, spread), err), ru_add(ru_mul(hx * hx, fabsf(T.q11)), ru_mul(hy * hy, fabsf(T.q22))));
    if (!(q_lo > 0.0f) || !(q_hi < INFINITY)) {
        // |N| can vanish over the rectangle: a unit normal maps into |m_i| <= sum_j |A_ij|
        m.x = F{0.0f, 0.0f, 0.0f, T.rowsum[0]};
        m.y = F{0.0f, 0.0f, 0.0f, T.rowsum[1]};
        m.z = F{0.0f, 0.0f, 0.0f, T.rowsum[2]};
        return;
    }
    const float up = 1.0f + 9.5367431640625e-07f, dn = 1.0f - 9.5367431640625e-07f;
    float r_lo = rd_mul(rsqrtf(q_hi), dn), r_hi = ru_mul(rsqrtf(q_lo), up);
    float rm = 0.5f * (r_lo + r_hi);
    float rr = fmaxf(__fsub_ru(r_hi, rm), __fsub_ru(rm, r_lo));
    F *out[3] = {&m.x, &m.y, &m.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float tu = cx * T.au[k], tv = cy * T.av[k];
        float c = __fmaf_rn(cy, T.av[k], __fmaf_rn(cx, T.au[k], T.a0[k]));
        float a = hx * T.au[k], b = hy * T.av[k];
        float k0 = ru_mul(G, ru_add(mag3(T.a0[k], tu, tv), ru_add(fabsf(a), fabsf(b))));
        F &f = *out[k];
        f.c = rm * c;
        f.a = rm * a;
        f.b = rm * b;
        float magm = ru_add(mag3(c, a, b), k0);
        f.k = ru_fma(G, mag3(f.c, f.a, f.b), ru_fma(rr, magm, ru_mul(rm, k0)));
    }
}

// The node test of one cell: box, and the slab at levels <= slab_max_level.
__device__ inline bool node_test32(const TriDev32 &T, const AssetDev &a, const Ray32 &r, int level, int i, int j,
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
    F3 m;
    tangent_normal_bound(T, cx, cy, hx, hy, m);
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

__device__ __noinline__ inline bool leaf64(const TriDev &T, const AssetDev &g, const double *o, const double *d,
                                    double t_min, double t_max, int i, int j, d64::hit64 &h, int64_t *st)
{
    return d64::intersect_newton(T, g, d64::V3(o[0], o[1], o[2]), d64::V3(d[0], d[1], d[2]), t_min, t_max, i, j,
                                 h, st);
}

} // namespace d32
