// The certified Newton leaf in double with the reference's operation order
// (displaced_intersector.cpp:22-27,239-440: plane_basis, newton_from,
// sub_square_bound, search_leaf, intersect_newton, the two-triangle leaf).
// Included by translation units compiled with -fmad=false.
#pragma once
#include "device_types.cuh"
#include "f64_math.cuh"

namespace d64
{

struct hit64 { double t; v2 st, bary; v3 ng; int64_t i, j; };

__device__ inline void plane_basis(v3 n, v3 &d1, v3 &d2) // :22-27
{
    v3 a = fabs(n.x) < 0.9 ? V3(1.0, 0.0, 0.0) : V3(0.0, 1.0, 0.0);
    d1 = normalized3(cross3(a, n));
    d2 = cross3(n, d1);
}

__device__ inline bool newton_from(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max, int64_t i,
                            int64_t j, v2 guess, hit64 &hit, int64_t &iters) // :325-388
{
    double w = cell_width(g, 0);
    v2 lo = {i * w, j * w}, hi = {(i + 1) * w, (j + 1) * w};
    double d_len = norm3(d);
    v3 dn = div3(d, d_len), d1, d2;
    plane_basis(dn, d1, d2);
    double prev_err2 = INFINITY;
    int err_streak = 0, behind_streak = 0, invalid_streak = 0;
    for (int iter = 0; iter < 20; ++iter) {
        ++iters;
        double s = guess.x, t = guess.y;
        nframe f = normal_frame_at(T, s, t);
        double h;
        v2 gh;
        grid_h_grad(g, s, t, h, gh);
        v3 S = add3(tri_P(T, s, t), mul3(h, f.N));
        v3 delta = sub3(S, o);
        v2 F = {dot3(delta, d1), dot3(delta, d2)};
        double err2 = F.x * F.x + F.y * F.y;
        double along = dot3(delta, dn);
        err_streak = err2 > prev_err2 ? err_streak + 1 : 0;
        behind_streak = along < 0.0 ? behind_streak + 1 : 0;
        if (err_streak >= 2 || behind_streak >= 2)
            return false;
        prev_err2 = err2;
        v3 Su = add3(add3(L3(T.e1), mul3(gh.x, f.N)), mul3(h, f.Nu));
        v3 Sv = add3(add3(L3(T.e2), mul3(gh.y, f.N)), mul3(h, f.Nv));
        if (err2 < T.residual_tol * T.residual_tol) {
            if (along < 0.0 || !uv_inside(T, guess))
                return false;
            double t_hit = along / d_len;
            if (t_hit <= t_min || t_hit >= t_max)
                return false;
            hit.t = t_hit;
            hit.st = guess;
            hit.bary = tri_bary(T, s, t);
            hit.ng = normalized3(cross3(Su, Sv));
            hit.i = i;
            hit.j = j;
            return true;
        }
        double J00 = dot3(d1, Su), J01 = dot3(d1, Sv), J10 = dot3(d2, Su), J11 = dot3(d2, Sv);
        double det = J00 * J11 - J01 * J10;
        if (det == 0.0)
            return false;
        v2 step = {(J11 * F.x - J01 * F.y) / det, (-J10 * F.x + J00 * F.y) / det};
        guess = sub2(guess, step);
        bool outside = guess.x < lo.x || guess.x > hi.x || guess.y < lo.y || guess.y > hi.y || !uv_inside(T, guess);
        if (outside) {
            if (++invalid_streak >= 3)
                return false;
            guess = min2(max2(guess, lo), hi);
        } else {
            invalid_streak = 0;
        }
    }
    return false;
}

struct leafbound { v2 lo; double w, h00, h10, h01, h11; af3 N_hat; v3 o, dn, d1, d2; double d_len; };

__device__ __forceinline__ af restricted(af f, double a, double b, double rho) // :72-76
{
    double alpha = 2.0 * a - 1.0, beta = 2.0 * b - 1.0, r = 2.0 * rho;
    return {(f.c + f.a * alpha) + f.b * beta, f.a * r, f.b * r, f.k};
}

__device__ inline bool sub_square_bound(const TriDev &T, const leafbound &L, double a, double b, double rho, double t_min,
                                 double t_max, double &t_lo) // :266-290
{
    v2 c = add2(L.lo, mul2(L.w, V2(a, b)));
    if (classify_square(T, c, L.w * rho) == OUTSIDE)
        return false;
    double Tw = ((L.h11 - L.h10) - L.h01) + L.h00;
    double ha = L.h10 - L.h00, hb = L.h01 - L.h00;
    af h = AF(((L.h00 + ha * a) + hb * b) + Tw * a * b, (ha + Tw * b) * rho, (hb + Tw * a) * rho, fabs(Tw) * rho * rho);
    double wr = L.w * rho;
    af3 P = AF3(tri_P(T, c.x, c.y), mul3(wr, L3(T.e1)), mul3(wr, L3(T.e2)));
    af3 Nr = {restricted(L.N_hat.x, a, b, rho), restricted(L.N_hat.y, a, b, rho), restricted(L.N_hat.z, a, b, rho)};
    af3 S = add(P, scale_form(h, Nr));
    af F1 = dot(L.d1, S), F2 = dot(L.d2, S);
    F1.c -= dot3(L.d1, L.o);
    F2.c -= dot3(L.d2, L.o);
    ivl i1 = interval(F1), i2 = interval(F2);
    if (!(i1.lo <= 0.0 && 0.0 <= i1.hi) || !(i2.lo <= 0.0 && 0.0 <= i2.hi))
        return false;
    af along = dot(L.dn, S);
    along.c -= dot3(L.dn, L.o);
    ivl range = interval(along);
    t_lo = range.lo / L.d_len;
    return t_lo < t_max && range.hi / L.d_len > t_min;
}

struct leafent { double a, b, t_lo; int depth; };

// intersect_newton + search_leaf (:239-264, :292-323) with an explicit
// stack: a popped entry is a call of search_leaf at its depth; siblings are
// pushed in reverse sorted order so the nearest comes off first, and the
// t_lo >= t_max test at the pop equals the sorted loop's break, since t_max
// only shrinks.
__device__ inline bool intersect_newton(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max,
                                 int64_t i, int64_t j, hit64 &hit, int64_t *st)
{
    constexpr int kDepth = 5; // subdivision_depth
    leafbound L;
    L.w = cell_width(g, 0);
    L.lo = {i * L.w, j * L.w};
    L.h00 = grid_h(g, L.lo.x, L.lo.y);
    L.h10 = grid_h(g, L.lo.x + L.w, L.lo.y);
    L.h01 = grid_h(g, L.lo.x, L.lo.y + L.w);
    L.h11 = grid_h(g, L.lo.x + L.w, L.lo.y + L.w);
    v2 c = add2(L.lo, V2(0.5 * L.w, 0.5 * L.w));
    double hw = 0.5 * L.w;
    L.N_hat = AF3(add3(add3(L3(T.m0), mul3(c.x, L3(T.Mu))), mul3(c.y, L3(T.Mv))), mul3(hw, L3(T.Mu)),
                  mul3(hw, L3(T.Mv)));
    normalize(L.N_hat);
    L.o = o;
    L.d_len = norm3(d);
    L.dn = div3(d, L.d_len);
    plane_basis(L.dn, L.d1, L.d2);

    bool found = false;
    int64_t subs = 0, iters = 0;
    leafent stack[4 * kDepth + 4];
    int sp = 0;
    stack[sp++] = {0.5, 0.5, -INFINITY, 0};
    bool first = true;
    while (sp > 0) {
        leafent e = stack[--sp];
        if (!first && e.t_lo >= t_max)
            continue;
        first = false;
        double rho = ldexp(0.5, -e.depth);
        if (e.depth == kDepth) {
            hit64 h;
            if (newton_from(T, g, o, d, t_min, t_max, i, j, add2(L.lo, mul2(L.w, V2(e.a, e.b))), h, iters)) {
                hit = h;
                t_max = h.t;
                found = true;
            }
            continue;
        }
        leafent ch[4];
        int n = 0;
        double r = 0.5 * rho;
        for (int q = 0; q < 4; ++q) {
            double ca = e.a + ((q & 1) ? r : -r), cb = e.b + ((q & 2) ? r : -r), t_lo;
            ++subs;
            if (sub_square_bound(T, L, ca, cb, r, t_min, t_max, t_lo))
                ch[n++] = {ca, cb, t_lo, e.depth + 1};
        }
        for (int p = 1; p < n; ++p)
            for (int q = p; q > 0 && ch[q].t_lo < ch[q - 1].t_lo; --q) {
                leafent x = ch[q];
                ch[q] = ch[q - 1];
                ch[q - 1] = x;
            }
        for (int q = n - 1; q >= 0; --q)
            stack[sp++] = ch[q];
    }
    if (st) {
        st[DMAP_ST_SUB] += subs;
        st[DMAP_ST_NEWTON] += iters;
    }
    return found;
}

__device__ inline bool ray_triangle(v3 o, v3 d, double t_min, double t_max, v3 A, v3 B, v3 C, double &t, double &b1,
                             double &b2) // :30-49
{
    v3 e1 = sub3(B, A), e2 = sub3(C, A);
    v3 p = cross3(d, e2);
    double det = dot3(e1, p);
    if (det == 0.0)
        return false;
    double inv = 1.0 / det;
    v3 s = sub3(o, A);
    b1 = dot3(s, p) * inv;
    if (b1 < 0.0 || b1 > 1.0)
        return false;
    v3 q = cross3(s, e1);
    b2 = dot3(d, q) * inv;
    if (b2 < 0.0 || b1 + b2 > 1.0)
        return false;
    t = dot3(e2, q) * inv;
    return t > t_min && t < t_max;
}

__device__ inline bool intersect_two_triangle(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max,
                                       int64_t i, int64_t j, hit64 &hit) // :390-426
{
    double w = cell_width(g, 0);
    v2 st00 = {i * w, j * w}, st10 = {(i + 1) * w, j * w}, st01 = {i * w, (j + 1) * w},
       st11 = {(i + 1) * w, (j + 1) * w};
    v3 S00 = displaced_position(T, g, st00.x, st00.y), S10 = displaced_position(T, g, st10.x, st10.y);
    v3 S01 = displaced_position(T, g, st01.x, st01.y), S11 = displaced_position(T, g, st11.x, st11.y);
    v3 A[2] = {S00, S10}, B[2] = {S10, S11}, C[2] = {S01, S01};
    v2 a[2] = {st00, st10}, b[2] = {st10, st11}, c[2] = {st01, st01};
    bool found = false;
    for (int k = 0; k < 2; ++k) {
        double t, b1, b2;
        if (!ray_triangle(o, d, t_min, t_max, A[k], B[k], C[k], t, b1, b2))
            continue;
        v2 st = add2(add2(mul2((1.0 - b1) - b2, a[k]), mul2(b1, b[k])), mul2(b2, c[k]));
        if (!uv_inside(T, st))
            continue;
        hit.t = t;
        hit.st = st;
        hit.bary = tri_bary(T, st.x, st.y);
        hit.ng = normalized3(cross3(sub3(B[k], A[k]), sub3(C[k], A[k])));
        hit.i = i;
        hit.j = j;
        t_max = t;
        found = true;
    }
    return found;
}


} // namespace d64
