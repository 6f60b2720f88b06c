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

struct hit64 { double t; v2 st, bary; v3 ng; int64_t i, j; };

__device__ void plane_basis(v3 n, v3 &d1, v3 &d2) // :222-227
{
    v3 a = fabs(n.x) < 0.9 ? V3(1.0, 0.0, 0.0) : V3(0.0, 1.0, 0.0);
    d1 = normalized3(cross3(a, n));
    d2 = cross3(n, d1);
}

__device__ bool newton_from(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max, int64_t i,
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

__device__ __forceinline__ af restricted(af f, double a, double b, double rho) // :272-276
{
    double alpha = 2.0 * a - 1.0, beta = 2.0 * b - 1.0, r = 2.0 * rho;
    return {(f.c + f.a * alpha) + f.b * beta, f.a * r, f.b * r, f.k};
}

__device__ bool sub_square_bound(const TriDev &T, const leafbound &L, double a, double b, double rho, double t_min,
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
__device__ bool intersect_newton(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max,
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

__device__ bool ray_triangle(v3 o, v3 d, double t_min, double t_max, v3 A, v3 B, v3 C, double &t, double &b1,
                             double &b2) // :230-249
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

__device__ bool intersect_two_triangle(const TriDev &T, const AssetDev &g, v3 o, v3 d, double t_min, double t_max,
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
