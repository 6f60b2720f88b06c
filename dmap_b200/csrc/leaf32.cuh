// The certified Newton leaf (displaced_intersector.cpp:239-388) in FP32,
// with an FP64 Newton polish of roots whose Jacobian is ill-conditioned.
//
// The leaf's setup runs once per leaf in double: the texel's corner heights
// (HeightGrid::h at the four corners, as the reference reads them), the
// reference's normal form N_hat over the texel (normalized in double with
// the reference's arithmetic), the ray's plane basis (d1, d2) and direction
// dn. Everything the search and Newton evaluate per step is then written
// relative to the point X0 = P(c0) + h_mid N(c0) at the texel centre c0,
// projected on d1, d2 and dn and rounded to float once: the constant
// projections of X0 - o, the half-texel chart vectors e1 w/2 and e2 w/2,
// the normal form's coefficients, and the heights as h_mid plus the
// bilinear deviation from it. Every per-step quantity is then of the order
// of a texel (no cancellation against the ray's distance, which stays in
// double in Q3), so FP32 keeps about 1e-10 of absolute accuracy on the
// residual of the cube-sphere maps.
//
// sub_square_bound32 is the reference's bound with every interval widened
// outward (2G of the magnitudes of the terms that entered it, G = 2^-20),
// so a sub-square the reference keeps is kept here: the FP32 forms are the
// reference's forms term for term (h N = h_mid N + (h - h_mid) N, with
// |h_mid| k + |h - h_mid| k >= |h| k in the remainder). The search is
// intersect_newton's nearest-first order with pruning by t_max.
//
// newton32 runs newton_from's iteration (the same streak rules, clamping
// and acceptance tests) on F(a, b) in texel coordinates, with the normal's
// deviation from N(c0) evaluated without cancellation (N - N0 = dM / |M| -
// M0 D / (|M| |M0| (|M| + |M0|)), D = |M|^2 - |M0|^2). It accepts a residual
// below max(residual_tolerance, the FP32 noise of the leaf's terms). An
// accepted root is reported in double (t from Q3, the texture coordinate
// and barycentrics from the texel coordinates, the normal from the
// reference's Su x Sv at that point); when its Jacobian's condition number
// exceeds the query's polish_cond, newton_from in double restarts from it.
#pragma once
#include "f32_node.cuh"

namespace l32
{
using dmapdev::AssetDev;
using dmapdev::TriDev;
using dmapdev::TriDev32;
using namespace d64;

constexpr float kG2 = 2.0f * d32::G; // margin factor of the bound's terms

struct Leaf32
{
    double lo_s, lo_t, w; // the texel in chart coordinates
    double Q3, inv_dlen;  // dn . (X0 - o) and 1 / |d|, in double
    float q0, q1;         // d1 . (X0 - o), d2 . (X0 - o)
    // along d1, d2, dn (index k): P(a, b) - P(c0) = alpha pe1 + beta pe2
    float pe1[3], pe2[3];
    float n0[3];          // N(c0)
    float dnc[3];         // centre of N_hat minus N(c0)
    float na[3], nb[3], nk[3]; // N_hat's coefficients (texel-wide symbols) and remainder
    float mu[3], mv[3];   // Mu w/2, Mv w/2
    float Mcu, Mcv, Muu, Muv, Mvv, Mcc, Mlc; // M0 . Mu w/2, ..., |M0|^2, |M0|
    float hmid, d00, ha, hb, tw; // h(a, b) = hmid + d00 + ha a + hb b + tw a b
    float tol2;           // Newton acceptance: residual^2 below this
};

// intersect_newton's setup (:239-264) and the leaf's FP32 terms.
__device__ inline void leaf_setup32(const TriDev &T, const AssetDev &g, v3 o, v3 d, int64_t i, int64_t j, Leaf32 &L)
{
    double w = cell_width(g, 0);
    double los = i * w, lot = j * w;
    L.lo_s = los;
    L.lo_t = lot;
    L.w = w;
    double h00 = grid_h(g, los, lot), h10 = grid_h(g, los + w, lot);
    double h01 = grid_h(g, los, lot + w), h11 = grid_h(g, los + w, lot + w);
    double hm = 0.25 * ((h00 + h10) + (h01 + h11));
    L.hmid = (float)hm;
    L.d00 = (float)(h00 - hm);
    L.ha = (float)(h10 - h00);
    L.hb = (float)(h01 - h00);
    L.tw = (float)(((h11 - h10) - h01) + h00);
    double cs = los + 0.5 * w, ct = lot + 0.5 * w, hw = 0.5 * w;
    // the reference's N_hat over the texel
    af3 Nh = AF3(add3(add3(L3(T.m0), mul3(cs, L3(T.Mu))), mul3(ct, L3(T.Mv))), mul3(hw, L3(T.Mu)), mul3(hw, L3(T.Mv)));
    normalize(Nh);
    v3 M0 = tri_M(T, cs, ct);
    double Ml0 = norm3(M0);
    v3 N0 = div3(M0, Ml0);
    v3 X0 = add3(tri_P(T, cs, ct), mul3(hm, N0));
    double dlen = norm3(d);
    v3 dn = div3(d, dlen), d1, d2;
    plane_basis(dn, d1, d2);
    v3 rel = sub3(X0, o);
    L.Q3 = dot3(dn, rel);
    L.inv_dlen = 1.0 / dlen;
    L.q0 = (float)dot3(d1, rel);
    L.q1 = (float)dot3(d2, rel);
    v3 e1h = mul3(hw, L3(T.e1)), e2h = mul3(hw, L3(T.e2));
    v3 muh = mul3(hw, L3(T.Mu)), mvh = mul3(hw, L3(T.Mv));
    v3 dc = V3(Nh.x.c - N0.x, Nh.y.c - N0.y, Nh.z.c - N0.z);
    v3 na = V3(Nh.x.a, Nh.y.a, Nh.z.a), nb = V3(Nh.x.b, Nh.y.b, Nh.z.b);
    v3 basis[3] = {d1, d2, dn};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v3 e = basis[k];
        L.pe1[k] = (float)dot3(e, e1h);
        L.pe2[k] = (float)dot3(e, e2h);
        L.n0[k] = (float)dot3(e, N0);
        L.dnc[k] = (float)dot3(e, dc);
        L.na[k] = (float)dot3(e, na);
        L.nb[k] = (float)dot3(e, nb);
        // the remainder of a dot product with a unit vector: sum |e_i| k_i
        L.nk[k] = __double2float_ru((fabs(e.x) * Nh.x.k + fabs(e.y) * Nh.y.k) + fabs(e.z) * Nh.z.k);
        L.mu[k] = (float)dot3(e, muh);
        L.mv[k] = (float)dot3(e, mvh);
    }
    L.Mcu = (float)dot3(M0, muh);
    L.Mcv = (float)dot3(M0, mvh);
    L.Muu = (float)dot3(muh, muh);
    L.Muv = (float)dot3(muh, mvh);
    L.Mvv = (float)dot3(mvh, mvh);
    L.Mcc = (float)dot3(M0, M0);
    L.Mlc = (float)Ml0;
    // the FP32 noise of F: a few units in the last place of the terms of
    // the residual (the texel's own scale), or the reference's tolerance
    double scale = fabs(dot3(d1, rel)) + fabs(dot3(d2, rel)) + norm3(e1h) + norm3(e2h) +
                   fabs(hm) * (norm3(muh) + norm3(mvh)) / Ml0 +
                   (fabs(h00 - hm) + fabs(h10 - h00) + fabs(h01 - h00) + fabs(h11 - h10 - h01 + h00));
    double tol = fmax(T.residual_tol, 2.384185791015625e-07 * scale); // 2^-22
    L.tol2 = (float)(tol * tol);
}

// sub_square_bound (:266-290) over the sub-square (a, b) +- rho of the texel,
// every interval widened outward. On a pass, t_lo is the lower end of the
// sub-square's t range (rounded down to float).
__device__ inline bool sub_square_bound32(const TriDev32 &T32, const Leaf32 &L, float a, float b, float rho,
                                          double t_min, double t_max, float &t_lo)
{
    using namespace d32;
    float wf = (float)L.w;
    if (!square_meets_domain(T32, (float)L.lo_s + wf * a, (float)L.lo_t + wf * b, wf * rho))
        return false;
    const float al = 2.0f * a - 1.0f, be = 2.0f * b - 1.0f, r = 2.0f * rho;
    // the height's deviation from h_mid over the sub-square
    float tb = L.tw * b, ta = L.tw * a;
    float hc = __fmaf_rn(ta, b, __fmaf_rn(L.hb, b, __fmaf_rn(L.ha, a, L.d00)));
    float hA = (L.ha + tb) * rho, hB = (L.hb + ta) * rho;
    float hK = ru_mul(ru_mul(fabsf(L.tw), rho), rho);
    float hmag = ru_add(ru_add(fabsf(L.d00), fabsf(L.ha * a)), ru_add(fabsf(L.hb * b), fabsf(ta * b)));
    hmag = ru_add(hmag, ru_add(fabsf(L.ha), ru_add(fabsf(L.hb), fabsf(L.tw)))); // hA, hB's own terms
    const float hm = L.hmid, ahm = fabsf(hm);
    float lo3 = 0.0f, hi3 = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float dn_ = __fmaf_rn(L.nb[k], be, __fmaf_rn(L.na[k], al, L.dnc[k])); // N_r centre - N(c0)
        float ncr = L.n0[k] + dn_;
        float nar = L.na[k] * r, nbr = L.nb[k] * r, nkr = L.nk[k];
        float p = __fmaf_rn(be, L.pe2[k], al * L.pe1[k]);
        float c = __fmaf_rn(hc, ncr, __fmaf_rn(hm, dn_, p));
        float A = __fmaf_rn(ncr, hA, __fmaf_rn(hc, nar, __fmaf_rn(hm, nar, r * L.pe1[k])));
        float B = __fmaf_rn(ncr, hB, __fmaf_rn(hc, nbr, __fmaf_rn(hm, nbr, r * L.pe2[k])));
        float u = ru_add(ru_add(fabsf(hA), fabsf(hB)), hK);
        float v = ru_add(ru_add(fabsf(nar), fabsf(nbr)), nkr);
        float K = ru_add(ru_add(ru_mul(ahm, nkr), ru_mul(fabsf(ncr), hK)), ru_add(ru_mul(fabsf(hc), nkr), ru_mul(u, v)));
        // magnitudes of every term that entered c, A and B
        float mag = ru_add(ru_add(fabsf(al * L.pe1[k]), fabsf(be * L.pe2[k])),
                           ru_mul(ahm, ru_add(ru_add(fabsf(L.dnc[k]), fabsf(L.na[k] * al)), fabsf(L.nb[k] * be))));
        mag = ru_add(mag, ru_mul(ru_add(hmag, fabsf(hc)), ru_add(ru_add(fabsf(L.n0[k]), fabsf(dn_)), v)));
        mag = ru_add(mag, ru_add(ru_mul(r, ru_add(fabsf(L.pe1[k]), fabsf(L.pe2[k]))), ru_mul(ahm, v)));
        float half = ru_add(ru_add(fabsf(A), fabsf(B)), ru_fma(kG2, mag, K));
        if (k < 2) {
            float q = k == 0 ? L.q0 : L.q1;
            float f = q + c;
            half = ru_fma(kG2, ru_add(fabsf(q), fabsf(c)), half);
            if (!(fabsf(f) <= half)) // F_k's interval misses 0 (NaN fails too)
                return false;
        } else {
            lo3 = __fsub_rd(c, half);
            hi3 = __fadd_ru(c, half);
        }
    }
    double tl = (L.Q3 + (double)lo3) * L.inv_dlen, th = (L.Q3 + (double)hi3) * L.inv_dlen;
    t_lo = __double2float_rd(tl);
    return tl < t_max && th > t_min;
}

struct Root32
{
    float a, b;
    float along_rel;   // along - Q3
    float J00, J01, J10, J11;
};

// newton_from (:325-388) in texel coordinates from (a, b).
__device__ inline bool newton32(const TriDev &T, const Leaf32 &L, float a, float b, Root32 &root, int64_t &iters)
{
    float prev = INFINITY;
    int err_streak = 0, behind_streak = 0, invalid_streak = 0;
    for (int iter = 0; iter < 20; ++iter) {
        ++iters;
        const float al = 2.0f * a - 1.0f, be = 2.0f * b - 1.0f;
        // N(a, b) - N(c0) without cancellation
        float D = __fmaf_rn(2.0f, __fmaf_rn(be, L.Mcv, al * L.Mcu),
                            __fmaf_rn(be * be, L.Mvv, __fmaf_rn(2.0f * al * be, L.Muv, al * al * L.Muu)));
        float Ml = sqrtf(L.Mcc + D);
        float iM = 1.0f / Ml;
        float cD = D * iM / (L.Mlc * (Ml + L.Mlc));
        float NMu = (L.Mcu + __fmaf_rn(be, L.Muv, al * L.Muu)) * iM; // N . Mu w/2
        float NMv = (L.Mcv + __fmaf_rn(be, L.Mvv, al * L.Muv)) * iM;
        float dh = __fmaf_rn(L.tw * a, b, __fmaf_rn(L.hb, b, __fmaf_rn(L.ha, a, L.d00)));
        float dha = L.ha + L.tw * b, dhb = L.hb + L.tw * a; // dh/da, dh/db
        float hfull = L.hmid + dh;
        float F[3], Ja[3], Jb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float dM = __fmaf_rn(be, L.mv[k], al * L.mu[k]);
            float dN = __fmaf_rn(-L.n0[k] * L.Mlc, cD, dM * iM); // N_k - N0_k
            float Nk = L.n0[k] + dN;
            F[k] = __fmaf_rn(dh, Nk, __fmaf_rn(L.hmid, dN, __fmaf_rn(be, L.pe2[k], al * L.pe1[k])));
            // dN/da = (2 mu - N (N . 2 mu)) / |M|, the same for b
            float dNa = 2.0f * (L.mu[k] - Nk * NMu) * iM, dNb = 2.0f * (L.mv[k] - Nk * NMv) * iM;
            Ja[k] = __fmaf_rn(hfull, dNa, __fmaf_rn(dha, Nk, 2.0f * L.pe1[k]));
            Jb[k] = __fmaf_rn(hfull, dNb, __fmaf_rn(dhb, Nk, 2.0f * L.pe2[k]));
        }
        float F0 = L.q0 + F[0], F1 = L.q1 + F[1];
        float err2 = __fmaf_rn(F1, F1, F0 * F0);
        double along = L.Q3 + (double)F[2];
        err_streak = err2 > prev ? err_streak + 1 : 0;
        behind_streak = along < 0.0 ? behind_streak + 1 : 0;
        if (err_streak >= 2 || behind_streak >= 2)
            return false;
        prev = err2;
        if (err2 < L.tol2) {
            root = {a, b, F[2], Ja[0], Jb[0], Ja[1], Jb[1]};
            return true;
        }
        float det = Ja[0] * Jb[1] - Jb[0] * Ja[1];
        if (det == 0.0f)
            return false;
        float id = 1.0f / det;
        a -= (Jb[1] * F0 - Jb[0] * F1) * id;
        b -= (-Ja[1] * F0 + Ja[0] * F1) * id;
        bool outside = !(a >= 0.0f && a <= 1.0f && b >= 0.0f && b <= 1.0f) ||
                       !uv_inside(T, V2(L.lo_s + L.w * (double)a, L.lo_t + L.w * (double)b));
        if (outside) {
            if (++invalid_streak >= 3)
                return false;
            a = fminf(fmaxf(a, 0.0f), 1.0f);
            b = fminf(fmaxf(b, 0.0f), 1.0f);
        } else {
            invalid_streak = 0;
        }
    }
    return false;
}

// An FP32 root as a hit (newton_from's acceptance tests, :350-364), with the
// FP64 polish when the Jacobian is ill-conditioned. The texel (lo_s, lo_t,
// w) and the ray's Q3 and 1/|d| come from the leaf's setup. flags gets
// DMAP_HIT_FP64_LEAF | DMAP_HIT_POLISHED when the reported root is the FP64
// Newton root. Kept out of line: it runs once per accepted root.
static __device__ __noinline__ bool accept_root(const TriDev &T, const AssetDev &g, double lo_s, double lo_t, double w,
                                         double Q3, double inv_dlen, v3 o, v3 d, double t_min, double t_max,
                                         int64_t i, int64_t j, Root32 R, double polish_cond, hit64 &hit, int &flags,
                                         int64_t &iters)
{
    double along = Q3 + (double)R.along_rel;
    v2 st = V2(lo_s + w * (double)R.a, lo_t + w * (double)R.b);
    if (along < 0.0 || !uv_inside(T, st))
        return false;
    double t_hit = along * inv_dlen;
    if (t_hit <= t_min || t_hit >= t_max)
        return false;
    float fro = R.J00 * R.J00 + R.J01 * R.J01 + R.J10 * R.J10 + R.J11 * R.J11;
    float det = fabsf(R.J00 * R.J11 - R.J01 * R.J10);
    if (fro > (float)polish_cond * det) { // cond(J) <= |J|_F^2 / |det J|
        // the reference's Newton from the FP32 root, its t judged here: a
        // root at or beyond t_max is the one the search already holds (found
        // again from another start) or a farther one
        hit64 h;
        int64_t it = 0;
        bool ok = newton_from(T, g, o, d, t_min, INFINITY, i, j, st, h, it);
        iters += it;
        if (ok) {
            if (h.t >= t_max)
                return false;
            hit = h;
            flags = DMAP_HIT_FP64_LEAF | DMAP_HIT_POLISHED;
            return true;
        }
    }
    hit.t = t_hit;
    hit.st = st;
    hit.bary = tri_bary(T, st.x, st.y);
    // the reference's normal, Su x Sv, at the root
    nframe f = normal_frame_at(T, st.x, st.y);
    double h;
    v2 gh;
    grid_h_grad(g, st.x, st.y, h, gh);
    v3 Su = add3(add3(L3(T.e1), mul3(gh.x, f.N)), mul3(h, f.Nu));
    v3 Sv = add3(add3(L3(T.e2), mul3(gh.y, f.N)), mul3(h, f.Nv));
    hit.ng = normalized3(cross3(Su, Sv));
    hit.i = i;
    hit.j = j;
    flags = 0;
    return true;
}

struct Ent32 { float a, b, t_lo; int depth; };

// intersect_newton + search_leaf (:239-264, :292-323) in FP32, with the
// explicit stack of the FP64 leaf (siblings pushed in reverse sorted order).
__device__ inline bool intersect_newton32(const TriDev &T, const TriDev32 &T32, const AssetDev &g, v3 o, v3 d,
                                          double t_min, double t_max, int64_t i, int64_t j, double polish_cond,
                                          hit64 &hit, int &flags, int64_t *st)
{
    constexpr int kDepth = 5; // subdivision_depth
    Leaf32 L;
    leaf_setup32(T, g, o, d, i, j, L);
    bool found = false;
    int64_t subs = 0, iters = 0;
    Ent32 stack[4 * kDepth + 4];
    int sp = 0;
    stack[sp++] = {0.5f, 0.5f, -INFINITY, 0};
    bool first = true;
    while (sp > 0) {
        Ent32 e = stack[--sp];
        if (!first && (double)e.t_lo >= t_max)
            continue;
        first = false;
        if (e.depth == kDepth) {
            Root32 R;
            if (newton32(T, L, e.a, e.b, R, iters)) {
                hit64 h;
                int fl = 0;
                if (accept_root(T, g, L.lo_s, L.lo_t, L.w, L.Q3, L.inv_dlen, o, d, t_min, t_max, i, j, R,
                                polish_cond, h, fl, iters)) {
                    hit = h;
                    flags = fl;
                    t_max = h.t;
                    found = true;
                }
            }
            continue;
        }
        Ent32 ch[4];
        int n = 0;
        float r = __int_as_float((125 - e.depth) << 23); // half of the entry's rho = 0.5 * 2^-depth
        for (int q = 0; q < 4; ++q) {
            float ca = e.a + ((q & 1) ? r : -r), cb = e.b + ((q & 2) ? r : -r), tl;
            ++subs;
            if (sub_square_bound32(T32, L, ca, cb, r, t_min, t_max, tl))
                ch[n++] = {ca, cb, tl, e.depth + 1};
        }
        for (int p = 1; p < n; ++p)
            for (int q = p; q > 0 && ch[q].t_lo < ch[q - 1].t_lo; --q) {
                Ent32 x = ch[q];
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

} // namespace l32
