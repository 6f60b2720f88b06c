// Per-triangle setup (one thread per base triangle), in double with the
// reference's operation order (compiled with -fmad=false):
//   BaseTriangle general-chart constructor   displaced_surface.cpp:54-91
//   tangent_frame                             node_bounds.cpp:13-23
//   UvTriangle                                uv_clip.cpp:10-25
//   footprint_roots                           descent_sampler.cpp:66-83
//   DisplacedIntersector roots, tolerance     displaced_intersector.cpp:135-151
//   triangle_height_range (explicit stack)    node_bounds.cpp:218-249
//   triangle_aabb                             node_bounds.cpp:251-269
// and the FP32 record derived from it, rounded outward where it bounds.
#include "device_types.cuh"
#include "f64_math.cuh"
#include "launch.h"

namespace
{
using namespace d64;
using dmapdev::AssetDev;
using dmapdev::TriDev;
using dmapdev::TriDev32;

__device__ void footprint_roots(const TriDev &T, int n_leaf, int &level, int64_t &i0, int64_t &j0)
{
    for (level = 0; level < 60; ++level) {
        double w = ldexp(1.0, level) / n_leaf;
        int64_t ilo = (int64_t)floor(T.lo[0] / w), ihi = (int64_t)ceil(T.hi[0] / w) - 1;
        int64_t jlo = (int64_t)floor(T.lo[1] / w), jhi = (int64_t)ceil(T.hi[1] / w) - 1;
        if (ihi - ilo <= 1 && jhi - jlo <= 1) {
            i0 = ilo;
            j0 = jlo;
            return;
        }
    }
    i0 = j0 = 0;
}

// The height channel of a node: FP64 pyramid when resident, else the
// outward-rounded FP32 one (conservative, exact for f32 grids at scale 1).
__device__ void node_hrange(const AssetDev &a, int level, int64_t i, int64_t j, double &lo, double &hi)
{
    if (a.pyr64) {
        node n = pyramid_node(a, level, i, j);
        lo = n.h_min;
        hi = n.h_max;
        return;
    }
    int lv = level >= a.n_levels ? a.n_levels - 1 : level;
    int64_t m = a.n_leaf >> lv;
    int64_t ri = level >= a.n_levels ? 0 : ((i % m) + m) % m;
    int64_t rj = level >= a.n_levels ? 0 : ((j % m) + m) % m;
    const float *p = a.pyr32 + 8 * (a.level_off[lv] + rj * m + ri);
    lo = (double)p[6];
    hi = (double)p[7];
}

// The base triangle's chart. A vertex record (24 doubles: p0 p1 p2 m0 m1 m2
// t0 t1 t2) runs the general-chart constructor; a chart record (37 doubles:
// p0 p1 p2, q0 e1 e2, t0 t1 t2, m0 Mu Mv, J row-major) carries a
// BaseTriangle the caller already built, whose fields are taken as they are.
__device__ bool init_triangle(TriDev &T, const double *r, bool chart)
{
    v3 p0 = L3(r), p1 = L3(r + 3), p2 = L3(r + 6);
    v2 t0 = L2(r + 18), t1 = L2(r + 20), t2 = L2(r + 22);
    T.t0[0] = t0.x, T.t0[1] = t0.y, T.t1[0] = t1.x, T.t1[1] = t1.y, T.t2[0] = t2.x, T.t2[1] = t2.y;
    v3 eb1 = sub3(p1, p0), eb2 = sub3(p2, p0);
    v3 wn = cross3(eb1, eb2); // winding_normal (displaced_surface.cpp:158)
    T.wn[0] = wn.x, T.wn[1] = wn.y, T.wn[2] = wn.z;
    double T00 = t1.x - t0.x, T10 = t1.y - t0.y, T01 = t2.x - t0.x, T11 = t2.y - t0.y;
    double det = T00 * T11 - T10 * T01;
    if (!(fabs(det) > 1e-30))
        return false;
    if (chart) {
        for (int a = 0; a < 3; ++a) {
            T.q0[a] = r[9 + a];
            T.e1[a] = r[12 + a];
            T.e2[a] = r[15 + a];
            T.m0[a] = r[24 + a];
            T.Mu[a] = r[27 + a];
            T.Mv[a] = r[30 + a];
        }
        T.J[0][0] = r[33];
        T.J[0][1] = r[34];
        T.J[1][0] = r[35];
        T.J[1][1] = r[36];
    } else {
        v3 m0 = L3(r + 9), m1 = L3(r + 12), m2 = L3(r + 15);
        v3 Mb1 = sub3(m1, m0), Mb2 = sub3(m2, m0);
        double invdet = 1.0 / det;
        T.J[0][0] = T11 * invdet;
        T.J[1][0] = -T10 * invdet;
        T.J[0][1] = -T01 * invdet;
        T.J[1][1] = T00 * invdet;
        v2 c = {(-T.J[0][0]) * t0.x + (-T.J[0][1]) * t0.y, (-T.J[1][0]) * t0.x + (-T.J[1][1]) * t0.y};
        for (int a = 0; a < 3; ++a) {
            double E0 = comp(eb1, a), E1 = comp(eb2, a), D0 = comp(Mb1, a), D1 = comp(Mb2, a);
            T.q0[a] = comp(p0, a) + (E0 * c.x + E1 * c.y);
            T.e1[a] = E0 * T.J[0][0] + E1 * T.J[1][0];
            T.e2[a] = E0 * T.J[0][1] + E1 * T.J[1][1];
            T.m0[a] = comp(m0, a) + (D0 * c.x + D1 * c.y);
            T.Mu[a] = D0 * T.J[0][0] + D1 * T.J[1][0];
            T.Mv[a] = D0 * T.J[0][1] + D1 * T.J[1][1];
        }
    }
    // tangent frame: [e1 e2 ng]^-1 by cofactors
    v3 ng = normalized3(cross3(L3(T.e1), L3(T.e2)));
    T.ng[0] = ng.x, T.ng[1] = ng.y, T.ng[2] = ng.z;
    double F[3][3];
    for (int a = 0; a < 3; ++a) {
        F[a][0] = T.e1[a];
        F[a][1] = T.e2[a];
        F[a][2] = T.ng[a];
    }
    auto cof = [&](int i, int j) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        return F[i1][j1] * F[i2][j2] - F[i1][j2] * F[i2][j1];
    };
    double c0 = cof(0, 0), c1 = cof(1, 0), c2 = cof(2, 0);
    double fdet = (c0 * F[0][0] + c1 * F[1][0]) + c2 * F[2][0];
    double finv = 1.0 / fdet;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            T.A[i][j] = cof(j, i) * finv;
    // uv domain
    v2 a = sub2(t1, t0), b = sub2(t2, t0);
    double signed_area = 0.5 * (a.x * b.y - a.y * b.x);
    double orient = signed_area >= 0.0 ? 1.0 : -1.0;
    v2 tt[3] = {t0, t1, t2};
    for (int k = 0; k < 3; ++k) {
        v2 e = sub2(tt[(k + 1) % 3], tt[k]);
        T.un[k][0] = orient * -e.y;
        T.un[k][1] = orient * e.x;
        T.ud[k] = T.un[k][0] * tt[k].x + T.un[k][1] * tt[k].y;
    }
    v2 lo = min2(min2(t0, t1), t2), hi = max2(max2(t0, t1), t2);
    T.lo[0] = lo.x, T.lo[1] = lo.y, T.hi[0] = hi.x, T.hi[1] = hi.y;
    double me = ((norm3(sub3(p1, p0)) + norm3(sub3(p2, p0))) + norm3(sub3(p2, p1))) / 3.0;
    T.residual_tol = 1e-10 * me;
    return true;
}

struct StackCell { int level; int64_t i, j; };

__device__ void setup_one(TriDev &T, const AssetDev &a, unsigned *status)
{
    int level;
    int64_t i0, j0;
    footprint_roots(T, a.n_leaf, level, i0, j0);
    T.root_level = level;
    // DisplacedIntersector roots: the block's cells meeting the domain's box, j outer
    double w = cell_width(a, level);
    int64_t i_lo = (int64_t)floor(T.lo[0] / w), i_hi = (int64_t)ceil(T.hi[0] / w) - 1;
    int64_t j_lo = (int64_t)floor(T.lo[1] / w), j_hi = (int64_t)ceil(T.hi[1] / w) - 1;
    int n = 0;
    for (int64_t j = j_lo; j <= j_hi && n < 4; ++j)
        for (int64_t i = i_lo; i <= i_hi && n < 4; ++i) {
            T.roots_i[n] = (int)i;
            T.roots_j[n] = (int)j;
            ++n;
        }
    T.n_roots = n;
    // triangle_height_range: depth-first over the footprint, explicit stack
    double h_min = INFINITY, h_max = -INFINITY;
    StackCell st[96];
    int sp = 0;
    for (int ch = 3; ch >= 0; --ch)
        st[sp++] = {level, i0 + (ch & 1), j0 + (ch >> 1)};
    int guard = 0;
    while (sp > 0) {
        if (++guard > (1 << 26)) {
            atomicOr(status, dmapdev::kStatusCapped);
            break;
        }
        StackCell c = st[--sp];
        double cw = cell_width(a, c.level);
        v2 cc = {(c.i + 0.5) * cw, (c.j + 0.5) * cw};
        int ov = classify_square(T, cc, 0.5 * cw);
        if (ov == OUTSIDE)
            continue;
        if (ov == INSIDE || c.level == 0) {
            double lo, hi;
            node_hrange(a, c.level, c.i, c.j, lo, hi);
            h_min = dmin(h_min, lo);
            h_max = dmax(h_max, hi);
            continue;
        }
        if (sp + 4 > 96) {
            atomicOr(status, dmapdev::kStatusCapped);
            break;
        }
        for (int ch = 3; ch >= 0; --ch)
            st[sp++] = {c.level - 1, 2 * c.i + (ch & 1), 2 * c.j + (ch >> 1)};
    }
    T.h_min = h_min;
    T.h_max = h_max;
    // triangle_aabb: three parallelograms
    v2 tv[3] = {L2(T.t0), L2(T.t1), L2(T.t2)};
    af h = AF(0.5 * (h_min + h_max), 0.0, 0.0, 0.5 * (h_max - h_min));
    box3 box = {{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
    for (int k = 0; k < 3; ++k) {
        v2 tk = tv[k], tk1 = tv[(k + 1) % 3], tk2 = tv[(k + 2) % 3];
        v2 c = add2(add2(mul2(0.5, tk), mul2(0.25, tk1)), mul2(0.25, tk2));
        v2 du = mul2(0.25, sub2(tk1, tk)), dv = mul2(0.25, sub2(tk2, tk));
        af3 P = AF3(tri_P(T, c.x, c.y), add3(mul3(du.x, L3(T.e1)), mul3(du.y, L3(T.e2))),
                    add3(mul3(dv.x, L3(T.e1)), mul3(dv.y, L3(T.e2))));
        af3 N = AF3(tri_M(T, c.x, c.y), add3(mul3(du.x, L3(T.Mu)), mul3(du.y, L3(T.Mv))),
                    add3(mul3(dv.x, L3(T.Mu)), mul3(dv.y, L3(T.Mv))));
        normalize(N);
        box3 b = hull(add(P, scale_form(h, N)));
        box.lo = {dmin(box.lo.x, b.lo.x), dmin(box.lo.y, b.lo.y), dmin(box.lo.z, b.lo.z)};
        box.hi = {dmax(box.hi.x, b.hi.x), dmax(box.hi.y, b.hi.y), dmax(box.hi.z, b.hi.z)};
    }
    T.box_lo[0] = box.lo.x, T.box_lo[1] = box.lo.y, T.box_lo[2] = box.lo.z;
    T.box_hi[0] = box.hi.x, T.box_hi[1] = box.hi.y, T.box_hi[2] = box.hi.z;
}

__device__ float fdown(double x) { return __double2float_rd(x); }
__device__ float fup(double x) { return __double2float_ru(x); }

__device__ void derive32(const TriDev &T, TriDev32 &S)
{
    for (int a = 0; a < 3; ++a) {
        S.e1[a] = (float)T.e1[a];
        S.e2[a] = (float)T.e2[a];
        S.m0[a] = (float)T.m0[a];
        S.Mu[a] = (float)T.Mu[a];
        S.Mv[a] = (float)T.Mv[a];
        S.q0f[a] = (float)T.q0[a];
        S.q0[a] = T.q0[a];
        for (int b = 0; b < 3; ++b) {
            S.Af[a][b] = (float)T.A[a][b];
            S.A[a][b] = T.A[a][b];
        }
        // object AABB widened by a few float ulps of its magnitude
        double pad = 4.0 * 1.1920928955078125e-7 * (1.0 + fmax(fabs(T.box_lo[a]), fabs(T.box_hi[a])));
        S.box_lo[a] = fdown(T.box_lo[a] - pad);
        S.box_hi[a] = fup(T.box_hi[a] + pad);
    }
    S.t0[0] = (float)T.t0[0], S.t0[1] = (float)T.t0[1];
    S.t1[0] = (float)T.t1[0], S.t1[1] = (float)T.t1[1];
    S.t2[0] = (float)T.t2[0], S.t2[1] = (float)T.t2[1];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            S.J[a][b] = (float)T.J[a][b];
    for (int k = 0; k < 3; ++k) {
        S.un[k][0] = (float)T.un[k][0];
        S.un[k][1] = (float)T.un[k][1];
        S.ud[k] = (float)T.ud[k];
    }
    S.lo[0] = fdown(T.lo[0]), S.lo[1] = fdown(T.lo[1]);
    S.hi[0] = fup(T.hi[0]), S.hi[1] = fup(T.hi[1]);
    S.residual_tol = (float)T.residual_tol;
    S.mean_edge = (float)(T.residual_tol * 1e10);
    S.newton_tol = 0.0f; // set by the FP32 path from the ray scale
    S.root_level = T.root_level;
    S.n_roots = T.n_roots;
    S.asset = T.asset;
    S.pad = 0;
    for (int k = 0; k < 4; ++k) {
        S.roots_i[k] = T.roots_i[k];
        S.roots_j[k] = T.roots_j[k];
    }
    v3 m0 = L3(T.m0), Mu = L3(T.Mu), Mv = L3(T.Mv);
    v3 a0 = mat3mul(T.A, m0), au = mat3mul(T.A, Mu), av = mat3mul(T.A, Mv);
    for (int a = 0; a < 3; ++a) {
        S.a0[a] = (float)comp(a0, a);
        S.au[a] = (float)comp(au, a);
        S.av[a] = (float)comp(av, a);
        S.rowsum[a] = fup((fabs(T.A[a][0]) + fabs(T.A[a][1])) + fabs(T.A[a][2]));
    }
    S.qc = (float)dot3(m0, m0);
    S.q1 = (float)dot3(m0, Mu);
    S.q2 = (float)dot3(m0, Mv);
    S.q11 = (float)dot3(Mu, Mu);
    S.q12 = (float)dot3(Mu, Mv);
    S.q22 = (float)dot3(Mv, Mv);
}

__global__ void setup_kernel(const double *__restrict__ tris, int stride, const int *__restrict__ tri_asset,
                             const AssetDev *__restrict__ assets, int n_tri, TriDev *out, TriDev32 *out32,
                             unsigned *status)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_tri)
        return;
    TriDev T;
    T.asset = tri_asset[k];
    T.status = 0;
    T.inst = 0;
    T.inst_pad = 0;
    if (!init_triangle(T, tris + stride * (size_t)k, stride == dmapk::kChartRecord)) {
        T.status = 1;
        atomicOr(status, dmapdev::kStatusBadInput);
        out[k] = T;
        return;
    }
    setup_one(T, assets[T.asset], status);
    out[k] = T;
    TriDev32 S;
    derive32(T, S);
    out32[k] = S;
}

} // namespace

namespace dmapk
{
cudaError_t launch_setup(const double *tris_dev, int stride, const int *tri_asset_dev,
                         const dmapdev::AssetDev *assets_dev, int n_tri, dmapdev::TriDev *out,
                         dmapdev::TriDev32 *out32, unsigned *status, cudaStream_t stream)
{
    int threads = 64;
    int blocks = (n_tri + threads - 1) / threads;
    setup_kernel<<<blocks, threads, 0, stream>>>(tris_dev, stride, tri_asset_dev, assets_dev, n_tri, out, out32,
                                                 status);
    return cudaGetLastError();
}
} // namespace dmapk
