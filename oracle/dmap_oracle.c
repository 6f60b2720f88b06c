/*
 * CPU oracle of the ray vs displaced-surface query. TEST INFRASTRUCTURE ONLY:
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker, never by the product.
 *
 * A double-precision restatement of MangoSister/dmap's hot path
 * (code/cpp/src, cited below by file:line). Parity is pinned two ways:
 * against the reference sources compiled here with shim headers
 * (oracle/_ref, built by oracle/Makefile) and against golden vectors of the
 * reference's numpy pyramid (tests/golden). Operation order follows the
 * reference; see dmap_oracle.h for the conventions.
 */
#include "dmap_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* Small vector helpers (the Eigen subset the reference uses).               */
/* ------------------------------------------------------------------------ */

typedef struct { double x, y; } v2;
typedef struct { double x, y, z; } v3;

static inline double dmin(double a, double b) { return b < a ? b : a; } /* std::min */
static inline double dmax(double a, double b) { return a < b ? b : a; } /* std::max */
static inline v2 V2(double x, double y) { v2 r = {x, y}; return r; }
static inline v3 V3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v2 sub2(v2 a, v2 b) { return V2(a.x - b.x, a.y - b.y); }
static inline v2 add2(v2 a, v2 b) { return V2(a.x + b.x, a.y + b.y); }
static inline v2 mul2(double s, v2 a) { return V2(s * a.x, s * a.y); }
static inline v2 min2(v2 a, v2 b) { return V2(dmin(a.x, b.x), dmin(a.y, b.y)); }
static inline v2 max2(v2 a, v2 b) { return V2(dmax(a.x, b.x), dmax(a.y, b.y)); }
static inline double dot2(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline v3 add3(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul3(double s, v3 a) { return V3(s * a.x, s * a.y, s * a.z); }
static inline v3 div3(v3 a, double s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline double dot3(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline v3 cross3(v3 a, v3 b)
{
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double norm3(v3 a) { return sqrt(dot3(a, a)); }
static inline v3 normalized3(v3 a)
{
    double z = dot3(a, a);
    if (z > 0.0)
        return div3(a, sqrt(z));
    return a;
}
static inline double comp3(v3 a, int k) { return k == 0 ? a.x : k == 1 ? a.y : a.z; }
static inline void set3(v3 *a, int k, double v)
{
    if (k == 0)
        a->x = v;
    else if (k == 1)
        a->y = v;
    else
        a->z = v;
}
typedef struct { double m[3][3]; } m3;
static inline v3 m3mul(const m3 *A, v3 v)
{
    return V3((A->m[0][0] * v.x + A->m[0][1] * v.y) + A->m[0][2] * v.z,
              (A->m[1][0] * v.x + A->m[1][1] * v.y) + A->m[1][2] * v.z,
              (A->m[2][0] * v.x + A->m[2][1] * v.y) + A->m[2][2] * v.z);
}
/* 3x3 inverse by cofactors (the Eigen fixed-size routine's structure). */
static inline double cof3(const m3 *M, int i, int j)
{
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return M->m[i1][j1] * M->m[i2][j2] - M->m[i1][j2] * M->m[i2][j1];
}
static m3 m3inverse(const m3 *M)
{
    m3 R;
    double c0 = cof3(M, 0, 0), c1 = cof3(M, 1, 0), c2 = cof3(M, 2, 0);
    double det = (c0 * M->m[0][0] + c1 * M->m[1][0]) + c2 * M->m[2][0];
    double invdet = 1.0 / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            R.m[i][j] = cof3(M, j, i) * invdet;
    return R;
}

/* ------------------------------------------------------------------------ */
/* Affine forms, affine_form.cpp.                                            */
/* ------------------------------------------------------------------------ */

typedef struct { double c, a, b, k; } af;
typedef struct { af x, y, z; } af3;
typedef struct { double lo, hi; } ivl;

static inline af AF(double c, double a, double b, double k) { af r = {c, a, b, k}; return r; }
static inline ivl af_interval(af f) /* affine_form.h:50-54 */
{
    double e = (fabs(f.a) + fabs(f.b)) + f.k;
    ivl r = {f.c - e, f.c + e};
    return r;
}
static inline af af_add(af x, af y) /* affine_form.cpp:17-24 */
{
    return AF(x.c + y.c, x.a + y.a, x.b + y.b, x.k + y.k);
}
static inline af af_scale(double s, af x) /* affine_form.cpp:49-56 */
{
    return AF(x.c * s, x.a * s, x.b * s, x.k * fabs(s));
}
static inline af af_mul(af x, af r) /* affine_form.cpp:35-47 */
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
static inline double g_rsqrt(double x) { return 1.0 / sqrt(x); }
static af af_rsqrt(af f) /* affine_form.cpp:64-76, Min-Range */
{
    ivl range = af_interval(f);
    double lo = range.lo, hi = range.hi;
    double alpha = -0.5 * g_rsqrt(hi) * g_rsqrt(hi) * g_rsqrt(hi);
    double beta = 0.5 * (g_rsqrt(lo) + g_rsqrt(hi) - alpha * (lo + hi));
    double delta = 0.5 * fabs(g_rsqrt(lo) - g_rsqrt(hi) - alpha * (lo - hi));
    return AF(alpha * f.c + beta, alpha * f.a, alpha * f.b, fabs(alpha) * f.k + delta);
}
static inline af3 AF3(v3 c, v3 a, v3 b)
{
    af3 r = {AF(c.x, a.x, b.x, 0.0), AF(c.y, a.y, b.y, 0.0), AF(c.z, a.z, b.z, 0.0)};
    return r;
}
static inline af *af3_comp(af3 *v, int k) { return k == 0 ? &v->x : k == 1 ? &v->y : &v->z; }
static af af3_sq_length(const af3 *v) /* affine_form.cpp:78-85 */
{
    v3 xc = V3(v->x.c, v->y.c, v->z.c), xu = V3(v->x.a, v->y.a, v->z.a);
    v3 xv = V3(v->x.b, v->y.b, v->z.b), xk = V3(v->x.k, v->y.k, v->z.k);
    v3 dev = V3((fabs(xu.x) + fabs(xv.x)) + xk.x, (fabs(xu.y) + fabs(xv.y)) + xk.y,
                (fabs(xu.z) + fabs(xv.z)) + xk.z);
    double offset = 0.5 * dot3(dev, dev);
    return AF(dot3(xc, xc) + offset, 2.0 * dot3(xc, xu), 2.0 * dot3(xc, xv), 2.0 * fabs(dot3(xc, xk)) + offset);
}
static void af3_normalize(af3 *v) /* affine_form.cpp:87-95 */
{
    af l = af3_sq_length(v);
    if (af_interval(l).lo <= 0.0) {
        v->x = v->y = v->z = AF(0.0, 0.0, 0.0, 1.0);
        return;
    }
    af r = af_rsqrt(l);
    v->x = af_mul(r, v->x);
    v->y = af_mul(r, v->y);
    v->z = af_mul(r, v->z);
}
static inline af3 af3_add(af3 a, af3 b) /* affine_form.cpp:97 */
{
    af3 r = {af_add(a.x, b.x), af_add(a.y, b.y), af_add(a.z, b.z)};
    return r;
}
static inline af af_dot(v3 a, af3 b) /* affine_form.cpp:101 */
{
    return af_add(af_add(af_scale(a.x, b.x), af_scale(a.y, b.y)), af_scale(a.z, b.z));
}
static inline af3 af3_matmul(const m3 *A, af3 v) /* affine_form.cpp:103-106 */
{
    af3 r;
    r.x = af_dot(V3(A->m[0][0], A->m[0][1], A->m[0][2]), v);
    r.y = af_dot(V3(A->m[1][0], A->m[1][1], A->m[1][2]), v);
    r.z = af_dot(V3(A->m[2][0], A->m[2][1], A->m[2][2]), v);
    return r;
}
static inline af3 af3_scale_form(af s, af3 v) /* affine_form.h:100 */
{
    af3 r = {af_mul(s, v.x), af_mul(s, v.y), af_mul(s, v.z)};
    return r;
}

/* ------------------------------------------------------------------------ */
/* Taylor pyramid, taylor_pyramid.cpp.                                       */
/* ------------------------------------------------------------------------ */

enum { CH_H0, CH_GU, CH_GV, CH_R, CH_RU, CH_RV, CH_HMIN, CH_HMAX, N_CH };

typedef struct {
    int m;
    double *ch[N_CH];
} o_level;

struct o_pyramid {
    int n_leaf, n_levels, build;
    o_level *levels;
};

static void level_alloc(o_level *l, int m)
{
    l->m = m;
    for (int c = 0; c < N_CH; ++c)
        l->ch[c] = (double *)calloc((size_t)m * m, sizeof(double));
}

static void leaf_level(o_level *out, const double *V, int nodes, int n_leaf) /* taylor_pyramid.cpp:45-67 */
{
    level_alloc(out, n_leaf);
    double w = 1.0 / n_leaf;
    double s = 0.5 * w;
    for (int j = 0; j < n_leaf; ++j) {
        for (int i = 0; i < n_leaf; ++i) {
            double v00 = V[(size_t)j * nodes + i], v10 = V[(size_t)j * nodes + i + 1];
            double v01 = V[(size_t)(j + 1) * nodes + i], v11 = V[(size_t)(j + 1) * nodes + i + 1];
            size_t k = (size_t)j * n_leaf + i;
            out->ch[CH_H0][k] = 0.25 * (((v00 + v10) + v01) + v11);
            out->ch[CH_GU][k] = 0.5 * ((v10 - v00) + (v11 - v01)) / w;
            out->ch[CH_GV][k] = 0.5 * ((v01 - v00) + (v11 - v10)) / w;
            double c3 = (((v00 - v10) - v01) + v11) / (w * w);
            out->ch[CH_R][k] = fabs(c3) * s * s;
            out->ch[CH_RU][k] = fabs(c3) * s;
            out->ch[CH_RV][k] = fabs(c3) * s;
            out->ch[CH_HMIN][k] = dmin(dmin(v00, v10), dmin(v01, v11));
            out->ch[CH_HMAX][k] = dmax(dmax(v00, v10), dmax(v01, v11));
        }
    }
}

static void fold_level(o_level *out, const o_level *child) /* taylor_pyramid.cpp:77-138 */
{
    int m = child->m / 2;
    level_alloc(out, m);
    double s = 0.5 / m;
    const double off[2] = {-0.5 * s, 0.5 * s};
    const double corner_off[2] = {-0.5 * s, 0.5 * s};
    for (int J = 0; J < m; ++J) {
        for (int I = 0; I < m; ++I) {
            size_t kp = (size_t)J * m + I;
            double gu_hi = -INFINITY, gu_lo = INFINITY, gv_hi = -INFINITY, gv_lo = INFINITY;
            double h_min = INFINITY, h_max = -INFINITY;
            for (int a = 0; a < 2; ++a) {
                for (int b = 0; b < 2; ++b) {
                    size_t kc = (size_t)(2 * J + a) * child->m + (2 * I + b);
                    gu_hi = dmax(gu_hi, child->ch[CH_GU][kc] + child->ch[CH_RU][kc]);
                    gu_lo = dmin(gu_lo, child->ch[CH_GU][kc] - child->ch[CH_RU][kc]);
                    gv_hi = dmax(gv_hi, child->ch[CH_GV][kc] + child->ch[CH_RV][kc]);
                    gv_lo = dmin(gv_lo, child->ch[CH_GV][kc] - child->ch[CH_RV][kc]);
                    h_min = dmin(h_min, child->ch[CH_HMIN][kc]);
                    h_max = dmax(h_max, child->ch[CH_HMAX][kc]);
                }
            }
            double gu_p = 0.5 * (gu_hi + gu_lo);
            double gv_p = 0.5 * (gv_hi + gv_lo);
            out->ch[CH_GU][kp] = gu_p;
            out->ch[CH_RU][kp] = 0.5 * (gu_hi - gu_lo);
            out->ch[CH_GV][kp] = gv_p;
            out->ch[CH_RV][kp] = 0.5 * (gv_hi - gv_lo);
            out->ch[CH_HMIN][kp] = h_min;
            out->ch[CH_HMAX][kp] = h_max;
            double upper = -INFINITY, lower = INFINITY;
            for (int a = 0; a < 2; ++a) {
                for (int b = 0; b < 2; ++b) {
                    size_t kc = (size_t)(2 * J + a) * child->m + (2 * I + b);
                    double dx = off[b], dy = off[a];
                    double du_g = child->ch[CH_GU][kc] - gu_p;
                    double dv_g = child->ch[CH_GV][kc] - gv_p;
                    double base = (child->ch[CH_H0][kc] - child->ch[CH_GU][kc] * dx) - child->ch[CH_GV][kc] * dy;
                    for (int cu = 0; cu < 2; ++cu) {
                        for (int cv = 0; cv < 2; ++cv) {
                            double corner = (base + du_g * (dx + corner_off[cu])) + dv_g * (dy + corner_off[cv]);
                            upper = dmax(upper, corner + child->ch[CH_R][kc]);
                            lower = dmin(lower, corner - child->ch[CH_R][kc]);
                        }
                    }
                }
            }
            out->ch[CH_H0][kp] = 0.5 * (upper + lower);
            out->ch[CH_R][kp] = 0.5 * (upper - lower);
        }
    }
}

/* taylor_pyramid.cpp:20-43 and :151-202 (the direct construction). */
static void direct_level(o_level *out, const double *V, int nodes, int n_leaf, int level)
{
    int k = 1 << level;
    int m = n_leaf >> level;
    level_alloc(out, m);
    double w = 1.0 / n_leaf;
    double s_texel = 0.5 / n_leaf;
    for (int J = 0; J < m; ++J) {
        for (int I = 0; I < m; ++I) {
            size_t kp = (size_t)J * m + I;
            double gu_hi = -INFINITY, gu_lo = INFINITY, gv_hi = -INFINITY, gv_lo = INFINITY;
            for (int b = 0; b < k; ++b) {
                for (int a = 0; a < k; ++a) {
                    int tj = J * k + b, ti = I * k + a;
                    double v00 = V[(size_t)tj * nodes + ti], v10 = V[(size_t)tj * nodes + ti + 1];
                    double v01 = V[(size_t)(tj + 1) * nodes + ti], v11 = V[(size_t)(tj + 1) * nodes + ti + 1];
                    double c1 = 0.5 * ((v10 - v00) + (v11 - v01)) / w;
                    double c2 = 0.5 * ((v01 - v00) + (v11 - v10)) / w;
                    double c3 = (((v00 - v10) - v01) + v11) / (w * w);
                    double spread = fabs(c3) * s_texel;
                    gu_hi = dmax(gu_hi, c1 + spread);
                    gu_lo = dmin(gu_lo, c1 - spread);
                    gv_hi = dmax(gv_hi, c2 + spread);
                    gv_lo = dmin(gv_lo, c2 - spread);
                }
            }
            double gu = 0.5 * (gu_hi + gu_lo);
            double gv = 0.5 * (gv_hi + gv_lo);
            out->ch[CH_GU][kp] = gu;
            out->ch[CH_RU][kp] = 0.5 * (gu_hi - gu_lo);
            out->ch[CH_GV][kp] = gv;
            out->ch[CH_RV][kp] = 0.5 * (gv_hi - gv_lo);
            double upper = -INFINITY, lower = INFINITY, h_min = INFINITY, h_max = -INFINITY;
            for (int b = 0; b <= k; ++b) {
                double dv = (b - 0.5 * k) / n_leaf;
                for (int a = 0; a <= k; ++a) {
                    double du = (a - 0.5 * k) / n_leaf;
                    double value = V[(size_t)(J * k + b) * nodes + (I * k + a)];
                    double residual = (value - gu * du) - gv * dv;
                    upper = dmax(upper, residual);
                    lower = dmin(lower, residual);
                    h_min = dmin(h_min, value);
                    h_max = dmax(h_max, value);
                }
            }
            out->ch[CH_H0][kp] = 0.5 * (upper + lower);
            out->ch[CH_R][kp] = 0.5 * (upper - lower);
            out->ch[CH_HMIN][kp] = h_min;
            out->ch[CH_HMAX][kp] = h_max;
        }
    }
}

o_pyramid *o_pyramid_build(const double *values, int nodes, double scale, double offset, int build)
{
    /* taylor_pyramid.cpp:215-251 */
    int n = nodes - 1;
    if (!(n >= 1 && (n & (n - 1)) == 0))
        return NULL;
    o_pyramid *p = (o_pyramid *)calloc(1, sizeof(o_pyramid));
    p->n_leaf = n;
    p->n_levels = 1;
    while ((1 << p->n_levels) <= n)
        ++p->n_levels;
    p->build = build;
    p->levels = (o_level *)calloc((size_t)p->n_levels, sizeof(o_level));
    double *V = (double *)malloc((size_t)nodes * nodes * sizeof(double));
    for (size_t k = 0; k < (size_t)nodes * nodes; ++k)
        V[k] = values[k] * scale;
    if (build == O_BUILD_FOLD) {
        leaf_level(&p->levels[0], V, nodes, n);
        for (int l = 1; l < p->n_levels; ++l)
            fold_level(&p->levels[l], &p->levels[l - 1]);
    } else {
        for (int l = 0; l < p->n_levels; ++l)
            direct_level(&p->levels[l], V, nodes, n, l);
    }
    free(V);
    if (offset != 0.0) {
        for (int l = 0; l < p->n_levels; ++l) {
            size_t cells = (size_t)p->levels[l].m * p->levels[l].m;
            for (size_t k = 0; k < cells; ++k) {
                p->levels[l].ch[CH_H0][k] += offset;
                p->levels[l].ch[CH_HMIN][k] += offset;
                p->levels[l].ch[CH_HMAX][k] += offset;
            }
        }
    }
    return p;
}

void o_pyramid_free(o_pyramid *p)
{
    if (!p)
        return;
    for (int l = 0; l < p->n_levels; ++l)
        for (int c = 0; c < N_CH; ++c)
            free(p->levels[l].ch[c]);
    free(p->levels);
    free(p);
}

int o_pyramid_levels(const o_pyramid *p) { return p->n_levels; }
int o_pyramid_n_leaf(const o_pyramid *p) { return p->n_leaf; }

void o_pyramid_level(const o_pyramid *p, int level, double *out)
{
    size_t cells = (size_t)p->levels[level].m * p->levels[level].m;
    for (int c = 0; c < N_CH; ++c)
        memcpy(out + c * cells, p->levels[level].ch[c], cells * sizeof(double));
}

typedef struct { double h0, gu, gv, r, ru, rv, h_min, h_max; } o_node;

static o_node pyramid_node(const o_pyramid *p, int level, int64_t i, int64_t j) /* taylor_pyramid.cpp:259-274 */
{
    o_node n;
    if (level >= p->n_levels) {
        const o_level *root = &p->levels[p->n_levels - 1];
        double lo = root->ch[CH_HMIN][0], hi = root->ch[CH_HMAX][0];
        n.h0 = 0.5 * (lo + hi);
        n.gu = 0.0;
        n.gv = 0.0;
        n.r = 0.5 * (hi - lo);
        n.ru = root->ch[CH_RU][0];
        n.rv = root->ch[CH_RV][0];
        n.h_min = lo;
        n.h_max = hi;
        return n;
    }
    const o_level *l = &p->levels[level];
    int64_t ri = i % l->m, rj = j % l->m;
    if (ri < 0)
        ri += l->m;
    if (rj < 0)
        rj += l->m;
    size_t k = (size_t)rj * l->m + ri;
    n.h0 = l->ch[CH_H0][k];
    n.gu = l->ch[CH_GU][k];
    n.gv = l->ch[CH_GV][k];
    n.r = l->ch[CH_R][k];
    n.ru = l->ch[CH_RU][k];
    n.rv = l->ch[CH_RV][k];
    n.h_min = l->ch[CH_HMIN][k];
    n.h_max = l->ch[CH_HMAX][k];
    return n;
}

void o_pyramid_node(const o_pyramid *p, int level, int64_t i, int64_t j, double *out8)
{
    o_node n = pyramid_node(p, level, i, j);
    memcpy(out8, &n, sizeof(n));
}

static inline double cell_width(const o_pyramid *p, int level) /* taylor_pyramid.h:94 */
{
    return ldexp(1.0, level) / p->n_leaf;
}

/* ------------------------------------------------------------------------ */
/* Height grid and base triangle, displaced_surface.cpp.                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    int W, H;
    double scale;
    const double *values;
    double offset;
    int repeat;
} o_grid;

static inline double grid_value(const o_grid *g, int j, int i) { return g->values[(size_t)j * g->W + i]; }

static void grid_cell(const o_grid *g, double x, double y, int *i, int *j, double *s, double *t)
{
    /* displaced_surface.cpp:12-27 */
    if (g->repeat) {
        x -= floor(x);
        y -= floor(y);
    } else {
        x = x < 0.0 ? 0.0 : (1.0 < x ? 1.0 : x);
        y = y < 0.0 ? 0.0 : (1.0 < y ? 1.0 : y);
    }
    double fx = x * (g->W - 1);
    double fy = y * (g->H - 1);
    int ii = (int)fx, jj = (int)fy;
    *i = g->W - 2 < ii ? g->W - 2 : ii;
    *j = g->H - 2 < jj ? g->H - 2 : jj;
    *s = fx - *i;
    *t = fy - *j;
}

static double grid_h(const o_grid *g, double x, double y) /* displaced_surface.cpp:29-37 */
{
    int i, j;
    double s, t;
    grid_cell(g, x, y, &i, &j, &s, &t);
    return g->scale * (((((1.0 - s) * (1.0 - t)) * grid_value(g, j, i) + (s * (1.0 - t)) * grid_value(g, j, i + 1)) +
                        ((1.0 - s) * t) * grid_value(g, j + 1, i)) +
                       (s * t) * grid_value(g, j + 1, i + 1)) +
           g->offset;
}

static v2 grid_grad(const o_grid *g, double x, double y) /* displaced_surface.cpp:39-47 */
{
    int i, j;
    double s, t;
    grid_cell(g, x, y, &i, &j, &s, &t);
    double dh_ds = (1.0 - t) * (grid_value(g, j, i + 1) - grid_value(g, j, i)) +
                   t * (grid_value(g, j + 1, i + 1) - grid_value(g, j + 1, i));
    double dh_dt = (1.0 - s) * (grid_value(g, j + 1, i) - grid_value(g, j, i)) +
                   s * (grid_value(g, j + 1, i + 1) - grid_value(g, j, i + 1));
    return V2(g->scale * (dh_ds * (g->W - 1)), g->scale * (dh_dt * (g->H - 1)));
}

typedef struct {
    v3 q0, e1, e2, m0, Mu, Mv;
    v3 p0, p1, p2;
    v2 t0, t1, t2;
    double J[2][2];
} o_tri;

static int tri_init(o_tri *T, const double *r) /* displaced_surface.cpp:54-91 */
{
    v3 p0 = V3(r[0], r[1], r[2]), p1 = V3(r[3], r[4], r[5]), p2 = V3(r[6], r[7], r[8]);
    v3 m0 = V3(r[9], r[10], r[11]), m1 = V3(r[12], r[13], r[14]), m2 = V3(r[15], r[16], r[17]);
    v2 t0 = V2(r[18], r[19]), t1 = V2(r[20], r[21]), t2 = V2(r[22], r[23]);
    T->p0 = p0;
    T->p1 = p1;
    T->p2 = p2;
    T->t0 = t0;
    T->t1 = t1;
    T->t2 = t2;
    v3 eb1 = sub3(p1, p0), eb2 = sub3(p2, p0);
    v3 Mb1 = sub3(m1, m0), Mb2 = sub3(m2, m0);
    double T00 = t1.x - t0.x, T10 = t1.y - t0.y, T01 = t2.x - t0.x, T11 = t2.y - t0.y;
    double det = T00 * T11 - T10 * T01;
    if (!(fabs(det) > 1e-30))
        return 0;
    double invdet = 1.0 / det;
    T->J[0][0] = T11 * invdet;
    T->J[1][0] = -T10 * invdet;
    T->J[0][1] = -T01 * invdet;
    T->J[1][1] = T00 * invdet;
    double (*J)[2] = T->J;
    /* E = [eb1 eb2], D = [Mb1 Mb2]; EJ = E J, DJ = D J, c = -J t0. */
    v2 c = V2((-J[0][0]) * t0.x + (-J[0][1]) * t0.y, (-J[1][0]) * t0.x + (-J[1][1]) * t0.y);
    for (int a = 0; a < 3; ++a) {
        double E0 = comp3(eb1, a), E1 = comp3(eb2, a), D0 = comp3(Mb1, a), D1 = comp3(Mb2, a);
        set3(&T->q0, a, comp3(p0, a) + (E0 * c.x + E1 * c.y));
        set3(&T->e1, a, E0 * J[0][0] + E1 * J[1][0]);
        set3(&T->e2, a, E0 * J[0][1] + E1 * J[1][1]);
        set3(&T->m0, a, comp3(m0, a) + (D0 * c.x + D1 * c.y));
        set3(&T->Mu, a, D0 * J[0][0] + D1 * J[1][0]);
        set3(&T->Mv, a, D0 * J[0][1] + D1 * J[1][1]);
    }
    return 1;
}

static inline v3 tri_P(const o_tri *T, double s, double t) /* displaced_surface.h:83 */
{
    return add3(add3(T->q0, mul3(s, T->e1)), mul3(t, T->e2));
}
static inline v3 tri_M(const o_tri *T, double s, double t) /* displaced_surface.h:84 */
{
    return add3(add3(T->m0, mul3(s, T->Mu)), mul3(t, T->Mv));
}
static inline v2 tri_bary(const o_tri *T, double s, double t) /* displaced_surface.h:86 */
{
    double x = s - T->t0.x, y = t - T->t0.y;
    return V2(T->J[0][0] * x + T->J[0][1] * y, T->J[1][0] * x + T->J[1][1] * y);
}
static inline v2 tri_param(const o_tri *T, double u, double v) /* displaced_surface.h:87 */
{
    return add2(add2(T->t0, mul2(u, sub2(T->t1, T->t0))), mul2(v, sub2(T->t2, T->t0)));
}

typedef struct { v3 N, Nu, Nv; } o_nframe;

static o_nframe normal_frame_at(const o_tri *T, double s, double t) /* displaced_surface.cpp:99-108 */
{
    v3 M = tri_M(T, s, t);
    double Mlen = norm3(M);
    o_nframe f;
    f.N = div3(M, Mlen);
    f.Nu = div3(sub3(T->Mu, mul3(dot3(f.N, T->Mu), f.N)), Mlen);
    f.Nv = div3(sub3(T->Mv, mul3(dot3(f.N, T->Mv), f.N)), Mlen);
    return f;
}

static v3 displaced_position(const o_tri *T, const o_grid *g, double s, double t) /* displaced_surface.cpp:162-166 */
{
    o_nframe f = normal_frame_at(T, s, t);
    return add3(tri_P(T, s, t), mul3(grid_h(g, s, t), f.N));
}

static double mean_edge(const o_tri *T) /* displaced_surface.cpp:168-171 */
{
    return ((norm3(sub3(T->p1, T->p0)) + norm3(sub3(T->p2, T->p0))) + norm3(sub3(T->p2, T->p1))) / 3.0;
}

/* ------------------------------------------------------------------------ */
/* UV domain, uv_clip.cpp.                                                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    v2 t[3], n[3];
    double d[3];
    v2 lo, hi;
} o_uvtri;

enum { OUTSIDE = 0, INSIDE = 1, STRADDLE = 2 };

static void uvtri_init(o_uvtri *U, v2 t0, v2 t1, v2 t2) /* uv_clip.cpp:10-25 */
{
    U->t[0] = t0;
    U->t[1] = t1;
    U->t[2] = t2;
    v2 a = sub2(t1, t0), b = sub2(t2, t0);
    double signed_area = 0.5 * (a.x * b.y - a.y * b.x);
    double orient = signed_area >= 0.0 ? 1.0 : -1.0;
    for (int k = 0; k < 3; ++k) {
        v2 e = sub2(U->t[(k + 1) % 3], U->t[k]);
        U->n[k] = V2(orient * -e.y, orient * e.x);
        U->d[k] = dot2(U->n[k], U->t[k]);
    }
    U->lo = min2(min2(t0, t1), t2);
    U->hi = max2(max2(t0, t1), t2);
}

static inline int uvtri_inside(const o_uvtri *U, v2 p) /* uv_clip.h:28-34 */
{
    for (int k = 0; k < 3; ++k)
        if (dot2(U->n[k], p) < U->d[k])
            return 0;
    return 1;
}

static int classify_square(const o_uvtri *U, v2 c, double s) /* uv_clip.cpp:27-44 */
{
    if (c.x + s <= U->lo.x || c.x - s >= U->hi.x || c.y + s <= U->lo.y || c.y - s >= U->hi.y)
        return OUTSIDE;
    int all_inside = 1;
    for (int k = 0; k < 3; ++k) {
        double proj = dot2(U->n[k], c);
        double ext = (fabs(U->n[k].x) + fabs(U->n[k].y)) * s;
        if (proj + ext <= U->d[k])
            return OUTSIDE;
        if (proj - ext < U->d[k])
            all_inside = 0;
    }
    return all_inside ? INSIDE : STRADDLE;
}

/* descent_sampler.cpp:15-21,66-83 (TFDM's find_roots). */
static void footprint_roots(const o_uvtri *U, int n_leaf, int *level, int64_t *i0, int64_t *j0)
{
    *level = 0;
    for (;;) {
        double w = ldexp(1.0, *level) / n_leaf;
        int64_t ilo = (int64_t)floor(U->lo.x / w), ihi = (int64_t)ceil(U->hi.x / w) - 1;
        int64_t jlo = (int64_t)floor(U->lo.y / w), jhi = (int64_t)ceil(U->hi.y / w) - 1;
        if (ihi - ilo <= 1 && jhi - jlo <= 1) {
            *i0 = ilo;
            *j0 = jlo;
            return;
        }
        ++*level;
    }
}

/* ------------------------------------------------------------------------ */
/* Node bounds, node_bounds.cpp.                                             */
/* ------------------------------------------------------------------------ */

typedef struct {
    m3 to_tangent;
    v3 origin, ng;
} o_frame;

static void tangent_frame(o_frame *F, const o_tri *T) /* node_bounds.cpp:13-23 */
{
    F->origin = T->q0;
    F->ng = normalized3(cross3(T->e1, T->e2));
    m3 from;
    for (int a = 0; a < 3; ++a) {
        from.m[a][0] = comp3(T->e1, a);
        from.m[a][1] = comp3(T->e2, a);
        from.m[a][2] = comp3(F->ng, a);
    }
    F->to_tangent = m3inverse(&from);
}

typedef struct { v3 lo, hi; } o_box;

static inline double interval_tolerance(double t_scale) /* node_bounds.cpp:128 */
{
    return 1e-9 * dmax(1.0, t_scale);
}

static int box_clip(const o_box *B, v3 o, v3 d, double *t0, double *t1) /* node_bounds.cpp:25-44 */
{
    for (int a = 0; a < 3; ++a) {
        double da = comp3(d, a), oa = comp3(o, a);
        if (da != 0.0) {
            double ta = (comp3(B->lo, a) - oa) / da, tb = (comp3(B->hi, a) - oa) / da;
            if (ta > tb) {
                double x = ta;
                ta = tb;
                tb = x;
            }
            *t0 = dmax(*t0, ta);
            *t1 = dmin(*t1, tb);
        } else if (oa < comp3(B->lo, a) || oa > comp3(B->hi, a)) {
            return 0;
        }
    }
    if (*t0 > *t1 + interval_tolerance(dmax(fabs(*t0), fabs(*t1))))
        return 0;
    if (*t0 > *t1) {
        double x = *t0;
        *t0 = *t1;
        *t1 = x;
    }
    return 1;
}

static void box_expand(o_box *B, const o_box *o) /* node_bounds.cpp:54-58 */
{
    B->lo = V3(dmin(B->lo.x, o->lo.x), dmin(B->lo.y, o->lo.y), dmin(B->lo.z, o->lo.z));
    B->hi = V3(dmax(B->hi.x, o->hi.x), dmax(B->hi.y, o->hi.y), dmax(B->hi.z, o->hi.z));
}

static o_box hull(af3 S) /* node_bounds.cpp:70-79 */
{
    o_box b;
    for (int a = 0; a < 3; ++a) {
        ivl r = af_interval(*af3_comp(&S, a));
        set3(&b.lo, a, r.lo);
        set3(&b.hi, a, r.hi);
    }
    return b;
}

typedef struct {
    int level;
    int64_t i, j;
    o_node node;
    v2 centre;
    af3 m;
    o_box box;
} o_nodebound;

static void node_bound(o_nodebound *nb, const o_tri *T, const o_frame *F, const o_pyramid *P, int level, int64_t i,
                       int64_t j) /* node_bounds.cpp:83-109 */
{
    nb->level = level;
    nb->i = i;
    nb->j = j;
    nb->node = pyramid_node(P, level, i, j);
    double w = cell_width(P, level);
    nb->centre = V2((i + 0.5) * w, (j + 0.5) * w);
    v2 tri_lo = min2(min2(T->t0, T->t1), T->t2), tri_hi = max2(max2(T->t0, T->t1), T->t2);
    v2 rect_lo = max2(V2(i * w, j * w), tri_lo);
    v2 rect_hi = min2(V2((i + 1) * w, (j + 1) * w), tri_hi);
    v2 c = mul2(0.5, add2(rect_lo, rect_hi));
    v2 hh = mul2(0.5, sub2(rect_hi, rect_lo));
    v2 half = V2(dmax(hh.x, 0.0), dmax(hh.y, 0.0));
    /* normal_form, node_bounds.cpp:65-68 */
    af3 N = AF3(add3(add3(T->m0, mul3(c.x, T->Mu)), mul3(c.y, T->Mv)), mul3(half.x, T->Mu), mul3(half.y, T->Mv));
    af3_normalize(&N);
    nb->m = af3_matmul(&F->to_tangent, N);
    af h = AF(0.5 * (nb->node.h_min + nb->node.h_max), 0.0, 0.0, 0.5 * (nb->node.h_max - nb->node.h_min));
    af3 p = AF3(V3(c.x, c.y, 0.0), V3(half.x, 0.0, 0.0), V3(0.0, half.y, 0.0));
    nb->box = hull(af3_add(p, af3_scale_form(h, nb->m)));
}

static inline ivl IV(double lo, double hi) { ivl r = {lo, hi}; return r; }
static inline ivl iv_add(ivl a, ivl b) { return IV(a.lo + b.lo, a.hi + b.hi); }
static inline ivl iv_adds(ivl a, double b) { return IV(a.lo + b, a.hi + b); }
static inline ivl iv_scale(double s, ivl a) /* affine_form.cpp:12-15 */
{
    return s >= 0.0 ? IV(s * a.lo, s * a.hi) : IV(s * a.hi, s * a.lo);
}

typedef struct {
    ivl A, B, C, D;
    double R;
} o_slab;

static o_slab slab_form(const o_nodebound *nb) /* node_bounds.cpp:111-122 */
{
    const o_node *n = &nb->node;
    ivl mx = af_interval(nb->m.x), my = af_interval(nb->m.y), mz = af_interval(nb->m.z);
    o_slab f;
    f.A = iv_add(iv_add(IV(1.0, 1.0), iv_scale(n->gu, mx)), iv_scale(n->gv, my));
    f.B = iv_scale(-n->gu, mz);
    f.C = iv_scale(-n->gv, mz);
    f.D = iv_scale(-((n->h0 - n->gu * nb->centre.x) - n->gv * nb->centre.y), mz);
    f.R = n->r * dmax(fabs(mz.lo), fabs(mz.hi));
    return f;
}

typedef struct {
    v3 o, d;
    double t_min, t_max;
} o_tray;

static int box_interval(const o_nodebound *nb, const o_tray *ray, double *t0, double *t1) /* node_bounds.cpp:130-135 */
{
    *t0 = ray->t_min;
    *t1 = ray->t_max;
    return box_clip(&nb->box, ray->o, ray->d, t0, t1);
}

static int slab_interval(const o_nodebound *nb, const o_tray *ray, double *t0, double *t1) /* node_bounds.cpp:137-179 */
{
    o_box column = nb->box;
    column.lo.z = -INFINITY;
    column.hi.z = INFINITY;
    *t0 = ray->t_min;
    *t1 = ray->t_max;
    if (!box_clip(&column, ray->o, ray->d, t0, t1))
        return 0;
    v3 anchor = add3(ray->o, mul3(*t0, ray->d));
    double span = *t1 - *t0;
    o_slab f = slab_form(nb);
    ivl F0 = iv_add(iv_add(iv_add(iv_scale(anchor.z, f.A), iv_scale(anchor.x, f.B)), iv_scale(anchor.y, f.C)), f.D);
    ivl F1 = iv_add(iv_add(iv_scale(ray->d.z, f.A), iv_scale(ray->d.x, f.B)), iv_scale(ray->d.y, f.C));
    double s0 = 0.0, s1 = span;
    if (F1.lo > 0.0)
        s1 = dmin(s1, (f.R - F0.lo) / F1.lo);
    else if (F1.lo < 0.0)
        s0 = dmax(s0, (f.R - F0.lo) / F1.lo);
    else if (F0.lo > f.R)
        return 0;
    if (F1.hi > 0.0)
        s0 = dmax(s0, (-f.R - F0.hi) / F1.hi);
    else if (F1.hi < 0.0)
        s1 = dmin(s1, (-f.R - F0.hi) / F1.hi);
    else if (F0.hi < -f.R)
        return 0;
    if (s0 > s1 + interval_tolerance(fabs(*t0) + span))
        return 0;
    if (s0 > s1) {
        double x = s0;
        s0 = s1;
        s1 = x;
    }
    *t1 = *t0 + s1;
    *t0 = *t0 + s0;
    return 1;
}

static int both_interval(const o_nodebound *nb, const o_tray *ray, double *t0, double *t1) /* node_bounds.cpp:181-197 */
{
    double b0, b1, s0, s1;
    if (!box_interval(nb, ray, &b0, &b1) || !slab_interval(nb, ray, &s0, &s1))
        return 0;
    *t0 = dmax(b0, s0);
    *t1 = dmin(b1, s1);
    double tol = interval_tolerance(dmax(fabs(*t0), fabs(*t1)));
    if (*t0 > *t1 + tol)
        return 0;
    if (*t0 > *t1) {
        double x = *t0;
        *t0 = *t1;
        *t1 = x;
    }
    return 1;
}

static int node_interval(const o_nodebound *nb, const o_tray *ray, int bound, int slab_max_level, double *t0,
                         double *t1) /* node_bounds.cpp:199-211 */
{
    int read_slab = nb->level <= slab_max_level;
    switch (bound) {
    case O_BOUND_BOX:
        return box_interval(nb, ray, t0, t1);
    case O_BOUND_SLAB:
        return read_slab ? slab_interval(nb, ray, t0, t1) : box_interval(nb, ray, t0, t1);
    case O_BOUND_BOTH:
        return read_slab ? both_interval(nb, ray, t0, t1) : box_interval(nb, ray, t0, t1);
    }
    return 0;
}

static void height_range_walk(const o_uvtri *U, const o_pyramid *P, int level, int64_t i, int64_t j, double *h_min,
                              double *h_max) /* node_bounds.cpp:218-234 */
{
    double w = cell_width(P, level);
    v2 c = V2((i + 0.5) * w, (j + 0.5) * w);
    int overlap = classify_square(U, c, 0.5 * w);
    if (overlap == OUTSIDE)
        return;
    if (overlap == INSIDE || level == 0) {
        o_node n = pyramid_node(P, level, i, j);
        *h_min = dmin(*h_min, n.h_min);
        *h_max = dmax(*h_max, n.h_max);
        return;
    }
    for (int ch = 0; ch < 4; ++ch)
        height_range_walk(U, P, level - 1, 2 * i + (ch & 1), 2 * j + (ch >> 1), h_min, h_max);
}

static void triangle_height_range(const o_tri *T, const o_pyramid *P, double *h_min, double *h_max)
{
    /* node_bounds.cpp:238-249 */
    o_uvtri U;
    uvtri_init(&U, T->t0, T->t1, T->t2);
    int level;
    int64_t i0, j0;
    footprint_roots(&U, P->n_leaf, &level, &i0, &j0);
    *h_min = INFINITY;
    *h_max = -INFINITY;
    for (int ch = 0; ch < 4; ++ch)
        height_range_walk(&U, P, level, i0 + (ch & 1), j0 + (ch >> 1), h_min, h_max);
}

static o_box triangle_aabb(const o_tri *T, double h_min, double h_max) /* node_bounds.cpp:251-269 */
{
    const v2 t[3] = {T->t0, T->t1, T->t2};
    af h = AF(0.5 * (h_min + h_max), 0.0, 0.0, 0.5 * (h_max - h_min));
    o_box box = {V3(INFINITY, INFINITY, INFINITY), V3(-INFINITY, -INFINITY, -INFINITY)};
    for (int k = 0; k < 3; ++k) {
        v2 tk = t[k], tk1 = t[(k + 1) % 3], tk2 = t[(k + 2) % 3];
        v2 c = add2(add2(mul2(0.5, tk), mul2(0.25, tk1)), mul2(0.25, tk2));
        v2 du = mul2(0.25, sub2(tk1, tk)), dv = mul2(0.25, sub2(tk2, tk));
        af3 Pf = AF3(tri_P(T, c.x, c.y), add3(mul3(du.x, T->e1), mul3(du.y, T->e2)),
                     add3(mul3(dv.x, T->e1), mul3(dv.y, T->e2)));
        af3 Nf = AF3(tri_M(T, c.x, c.y), add3(mul3(du.x, T->Mu), mul3(du.y, T->Mv)),
                     add3(mul3(dv.x, T->Mu), mul3(dv.y, T->Mv)));
        af3_normalize(&Nf);
        o_box b = hull(af3_add(Pf, af3_scale_form(h, Nf)));
        box_expand(&box, &b);
    }
    return box;
}

/* ------------------------------------------------------------------------ */
/* The walk and the leaves, displaced_intersector.cpp.                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    int level;
    int64_t i, j;
} o_cell;

static inline int64_t floor_div2(int64_t x) { return x >= 0 ? x / 2 : -((-x + 1) / 2); } /* :18 */
static inline int floor_mod2(int64_t x) { return (int)(x - 2 * floor_div2(x)); }            /* :19 */
static inline void cell_up(o_cell *c)                                                       /* :85-90 */
{
    ++c->level;
    c->i = floor_div2(c->i);
    c->j = floor_div2(c->j);
}
static inline void cell_down(o_cell *c, int si, int sj) /* :92-97 */
{
    --c->level;
    c->i = 2 * c->i + (si ? 1 : 0);
    c->j = 2 * c->j + (sj ? 1 : 0);
}
static void cell_next(o_cell *c, int si, int sj, int root_level) /* :99-121 */
{
    for (;;) {
        int code = 2 * floor_mod2(c->i + (si ? 1 : 0)) + floor_mod2(c->j + (sj ? 1 : 0));
        switch (code) {
        case 1:
            c->j += sj ? 1 : -1;
            c->i += si ? -1 : 1;
            return;
        case 3:
            cell_up(c);
            if (c->level > root_level)
                return;
            break;
        default:
            c->j += sj ? -1 : 1;
            return;
        }
    }
}

typedef struct {
    const o_tri *tri;
    const o_pyramid *pyr;
    const o_grid *field;
    o_frame frame;
    o_uvtri domain;
    int root_level;
    o_cell roots[4];
    int n_roots;
    double residual_tolerance;
    int max_iterations, subdivision_depth;
    o_box box;
    double h_min, h_max;
} o_isect;

typedef struct {
    double t;
    v2 st, bary;
    v3 ng;
    int64_t i, j;
} o_hit;

static void isect_init(o_isect *X, const o_tri *T, const o_pyramid *P, const o_grid *g) /* :135-151 */
{
    X->tri = T;
    X->pyr = P;
    X->field = g;
    tangent_frame(&X->frame, T);
    uvtri_init(&X->domain, T->t0, T->t1, T->t2);
    int64_t i0, j0;
    footprint_roots(&X->domain, P->n_leaf, &X->root_level, &i0, &j0);
    double w = cell_width(P, X->root_level);
    int64_t i_lo = (int64_t)floor(X->domain.lo.x / w), i_hi = (int64_t)ceil(X->domain.hi.x / w) - 1;
    int64_t j_lo = (int64_t)floor(X->domain.lo.y / w), j_hi = (int64_t)ceil(X->domain.hi.y / w) - 1;
    X->n_roots = 0;
    for (int64_t j = j_lo; j <= j_hi; ++j)
        for (int64_t i = i_lo; i <= i_hi; ++i) {
            o_cell c = {X->root_level, i, j};
            X->roots[X->n_roots++] = c;
        }
    X->residual_tolerance = 1e-10 * mean_edge(T);
    X->max_iterations = 20;
    X->subdivision_depth = 5;
}

static void plane_basis(v3 n, v3 *d1, v3 *d2) /* :222-227 */
{
    v3 a = fabs(n.x) < 0.9 ? V3(1.0, 0.0, 0.0) : V3(0.0, 1.0, 0.0);
    *d1 = normalized3(cross3(a, n));
    *d2 = cross3(n, *d1);
}

static int ray_triangle(v3 o, v3 d, double t_min, double t_max, v3 A, v3 B, v3 C, double *t, double *b1,
                        double *b2) /* :230-249 */
{
    v3 e1 = sub3(B, A), e2 = sub3(C, A);
    v3 p = cross3(d, e2);
    double det = dot3(e1, p);
    if (det == 0.0)
        return 0;
    double inv = 1.0 / det;
    v3 s = sub3(o, A);
    *b1 = dot3(s, p) * inv;
    if (*b1 < 0.0 || *b1 > 1.0)
        return 0;
    v3 q = cross3(s, e1);
    *b2 = dot3(d, q) * inv;
    if (*b2 < 0.0 || *b1 + *b2 > 1.0)
        return 0;
    *t = dot3(e2, q) * inv;
    return *t > t_min && *t < t_max;
}

typedef struct {
    v2 lo;
    double w;
    double h00, h10, h01, h11;
    af3 N_hat;
    v3 o, d, dn, d1, d2;
    double d_len;
} o_leafbound;

static inline af restricted(af f, double a, double b, double rho) /* :272-276 */
{
    double alpha = 2.0 * a - 1.0, beta = 2.0 * b - 1.0, r = 2.0 * rho;
    return AF((f.c + f.a * alpha) + f.b * beta, f.a * r, f.b * r, f.k);
}

static int newton_from(const o_isect *X, v3 o, v3 d, double t_min, double t_max, int64_t i, int64_t j, v2 guess,
                       o_hit *hit, int64_t *iters) /* :325-388 */
{
    const o_tri *T = X->tri;
    double w = cell_width(X->pyr, 0);
    v2 lo = V2(i * w, j * w), hi = V2((i + 1) * w, (j + 1) * w);
    double d_len = norm3(d);
    v3 dn = div3(d, d_len), d1, d2;
    plane_basis(dn, &d1, &d2);
    double prev_err2 = INFINITY;
    int err_streak = 0, behind_streak = 0, invalid_streak = 0;
    for (int iter = 0; iter < X->max_iterations; ++iter) {
        if (iters)
            ++*iters;
        double s = guess.x, t = guess.y;
        o_nframe f = normal_frame_at(T, s, t);
        double h = grid_h(X->field, s, t);
        v2 gh = grid_grad(X->field, s, t);
        v3 S = add3(tri_P(T, s, t), mul3(h, f.N));
        v3 delta = sub3(S, o);
        v2 F = V2(dot3(delta, d1), dot3(delta, d2));
        double err2 = F.x * F.x + F.y * F.y;
        double along = dot3(delta, dn);
        err_streak = err2 > prev_err2 ? err_streak + 1 : 0;
        behind_streak = along < 0.0 ? behind_streak + 1 : 0;
        if (err_streak >= 2 || behind_streak >= 2)
            return 0;
        prev_err2 = err2;
        v3 Su = add3(add3(T->e1, mul3(gh.x, f.N)), mul3(h, f.Nu));
        v3 Sv = add3(add3(T->e2, mul3(gh.y, f.N)), mul3(h, f.Nv));
        if (err2 < X->residual_tolerance * X->residual_tolerance) {
            if (along < 0.0 || !uvtri_inside(&X->domain, guess))
                return 0;
            double t_hit = along / d_len;
            if (t_hit <= t_min || t_hit >= t_max)
                return 0;
            hit->t = t_hit;
            hit->st = guess;
            hit->bary = tri_bary(T, s, t);
            hit->ng = normalized3(cross3(Su, Sv));
            hit->i = i;
            hit->j = j;
            return 1;
        }
        double J00 = dot3(d1, Su), J01 = dot3(d1, Sv), J10 = dot3(d2, Su), J11 = dot3(d2, Sv);
        double det = J00 * J11 - J01 * J10;
        if (det == 0.0)
            return 0;
        v2 step = V2((J11 * F.x - J01 * F.y) / det, (-J10 * F.x + J00 * F.y) / det);
        guess = sub2(guess, step);
        int outside = guess.x < lo.x || guess.x > hi.x || guess.y < lo.y || guess.y > hi.y ||
                      !uvtri_inside(&X->domain, guess);
        if (outside) {
            if (++invalid_streak >= 3)
                return 0;
            guess = min2(max2(guess, lo), hi);
        } else {
            invalid_streak = 0;
        }
    }
    return 0;
}

static int sub_square_bound(const o_isect *X, const o_leafbound *L, double a, double b, double rho, double t_min,
                            double t_max, double *t_lo) /* :266-290 */
{
    const o_tri *T = X->tri;
    v2 c = add2(L->lo, mul2(L->w, V2(a, b)));
    if (classify_square(&X->domain, c, L->w * rho) == OUTSIDE)
        return 0;
    double Tw = ((L->h11 - L->h10) - L->h01) + L->h00;
    double ha = L->h10 - L->h00, hb = L->h01 - L->h00;
    af h = AF(((L->h00 + ha * a) + hb * b) + Tw * a * b, (ha + Tw * b) * rho, (hb + Tw * a) * rho,
              fabs(Tw) * rho * rho);
    double wr = L->w * rho;
    af3 P = AF3(tri_P(T, c.x, c.y), mul3(wr, T->e1), mul3(wr, T->e2));
    af3 Nr = {restricted(L->N_hat.x, a, b, rho), restricted(L->N_hat.y, a, b, rho),
              restricted(L->N_hat.z, a, b, rho)};
    af3 S = af3_add(P, af3_scale_form(h, Nr));
    af F1 = af_dot(L->d1, S), F2 = af_dot(L->d2, S);
    F1.c -= dot3(L->d1, L->o);
    F2.c -= dot3(L->d2, L->o);
    ivl i1 = af_interval(F1), i2 = af_interval(F2);
    if (!(i1.lo <= 0.0 && 0.0 <= i1.hi) || !(i2.lo <= 0.0 && 0.0 <= i2.hi))
        return 0;
    af along = af_dot(L->dn, S);
    along.c -= dot3(L->dn, L->o);
    ivl range = af_interval(along);
    *t_lo = range.lo / L->d_len;
    return *t_lo < t_max && range.hi / L->d_len > t_min;
}

static void search_leaf(const o_isect *X, const o_leafbound *L, int64_t i, int64_t j, int depth, double a, double b,
                        double rho, double t_min, double *t_max, o_hit *hit, int *found, int64_t *sub_squares,
                        int64_t *iters) /* :292-323 */
{
    if (depth == X->subdivision_depth) {
        o_hit h;
        if (newton_from(X, L->o, L->d, t_min, *t_max, i, j, add2(L->lo, mul2(L->w, V2(a, b))), &h, iters)) {
            *hit = h;
            *t_max = h.t;
            *found = 1;
        }
        return;
    }
    struct { double a, b, t_lo; } ch[4];
    int n = 0;
    double r = 0.5 * rho;
    for (int q = 0; q < 4; ++q) {
        double ca = a + ((q & 1) ? r : -r), cb = b + ((q & 2) ? r : -r), t_lo;
        ++*sub_squares;
        if (sub_square_bound(X, L, ca, cb, r, t_min, *t_max, &t_lo)) {
            ch[n].a = ca;
            ch[n].b = cb;
            ch[n].t_lo = t_lo;
            ++n;
        }
    }
    /* std::sort of at most four: stable insertion by t_lo. */
    for (int p = 1; p < n; ++p) {
        for (int q = p; q > 0 && ch[q].t_lo < ch[q - 1].t_lo; --q) {
            double ta = ch[q].a, tb = ch[q].b, tt = ch[q].t_lo;
            ch[q] = ch[q - 1];
            ch[q - 1].a = ta;
            ch[q - 1].b = tb;
            ch[q - 1].t_lo = tt;
        }
    }
    for (int q = 0; q < n; ++q) {
        if (ch[q].t_lo >= *t_max)
            break;
        search_leaf(X, L, i, j, depth + 1, ch[q].a, ch[q].b, r, t_min, t_max, hit, found, sub_squares, iters);
    }
}

static int intersect_newton(const o_isect *X, v3 o, v3 d, double t_min, double t_max, int64_t i, int64_t j,
                            o_hit *hit, int64_t *sub_squares, int64_t *iters) /* :239-264 */
{
    const o_tri *T = X->tri;
    o_leafbound L;
    L.w = cell_width(X->pyr, 0);
    L.lo = V2(i * L.w, j * L.w);
    L.h00 = grid_h(X->field, L.lo.x, L.lo.y);
    L.h10 = grid_h(X->field, L.lo.x + L.w, L.lo.y);
    L.h01 = grid_h(X->field, L.lo.x, L.lo.y + L.w);
    L.h11 = grid_h(X->field, L.lo.x + L.w, L.lo.y + L.w);
    v2 c = add2(L.lo, V2(0.5 * L.w, 0.5 * L.w));
    double hw = 0.5 * L.w;
    L.N_hat = AF3(add3(add3(T->m0, mul3(c.x, T->Mu)), mul3(c.y, T->Mv)), mul3(hw, T->Mu), mul3(hw, T->Mv));
    af3_normalize(&L.N_hat);
    L.o = o;
    L.d = d;
    L.d_len = norm3(d);
    L.dn = div3(d, L.d_len);
    plane_basis(L.dn, &L.d1, &L.d2);
    int found = 0;
    int64_t count = 0;
    search_leaf(X, &L, i, j, 0, 0.5, 0.5, 0.5, t_min, &t_max, hit, &found, &count, iters);
    if (sub_squares)
        *sub_squares += count;
    return found;
}

static int intersect_two_triangle(const o_isect *X, v3 o, v3 d, double t_min, double t_max, int64_t i, int64_t j,
                                  o_hit *hit) /* :390-426 */
{
    const o_tri *T = X->tri;
    double w = cell_width(X->pyr, 0);
    v2 st00 = V2(i * w, j * w), st10 = V2((i + 1) * w, j * w), st01 = V2(i * w, (j + 1) * w),
       st11 = V2((i + 1) * w, (j + 1) * w);
    v3 S00 = displaced_position(T, X->field, st00.x, st00.y);
    v3 S10 = displaced_position(T, X->field, st10.x, st10.y);
    v3 S01 = displaced_position(T, X->field, st01.x, st01.y);
    v3 S11 = displaced_position(T, X->field, st11.x, st11.y);
    v3 A[2] = {S00, S10}, B[2] = {S10, S11}, C[2] = {S01, S01};
    v2 a[2] = {st00, st10}, b[2] = {st10, st11}, c[2] = {st01, st01};
    int found = 0;
    for (int k = 0; k < 2; ++k) {
        double t, b1, b2;
        if (!ray_triangle(o, d, t_min, t_max, A[k], B[k], C[k], &t, &b1, &b2))
            continue;
        v2 st = add2(add2(mul2((1.0 - b1) - b2, a[k]), mul2(b1, b[k])), mul2(b2, c[k]));
        if (!uvtri_inside(&X->domain, st))
            continue;
        hit->t = t;
        hit->st = st;
        hit->bary = tri_bary(T, st.x, st.y);
        hit->ng = normalized3(cross3(sub3(B[k], A[k]), sub3(C[k], A[k])));
        hit->i = i;
        hit->j = j;
        t_max = t;
        found = 1;
    }
    return found;
}

static int isect_intersect(const o_isect *X, v3 o, v3 d, double t_min, double t_max, int bound, int slab_max_level,
                           int leaf, o_hit *hit, int64_t *st, int64_t *level_stats) /* :175-237 */
{
    o_tray ray = {m3mul(&X->frame.to_tangent, sub3(o, X->frame.origin)), m3mul(&X->frame.to_tangent, d), t_min,
                  t_max};
    int si = ray.d.x < 0.0, sj = ray.d.y < 0.0;
    int found = 0;
    int64_t nah = 0, lah = 0;
    for (int r = 0; r < X->n_roots; ++r) {
        o_cell cur = X->roots[r], end = X->roots[r];
        cell_next(&end, si, sj, X->root_level);
        while (!(cur.level == end.level && cur.i == end.i && cur.j == end.j)) {
            double w = cell_width(X->pyr, cur.level);
            v2 c = V2((cur.i + 0.5) * w, (cur.j + 0.5) * w);
            if (classify_square(&X->domain, c, 0.5 * w) == OUTSIDE) {
                cell_next(&cur, si, sj, X->root_level);
                continue;
            }
            if (st) {
                ++st[O_ST_NODE_TESTS];
                ++nah;
            }
            if (level_stats)
                ++level_stats[cur.level < 31 ? cur.level : 31];
            o_nodebound nb;
            node_bound(&nb, X->tri, &X->frame, X->pyr, cur.level, cur.i, cur.j);
            ray.t_max = t_max;
            double t0, t1;
            if (!node_interval(&nb, &ray, bound, slab_max_level, &t0, &t1)) {
                cell_next(&cur, si, sj, X->root_level);
                continue;
            }
            if (cur.level > 0) {
                cell_down(&cur, si, sj);
                continue;
            }
            if (st) {
                ++st[O_ST_LEAF_TESTS];
                ++lah;
            }
            o_hit lh;
            int lf;
            if (leaf == O_LEAF_NEWTON)
                lf = intersect_newton(X, o, d, t_min, t_max, cur.i, cur.j, &lh, st ? &st[O_ST_SUB_SQUARES] : NULL,
                                      st ? &st[O_ST_NEWTON_ITERS] : NULL);
            else
                lf = intersect_two_triangle(X, o, d, t_min, t_max, cur.i, cur.j, &lh);
            if (lf && lh.t < t_max) {
                *hit = lh;
                t_max = lh.t;
                found = 1;
                nah = 0;
                lah = 0;
            }
            cell_next(&cur, si, sj, X->root_level);
        }
    }
    if (st && found) {
        st[O_ST_NODE_AFTER_HIT] += nah;
        st[O_ST_LEAF_AFTER_HIT] += lah;
    }
    return found;
}

/* ------------------------------------------------------------------------ */
/* Objects and scenes.                                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    double *values;
    o_grid *grid; /* heap: the triangles' intersectors point at it while obj[] grows */
    o_pyramid *pyr;
    int n_tri, first_tri;
    o_tri *tris;
    o_isect *isects;
} o_object;

struct o_scene {
    int n_obj, cap;
    o_object *obj;
    int n_tri;
    /* the opacity filter (o_scene_set_opacity); op_mask NULL: none */
    uint8_t *op_mask, *op_tri;
    int op_w, op_h, op_flip;
    double op_scale[2], op_offset[2];
};

o_scene *o_scene_create(void) { return (o_scene *)calloc(1, sizeof(o_scene)); }

void o_scene_free(o_scene *s)
{
    if (!s)
        return;
    for (int k = 0; k < s->n_obj; ++k) {
        free(s->obj[k].values);
        free(s->obj[k].grid);
        o_pyramid_free(s->obj[k].pyr);
        free(s->obj[k].tris);
        free(s->obj[k].isects);
    }
    free(s->obj);
    free(s->op_mask);
    free(s->op_tri);
    free(s);
}

void o_scene_set_opacity(o_scene *s, const uint8_t *mask, int w, int h, const double *map5, const uint8_t *tri_flags)
{
    free(s->op_mask);
    free(s->op_tri);
    s->op_mask = s->op_tri = NULL;
    if (!mask || w <= 0 || h <= 0)
        return;
    s->op_mask = (uint8_t *)malloc((size_t)w * h);
    memcpy(s->op_mask, mask, (size_t)w * h);
    if (tri_flags) {
        s->op_tri = (uint8_t *)malloc((size_t)(s->n_tri > 0 ? s->n_tri : 1));
        memcpy(s->op_tri, tri_flags, (size_t)s->n_tri);
    }
    s->op_w = w;
    s->op_h = h;
    s->op_scale[0] = map5 ? map5[0] : 1.0;
    s->op_scale[1] = map5 ? map5[1] : 1.0;
    s->op_offset[0] = map5 ? map5[2] : 0.0;
    s->op_offset[1] = map5 ? map5[3] : 0.0;
    s->op_flip = map5 ? map5[4] != 0.0 : 0;
}

int o_scene_add_object(o_scene *s, const double *values, int W, double scale, double offset, int repeat, int build,
                       const double *tris, int n_tri)
{
    if (s->n_obj == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 8;
        s->obj = (o_object *)realloc(s->obj, (size_t)s->cap * sizeof(o_object));
    }
    o_object *O = &s->obj[s->n_obj];
    memset(O, 0, sizeof(*O));
    O->values = (double *)malloc((size_t)W * W * sizeof(double));
    memcpy(O->values, values, (size_t)W * W * sizeof(double));
    O->grid = (o_grid *)calloc(1, sizeof(o_grid));
    O->grid->W = W;
    O->grid->H = W;
    O->grid->scale = scale;
    O->grid->values = O->values;
    O->grid->offset = offset;
    O->grid->repeat = repeat;
    O->pyr = o_pyramid_build(O->values, W, scale, offset, build);
    if (!O->pyr) {
        free(O->values);
        free(O->grid);
        return -1;
    }
    O->n_tri = n_tri;
    O->first_tri = s->n_tri;
    O->tris = (o_tri *)calloc((size_t)n_tri, sizeof(o_tri));
    O->isects = (o_isect *)calloc((size_t)n_tri, sizeof(o_isect));
    for (int k = 0; k < n_tri; ++k) {
        if (!tri_init(&O->tris[k], tris + 24 * (size_t)k)) {
            o_pyramid_free(O->pyr);
            free(O->values);
            free(O->grid);
            free(O->tris);
            free(O->isects);
            return -1;
        }
    }
    for (int k = 0; k < n_tri; ++k) { /* displaced_intersector.cpp:466-479 */
        o_isect *X = &O->isects[k];
        isect_init(X, &O->tris[k], O->pyr, O->grid);
        triangle_height_range(&O->tris[k], O->pyr, &X->h_min, &X->h_max);
        X->box = triangle_aabb(&O->tris[k], X->h_min, X->h_max);
    }
    s->n_tri += n_tri;
    return s->n_obj++;
}

int o_scene_triangle_count(const o_scene *s) { return s->n_tri; }

static const o_isect *find_tri(const o_scene *s, int tri, int *obj)
{
    for (int k = 0; k < s->n_obj; ++k) {
        if (tri < s->obj[k].first_tri + s->obj[k].n_tri) {
            if (obj)
                *obj = k;
            return &s->obj[k].isects[tri - s->obj[k].first_tri];
        }
    }
    return NULL;
}

void o_scene_triangle_info(const o_scene *s, int tri, double *out)
{
    const o_isect *X = find_tri(s, tri, NULL);
    out[0] = X->root_level;
    out[1] = X->n_roots;
    out[2] = X->residual_tolerance;
    out[3] = X->box.lo.x;
    out[4] = X->box.lo.y;
    out[5] = X->box.lo.z;
    out[6] = X->box.hi.x;
    out[7] = X->box.hi.y;
    out[8] = X->box.hi.z;
    out[9] = X->h_min;
    out[10] = X->h_max;
}

void o_scene_triangle_frame(const o_scene *s, int tri, double *out)
{
    const o_isect *X = find_tri(s, tri, NULL);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            out[3 * i + j] = X->frame.to_tangent.m[i][j];
    out[9] = X->frame.ng.x;
    out[10] = X->frame.ng.y;
    out[11] = X->frame.ng.z;
}

static void write_hit(double *out, const o_hit *h, int tri, int obj)
{
    out[0] = h->t;
    out[1] = h->st.x;
    out[2] = h->st.y;
    out[3] = h->bary.x;
    out[4] = h->bary.y;
    out[5] = h->ng.x;
    out[6] = h->ng.y;
    out[7] = h->ng.z;
    out[8] = (double)h->i;
    out[9] = (double)h->j;
    out[10] = tri;
    out[11] = obj;
}

static void write_miss(double *out)
{
    for (int k = 0; k < O_HIT_DOUBLES; ++k)
        out[k] = 0.0;
    out[0] = INFINITY;
    out[10] = -1.0;
    out[11] = -1.0;
}

/* A candidate of the nearest-first order: the triangle's box entry key and
 * its scene-global index. */
typedef struct {
    double key;
    int ob, k, g;
} o_cand;

static int cand_cmp(const void *pa, const void *pb)
{
    const o_cand *a = (const o_cand *)pa, *b = (const o_cand *)pb;
    if (a->key != b->key)
        return a->key < b->key ? -1 : 1;
    return (a->g > b->g) - (a->g < b->g);
}

/* The nearest-first key (not in the reference: the order a BVH over the
 * embree callbacks gives, displaced_geometry.cpp:49-106, made exact):
 * max(t_min, max over axes with d != 0 of min(ta, tb)), ta = (lo - o) * (1 / d). */
static double entry_key(const o_box *B, v3 o, v3 d, const double *inv, double t_min)
{
    double key = t_min;
    for (int a = 0; a < 3; ++a)
        if (comp3(d, a) != 0.0) {
            double ta = (comp3(B->lo, a) - comp3(o, a)) * inv[a], tb = (comp3(B->hi, a) - comp3(o, a)) * inv[a];
            key = dmax(key, dmin(ta, tb));
        }
    return key;
}

/* The opacity filter (not in the reference's sources: ks's opacity map
 * behind embree's filter functions, reduced to a binary texel mask): the
 * crossing's texture coordinate as compute_hit_texcoord forms it
 * (displaced_geometry.cpp:189-193) from the float barycentrics of
 * potential_hit (:21-34), BaseTriangle::param (displaced_surface.h:87) and
 * DisplacedObject::object_uv (scene_spec.cpp:382-388) rounded to float,
 * then the mask texel under it with repeat; 0 rejects. */
static int crossing_opaque(const o_scene *s, const o_tri *T, int g, const o_hit *h)
{
    if (!s->op_mask || (s->op_tri && !s->op_tri[g]))
        return 1;
    double u = (double)(float)h->bary.x, v = (double)(float)h->bary.y;
    double ps = (T->t0.x + u * (T->t1.x - T->t0.x)) + v * (T->t2.x - T->t0.x);
    double pt = (T->t0.y + u * (T->t1.y - T->t0.y)) + v * (T->t2.y - T->t0.y);
    double x = (ps - s->op_offset[0]) / s->op_scale[0], y = (pt - s->op_offset[1]) / s->op_scale[1];
    if (s->op_flip)
        y = 1.0 - y;
    double fx = (double)(float)x * s->op_w, fy = (double)(float)y * s->op_h;
    if (!(fabs(fx) < 1e15 && fabs(fy) < 1e15))
        return 1;
    long long i = (long long)floor(fx) % s->op_w, j = (long long)floor(fy) % s->op_h;
    if (i < 0)
        i += s->op_w;
    if (j < 0)
        j += s->op_h;
    return s->op_mask[j * s->op_w + i] != 0;
}

/* The intersect / occluded callback's passes (displaced_geometry.cpp:53-106):
 * a crossing the filter rejects raises t_min to its t and the triangle is
 * walked again, at most max_filter_passes = 64 times (displaced_geometry.h:64). */
static int isect_filtered(const o_scene *s, const o_isect *X, int g, v3 o, v3 d, double t_min, double t_max,
                          int bound, int slab_max_level, int leaf, o_hit *h, int64_t *st, int64_t *level_stats)
{
    if (!s->op_mask)
        return isect_intersect(X, o, d, t_min, t_max, bound, slab_max_level, leaf, h, st, level_stats);
    double t_lo = t_min;
    for (int pass = 0; pass < 64; ++pass) {
        if (!isect_intersect(X, o, d, t_lo, t_max, bound, slab_max_level, leaf, h, st, level_stats))
            return 0;
        if (crossing_opaque(s, X->tri, g, h))
            return 1;
        t_lo = h->t; /* the walk accepts t > t_min only */
    }
    return 0;
}

/* The flat loop of ObjectIntersector::intersect_flat (:578-599) over every
 * object (order O_ORDER_INDEX); or (O_ORDER_NEAREST) the same loop over the
 * triangles whose boxes the ray meets, sorted by (key, index), each still
 * box-tested with the t_max of the ones before it. cand: n_tri scratch. */
static int scene_intersect1(const o_scene *s, const double *ray, int bound, int slab_max_level, int leaf,
                            double *out, int64_t *st, int64_t *level_stats, int order, o_cand *cand)
{
    v3 o = V3(ray[0], ray[1], ray[2]), d = V3(ray[3], ray[4], ray[5]);
    double t_min = ray[6], t_max = ray[7];
    int found = 0;
    write_miss(out);
    if (order == O_ORDER_NEAREST) {
        double inv[3];
        for (int a = 0; a < 3; ++a)
            inv[a] = comp3(d, a) != 0.0 ? 1.0 / comp3(d, a) : 0.0;
        int nc = 0;
        for (int ob = 0; ob < s->n_obj; ++ob) {
            const o_object *O = &s->obj[ob];
            for (int k = 0; k < O->n_tri; ++k) {
                double t0 = t_min, t1 = t_max;
                if (!box_clip(&O->isects[k].box, o, d, &t0, &t1))
                    continue;
                o_cand c = {entry_key(&O->isects[k].box, o, d, inv, t_min), ob, k, O->first_tri + k};
                cand[nc++] = c;
            }
        }
        qsort(cand, (size_t)nc, sizeof(o_cand), cand_cmp);
        for (int c = 0; c < nc; ++c) {
            const o_object *O = &s->obj[cand[c].ob];
            const o_isect *X = &O->isects[cand[c].k];
            double t0 = t_min, t1 = t_max;
            if (!box_clip(&X->box, o, d, &t0, &t1))
                continue;
            if (st)
                ++st[O_ST_TRIANGLE_TESTS];
            o_hit h;
            if (isect_filtered(s, X, cand[c].g, o, d, t_min, t_max, bound, slab_max_level, leaf, &h, st,
                               level_stats)) {
                write_hit(out, &h, cand[c].g, cand[c].ob);
                t_max = h.t;
                found = 1;
            }
        }
        return found;
    }
    for (int ob = 0; ob < s->n_obj; ++ob) {
        const o_object *O = &s->obj[ob];
        for (int k = 0; k < O->n_tri; ++k) {
            double t0 = t_min, t1 = t_max;
            if (!box_clip(&O->isects[k].box, o, d, &t0, &t1))
                continue;
            if (st)
                ++st[O_ST_TRIANGLE_TESTS];
            o_hit h;
            if (isect_filtered(s, &O->isects[k], O->first_tri + k, o, d, t_min, t_max, bound, slab_max_level, leaf,
                               &h, st, level_stats)) {
                write_hit(out, &h, O->first_tri + k, ob);
                t_max = h.t;
                found = 1;
            }
        }
    }
    return found;
}

typedef struct {
    const o_scene *s;
    const double *rays;
    int64_t n;
    int bound, slab_max_level, leaf, order, threads;
    double *hits;
    int64_t *stats;
    atomic_llong next;
    atomic_llong n_hit;
    int64_t level_stats[32];
    pthread_mutex_t mu;
    int64_t *level_out;
} o_job;

static void *worker(void *arg)
{
    o_job *J = (o_job *)arg;
    int64_t local_levels[32] = {0};
    int64_t local_hits = 0;
    /* chunks of at most 4096 rays, small enough that every thread gets work */
    int64_t chunk = J->n / (8 * (int64_t)J->threads);
    chunk = chunk < 1 ? 1 : chunk > 4096 ? 4096 : chunk;
    o_cand *cand = (o_cand *)malloc(sizeof(o_cand) * (size_t)(J->s->n_tri > 0 ? J->s->n_tri : 1));
    for (;;) {
        int64_t b = atomic_fetch_add(&J->next, chunk);
        if (b >= J->n)
            break;
        int64_t e = b + chunk < J->n ? b + chunk : J->n;
        for (int64_t r = b; r < e; ++r) {
            int64_t *st = J->stats ? J->stats + r * O_ST_COUNT : NULL;
            if (st)
                memset(st, 0, O_ST_COUNT * sizeof(int64_t));
            local_hits += scene_intersect1(J->s, J->rays + 8 * r, J->bound, J->slab_max_level, J->leaf,
                                           J->hits + O_HIT_DOUBLES * r, st, J->level_out ? local_levels : NULL,
                                           J->order, cand);
        }
    }
    free(cand);
    atomic_fetch_add(&J->n_hit, local_hits);
    if (J->level_out) {
        pthread_mutex_lock(&J->mu);
        for (int l = 0; l < 32; ++l)
            J->level_out[l] += local_levels[l];
        pthread_mutex_unlock(&J->mu);
    }
    return NULL;
}

int64_t o_scene_intersect(const o_scene *s, const double *rays, int64_t n, int bound, int slab_max_level, int leaf,
                          double *hits, int64_t *stats, int64_t *level_stats, int threads, int order)
{
    if (threads <= 0)
        threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1)
        threads = 1;
    o_job J;
    memset(&J, 0, sizeof(J));
    J.s = s;
    J.rays = rays;
    J.n = n;
    J.bound = bound;
    J.slab_max_level = slab_max_level;
    J.leaf = leaf;
    J.order = order;
    J.threads = threads;
    J.hits = hits;
    J.stats = stats;
    J.level_out = level_stats;
    atomic_init(&J.next, 0);
    atomic_init(&J.n_hit, 0);
    pthread_mutex_init(&J.mu, NULL);
    if (threads == 1) {
        worker(&J);
    } else {
        pthread_t *th = (pthread_t *)malloc((size_t)threads * sizeof(pthread_t));
        for (int k = 0; k < threads; ++k)
            pthread_create(&th[k], NULL, worker, &J);
        for (int k = 0; k < threads; ++k)
            pthread_join(th[k], NULL);
        free(th);
    }
    pthread_mutex_destroy(&J.mu);
    return (int64_t)atomic_load(&J.n_hit);
}

int o_triangle_intersect(const o_scene *s, int tri, const double *ray, int bound, int slab_max_level, int leaf,
                         double *out, int64_t *stats)
{
    int ob = -1;
    const o_isect *X = find_tri(s, tri, &ob);
    o_hit h;
    write_miss(out);
    if (stats)
        memset(stats, 0, O_ST_COUNT * sizeof(int64_t));
    int f = isect_intersect(X, V3(ray[0], ray[1], ray[2]), V3(ray[3], ray[4], ray[5]), ray[6], ray[7], bound,
                            slab_max_level, leaf, &h, stats, NULL);
    if (f)
        write_hit(out, &h, tri, ob);
    return f;
}

void o_node_bound(const o_scene *s, int tri, int level, int64_t i, int64_t j, const double *ray, int bound,
                  int slab_max_level, double *out)
{
    const o_isect *X = find_tri(s, tri, NULL);
    o_nodebound nb;
    node_bound(&nb, X->tri, &X->frame, X->pyr, level, i, j);
    o_tray tr = {m3mul(&X->frame.to_tangent, sub3(V3(ray[0], ray[1], ray[2]), X->frame.origin)),
                 m3mul(&X->frame.to_tangent, V3(ray[3], ray[4], ray[5])), ray[6], ray[7]};
    out[0] = nb.box.lo.x;
    out[1] = nb.box.lo.y;
    out[2] = nb.box.lo.z;
    out[3] = nb.box.hi.x;
    out[4] = nb.box.hi.y;
    out[5] = nb.box.hi.z;
    ivl mx = af_interval(nb.m.x), my = af_interval(nb.m.y), mz = af_interval(nb.m.z);
    out[6] = mx.lo;
    out[7] = mx.hi;
    out[8] = my.lo;
    out[9] = my.hi;
    out[10] = mz.lo;
    out[11] = mz.hi;
    double t0, t1;
    out[12] = box_interval(&nb, &tr, &t0, &t1);
    out[13] = slab_interval(&nb, &tr, &t0, &t1);
    int pass = node_interval(&nb, &tr, bound, slab_max_level, &t0, &t1);
    out[14] = pass ? t0 : NAN;
    out[15] = pass ? t1 : NAN;
}

void o_displaced_position(const o_scene *s, int tri, double sp, double tp, double *out)
{
    const o_isect *X = find_tri(s, tri, NULL);
    v3 S = displaced_position(X->tri, X->field, sp, tp);
    out[0] = S.x;
    out[1] = S.y;
    out[2] = S.z;
}

void o_triangle_param(const o_scene *s, int tri, double u, double v, double *out)
{
    const o_isect *X = find_tri(s, tri, NULL);
    v2 p = tri_param(X->tri, u, v);
    out[0] = p.x;
    out[1] = p.y;
}

/* DisplacedGeometry::surface_point (displaced_geometry.cpp:126-152) on
 * triangle tri at barycentrics (u, v), with the object's uv map
 * (DisplacedObject::object_uv, scene_spec.cpp:382-388): out14 = p, ng, dpdu,
 * dpdv, uv. Eigen's normalize() leaves a zero vector as it is. */
static v3 eigen_normalized(v3 a)
{
    double z = dot3(a, a);
    return z > 0.0 ? div3(a, sqrt(z)) : a;
}

void o_surface_point(const o_scene *s, int tri, double u, double v, const double *uv_scale, const double *uv_offset,
                     int flip_v, double *out)
{
    const o_isect *X = find_tri(s, tri, NULL);
    const o_tri *T = X->tri;
    v2 st = tri_param(T, u, v);
    double sp = st.x, tp = st.y;
    o_nframe f = normal_frame_at(T, sp, tp);
    double h = grid_h(X->field, sp, tp);
    v2 gh = grid_grad(X->field, sp, tp);
    v3 Ss = add3(add3(T->e1, mul3(gh.x, f.N)), mul3(h, f.Nu));
    v3 St = add3(add3(T->e2, mul3(gh.y, f.N)), mul3(h, f.Nv));
    v3 p = add3(tri_P(T, sp, tp), mul3(h, f.N));
    v3 wn = cross3(sub3(T->p1, T->p0), sub3(T->p2, T->p0));
    v3 ng = cross3(Ss, St);
    if (dot3(ng, wn) < 0.0)
        ng = V3(-ng.x, -ng.y, -ng.z);
    ng = eigen_normalized(ng);
    if (!(isfinite(ng.x) && isfinite(ng.y) && isfinite(ng.z)))
        ng = eigen_normalized(wn);
    double su = uv_scale[0], sv = flip_v ? -uv_scale[1] : uv_scale[1];
    v3 dpdu = mul3(su, Ss), dpdv = mul3(sv, St);
    double uvx = (sp - uv_offset[0]) / uv_scale[0], uvy = (tp - uv_offset[1]) / uv_scale[1];
    if (flip_v)
        uvy = 1.0 - uvy;
    double o[14] = {p.x, p.y, p.z, ng.x, ng.y, ng.z, dpdu.x, dpdu.y, dpdu.z, dpdv.x, dpdv.y, dpdv.z, uvx, uvy};
    memcpy(out, o, sizeof(o));
}

/* ------------------------------------------------------------------------ */
/* Oracle meshes, displaced_tessellation.cpp.                                */
/* ------------------------------------------------------------------------ */

/* pointwise_fields(tri, field, s, t).n (displaced_surface.cpp:110-158): the
 * unnormalized surface normal Su x Sv, h and its gradient from the grid. */
static v3 pointwise_normal(const o_tri *T, const o_grid *g, double s, double t)
{
    v2 gh = grid_grad(g, s, t);
    double h = grid_h(g, s, t);
    o_nframe f = normal_frame_at(T, s, t);
    v3 Su = add3(add3(T->e1, mul3(gh.x, f.N)), mul3(h, f.Nu));
    v3 Sv = add3(add3(T->e2, mul3(gh.y, f.N)), mul3(h, f.Nv));
    return cross3(Su, Sv);
}

/* chart_mirrored (displaced_surface.cpp:160). */
static int chart_mirrored(const o_tri *T)
{
    v3 wn = cross3(sub3(T->p1, T->p0), sub3(T->p2, T->p0));
    return dot3(cross3(T->e1, T->e2), wn) < 0.0;
}

static void put_vertex(v3 S, v2 st, v3 n, float *pos, float *uv, float *nrm)
{
    pos[0] = (float)S.x;
    pos[1] = (float)S.y;
    pos[2] = (float)S.z;
    uv[0] = (float)st.x;
    uv[1] = (float)st.y;
    nrm[0] = (float)n.x;
    nrm[1] = (float)n.y;
    nrm[2] = (float)n.z;
}

void o_tessellate_uniform(const o_scene *s, int tri, int n, float *pos, float *uv, float *nrm, uint32_t *idx)
{
    /* tessellation_grid (:11-30) and append_displaced_triangle (:32-56),
     * vertex indices relative to the triangle's first vertex */
    const o_isect *X = find_tri(s, tri, NULL);
    const o_tri *T = X->tri;
    int64_t k = 0;
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n - j; ++i, ++k) {
            v2 st = tri_param(T, (double)i / n, (double)j / n);
            v3 S = displaced_position(T, X->field, st.x, st.y);
            v3 nr = eigen_normalized(pointwise_normal(T, X->field, st.x, st.y));
            put_vertex(S, st, nr, pos + 3 * k, uv + 2 * k, nrm + 3 * k);
        }
#define TESS_INDEX(i, j) ((uint32_t)((j) * (n + 1) - (j) * ((j)-1) / 2 + (i)))
    int64_t f = 0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n - j; ++i) {
            idx[3 * f] = TESS_INDEX(i, j);
            idx[3 * f + 1] = TESS_INDEX(i + 1, j);
            idx[3 * f + 2] = TESS_INDEX(i, j + 1);
            ++f;
            if (i + j < n - 1) {
                idx[3 * f] = TESS_INDEX(i + 1, j);
                idx[3 * f + 1] = TESS_INDEX(i + 1, j + 1);
                idx[3 * f + 2] = TESS_INDEX(i, j + 1);
                ++f;
            }
        }
#undef TESS_INDEX
}

typedef struct {
    int n;
    v2 p[8];
} o_clip;

/* clip_square (uv_clip.cpp:56-83): Sutherland-Hodgman of the square (c, s)
 * against the domain's three inward half-planes. */
static o_clip clip_square(const o_uvtri *U, v2 c, double s)
{
    o_clip in;
    in.n = 4;
    in.p[0] = add2(c, V2(-s, -s));
    in.p[1] = add2(c, V2(s, -s));
    in.p[2] = add2(c, V2(s, s));
    in.p[3] = add2(c, V2(-s, s));
    for (int k = 0; k < 3; ++k) {
        o_clip out;
        out.n = 0;
        for (int a = 0; a < in.n; ++a) {
            v2 pa = in.p[a], pb = in.p[(a + 1) % in.n];
            double fa = dot2(U->n[k], pa) - U->d[k], fb = dot2(U->n[k], pb) - U->d[k];
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

typedef struct {
    const o_isect *X;
    int mirrored;
    int64_t n, cap;
    float *pos, *uv, *nrm;
    double *st6;
    int *interior;
} o_texel_out;

/* append_face / append_vertex (displaced_tessellation.cpp:61-99): three
 * unshared vertices per face, the normal oriented along the base face's
 * winding, b and c swapped under a mirrored chart. */
static void texel_face(o_texel_out *o, v2 a, v2 b, v2 c, int interior)
{
    if (o->mirrored) {
        v2 x = b;
        b = c;
        c = x;
    }
    if (o->n < o->cap) {
        const o_tri *T = o->X->tri;
        v2 v[3] = {a, b, c};
        for (int q = 0; q < 3; ++q) {
            int64_t k = 3 * o->n + q;
            v3 S = displaced_position(T, o->X->field, v[q].x, v[q].y);
            v3 nr = eigen_normalized(pointwise_normal(T, o->X->field, v[q].x, v[q].y));
            if (o->mirrored)
                nr = V3(-nr.x, -nr.y, -nr.z);
            put_vertex(S, v[q], nr, o->pos + 3 * k, o->uv + 2 * k, o->nrm + 3 * k);
            o->st6[6 * o->n + 2 * q] = v[q].x;
            o->st6[6 * o->n + 2 * q + 1] = v[q].y;
        }
        o->interior[o->n] = interior;
    }
    ++o->n;
}

int64_t o_tessellate_texel(const o_scene *s, int tri, int m, int64_t cap, float *pos, float *uv, float *nrm,
                           double *st6, int *interior)
{
    /* append_texel_tessellation (displaced_tessellation.cpp:101-136) */
    const o_isect *X = find_tri(s, tri, NULL);
    const o_uvtri *U = &X->domain;
    o_texel_out o = {X, chart_mirrored(X->tri), 0, cap, pos, uv, nrm, st6, interior};
    double w = 1.0 / X->pyr->n_leaf;
    int64_t i_lo = (int64_t)floor(U->lo.x / w), i_hi = (int64_t)ceil(U->hi.x / w) - 1;
    int64_t j_lo = (int64_t)floor(U->lo.y / w), j_hi = (int64_t)ceil(U->hi.y / w) - 1;
    for (int64_t j = j_lo; j <= j_hi; ++j)
        for (int64_t i = i_lo; i <= i_hi; ++i) {
            v2 c = V2((i + 0.5) * w, (j + 0.5) * w);
            int overlap = classify_square(U, c, 0.5 * w);
            if (overlap == OUTSIDE)
                continue;
            double ws = w / m;
            for (int b = 0; b < m; ++b)
                for (int a = 0; a < m; ++a) {
                    v2 p00 = V2(i * w + a * ws, j * w + b * ws);
                    v2 p10 = add2(p00, V2(ws, 0.0)), p01 = add2(p00, V2(0.0, ws)), p11 = add2(p00, V2(ws, ws));
                    v2 sc = add2(p00, V2(0.5 * ws, 0.5 * ws));
                    int sub = overlap == INSIDE ? INSIDE : classify_square(U, sc, 0.5 * ws);
                    if (sub == OUTSIDE)
                        continue;
                    if (sub == STRADDLE) {
                        o_clip poly = clip_square(U, sc, 0.5 * ws);
                        for (int k = 1; k + 1 < poly.n; ++k)
                            texel_face(&o, poly.p[0], poly.p[k], poly.p[k + 1], 0);
                        continue;
                    }
                    texel_face(&o, p00, p10, p01, 1);
                    texel_face(&o, p10, p11, p01, 1);
                }
        }
    return o.n;
}

/* ------------------------------------------------------------------------ */
/* Displaced-emitter sampling: emission_tile.cpp, descent_sampler.cpp.      */
/* ------------------------------------------------------------------------ */

/* EmissionTile over the texture's own tile (emission_tile.cpp:30-33,
 * 43-78, 80-130; the repeating layout): per level the mean of the texels
 * below each cell. */
typedef struct {
    int n_leaf, n_levels;
    int *m;
    double **mean;
} o_tile;

static void tile_build(o_tile *E, const double *texels, int n)
{
    E->n_leaf = n;
    E->n_levels = 1;
    while ((1 << E->n_levels) <= n)
        ++E->n_levels;
    E->m = (int *)malloc(sizeof(int) * (size_t)E->n_levels);
    E->mean = (double **)malloc(sizeof(double *) * (size_t)E->n_levels);
    E->m[0] = n;
    E->mean[0] = (double *)malloc(sizeof(double) * (size_t)n * n);
    memcpy(E->mean[0], texels, sizeof(double) * (size_t)n * n);
    for (int l = 1; l < E->n_levels; ++l) {
        int cm = E->m[l - 1], pm = cm / 2;
        E->m[l] = pm;
        E->mean[l] = (double *)malloc(sizeof(double) * (size_t)pm * pm);
        for (int J = 0; J < pm; ++J)
            for (int I = 0; I < pm; ++I) {
                double sum = 0.0;
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        sum += E->mean[l - 1][(size_t)(2 * J + a) * cm + (2 * I + b)];
                E->mean[l][(size_t)J * pm + I] = 0.25 * sum;
            }
    }
}

static void tile_free(o_tile *E)
{
    for (int l = 0; l < E->n_levels; ++l)
        free(E->mean[l]);
    free(E->mean);
    free(E->m);
}

static int64_t wrap_index(int64_t i, int m)
{
    int64_t r = i % m;
    return r < 0 ? r + m : r;
}

static double tile_mean(const o_tile *E, int level, int64_t i, int64_t j) /* emission_tile.cpp:99-118 */
{
    if (level >= E->n_levels)
        return E->mean[E->n_levels - 1][0];
    int m = E->m[level];
    return E->mean[level][(size_t)wrap_index(j, m) * m + wrap_index(i, m)];
}

static double tile_sum(const o_tile *E, int level, int64_t i, int64_t j) /* emission_tile.h:73-74 */
{
    double w = ldexp(1.0, level) / E->n_leaf;
    return tile_mean(E, level, i, j) * (w * w);
}

/* FootprintChild / FootprintNode (descent_sampler.h:71-84). */
typedef struct {
    int overlap;
    double area, mass;
    int32_t node;
} o_fpchild;

typedef struct {
    o_fpchild child[4];
} o_fpnode;

enum { O_DESCENT_AREA = 0, O_DESCENT_PRODUCT = 1, O_DESCENT_PRODUCT_GEOMETRY = 2 };

struct o_emitter {
    const o_isect *X;
    o_tile tile;
    int variant, emitter_cosine;
    double beta;
    int root_level;
    int64_t root_i0, root_j0;
    o_fpchild roots[4];
    o_fpnode *nodes;
    int n_nodes, cap_nodes;
    double total_area, total_mass;
};

static double clip_area(const o_clip *P) /* uv_clip.cpp:46-54 */
{
    double a = 0.0;
    for (int k = 0; k < P->n; ++k) {
        v2 p0 = P->p[k], p1 = P->p[(k + 1) % P->n];
        a += p0.x * p1.y - p1.x * p0.y;
    }
    return 0.5 * fabs(a);
}

static o_fpchild build_child(o_emitter *e, int level, int64_t i, int64_t j) /* descent_sampler.cpp:33-63 */
{
    int n_leaf = e->tile.n_leaf;
    double w = ldexp(1.0, level) / n_leaf;
    v2 c = V2((i + 0.5) * w, (j + 0.5) * w);
    o_fpchild out = {OUTSIDE, 0.0, 0.0, -1};
    out.overlap = classify_square(&e->X->domain, c, 0.5 * w);
    if (out.overlap == OUTSIDE)
        return out;
    if (out.overlap == INSIDE) {
        out.area = w * w;
        out.mass = tile_sum(&e->tile, level, i, j);
        return out;
    }
    if (level == 0) {
        o_clip poly = clip_square(&e->X->domain, c, 0.5 * w);
        out.area = clip_area(&poly);
        out.mass = tile_mean(&e->tile, 0, i, j) * out.area;
        return out;
    }
    int32_t index = e->n_nodes;
    if (e->n_nodes == e->cap_nodes) {
        e->cap_nodes = e->cap_nodes ? 2 * e->cap_nodes : 64;
        e->nodes = (o_fpnode *)realloc(e->nodes, sizeof(o_fpnode) * (size_t)e->cap_nodes);
    }
    ++e->n_nodes;
    o_fpnode node;
    for (int ch = 0; ch < 4; ++ch) {
        node.child[ch] = build_child(e, level - 1, 2 * i + (ch & 1), 2 * j + (ch >> 1));
        out.area += node.child[ch].area;
        out.mass += node.child[ch].mass;
    }
    e->nodes[index] = node;
    out.node = index;
    return out;
}

o_emitter *o_emitter_create(const o_scene *s, int tri, const double *texels, int n, int variant, double beta,
                            int emitter_cosine)
{
    /* DescentSampler's constructor and build_footprint (descent_sampler.cpp:85-113) */
    const o_isect *X = find_tri(s, tri, NULL);
    if (!X || n != X->pyr->n_leaf)
        return NULL;
    o_emitter *e = (o_emitter *)calloc(1, sizeof(o_emitter));
    e->X = X;
    tile_build(&e->tile, texels, n);
    e->variant = variant;
    e->beta = beta;
    e->emitter_cosine = emitter_cosine;
    footprint_roots(&X->domain, n, &e->root_level, &e->root_i0, &e->root_j0);
    for (int ch = 0; ch < 4; ++ch) {
        e->roots[ch] = build_child(e, e->root_level, e->root_i0 + (ch & 1), e->root_j0 + (ch >> 1));
        e->total_area += e->roots[ch].area;
        e->total_mass += e->roots[ch].mass;
    }
    return e;
}

void o_emitter_free(o_emitter *e)
{
    if (!e)
        return;
    tile_free(&e->tile);
    free(e->nodes);
    free(e);
}

void o_emitter_info(const o_emitter *e, double *out)
{
    out[0] = e->root_level;
    out[1] = (double)e->root_i0;
    out[2] = (double)e->root_j0;
    out[3] = e->total_area;
    out[4] = e->total_mass;
    out[5] = e->n_nodes;
}

/* pointwise_fields(tri, s, t, h, hu, hv) (displaced_surface.cpp:116-158):
 * the metric's sqrt(det G) and the unnormalized normal Su x Sv. */
static void pointwise_metric(const o_tri *T, double s, double t, double h, double hu, double hv, double *sqrt_det,
                             v3 *n)
{
    o_nframe f = normal_frame_at(T, s, t);
    v3 e1 = T->e1, e2 = T->e2;
    double bt00 = -dot3(f.Nu, e1), bt01 = -dot3(f.Nv, e1);
    double bt10 = -dot3(f.Nu, e2), bt11 = -dot3(f.Nv, e2);
    double B00 = bt00, B01 = 0.5 * (bt01 + bt10), B11 = bt11;
    double C00 = dot3(f.Nu, f.Nu), C01 = dot3(f.Nu, f.Nv), C11 = dot3(f.Nv, f.Nv);
    double a0 = dot3(f.N, e1), a1 = dot3(f.N, e2);
    double G0_00 = dot3(e1, e1), G0_01 = dot3(e1, e2), G0_11 = dot3(e2, e2); /* displaced_surface.cpp:87-90 */
    double G00 = (((G0_00 - 2.0 * h * B00) + h * h * C00) + hu * hu) + 2.0 * hu * a0;
    double G01 = ((((G0_01 - 2.0 * h * B01) + h * h * C01) + hu * hv) + hu * a1) + hv * a0;
    double G11 = (((G0_11 - 2.0 * h * B11) + h * h * C11) + hv * hv) + 2.0 * hv * a1;
    double det = G00 * G11 - G01 * G01;
    *sqrt_det = sqrt(dmax(det, 0.0));
    v3 Su = add3(add3(e1, mul3(hu, f.N)), mul3(h, f.Nu));
    v3 Sv = add3(add3(e2, mul3(hv, f.N)), mul3(h, f.Nv));
    *n = cross3(Su, Sv);
}

static int admissible(const o_emitter *e, const o_fpchild *info) /* descent_sampler.cpp:115-122 */
{
    if (info->overlap == OUTSIDE)
        return 0;
    return e->variant == O_DESCENT_AREA ? info->area > 0.0 : info->mass > 0.0;
}

static o_fpchild child_info(const o_emitter *e, int level, int64_t pi, int64_t pj, const o_fpchild *parent, int c)
{
    /* descent_sampler.cpp:124-138 */
    o_fpchild out = {OUTSIDE, 0.0, 0.0, -1};
    if (parent->node >= 0)
        return e->nodes[parent->node].child[c];
    if (parent->overlap != INSIDE)
        return out;
    int64_t i = 2 * pi + (c & 1), j = 2 * pj + (c >> 1);
    double w = cell_width(e->X->pyr, level);
    out.overlap = INSIDE;
    out.area = w * w;
    out.mass = tile_sum(&e->tile, level, i, j);
    return out;
}

typedef struct {
    v3 x, n;
} o_receiver;

static double node_weight(const o_emitter *e, int level, int64_t i, int64_t j, const o_fpchild *info,
                          const o_receiver *rcv) /* descent_sampler.cpp:140-170 */
{
    const o_tri *T = e->X->tri;
    o_node nd = pyramid_node(e->X->pyr, level, i, j);
    double w = ldexp(1.0, level) / e->X->pyr->n_leaf;
    double u0 = (i + 0.5) * w, v0 = (j + 0.5) * w;
    double sqrt_det;
    v3 fn;
    pointwise_metric(T, u0, v0, nd.h0, nd.gu, nd.gv, &sqrt_det, &fn);
    double base = e->variant == O_DESCENT_AREA ? info->area : info->mass;
    double weight = base * sqrt_det;
    if (e->variant == O_DESCENT_PRODUCT_GEOMETRY && rcv) {
        o_nframe nf = normal_frame_at(T, u0, v0);
        v3 y = add3(tri_P(T, u0, v0), mul3(nd.h0, nf.N));
        v3 d = sub3(y, rcv->x);
        double r2 = dmax(dot3(d, d), 1e-12);
        v3 omega = div3(d, sqrt(r2));
        double cos_r = dmax(dot3(rcv->n, omega), 0.0);
        double cos_e = e->emitter_cosine ? fabs(dot3(eigen_normalized(fn), omega)) : 1.0;
        weight *= cos_r * cos_e / r2;
    }
    return weight;
}

static void child_probs(const o_emitter *e, int level, int64_t pi, int64_t pj, const o_fpchild *parent,
                        const o_receiver *rcv, double p[4], o_fpchild info[4]) /* descent_sampler.cpp:172-206 */
{
    double w[4];
    int adm[4];
    int n_adm = 0;
    double sumw = 0.0;
    int virtual_root = level > e->root_level;
    for (int c = 0; c < 4; ++c) {
        int child_level = level - 1;
        int64_t i, j;
        if (virtual_root) {
            info[c] = e->roots[c];
            i = e->root_i0 + (c & 1);
            j = e->root_j0 + (c >> 1);
        } else {
            info[c] = child_info(e, child_level, pi, pj, parent, c);
            i = 2 * pi + (c & 1);
            j = 2 * pj + (c >> 1);
        }
        adm[c] = admissible(e, &info[c]);
        w[c] = adm[c] ? node_weight(e, child_level, i, j, &info[c], rcv) : 0.0;
        if (adm[c])
            ++n_adm;
        sumw += w[c];
    }
    for (int c = 0; c < 4; ++c) {
        if (!adm[c])
            p[c] = 0.0;
        else if (sumw > 0.0)
            p[c] = (1.0 - e->beta) * w[c] / sumw + e->beta / n_adm;
        else
            p[c] = 1.0 / n_adm;
    }
}

typedef struct {
    const float *u;
    int n, k;
} o_rng;

static double rng_next(o_rng *r) { return r->k < r->n ? (double)r->u[r->k++] : 0.5; }

static v2 sample_polygon(const o_clip *poly, double xi_tri, double xi1, double xi2) /* uv_clip.cpp:85-108 */
{
    double areas[8];
    double total = 0.0;
    for (int k = 1; k + 1 < poly->n; ++k) {
        v2 a = sub2(poly->p[k], poly->p[0]), b = sub2(poly->p[k + 1], poly->p[0]);
        areas[k] = 0.5 * fabs(a.x * b.y - a.y * b.x);
        total += areas[k];
    }
    double target = xi_tri * total, acc = 0.0;
    int chosen = poly->n - 2;
    for (int k = 1; k + 1 < poly->n; ++k) {
        acc += areas[k];
        if (target < acc) {
            chosen = k;
            break;
        }
    }
    double r = sqrt(xi1);
    double b1 = 1.0 - r, b2 = r * xi2;
    return add2(add2(poly->p[0], mul2(b1, sub2(poly->p[chosen], poly->p[0]))),
                mul2(b2, sub2(poly->p[chosen + 1], poly->p[0])));
}

int o_emitter_sample(const o_emitter *e, const float *u, int n_u, const double *recv, double *out)
{
    /* DescentSampler::sample (descent_sampler.cpp:208-290) */
    o_rng rng = {u, n_u, 0};
    o_receiver R, *rcv = NULL;
    if (recv) {
        R.x = V3(recv[0], recv[1], recv[2]);
        R.n = V3(recv[3], recv[4], recv[5]);
        rcv = &R;
    }
    int level = e->root_level + 1;
    int64_t i = 0, j = 0;
    o_fpchild cur = {OUTSIDE, 0.0, 0.0, -1};
    double P = 1.0;
    for (; level >= 1; --level) {
        double p[4];
        o_fpchild info[4];
        child_probs(e, level, i, j, &cur, rcv, p, info);
        double xi = rng_next(&rng);
        int c = -1;
        double cum = 0.0;
        for (int k = 0; k < 4; ++k) {
            cum += p[k];
            if (xi < cum) {
                c = k;
                break;
            }
        }
        if (c < 0 || p[c] == 0.0) {
            for (int k = 3; k >= 0; --k)
                if (p[k] > 0.0) {
                    c = k;
                    break;
                }
        }
        P *= p[c];
        if (level > e->root_level) {
            i = e->root_i0 + (c & 1);
            j = e->root_j0 + (c >> 1);
        } else {
            i = 2 * i + (c & 1);
            j = 2 * j + (c >> 1);
        }
        cur = info[c];
    }
    int n = e->X->pyr->n_leaf;
    double wl = 1.0 / n;
    double uu, vv;
    int inside_leaf = cur.overlap == INSIDE;
    for (int tries = 0;;) {
        uu = (i + rng_next(&rng)) * wl;
        vv = (j + rng_next(&rng)) * wl;
        if (inside_leaf || uvtri_inside(&e->X->domain, V2(uu, vv)))
            break;
        if (++tries == 32) {
            o_clip poly = clip_square(&e->X->domain, V2((i + 0.5) * wl, (j + 0.5) * wl), 0.5 * wl);
            /* sample_polygon(poly, rng.next(), rng.next(), rng.next()): g++
             * evaluates these arguments right to left */
            double x3 = rng_next(&rng), x2 = rng_next(&rng), x1 = rng_next(&rng);
            v2 s = sample_polygon(&poly, x1, x2, x3);
            uu = s.x;
            vv = s.y;
            break;
        }
    }
    const o_tri *T = e->X->tri;
    double h = grid_h(e->X->field, uu, vv);
    v2 gh = grid_grad(e->X->field, uu, vv);
    double sqrt_det;
    v3 fn;
    pointwise_metric(T, uu, vv, h, gh.x, gh.y, &sqrt_det, &fn);
    v3 p = add3(tri_P(T, uu, vv), mul3(h, normal_frame_at(T, uu, vv).N));
    v3 nn = eigen_normalized(fn);
    double pdf_uv = P / cur.area;
    double o[11] = {uu, vv, p.x, p.y, p.z, nn.x, nn.y, nn.z, sqrt_det, pdf_uv, pdf_uv / sqrt_det};
    memcpy(out, o, sizeof(o));
    return rng.k;
}

static o_receiver *receiver_of(const double *recv, o_receiver *R)
{
    if (!recv)
        return NULL;
    R->x = V3(recv[0], recv[1], recv[2]);
    R->n = V3(recv[3], recv[4], recv[5]);
    return R;
}

static double leaf_prob(const o_emitter *e, int64_t i, int64_t j, const o_receiver *rcv, o_fpchild *leaf)
{
    /* DescentSampler::leaf_prob (descent_sampler.cpp:290-325) */
    int L = e->root_level;
    int64_t ri = i >> L, rj = j >> L;
    int64_t di = ri - e->root_i0, dj = rj - e->root_j0;
    if (di < 0 || di > 1 || dj < 0 || dj > 1)
        return 0.0;
    o_fpchild cur = {OUTSIDE, 0.0, 0.0, -1};
    double P = 1.0;
    int64_t pi = 0, pj = 0;
    for (int level = L + 1; level >= 1; --level) {
        double p[4];
        o_fpchild info[4];
        child_probs(e, level, pi, pj, &cur, rcv, p, info);
        int c;
        if (level > L) {
            c = (int)(di | (dj << 1));
            pi = ri;
            pj = rj;
        } else {
            int64_t ci = i >> (level - 1), cj = j >> (level - 1);
            c = (int)((ci - 2 * pi) | ((cj - 2 * pj) << 1));
            pi = ci;
            pj = cj;
        }
        P *= p[c];
        cur = info[c];
        if (P == 0.0)
            return 0.0;
    }
    if (leaf)
        *leaf = cur;
    return P;
}

double o_emitter_leaf_prob(const o_emitter *e, int64_t i, int64_t j, const double *recv)
{
    o_receiver R;
    return leaf_prob(e, i, j, receiver_of(recv, &R), NULL);
}

double o_emitter_pdf_uv(const o_emitter *e, double u, double v, const double *recv)
{
    /* DescentSampler::pdf_uv (descent_sampler.cpp:346-356) */
    int n = e->X->pyr->n_leaf;
    int64_t i = (int64_t)floor(u / (1.0 / n)), j = (int64_t)floor(v / (1.0 / n));
    o_receiver R;
    o_fpchild leaf;
    double P = leaf_prob(e, i, j, receiver_of(recv, &R), &leaf);
    if (P == 0.0)
        return 0.0;
    return P / leaf.area;
}

double o_emitter_pdf_area(const o_emitter *e, double u, double v, const double *recv)
{
    /* DescentSampler::pdf_area (descent_sampler.cpp:358-364) */
    double p = o_emitter_pdf_uv(e, u, v, recv);
    if (p == 0.0)
        return 0.0;
    double h = grid_h(e->X->field, u, v);
    v2 gh = grid_grad(e->X->field, u, v);
    double sqrt_det;
    v3 fn;
    pointwise_metric(e->X->tri, u, v, h, gh.x, gh.y, &sqrt_det, &fn);
    return p / sqrt_det;
}

/* ---- DisplacedEmitterLight (displaced_emitter_light.cpp:20-116) ---------
 * The descent sampler as a light seen from a shading point (p, n): a sample
 * converted to a direction, distance and solid-angle pdf, and the pdf of a
 * direction from the (u, v) it reaches. The light's sampler is the
 * emitter's: AreaDescent / ProductDescent / ReceiverDescent for variants
 * 0 / 1 / 2, the receiver read only by the last (whose emitter cosine the
 * light turns off: create the emitter with emitter_cosine 0). */
#define O_MIN_COS_Y 1e-7 /* displaced_emitter_light.cpp:16 */

int o_emitter_light_sample(const o_emitter *e, const float *u, int n_u, const double *shade6, double *out16)
{
    /* DisplacedEmitterLight::sample (:58-90) */
    double s[11];
    o_emitter_sample(e, u, n_u, e->variant == 2 ? shade6 : NULL, s);
    v3 p = V3(shade6[0], shade6[1], shade6[2]);
    v3 y = V3(s[2], s[3], s[4]), ny = V3(s[5], s[6], s[7]);
    v3 d = sub3(y, p);
    double dist = sqrt(dot3(d, d));
    v3 wi = div3(d, dist);
    double cos_y = fabs(dot3(ny, wi));
    double o[16] = {s[0], s[1], y.x, y.y, y.z, ny.x, ny.y, ny.z, wi.x, wi.y, wi.z, dist, 0.0, 0.0, 0.0, 0.0};
    if (!(cos_y < O_MIN_COS_Y)) {
        int n = e->tile.n_leaf;
        o[12] = s[10];
        o[13] = s[10] * dist * dist / cos_y;
        o[14] = tile_mean(&e->tile, 0, (int64_t)floor(s[0] * n), (int64_t)floor(s[1] * n)); /* Le_at, :47-51 */
        o[15] = 1.0;
    }
    memcpy(out16, o, sizeof(o));
    return o[15] != 0.0;
}

double o_emitter_light_pdf_uv(const o_emitter *e, const double *shade6, double u, double v)
{
    /* DisplacedEmitterLight::pdf_omega_from_uv (:103-117) */
    double pa = o_emitter_pdf_area(e, u, v, e->variant == 2 ? shade6 : NULL);
    if (pa <= 0.0)
        return 0.0;
    const o_tri *T = e->X->tri;
    double h = grid_h(e->X->field, u, v);
    v2 gh = grid_grad(e->X->field, u, v);
    double sqrt_det;
    v3 fn;
    pointwise_metric(T, u, v, h, gh.x, gh.y, &sqrt_det, &fn);
    v3 y = add3(tri_P(T, u, v), mul3(h, normal_frame_at(T, u, v).N));
    v3 d = sub3(y, V3(shade6[0], shade6[1], shade6[2]));
    double dist2 = dot3(d, d);
    double cos_y = fabs(dot3(eigen_normalized(fn), div3(d, sqrt(dist2))));
    if (cos_y < O_MIN_COS_Y)
        return 0.0;
    return pa * dist2 / cos_y;
}

double o_emitter_light_pdf_walk(const o_emitter *e, const double *shade6, const double *wi3, double *uv_out)
{
    /* the pdf of a direction by its walk (DisplacedAreaLight::pdf,
     * displaced_area_light.cpp:174-186, in object space): the triangle's
     * walk from p along wi, then the pdf at the crossing's (s, t) */
    o_hit h;
    uv_out[0] = uv_out[1] = NAN;
    if (!isect_intersect(e->X, V3(shade6[0], shade6[1], shade6[2]), V3(wi3[0], wi3[1], wi3[2]), 0.0, INFINITY, 2, 1,
                         0, &h, NULL, NULL))
        return 0.0;
    uv_out[0] = h.st.x;
    uv_out[1] = h.st.y;
    return o_emitter_light_pdf_uv(e, shade6, h.st.x, h.st.y);
}
