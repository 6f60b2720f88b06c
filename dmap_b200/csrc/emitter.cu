// Displaced-emitter sampling on the device (include/dmap_b200.h,
// dmap_emitter_*): the DescentSampler of every scene triangle
// (descent_sampler.cpp:85-362) over an EmissionTile per asset
// (emission_tile.cpp, the repeating tile layout), with the reference's
// operation order in double (compiled with -fmad=false), so samples and
// pdfs equal the reference's bit for bit when both draw the same uniforms.
//
// Set-up on the host (once per emitter): each asset's emission levels (the
// mean of the texels below each cell, folded level by level) and each
// triangle's footprint (its 2 x 2 root block and the tree of straddling
// cells with their exact clipped areas and masses), uploaded flat. Queries
// on the device, one thread per sample or pdf: the descent draws one uniform
// per level and weighs the four children of each cell by the node's Taylor
// plane through the exact metric (sqrt det G at the cell centre), times the
// clipped area or emission mass, times (ProductGeometry) the receiver's
// cosines over r^2; the point inside the chosen leaf is drawn by rejection,
// with the clipped polygon sampled after 32 misses.
#include "api_internal.h"
#include "f64_math.cuh"
#include "f64_walk.cuh"

#include <algorithm>
#include <cmath>
#include <memory>

using namespace dmapi;

namespace
{
using namespace d64;

// FootprintChild (descent_sampler.h:71-78)
struct FpChild
{
    int overlap; // OUTSIDE / INSIDE / STRADDLE
    int node;    // the straddling cell's own node, or -1
    double area, mass;
};

// One triangle's footprint: the roots' block and its first node.
struct TriEmit
{
    int root_level, node_base;
    int64_t root_i0, root_j0;
    FpChild roots[4];
    double total_area, total_mass;
};

// Emission levels of one asset: level l holds (n_leaf >> l)^2 means at off[l].
struct TileDev
{
    const double *mean;
    int n_leaf, n_levels;
    int64_t off[dmapdev::kMaxLevels];
};

} // namespace

struct dmap_emitter
{
    dmap_scene *scene = nullptr;  // queries only; destruction needs just the context
    dmap_context *ctx = nullptr;
    int variant = 1, emitter_cosine = 1;
    double beta = 0.05;
    double *means_dev = nullptr;
    FpChild *nodes_dev = nullptr;
    TriEmit *tris_dev = nullptr;
    TileDev *tiles_dev = nullptr;
    std::vector<TriEmit> tris_host;
    std::vector<int> nodes_per_tri;
};

namespace
{

// ---- host set-up: tiles and footprints ------------------------------------

struct HostTile
{
    int n_leaf = 0, n_levels = 0;
    std::vector<std::vector<double>> mean;

    double mean_at(int level, int64_t i, int64_t j) const // emission_tile.cpp:99-118 (repeat)
    {
        if (level >= n_levels)
            return mean.back()[0];
        const int m = n_leaf >> level;
        int64_t ri = i % m, rj = j % m;
        if (ri < 0)
            ri += m;
        if (rj < 0)
            rj += m;
        return mean[level][(size_t)rj * m + ri];
    }
    double sum(int level, int64_t i, int64_t j) const // emission_tile.h:73-74
    {
        double w = std::ldexp(1.0, level) / n_leaf;
        return mean_at(level, i, j) * (w * w);
    }
};

HostTile build_tile(const double *texels, int n) // emission_tile.cpp:43-78
{
    HostTile E;
    E.n_leaf = n;
    E.n_levels = 1;
    while ((1 << E.n_levels) <= n)
        ++E.n_levels;
    E.mean.emplace_back(texels ? std::vector<double>(texels, texels + (size_t)n * n)
                               : std::vector<double>((size_t)n * n, 1.0));
    for (int l = 1; l < E.n_levels; ++l) {
        const std::vector<double> &c = E.mean[l - 1];
        const int cm = n >> (l - 1), pm = cm / 2;
        std::vector<double> p((size_t)pm * pm);
        for (int J = 0; J < pm; ++J)
            for (int I = 0; I < pm; ++I) {
                double sum = 0.0;
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b)
                        sum += c[(size_t)(2 * J + a) * cm + (2 * I + b)];
                p[(size_t)J * pm + I] = 0.25 * sum;
            }
        E.mean.push_back(std::move(p));
    }
    return E;
}

// The domain tests of uv_clip.cpp on the host, from the triangle record.
int host_classify(const TriDev &T, double cx, double cy, double s) // uv_clip.cpp:27-44
{
    if (cx + s <= T.lo[0] || cx - s >= T.hi[0] || cy + s <= T.lo[1] || cy - s >= T.hi[1])
        return OUTSIDE;
    bool all_inside = true;
    for (int k = 0; k < 3; ++k) {
        double proj = T.un[k][0] * cx + T.un[k][1] * cy;
        double ext = (std::fabs(T.un[k][0]) + std::fabs(T.un[k][1])) * s;
        if (proj + ext <= T.ud[k])
            return OUTSIDE;
        if (proj - ext < T.ud[k])
            all_inside = false;
    }
    return all_inside ? INSIDE : STRADDLE;
}

double host_clipped_area(const TriDev &T, double cx, double cy, double s) // uv_clip.cpp:46-83
{
    double px[8], py[8], qx[8], qy[8];
    int n = 4;
    px[0] = cx + -s, py[0] = cy + -s;
    px[1] = cx + s, py[1] = cy + -s;
    px[2] = cx + s, py[2] = cy + s;
    px[3] = cx + -s, py[3] = cy + s;
    for (int k = 0; k < 3; ++k) {
        int m = 0;
        for (int a = 0; a < n; ++a) {
            const int b = a + 1 == n ? 0 : a + 1;
            double fa = (T.un[k][0] * px[a] + T.un[k][1] * py[a]) - T.ud[k];
            double fb = (T.un[k][0] * px[b] + T.un[k][1] * py[b]) - T.ud[k];
            if (fa >= 0.0) {
                qx[m] = px[a];
                qy[m++] = py[a];
            }
            if ((fa >= 0.0) != (fb >= 0.0)) {
                double t = fa / (fa - fb);
                qx[m] = px[a] + t * (px[b] - px[a]);
                qy[m++] = py[a] + t * (py[b] - py[a]);
            }
        }
        n = m;
        for (int a = 0; a < n; ++a) {
            px[a] = qx[a];
            py[a] = qy[a];
        }
        if (n == 0)
            break;
    }
    double area = 0.0;
    for (int k = 0; k < n; ++k) {
        const int b = (k + 1) % n;
        area += px[k] * py[b] - px[b] * py[k];
    }
    return 0.5 * std::fabs(area);
}

// build_child (descent_sampler.cpp:33-63): nodes are appended in the
// reference's order (a straddling cell's node before its children's).
FpChild build_child(const TriDev &T, const HostTile &E, std::vector<FpChild> &nodes, int level, int64_t i, int64_t j)
{
    double w = std::ldexp(1.0, level) / E.n_leaf;
    double cx = (i + 0.5) * w, cy = (j + 0.5) * w;
    FpChild out = {OUTSIDE, -1, 0.0, 0.0};
    out.overlap = host_classify(T, cx, cy, 0.5 * w);
    if (out.overlap == OUTSIDE)
        return out;
    if (out.overlap == INSIDE) {
        out.area = w * w;
        out.mass = E.sum(level, i, j);
        return out;
    }
    if (level == 0) {
        out.area = host_clipped_area(T, cx, cy, 0.5 * w);
        out.mass = E.mean_at(0, i, j) * out.area;
        return out;
    }
    const size_t index = nodes.size() / 4;
    nodes.resize(nodes.size() + 4);
    FpChild ch[4];
    for (int c = 0; c < 4; ++c) {
        ch[c] = build_child(T, E, nodes, level - 1, 2 * i + (c & 1), 2 * j + (c >> 1));
        out.area += ch[c].area;
        out.mass += ch[c].mass;
    }
    for (int c = 0; c < 4; ++c)
        nodes[4 * index + c] = ch[c];
    out.node = (int)index;
    return out;
}

void footprint_roots_host(const TriDev &T, int n_leaf, int &level, int64_t &i0, int64_t &j0) // descent_sampler.cpp:66-83
{
    level = 0;
    for (;;) {
        double w = std::ldexp(1.0, level) / n_leaf;
        int64_t ilo = (int64_t)std::floor(T.lo[0] / w), ihi = (int64_t)std::ceil(T.hi[0] / w) - 1;
        int64_t jlo = (int64_t)std::floor(T.lo[1] / w), jhi = (int64_t)std::ceil(T.hi[1] / w) - 1;
        if (ihi - ilo <= 1 && jhi - jlo <= 1) {
            i0 = ilo;
            j0 = jlo;
            return;
        }
        ++level;
    }
}

// ---- device: the descent ---------------------------------------------------

struct Emit
{
    const TriDev *tris;
    const AssetDev *assets;
    const TriEmit *temit;
    const FpChild *nodes;
    const TileDev *tiles;
    int variant, emitter_cosine;
    double beta;
};

struct Receiver
{
    v3 x, n;
    bool on;
};

__device__ __forceinline__ double tile_sum(const TileDev &E, int level, int64_t i, int64_t j)
{
    double mean;
    if (level >= E.n_levels) {
        mean = E.mean[E.off[E.n_levels - 1]];
    } else {
        const int64_t m = E.n_leaf >> level;
        int64_t ri = i % m, rj = j % m;
        if (ri < 0)
            ri += m;
        if (rj < 0)
            rj += m;
        mean = E.mean[E.off[level] + rj * m + ri];
    }
    double w = ldexp(1.0, level) / E.n_leaf;
    return mean * (w * w);
}

// pointwise_fields(tri, s, t, h, hu, hv) (displaced_surface.cpp:116-158):
// sqrt(det G) and the unnormalized normal Su x Sv.
__device__ inline void pointwise_metric(const TriDev &T, double s, double t, double h, double hu, double hv,
                                        double &sqrt_det, v3 &n)
{
    nframe f = normal_frame_at(T, s, t);
    const v3 e1 = L3(T.e1), e2 = L3(T.e2);
    double bt00 = -dot3(f.Nu, e1), bt01 = -dot3(f.Nv, e1);
    double bt10 = -dot3(f.Nu, e2), bt11 = -dot3(f.Nv, e2);
    double B00 = bt00, B01 = 0.5 * (bt01 + bt10), B11 = bt11;
    double C00 = dot3(f.Nu, f.Nu), C01 = dot3(f.Nu, f.Nv), C11 = dot3(f.Nv, f.Nv);
    double a0 = dot3(f.N, e1), a1 = dot3(f.N, e2);
    double G0_00 = dot3(e1, e1), G0_01 = dot3(e1, e2), G0_11 = dot3(e2, e2); // displaced_surface.cpp:87-90
    double G00 = (((G0_00 - 2.0 * h * B00) + h * h * C00) + hu * hu) + 2.0 * hu * a0;
    double G01 = ((((G0_01 - 2.0 * h * B01) + h * h * C01) + hu * hv) + hu * a1) + hv * a0;
    double G11 = (((G0_11 - 2.0 * h * B11) + h * h * C11) + hv * hv) + 2.0 * hv * a1;
    double det = G00 * G11 - G01 * G01;
    sqrt_det = sqrt(dmax(det, 0.0));
    v3 Su = add3(add3(e1, mul3(hu, f.N)), mul3(h, f.Nu));
    v3 Sv = add3(add3(e2, mul3(hv, f.N)), mul3(h, f.Nv));
    n = cross3(Su, Sv);
}

__device__ __forceinline__ v3 eigen_normalized(v3 a)
{
    double z = dot3(a, a);
    return z > 0.0 ? div3(a, sqrt(z)) : a;
}

__device__ inline double node_weight(const Emit &E, const TriDev &T, const AssetDev &g, int level, int64_t i,
                                     int64_t j, const FpChild &info, const Receiver &rcv) // descent_sampler.cpp:140-170
{
    node nd = pyramid_node(g, level, i, j);
    double w = ldexp(1.0, level) / g.n_leaf;
    double u0 = (i + 0.5) * w, v0 = (j + 0.5) * w;
    double sqrt_det;
    v3 fn;
    pointwise_metric(T, u0, v0, nd.h0, nd.gu, nd.gv, sqrt_det, fn);
    double base = E.variant == DMAP_DESCENT_AREA ? info.area : info.mass;
    double weight = base * sqrt_det;
    if (E.variant == DMAP_DESCENT_PRODUCT_GEOMETRY && rcv.on) {
        nframe nf = normal_frame_at(T, u0, v0);
        v3 y = add3(tri_P(T, u0, v0), mul3(nd.h0, nf.N));
        v3 d = sub3(y, rcv.x);
        double r2 = dmax(dot3(d, d), 1e-12);
        v3 omega = div3(d, sqrt(r2));
        double cos_r = dmax(dot3(rcv.n, omega), 0.0);
        double cos_e = E.emitter_cosine ? fabs(dot3(eigen_normalized(fn), omega)) : 1.0;
        weight *= cos_r * cos_e / r2;
    }
    return weight;
}

__device__ inline void child_probs(const Emit &E, const TriDev &T, const AssetDev &g, const TriEmit &F, int level,
                                   int64_t pi, int64_t pj, const FpChild &parent, const Receiver &rcv, double p[4],
                                   FpChild info[4]) // descent_sampler.cpp:124-138, 172-206
{
    double w[4];
    bool adm[4];
    int n_adm = 0;
    double sumw = 0.0;
    const bool virtual_root = level > F.root_level;
    const TileDev &tile = E.tiles[T.asset];
    for (int c = 0; c < 4; ++c) {
        const int child_level = level - 1;
        int64_t i, j;
        if (virtual_root) {
            info[c] = F.roots[c];
            i = F.root_i0 + (c & 1);
            j = F.root_j0 + (c >> 1);
        } else {
            i = 2 * pi + (c & 1);
            j = 2 * pj + (c >> 1);
            if (parent.node >= 0) {
                info[c] = E.nodes[4 * (int64_t)(F.node_base + parent.node) + c];
            } else if (parent.overlap != INSIDE) {
                info[c] = {OUTSIDE, -1, 0.0, 0.0};
            } else {
                double cw = cell_width(g, child_level);
                info[c] = {INSIDE, -1, cw * cw, tile_sum(tile, child_level, i, j)};
            }
        }
        adm[c] = info[c].overlap != OUTSIDE &&
                 (E.variant == DMAP_DESCENT_AREA ? info[c].area > 0.0 : info[c].mass > 0.0);
        w[c] = adm[c] ? node_weight(E, T, g, child_level, i, j, info[c], rcv) : 0.0;
        if (adm[c])
            ++n_adm;
        sumw += w[c];
    }
    for (int c = 0; c < 4; ++c) {
        if (!adm[c])
            p[c] = 0.0;
        else if (sumw > 0.0)
            p[c] = (1.0 - E.beta) * w[c] / sumw + E.beta / n_adm;
        else
            p[c] = 1.0 / n_adm;
    }
}

__device__ __forceinline__ Receiver load_receiver(const double *r, int64_t k)
{
    Receiver R;
    R.on = r != nullptr;
    if (R.on) {
        const double *q = r + 6 * k;
        R.x = V3(q[0], q[1], q[2]);
        R.n = V3(q[3], q[4], q[5]);
    } else {
        R.x = R.n = V3(0.0, 0.0, 0.0);
    }
    return R;
}

__device__ inline v2 sample_polygon(const ClipPoly &poly, double xi_tri, double xi1, double xi2) // uv_clip.cpp:85-108
{
    double areas[8];
    double total = 0.0;
    for (int k = 1; k + 1 < poly.n; ++k) {
        v2 a = sub2(poly.p[k], poly.p[0]), b = sub2(poly.p[k + 1], poly.p[0]);
        areas[k] = 0.5 * fabs(a.x * b.y - a.y * b.x);
        total += areas[k];
    }
    double target = xi_tri * total, acc = 0.0;
    int chosen = poly.n - 2;
    for (int k = 1; k + 1 < poly.n; ++k) {
        acc += areas[k];
        if (target < acc) {
            chosen = k;
            break;
        }
    }
    double r = sqrt(xi1);
    double b1 = 1.0 - r, b2 = r * xi2;
    return add2(add2(poly.p[0], mul2(b1, sub2(poly.p[chosen], poly.p[0]))), mul2(b2, sub2(poly.p[chosen + 1], poly.p[0])));
}

__global__ void sample_kernel(Emit E, const int32_t *__restrict__ tri_of, const float *__restrict__ uni, int n_uni,
                              const double *__restrict__ recv, int64_t n, int n_tri, dmap_emitter_point *out)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        dmap_emitter_point o = {};
        const int tri = tri_of[k];
        o.tri = tri;
        if (tri < 0 || tri >= n_tri) {
            o.draws = -1;
            out[k] = o;
            continue;
        }
        const TriDev &T = E.tris[tri];
        const AssetDev &g = E.assets[T.asset];
        const TriEmit &F = E.temit[tri];
        const Receiver rcv = load_receiver(recv, k);
        const float *u = uni + (int64_t)n_uni * k;
        int ku = 0;
        auto next = [&]() { return ku < n_uni ? (double)u[ku++] : 0.5; };
        // DescentSampler::sample (descent_sampler.cpp:208-290)
        int64_t i = 0, j = 0;
        FpChild cur = {OUTSIDE, -1, 0.0, 0.0};
        double P = 1.0;
        for (int level = F.root_level + 1; level >= 1; --level) {
            double p[4];
            FpChild info[4];
            child_probs(E, T, g, F, level, i, j, cur, rcv, p, info);
            double xi = next();
            int c = -1;
            double cum = 0.0;
            for (int q = 0; q < 4; ++q) {
                cum += p[q];
                if (xi < cum) {
                    c = q;
                    break;
                }
            }
            if (c < 0 || p[c] == 0.0) {
                for (int q = 3; q >= 0; --q)
                    if (p[q] > 0.0) {
                        c = q;
                        break;
                    }
            }
            if (c < 0) { // no admissible child: an emitter without mass here
                o.draws = -1;
                break;
            }
            P *= p[c];
            if (level > F.root_level) {
                i = F.root_i0 + (c & 1);
                j = F.root_j0 + (c >> 1);
            } else {
                i = 2 * i + (c & 1);
                j = 2 * j + (c >> 1);
            }
            cur = info[c];
        }
        if (o.draws < 0) {
            out[k] = o;
            continue;
        }
        const double wl = 1.0 / g.n_leaf;
        double uu, vv;
        const bool inside_leaf = cur.overlap == INSIDE;
        for (int tries = 0;;) {
            uu = (i + next()) * wl;
            vv = (j + next()) * wl;
            if (inside_leaf || uv_inside(T, V2(uu, vv)))
                break;
            if (++tries == 32) {
                ClipPoly poly = clip_square(T, V2((i + 0.5) * wl, (j + 0.5) * wl), 0.5 * wl);
                // the reference's sample_polygon(poly, rng.next(), rng.next(), rng.next())
                // as its compiler orders the draws: right to left
                double x3 = next(), x2 = next(), x1 = next();
                v2 s = sample_polygon(poly, x1, x2, x3);
                uu = s.x;
                vv = s.y;
                break;
            }
        }
        double h;
        v2 gh;
        grid_h_grad(g, uu, vv, h, gh);
        double sqrt_det;
        v3 fn;
        pointwise_metric(T, uu, vv, h, gh.x, gh.y, sqrt_det, fn);
        v3 p = add3(tri_P(T, uu, vv), mul3(h, normal_frame_at(T, uu, vv).N));
        v3 nn = eigen_normalized(fn);
        o.u = uu;
        o.v = vv;
        o.p[0] = p.x, o.p[1] = p.y, o.p[2] = p.z;
        o.n[0] = nn.x, o.n[1] = nn.y, o.n[2] = nn.z;
        o.sqrt_det = sqrt_det;
        o.pdf_uv = P / cur.area;
        o.pdf_area = o.pdf_uv / sqrt_det;
        o.draws = ku;
        out[k] = o;
    }
}

// DescentSampler::pdf_uv and pdf_area at (u, v) of triangle tri
// (descent_sampler.cpp:290-364); 0 outside the footprint.
__device__ inline void pdf_at(const Emit &E, int tri, double u, double v, const Receiver &rcv, double &pu, double &pa)
{
    pu = pa = 0.0;
    const TriDev &T = E.tris[tri];
    const AssetDev &g = E.assets[T.asset];
    const TriEmit &F = E.temit[tri];
    // pdf_uv / leaf_prob (descent_sampler.cpp:290-356)
    const int n_leaf = g.n_leaf;
    const int64_t i = (int64_t)floor(u / (1.0 / n_leaf)), j = (int64_t)floor(v / (1.0 / n_leaf));
    const int L = F.root_level;
    const int64_t ri = i >> L, rj = j >> L, di = ri - F.root_i0, dj = rj - F.root_j0;
    double P = 0.0;
    FpChild cur = {OUTSIDE, -1, 0.0, 0.0};
    if (di >= 0 && di <= 1 && dj >= 0 && dj <= 1) {
        P = 1.0;
        int64_t pi = 0, pj = 0;
        for (int level = L + 1; level >= 1; --level) {
            double p[4];
            FpChild info[4];
            child_probs(E, T, g, F, level, pi, pj, cur, rcv, p, info);
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
                break;
        }
    }
    if (P != 0.0) {
        pu = P / cur.area;
        double h;
        v2 gh;
        grid_h_grad(g, u, v, h, gh);
        double sqrt_det;
        v3 fn;
        pointwise_metric(T, u, v, h, gh.x, gh.y, sqrt_det, fn);
        pa = pu / sqrt_det;
    }
}

__global__ void pdf_kernel(Emit E, const int32_t *__restrict__ tri_of, const double *__restrict__ uv,
                           const double *__restrict__ recv, int64_t n, int n_tri, double *pdf_uv, double *pdf_area)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int tri = tri_of[k];
        double pu = 0.0, pa = 0.0;
        if (tri >= 0 && tri < n_tri)
            pdf_at(E, tri, uv[2 * k], uv[2 * k + 1], load_receiver(recv, k), pu, pa);
        pdf_uv[k] = pu;
        if (pdf_area)
            pdf_area[k] = pa;
    }
}

// ---- DisplacedEmitterLight (displaced_emitter_light.cpp:20-116) ----------
// The sampler seen from a shading point (p, n): a sample as a direction,
// distance and solid-angle pdf, and the pdf of a direction from the (u, v)
// it reaches, directly or by the walk of the emitter's triangle
// (DisplacedAreaLight::pdf, displaced_area_light.cpp:174-186). The receiver
// is read by the receiver variant only, as the light passes it.
constexpr double kMinCosY = 1e-7; // displaced_emitter_light.cpp:16

__device__ inline Receiver shade_receiver(const Emit &E, const double *shade, int64_t k)
{
    Receiver R = load_receiver(shade, k);
    R.on = R.on && E.variant == DMAP_DESCENT_PRODUCT_GEOMETRY;
    return R;
}

// EmissionTile::texel (emission_tile.h:71): the level-0 mean, wrapped
__device__ inline double tile_texel(const TileDev &E, int64_t i, int64_t j)
{
    const int64_t m = E.n_leaf;
    int64_t ri = i % m, rj = j % m;
    if (ri < 0)
        ri += m;
    if (rj < 0)
        rj += m;
    return E.mean[E.off[0] + rj * m + ri];
}

// DisplacedEmitterLight::pdf_omega_from_uv (:103-117)
__device__ inline double pdf_omega_from_uv(const Emit &E, int tri, v3 p, const Receiver &rcv, double u, double v)
{
    double pu, pa;
    pdf_at(E, tri, u, v, rcv, pu, pa);
    if (pa <= 0.0)
        return 0.0;
    const TriDev &T = E.tris[tri];
    const AssetDev &g = E.assets[T.asset];
    double h;
    v2 gh;
    grid_h_grad(g, u, v, h, gh);
    double sqrt_det;
    v3 fn;
    pointwise_metric(T, u, v, h, gh.x, gh.y, sqrt_det, fn);
    v3 y = add3(tri_P(T, u, v), mul3(h, normal_frame_at(T, u, v).N));
    v3 d = sub3(y, p);
    double dist2 = dot3(d, d);
    double cos_y = fabs(dot3(eigen_normalized(fn), div3(d, sqrt(dist2))));
    if (cos_y < kMinCosY)
        return 0.0;
    return pa * dist2 / cos_y;
}

// DisplacedEmitterLight::sample (:58-90) on points the sampler drew
__global__ void light_kernel(Emit E, const dmap_emitter_point *__restrict__ pts, const double *__restrict__ shade,
                             int64_t n, int n_tri, dmap_emitter_light_sample *out)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const dmap_emitter_point s = pts[k];
        dmap_emitter_light_sample o = {};
        o.tri = s.tri;
        if (s.tri >= 0 && s.tri < n_tri && s.draws >= 0) {
            const double *q = shade + 6 * k;
            v3 y = V3(s.p[0], s.p[1], s.p[2]), ny = V3(s.n[0], s.n[1], s.n[2]);
            v3 d = sub3(y, V3(q[0], q[1], q[2]));
            double dist = sqrt(dot3(d, d));
            v3 wi = div3(d, dist);
            double cos_y = fabs(dot3(ny, wi));
            o.u = s.u;
            o.v = s.v;
            o.y[0] = y.x, o.y[1] = y.y, o.y[2] = y.z;
            o.n_y[0] = ny.x, o.n_y[1] = ny.y, o.n_y[2] = ny.z;
            o.wi[0] = wi.x, o.wi[1] = wi.y, o.wi[2] = wi.z;
            o.dist = dist;
            if (!(cos_y < kMinCosY)) {
                const TileDev &tile = E.tiles[E.tris[s.tri].asset];
                o.pdf_area = s.pdf_area;
                o.pdf_omega = s.pdf_area * dist * dist / cos_y;
                o.Le = tile_texel(tile, (int64_t)floor(s.u * tile.n_leaf), (int64_t)floor(s.v * tile.n_leaf));
                o.ok = 1;
            }
        }
        out[k] = o;
    }
}

// pdf_omega_from_uv at given (u, v), or (uv NULL) at the crossing of the
// triangle's walk from p along wi
__global__ void light_pdf_kernel(Emit E, const int32_t *__restrict__ tri_of, const double *__restrict__ shade,
                                 const double *__restrict__ uv, const double *__restrict__ wi, int64_t n, int n_tri,
                                 double *pdf_omega, double *uv_hit)
{
    dmapk::QueryOpts opt{}; // TraversalOptions(): both bounds, slab at levels <= 1, the Newton leaf
    opt.bound = DMAP_BOUND_BOTH;
    opt.slab_max_level = 1;
    opt.leaf = DMAP_LEAF_NEWTON;
    opt.mode = DMAP_MODE_CLOSEST;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int tri = tri_of[k];
        double pw = 0.0, hu = NAN, hv = NAN;
        if (tri >= 0 && tri < n_tri) {
            const double *q = shade + 6 * k;
            const v3 p = V3(q[0], q[1], q[2]);
            const Receiver rcv = shade_receiver(E, shade, k);
            if (uv) {
                hu = uv[2 * k];
                hv = uv[2 * k + 1];
                pw = pdf_omega_from_uv(E, tri, p, rcv, hu, hv);
            } else {
                const TriDev &T = E.tris[tri];
                hit64 h;
                if (triangle_intersect(T, E.assets[T.asset], p, V3(wi[3 * k], wi[3 * k + 1], wi[3 * k + 2]), 0.0,
                                       INFINITY, opt, h, nullptr)) {
                    hu = h.st.x;
                    hv = h.st.y;
                    pw = pdf_omega_from_uv(E, tri, p, rcv, hu, hv);
                }
            }
        }
        pdf_omega[k] = pw;
        if (uv_hit) {
            uv_hit[2 * k] = hu;
            uv_hit[2 * k + 1] = hv;
        }
    }
}

unsigned grid_for(int64_t n)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, 148 * 32));
}

Emit emit_of(const dmap_emitter *e)
{
    Emit E;
    E.tris = e->scene->tris_dev;
    E.assets = e->scene->assets_dev;
    E.temit = e->tris_dev;
    E.nodes = e->nodes_dev;
    E.tiles = e->tiles_dev;
    E.variant = e->variant;
    E.emitter_cosine = e->emitter_cosine;
    E.beta = e->beta;
    return E;
}

} // namespace

extern "C" {

dmap_status dmap_emitter_create(dmap_scene *s, const double *const *texels_host, int variant, double beta,
                                int emitter_cosine, dmap_emitter **out)
{
    if (!s || !out || variant < DMAP_DESCENT_AREA || variant > DMAP_DESCENT_PRODUCT_GEOMETRY || !(beta >= 0.0) ||
        !(beta <= 1.0))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_create: bad argument");
    dmap_context *ctx = s->ctx;
    if (!s->all_f64)
        return fail(ctx, DMAP_ERR_UNSUPPORTED,
                    "dmap_emitter_create: the descent weights read the FP64 pyramid (assets with DMAP_ASSET_KEEP_F64)");
    auto e = std::make_unique<dmap_emitter>();
    e->scene = s;
    e->ctx = ctx;
    e->variant = variant;
    e->beta = beta;
    e->emitter_cosine = emitter_cosine ? 1 : 0;
    // tiles
    const int n_assets = (int)s->assets.size();
    std::vector<HostTile> tiles;
    std::vector<TileDev> tdev(n_assets);
    std::vector<double> means;
    for (int a = 0; a < n_assets; ++a) {
        const int n = s->assets[a]->dev.n_leaf;
        tiles.push_back(build_tile(texels_host ? texels_host[a] : nullptr, n));
        TileDev &t = tdev[a];
        t.n_leaf = n;
        t.n_levels = tiles.back().n_levels;
        for (int l = 0; l < t.n_levels; ++l) {
            t.off[l] = (int64_t)means.size();
            means.insert(means.end(), tiles.back().mean[l].begin(), tiles.back().mean[l].end());
        }
    }
    // footprints
    std::vector<FpChild> nodes;
    e->tris_host.resize(s->n_tri);
    e->nodes_per_tri.resize(s->n_tri);
    for (int t = 0; t < s->n_tri; ++t) {
        const TriDev &T = s->tris_host[t];
        const HostTile &E = tiles[T.asset];
        TriEmit &F = e->tris_host[t];
        std::vector<FpChild> own;
        footprint_roots_host(T, E.n_leaf, F.root_level, F.root_i0, F.root_j0);
        F.total_area = F.total_mass = 0.0;
        for (int c = 0; c < 4; ++c) {
            F.roots[c] = build_child(T, E, own, F.root_level, F.root_i0 + (c & 1), F.root_j0 + (c >> 1));
            F.total_area += F.roots[c].area;
            F.total_mass += F.roots[c].mass;
        }
        F.node_base = (int)(nodes.size() / 4);
        e->nodes_per_tri[t] = (int)(own.size() / 4);
        nodes.insert(nodes.end(), own.begin(), own.end());
    }
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    for (int a = 0; a < n_assets; ++a)
        tdev[a].mean = nullptr; // set below
    cudaError_t er;
    if ((er = cudaMalloc((void **)&e->means_dev, sizeof(double) * std::max<size_t>(1, means.size()))) ||
        (er = cudaMalloc((void **)&e->nodes_dev, sizeof(FpChild) * std::max<size_t>(1, nodes.size()))) ||
        (er = cudaMalloc((void **)&e->tris_dev, sizeof(TriEmit) * std::max(1, s->n_tri))) ||
        (er = cudaMalloc((void **)&e->tiles_dev, sizeof(TileDev) * std::max(1, n_assets)))) {
        dmap_emitter_destroy(e.release());
        return cuda_fail(ctx, er, "dmap_emitter_create: allocation");
    }
    for (int a = 0; a < n_assets; ++a)
        tdev[a].mean = e->means_dev;
    if ((er = cudaMemcpy(e->means_dev, means.data(), sizeof(double) * means.size(), cudaMemcpyHostToDevice)) ||
        (er = cudaMemcpy(e->nodes_dev, nodes.data(), sizeof(FpChild) * nodes.size(), cudaMemcpyHostToDevice)) ||
        (er = cudaMemcpy(e->tris_dev, e->tris_host.data(), sizeof(TriEmit) * s->n_tri, cudaMemcpyHostToDevice)) ||
        (er = cudaMemcpy(e->tiles_dev, tdev.data(), sizeof(TileDev) * n_assets, cudaMemcpyHostToDevice))) {
        dmap_emitter_destroy(e.release());
        return cuda_fail(ctx, er, "dmap_emitter_create: upload");
    }
    *out = e.release();
    return DMAP_OK;
}

void dmap_emitter_destroy(dmap_emitter *e)
{
    if (!e)
        return;
    cudaSetDevice(e->ctx->device);
    cudaStreamSynchronize(e->ctx->stream);
    cudaFree(e->means_dev);
    cudaFree(e->nodes_dev);
    cudaFree(e->tris_dev);
    cudaFree(e->tiles_dev);
    delete e;
}

dmap_status dmap_emitter_triangle_info(const dmap_emitter *e, int tri, double *out6)
{
    if (!e || !out6 || tri < 0 || tri >= e->scene->n_tri)
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_triangle_info: bad argument");
    const TriEmit &F = e->tris_host[tri];
    double v[6] = {(double)F.root_level, (double)F.root_i0, (double)F.root_j0, F.total_area, F.total_mass,
                   (double)e->nodes_per_tri[tri]};
    std::memcpy(out6, v, sizeof(v));
    return DMAP_OK;
}

dmap_status dmap_emitter_sample(dmap_emitter *e, const int32_t *tri_dev, const float *uniforms_dev,
                                int uniforms_per_sample, const double *receivers_dev, int64_t n,
                                dmap_emitter_point *out_dev, void *stream)
{
    if (!e || n < 0 || uniforms_per_sample < 0 || (n > 0 && (!tri_dev || !out_dev || (uniforms_per_sample > 0 &&
                                                                                      !uniforms_dev))))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_sample: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    sample_kernel<<<grid_for(n), 128, 0, st>>>(emit_of(e), tri_dev, uniforms_dev, uniforms_per_sample, receivers_dev,
                                                n, e->scene->n_tri, out_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return DMAP_OK;
}

dmap_status dmap_emitter_pdf(dmap_emitter *e, const int32_t *tri_dev, const double *uv_dev,
                             const double *receivers_dev, int64_t n, double *pdf_uv_dev, double *pdf_area_dev,
                             void *stream)
{
    if (!e || n < 0 || (n > 0 && (!tri_dev || !uv_dev || !pdf_uv_dev)))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_pdf: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    pdf_kernel<<<grid_for(n), 128, 0, st>>>(emit_of(e), tri_dev, uv_dev, receivers_dev, n, e->scene->n_tri,
                                             pdf_uv_dev, pdf_area_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return DMAP_OK;
}

dmap_status dmap_emitter_sample_host(dmap_emitter *e, const int32_t *tri, const float *uniforms,
                                     int uniforms_per_sample, const double *receivers, int64_t n,
                                     dmap_emitter_point *out)
{
    if (!e || n < 0 || uniforms_per_sample < 0 || (n > 0 && (!tri || !out || (uniforms_per_sample > 0 && !uniforms))))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_sample_host: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t bt = sizeof(int32_t) * n, bu = sizeof(float) * (size_t)uniforms_per_sample * n;
    const size_t br = receivers ? sizeof(double) * 6 * n : 0, bo = sizeof(dmap_emitter_point) * n;
    const size_t a = 256, ot = 0, ou = (bt + a - 1) / a * a, orr = ou + (bu + a - 1) / a * a,
                 oo = orr + (br + a - 1) / a * a;
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, oo + bo, st));
    dmap_status r = DMAP_OK;
    cudaError_t er = cudaMemcpyAsync(buf + ot, tri, bt, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess && bu)
        er = cudaMemcpyAsync(buf + ou, uniforms, bu, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess && br)
        er = cudaMemcpyAsync(buf + orr, receivers, br, cudaMemcpyHostToDevice, st);
    if (er != cudaSuccess)
        r = cuda_fail(ctx, er, "dmap_emitter_sample_host: copy");
    if (r == DMAP_OK)
        r = dmap_emitter_sample(e, (const int32_t *)(buf + ot), (const float *)(buf + ou), uniforms_per_sample,
                                br ? (const double *)(buf + orr) : nullptr, n, (dmap_emitter_point *)(buf + oo), st);
    if (r == DMAP_OK && (er = cudaMemcpyAsync(out, buf + oo, bo, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        r = cuda_fail(ctx, er, "dmap_emitter_sample_host: copy back");
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    return sync_and_check(ctx, "dmap_emitter_sample_host");
}

dmap_status dmap_emitter_pdf_host(dmap_emitter *e, const int32_t *tri, const double *uv, const double *receivers,
                                  int64_t n, double *pdf_uv, double *pdf_area)
{
    if (!e || n < 0 || (n > 0 && (!tri || !uv || !pdf_uv)))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_pdf_host: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t a = 256;
    const size_t bt = sizeof(int32_t) * n, buv = sizeof(double) * 2 * n, br = receivers ? sizeof(double) * 6 * n : 0,
                 bp = sizeof(double) * n;
    const size_t ouv = (bt + a - 1) / a * a, orr = ouv + (buv + a - 1) / a * a, op = orr + (br + a - 1) / a * a,
                 opa = op + (bp + a - 1) / a * a;
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, opa + bp, st));
    dmap_status r = DMAP_OK;
    cudaError_t er = cudaMemcpyAsync(buf, tri, bt, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess)
        er = cudaMemcpyAsync(buf + ouv, uv, buv, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess && br)
        er = cudaMemcpyAsync(buf + orr, receivers, br, cudaMemcpyHostToDevice, st);
    if (er != cudaSuccess)
        r = cuda_fail(ctx, er, "dmap_emitter_pdf_host: copy");
    if (r == DMAP_OK)
        r = dmap_emitter_pdf(e, (const int32_t *)buf, (const double *)(buf + ouv),
                             br ? (const double *)(buf + orr) : nullptr, n, (double *)(buf + op),
                             (double *)(buf + opa), st);
    if (r == DMAP_OK && ((er = cudaMemcpyAsync(pdf_uv, buf + op, bp, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                         (pdf_area && (er = cudaMemcpyAsync(pdf_area, buf + opa, bp, cudaMemcpyDeviceToHost, st)) !=
                                          cudaSuccess)))
        r = cuda_fail(ctx, er, "dmap_emitter_pdf_host: copy back");
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    return sync_and_check(ctx, "dmap_emitter_pdf_host");
}


dmap_status dmap_emitter_light(dmap_emitter *e, const dmap_emitter_point *points_dev, const double *shade_dev,
                               int64_t n, dmap_emitter_light_sample *out_dev, void *stream)
{
    if (!e || n < 0 || (n > 0 && (!points_dev || !shade_dev || !out_dev)))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_light: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    light_kernel<<<grid_for(n), 128, 0, st>>>(emit_of(e), points_dev, shade_dev, n, e->scene->n_tri, out_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return DMAP_OK;
}

dmap_status dmap_emitter_light_pdf(dmap_emitter *e, const int32_t *tri_dev, const double *shade_dev,
                                   const double *uv_dev, const double *wi_dev, int64_t n, double *pdf_omega_dev,
                                   double *uv_hit_dev, void *stream)
{
    if (!e || n < 0 || (n > 0 && (!tri_dev || !shade_dev || !pdf_omega_dev || (!uv_dev && !wi_dev))))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_light_pdf: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    light_pdf_kernel<<<grid_for(n), 128, 0, st>>>(emit_of(e), tri_dev, shade_dev, uv_dev, wi_dev, n,
                                                   e->scene->n_tri, pdf_omega_dev, uv_hit_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return DMAP_OK;
}

// Host forms: inputs and outputs staged through one stream-ordered block.
dmap_status dmap_emitter_light_host(dmap_emitter *e, const dmap_emitter_point *points, const double *shade,
                                    int64_t n, dmap_emitter_light_sample *out)
{
    if (!e || n < 0 || (n > 0 && (!points || !shade || !out)))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_light_host: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t a = 256, bp = sizeof(dmap_emitter_point) * n, bs = sizeof(double) * 6 * n,
                 bo = sizeof(dmap_emitter_light_sample) * n;
    const size_t os = (bp + a - 1) / a * a, oo = os + (bs + a - 1) / a * a;
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, oo + bo, st));
    dmap_status r = DMAP_OK;
    cudaError_t er = cudaMemcpyAsync(buf, points, bp, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess)
        er = cudaMemcpyAsync(buf + os, shade, bs, cudaMemcpyHostToDevice, st);
    if (er != cudaSuccess)
        r = cuda_fail(ctx, er, "dmap_emitter_light_host: copy");
    if (r == DMAP_OK)
        r = dmap_emitter_light(e, (const dmap_emitter_point *)buf, (const double *)(buf + os), n,
                               (dmap_emitter_light_sample *)(buf + oo), st);
    if (r == DMAP_OK && (er = cudaMemcpyAsync(out, buf + oo, bo, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        r = cuda_fail(ctx, er, "dmap_emitter_light_host: copy back");
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    return sync_and_check(ctx, "dmap_emitter_light_host");
}

dmap_status dmap_emitter_light_pdf_host(dmap_emitter *e, const int32_t *tri, const double *shade, const double *uv,
                                        const double *wi, int64_t n, double *pdf_omega, double *uv_hit)
{
    if (!e || n < 0 || (n > 0 && (!tri || !shade || !pdf_omega || (!uv && !wi))))
        return fail(e ? e->scene->ctx : nullptr, DMAP_ERR_INVALID, "dmap_emitter_light_pdf_host: bad argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = e->scene->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t a = 256, bt = sizeof(int32_t) * n, bs = sizeof(double) * 6 * n,
                 bu = uv ? sizeof(double) * 2 * n : 0, bw = wi ? sizeof(double) * 3 * n : 0, bp = sizeof(double) * n,
                 bh = sizeof(double) * 2 * n;
    auto up = [&](size_t x) { return (x + a - 1) / a * a; };
    const size_t os = up(bt), ou = os + up(bs), ow = ou + up(bu), op = ow + up(bw), oh = op + up(bp);
    char *buf = nullptr;
    DMAP_CUDA(ctx, cudaMallocAsync((void **)&buf, oh + bh, st));
    dmap_status r = DMAP_OK;
    cudaError_t er = cudaMemcpyAsync(buf, tri, bt, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess)
        er = cudaMemcpyAsync(buf + os, shade, bs, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess && bu)
        er = cudaMemcpyAsync(buf + ou, uv, bu, cudaMemcpyHostToDevice, st);
    if (er == cudaSuccess && bw)
        er = cudaMemcpyAsync(buf + ow, wi, bw, cudaMemcpyHostToDevice, st);
    if (er != cudaSuccess)
        r = cuda_fail(ctx, er, "dmap_emitter_light_pdf_host: copy");
    if (r == DMAP_OK)
        r = dmap_emitter_light_pdf(e, (const int32_t *)buf, (const double *)(buf + os),
                                   bu ? (const double *)(buf + ou) : nullptr, bw ? (const double *)(buf + ow) : nullptr,
                                   n, (double *)(buf + op), (double *)(buf + oh), st);
    if (r == DMAP_OK && ((er = cudaMemcpyAsync(pdf_omega, buf + op, bp, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                         (uv_hit && (er = cudaMemcpyAsync(uv_hit, buf + oh, bh, cudaMemcpyDeviceToHost, st)) !=
                                        cudaSuccess)))
        r = cuda_fail(ctx, er, "dmap_emitter_light_pdf_host: copy back");
    cudaFreeAsync(buf, st);
    if (r != DMAP_OK)
        return r;
    return sync_and_check(ctx, "dmap_emitter_light_pdf_host");
}

} // extern "C"
