// C entry points over the reference's own hot-path classes, compiled from the
// reference sources in place (oracle/Makefile) into oracle/_ref. TEST
// INFRASTRUCTURE ONLY: the tests use it to pin the C oracle (same entry
// points as dmap_oracle.h, prefixed r_ instead of o_).
#include "displaced_intersector.h"
#include "node_bounds.h"
#include "taylor_pyramid.h"
#include "displaced_tessellation.h"
#include "descent_sampler.h"
#include "displaced_emitter_light.h"

#include "../dmap_oracle.h"

#include <cmath>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <memory>
#include <thread>
#include <vector>

using dmap::BaseTriangle;
using ks::vec2d;
using ks::vec3d;

namespace
{

struct RefObject
{
    std::vector<double> values;
    dmap::HeightGrid field;
    std::unique_ptr<dmap::TaylorPyramid> pyramid;
    std::vector<BaseTriangle> tris;
    std::unique_ptr<dmap::ObjectIntersector> obj;
    int first_tri = 0;
};

} // namespace

struct r_scene
{
    std::vector<std::unique_ptr<RefObject>> objects;
    int n_tri = 0;
    // the opacity filter (r_scene_set_opacity); empty mask: none
    std::vector<uint8_t> op_mask, op_tri;
    int op_w = 0, op_h = 0, op_flip = 0;
    double op_scale[2] = {1.0, 1.0}, op_offset[2] = {0.0, 0.0};
};

struct r_pyramid
{
    std::unique_ptr<dmap::TaylorPyramid> p;
};

extern "C" {

r_pyramid *r_pyramid_build(const double *values, int nodes, double scale, double offset, int build)
{
    auto *r = new r_pyramid;
    r->p = std::make_unique<dmap::TaylorPyramid>(values, nodes, scale,
                                                 build == O_BUILD_FOLD ? dmap::PyramidBuild::Fold
                                                                       : dmap::PyramidBuild::Direct,
                                                 offset);
    return r;
}
void r_pyramid_free(r_pyramid *p) { delete p; }
int r_pyramid_levels(const r_pyramid *p) { return p->p->n_levels; }
void r_pyramid_level(const r_pyramid *p, int level, double *out)
{
    const dmap::TaylorLevel &l = p->p->levels[level];
    size_t cells = (size_t)l.m * l.m;
    const std::vector<double> *ch[8] = {&l.h0, &l.gu, &l.gv, &l.r, &l.ru, &l.rv, &l.h_min, &l.h_max};
    for (int c = 0; c < 8; ++c)
        std::memcpy(out + c * cells, ch[c]->data(), cells * sizeof(double));
}
void r_pyramid_node(const r_pyramid *p, int level, int64_t i, int64_t j, double *out8)
{
    dmap::TaylorNode n = p->p->node(level, i, j);
    std::memcpy(out8, &n, sizeof(n));
}

r_scene *r_scene_create(void) { return new r_scene; }
void r_scene_free(r_scene *s) { delete s; }

int r_scene_add_object(r_scene *s, const double *values, int W, double scale, double offset, int repeat, int build,
                       const double *tris, int n_tri)
{
    auto o = std::make_unique<RefObject>();
    o->values.assign(values, values + (size_t)W * W);
    o->field = dmap::HeightGrid{W, W, scale, o->values.data(), offset, repeat != 0};
    o->pyramid = std::make_unique<dmap::TaylorPyramid>(
        o->field, build == O_BUILD_FOLD ? dmap::PyramidBuild::Fold : dmap::PyramidBuild::Direct);
    for (int k = 0; k < n_tri; ++k) {
        const double *r = tris + 24 * (size_t)k;
        o->tris.emplace_back(vec3d(r[0], r[1], r[2]), vec3d(r[3], r[4], r[5]), vec3d(r[6], r[7], r[8]),
                             vec3d(r[9], r[10], r[11]), vec3d(r[12], r[13], r[14]), vec3d(r[15], r[16], r[17]),
                             vec2d(r[18], r[19]), vec2d(r[20], r[21]), vec2d(r[22], r[23]));
    }
    o->obj = std::make_unique<dmap::ObjectIntersector>(o->tris, *o->pyramid, o->field);
    o->first_tri = s->n_tri;
    s->n_tri += n_tri;
    s->objects.push_back(std::move(o));
    return (int)s->objects.size() - 1;
}

int r_scene_triangle_count(const r_scene *s) { return s->n_tri; }

static const dmap::DisplacedIntersector *find_tri(const r_scene *s, int tri, int *ob, int *local)
{
    for (size_t k = 0; k < s->objects.size(); ++k) {
        const RefObject &o = *s->objects[k];
        if (tri < o.first_tri + (int)o.tris.size()) {
            *ob = (int)k;
            *local = tri - o.first_tri;
            return &o.obj->triangles[*local];
        }
    }
    return nullptr;
}

void r_scene_triangle_info(const r_scene *s, int tri, double *out)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    const dmap::Aabb3 &b = s->objects[ob]->obj->boxes[local];
    double h_min, h_max;
    dmap::triangle_height_range(*X->tri, *X->pyramid, h_min, h_max);
    double v[11] = {(double)X->root_level, (double)X->n_roots, X->residual_tolerance, b.lo[0], b.lo[1], b.lo[2],
                    b.hi[0], b.hi[1], b.hi[2], h_min, h_max};
    std::memcpy(out, v, sizeof(v));
}

void r_scene_triangle_frame(const r_scene *s, int tri, double *out)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            out[3 * i + j] = X->frame.to_tangent(i, j);
    out[9] = X->frame.ng[0];
    out[10] = X->frame.ng[1];
    out[11] = X->frame.ng[2];
}

static dmap::TraversalOptions options_of(int bound, int slab_max_level, int leaf)
{
    dmap::TraversalOptions o;
    o.bound = bound == O_BOUND_BOX ? dmap::BoundMode::Box
                                   : bound == O_BOUND_SLAB ? dmap::BoundMode::Slab : dmap::BoundMode::Both;
    o.slab_max_level = slab_max_level;
    o.leaf = leaf == O_LEAF_NEWTON ? dmap::LeafMode::Newton : dmap::LeafMode::TwoTriangle;
    return o;
}

static void write_hit(double *out, const dmap::DisplacedHit &h, int tri, int ob)
{
    double v[O_HIT_DOUBLES] = {h.t,       h.st[0],   h.st[1],   h.bary[0],      h.bary[1],      h.ng[0],
                               h.ng[1],   h.ng[2],   (double)h.i, (double)h.j, (double)tri, (double)ob};
    std::memcpy(out, v, sizeof(v));
}

static void write_miss(double *out)
{
    for (int k = 0; k < O_HIT_DOUBLES; ++k)
        out[k] = 0.0;
    out[0] = INFINITY;
    out[10] = -1.0;
    out[11] = -1.0;
}

static void fill_stats(int64_t *out, const dmap::TraversalStats &st)
{
    std::memset(out, 0, O_ST_COUNT * sizeof(int64_t));
    out[O_ST_TRIANGLE_TESTS] = st.triangle_tests;
    out[O_ST_NODE_TESTS] = st.node_tests;
    out[O_ST_LEAF_TESTS] = st.leaf_tests;
    out[O_ST_SUB_SQUARES] = st.sub_squares;
    out[O_ST_NEWTON_ITERS] = -1; // the reference keeps no such counter
    out[O_ST_NODE_AFTER_HIT] = st.node_tests_after_hit;
    out[O_ST_LEAF_AFTER_HIT] = st.leaf_tests_after_hit;
}

// The object loop carries t_max the way intersect_flat does. The reference's
// intersect is const and re-entrant, so rays are split over `threads`
// std::threads in chunks of at most 4096, small enough that every thread gets
// work (threads <= 0: every core).
static int64_t intersect_range(const r_scene *s, const double *rays, int64_t b, int64_t e,
                               const dmap::TraversalOptions &opt, double *hits, int64_t *stats);

int64_t r_scene_intersect(const r_scene *s, const double *rays, int64_t n, int bound, int slab_max_level, int leaf,
                          double *hits, int64_t *stats, int threads)
{
    dmap::TraversalOptions opt = options_of(bound, slab_max_level, leaf);
    if (threads <= 0)
        threads = (int)std::thread::hardware_concurrency();
    if (threads <= 1)
        return intersect_range(s, rays, 0, n, opt, hits, stats);
    std::atomic<int64_t> next{0}, n_hit{0};
    std::vector<std::thread> pool;
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(4096, n / (8 * (int64_t)threads)));
    for (int k = 0; k < threads; ++k)
        pool.emplace_back([&] {
            for (;;) {
                int64_t b = next.fetch_add(chunk);
                if (b >= n)
                    break;
                n_hit += intersect_range(s, rays, b, std::min<int64_t>(n, b + chunk), opt, hits, stats);
            }
        });
    for (auto &t : pool)
        t.join();
    return n_hit.load();
}

// The opacity filter standing in for rtcFilterIntersection: the crossing's
// texture coordinate as DisplacedGeometry::compute_hit_texcoord forms it
// (displaced_geometry.cpp:189-193, from potential_hit's float barycentrics,
// :21-34) with the reference's BaseTriangle::param, the object uv
// (scene_spec.cpp:382-388) rounded to float, and the mask texel under it.
static bool crossing_opaque(const r_scene *s, const BaseTriangle &tri, int g, const dmap::DisplacedHit &h)
{
    if (s->op_mask.empty() || (!s->op_tri.empty() && !s->op_tri[g]))
        return true;
    float fu = (float)h.bary[0], fv = (float)h.bary[1];
    vec2d st = tri.param(fu, fv);
    double x = (st[0] - s->op_offset[0]) / s->op_scale[0], y = (st[1] - s->op_offset[1]) / s->op_scale[1];
    if (s->op_flip)
        y = 1.0 - y;
    double fx = (double)(float)x * s->op_w, fy = (double)(float)y * s->op_h;
    if (!(std::fabs(fx) < 1e15 && std::fabs(fy) < 1e15))
        return true;
    long long i = (long long)std::floor(fx) % s->op_w, j = (long long)std::floor(fy) % s->op_h;
    if (i < 0)
        i += s->op_w;
    if (j < 0)
        j += s->op_h;
    return s->op_mask[(size_t)(j * s->op_w + i)] != 0;
}

// A filtered scene: intersect_flat's loop (displaced_intersector.cpp:578-599)
// with each triangle behind intersect_callback's passes
// (displaced_geometry.cpp:53-78, max_filter_passes = 64 at displaced_geometry.h:64).
static bool intersect_filtered(const r_scene *s, const RefObject &ob, const vec3d &o, const vec3d &d, double t_min,
                               double &t_max, const dmap::TraversalOptions &opt, dmap::DisplacedHit &hit, int &tri,
                               dmap::TraversalStats *st)
{
    bool found = false;
    for (size_t k = 0; k < ob.obj->triangles.size(); ++k) {
        double t0 = t_min, t1 = t_max;
        if (!ob.obj->boxes[k].clip(o, d, t0, t1))
            continue;
        if (st)
            ++st->triangle_tests;
        double t_lo = t_min;
        for (int pass = 0; pass < 64; ++pass) {
            dmap::DisplacedHit h;
            if (!ob.obj->triangles[k].intersect(o, d, t_lo, t_max, opt, h, st))
                break;
            if (crossing_opaque(s, ob.tris[k], ob.first_tri + (int)k, h)) {
                hit = h;
                tri = (int)k;
                t_max = h.t;
                found = true;
                break;
            }
            t_lo = h.t;
        }
    }
    return found;
}

static int64_t intersect_range(const r_scene *s, const double *rays, int64_t b, int64_t e,
                               const dmap::TraversalOptions &opt, double *hits, int64_t *stats)
{
    int64_t n_hit = 0;
    for (int64_t r = b; r < e; ++r) {
        const double *q = rays + 8 * r;
        vec3d o(q[0], q[1], q[2]), d(q[3], q[4], q[5]);
        double t_min = q[6], t_max = q[7];
        double *out = hits + O_HIT_DOUBLES * r;
        write_miss(out);
        dmap::TraversalStats st;
        bool found = false;
        for (size_t k = 0; k < s->objects.size(); ++k) {
            const RefObject &ob = *s->objects[k];
            dmap::DisplacedHit h;
            int tri = -1;
            if (!s->op_mask.empty()) {
                if (intersect_filtered(s, ob, o, d, t_min, t_max, opt, h, tri, stats ? &st : nullptr)) {
                    write_hit(out, h, ob.first_tri + tri, (int)k);
                    found = true;
                }
                continue;
            }
            if (ob.obj->intersect(o, d, t_min, t_max, opt, h, tri, stats ? &st : nullptr)) {
                write_hit(out, h, ob.first_tri + tri, (int)k);
                t_max = h.t;
                found = true;
            }
        }
        n_hit += found;
        if (stats)
            fill_stats(stats + O_ST_COUNT * r, st);
    }
    return n_hit;
}

void r_scene_set_opacity(r_scene *s, const uint8_t *mask, int w, int h, const double *map5, const uint8_t *tri_flags)
{
    s->op_mask.clear();
    s->op_tri.clear();
    if (!mask || w <= 0 || h <= 0)
        return;
    s->op_mask.assign(mask, mask + (size_t)w * h);
    if (tri_flags)
        s->op_tri.assign(tri_flags, tri_flags + s->n_tri);
    s->op_w = w;
    s->op_h = h;
    s->op_scale[0] = map5 ? map5[0] : 1.0;
    s->op_scale[1] = map5 ? map5[1] : 1.0;
    s->op_offset[0] = map5 ? map5[2] : 0.0;
    s->op_offset[1] = map5 ? map5[3] : 0.0;
    s->op_flip = map5 ? map5[4] != 0.0 : 0;
}

int r_triangle_intersect(const r_scene *s, int tri, const double *q, int bound, int slab_max_level, int leaf,
                         double *out, int64_t *stats)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    dmap::DisplacedHit h;
    dmap::TraversalStats st;
    write_miss(out);
    bool f = X->intersect(vec3d(q[0], q[1], q[2]), vec3d(q[3], q[4], q[5]), q[6], q[7],
                          options_of(bound, slab_max_level, leaf), h, stats ? &st : nullptr);
    if (f)
        write_hit(out, h, tri, ob);
    if (stats)
        fill_stats(stats, st);
    return f;
}

void r_node_bound(const r_scene *s, int tri, int level, int64_t i, int64_t j, const double *q, int bound,
                  int slab_max_level, double *out)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    dmap::NodeBound nb = dmap::node_bound(*X->tri, X->frame, *X->pyramid, level, i, j);
    dmap::TangentRay ray{X->frame.point(vec3d(q[0], q[1], q[2])), X->frame.direction(vec3d(q[3], q[4], q[5])), q[6],
                         q[7]};
    for (int a = 0; a < 3; ++a) {
        out[a] = nb.box.lo[a];
        out[3 + a] = nb.box.hi[a];
        dmap::Interval m = nb.m.interval(a);
        out[6 + 2 * a] = m.lo;
        out[7 + 2 * a] = m.hi;
    }
    double t0, t1;
    out[12] = dmap::box_interval(nb, ray, t0, t1);
    out[13] = dmap::slab_interval(nb, ray, t0, t1);
    bool pass = dmap::node_interval(nb, ray, options_of(bound, slab_max_level, 0), t0, t1);
    out[14] = pass ? t0 : NAN;
    out[15] = pass ? t1 : NAN;
}

void r_displaced_position(const r_scene *s, int tri, double sp, double tp, double *out)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    vec3d S = dmap::displaced_position(*X->tri, X->field, sp, tp);
    out[0] = S[0];
    out[1] = S[1];
    out[2] = S[2];
}

void r_tessellate_uniform(const r_scene *s, int tri, int n, float *pos, float *uv, float *nrm, uint32_t *idx)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    ks::MeshData m;
    dmap::append_displaced_triangle(m, *X->tri, X->field, n);
    std::copy(m.vertices.begin(), m.vertices.end(), pos);
    std::copy(m.texcoords.begin(), m.texcoords.end(), uv);
    std::copy(m.vertex_normals.begin(), m.vertex_normals.end(), nrm);
    std::copy(m.indices.begin(), m.indices.end(), idx);
}

int64_t r_tessellate_texel(const r_scene *s, int tri, int m, int64_t cap, float *pos, float *uv, float *nrm,
                           double *st6, int *interior)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    ks::MeshData md;
    std::vector<dmap::TexelFace> faces;
    dmap::append_texel_tessellation(md, *X->tri, X->field, X->pyramid->n_leaf, m, tri, faces);
    int64_t n = (int64_t)faces.size();
    for (int64_t f = 0; f < n && f < cap; ++f) {
        for (int q = 0; q < 3; ++q) {
            uint32_t v = md.indices[3 * f + q];
            for (int c = 0; c < 3; ++c) {
                pos[9 * f + 3 * q + c] = md.vertices[3 * v + c];
                nrm[9 * f + 3 * q + c] = md.vertex_normals[3 * v + c];
            }
            uv[6 * f + 2 * q] = md.texcoords[2 * v];
            uv[6 * f + 2 * q + 1] = md.texcoords[2 * v + 1];
            st6[6 * f + 2 * q] = faces[f].st[q][0];
            st6[6 * f + 2 * q + 1] = faces[f].st[q][1];
        }
        interior[f] = faces[f].interior ? 1 : 0;
    }
    return n;
}

struct r_emitter
{
    std::unique_ptr<dmap::EmissionTile> tile;
    std::unique_ptr<dmap::DescentSampler> s;
    // the same sampler as the reference's light wrapper builds it
    std::unique_ptr<dmap::DisplacedEmitterLight> light;
    const dmap::DisplacedIntersector *X = nullptr;
};

static dmap::Receiver receiver_of(const double *r)
{
    dmap::Receiver out;
    out.x = vec3d(r[0], r[1], r[2]);
    out.n = vec3d(r[3], r[4], r[5]);
    return out;
}

r_emitter *r_emitter_create(const r_scene *s, int tri, const double *texels, int n, int variant, double beta,
                            int emitter_cosine)
{
    int ob, local;
    const dmap::DisplacedIntersector *X = find_tri(s, tri, &ob, &local);
    auto *e = new r_emitter;
    dmap::TextureGrid tg;
    tg.W = tg.H = n;
    tg.values.assign(texels, texels + (size_t)n * n);
    e->tile = std::make_unique<dmap::EmissionTile>(tg);
    dmap::DescentWeight w = variant == 0   ? dmap::DescentWeight::AreaOnly
                            : variant == 1 ? dmap::DescentWeight::Product
                                           : dmap::DescentWeight::ProductGeometry;
    e->s = std::make_unique<dmap::DescentSampler>(*X->tri, X->field, *X->pyramid, *e->tile, w, beta);
    e->s->emitter_cosine = emitter_cosine != 0;
    dmap::EmitterSamplerKind kind = variant == 0   ? dmap::EmitterSamplerKind::AreaDescent
                                    : variant == 1 ? dmap::EmitterSamplerKind::ProductDescent
                                                   : dmap::EmitterSamplerKind::ReceiverDescent;
    e->light = std::make_unique<dmap::DisplacedEmitterLight>(*X->tri, X->field, *X->pyramid, *e->tile, kind, beta);
    e->X = X;
    return e;
}

void r_emitter_free(r_emitter *e) { delete e; }

void r_emitter_info(const r_emitter *e, double *out)
{
    const dmap::Footprint &fp = e->s->footprint;
    double v[6] = {(double)fp.root_level, (double)fp.root_i0, (double)fp.root_j0, fp.total_area, fp.total_mass,
                   (double)fp.nodes.size()};
    std::memcpy(out, v, sizeof(v));
}

int r_emitter_sample(const r_emitter *e, const float *u, int n_u, const double *recv, double *out)
{
    ks::RNG rng;
    rng.u = u;
    rng.n = n_u;
    dmap::Receiver r;
    if (recv)
        r = receiver_of(recv);
    dmap::DescentSample d = e->s->sample(rng, recv ? &r : nullptr);
    double v[11] = {d.u, d.v, d.p[0], d.p[1], d.p[2], d.n[0], d.n[1], d.n[2], d.sqrt_det, d.pdf_uv, d.pdf_area};
    std::memcpy(out, v, sizeof(v));
    return rng.k;
}

double r_emitter_pdf_uv(const r_emitter *e, double u, double v, const double *recv)
{
    dmap::Receiver r;
    if (recv)
        r = receiver_of(recv);
    return e->s->pdf_uv(u, v, recv ? &r : nullptr);
}

double r_emitter_pdf_area(const r_emitter *e, double u, double v, const double *recv)
{
    dmap::Receiver r;
    if (recv)
        r = receiver_of(recv);
    return e->s->pdf_area(u, v, recv ? &r : nullptr);
}

double r_emitter_leaf_prob(const r_emitter *e, int64_t i, int64_t j, const double *recv)
{
    dmap::Receiver r;
    if (recv)
        r = receiver_of(recv);
    return e->s->leaf_prob(i, j, recv ? &r : nullptr);
}

// DisplacedEmitterLight::sample (displaced_emitter_light.cpp:58-90) from
// shade6 = (p, n), its random numbers replayed from u.
int r_emitter_light_sample(const r_emitter *e, const float *u, int n_u, const double *shade6, double *out16)
{
    ks::RNG rng;
    rng.u = u;
    rng.n = n_u;
    dmap::EmitterLightSample s =
        e->light->sample(vec3d(shade6[0], shade6[1], shade6[2]), vec3d(shade6[3], shade6[4], shade6[5]), rng, nullptr);
    double v[16] = {s.u, s.v, s.y[0], s.y[1], s.y[2], s.n_y[0], s.n_y[1], s.n_y[2], s.wi[0], s.wi[1], s.wi[2],
                    s.dist, s.ok ? s.pdf_area : 0.0, s.ok ? s.pdf_omega : 0.0, s.ok ? s.Le : 0.0, s.ok ? 1.0 : 0.0};
    std::memcpy(out16, v, sizeof(v));
    return s.ok ? 1 : 0;
}

// DisplacedEmitterLight::pdf_omega_from_uv (displaced_emitter_light.cpp:103-116).
double r_emitter_light_pdf_uv(const r_emitter *e, const double *shade6, double u, double v)
{
    return e->light->pdf_omega_from_uv(vec3d(shade6[0], shade6[1], shade6[2]),
                                       vec3d(shade6[3], shade6[4], shade6[5]), u, v);
}

// DisplacedAreaLight::pdf's walk (displaced_area_light.cpp:174-186) in object
// space: the triangle's own DisplacedIntersector::intersect from p along wi,
// then pdf_omega_from_uv at the crossing.
double r_emitter_light_pdf_walk(const r_emitter *e, const double *shade6, const double *wi3, double *uv_out)
{
    dmap::DisplacedHit h;
    uv_out[0] = uv_out[1] = NAN;
    if (!e->X->intersect(vec3d(shade6[0], shade6[1], shade6[2]), vec3d(wi3[0], wi3[1], wi3[2]), 0.0, INFINITY,
                         dmap::TraversalOptions(), h))
        return 0.0;
    uv_out[0] = h.st[0];
    uv_out[1] = h.st[1];
    return e->light->pdf_omega_from_uv(vec3d(shade6[0], shade6[1], shade6[2]),
                                       vec3d(shade6[3], shade6[4], shade6[5]), h.st[0], h.st[1]);
}

} // extern "C"
