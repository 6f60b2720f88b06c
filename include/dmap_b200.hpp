// C++ adapter over the C ABI of dmap_b200.h with the shape of the
// reference's intersector API (code/cpp/src in the reference):
//
//   dmapgpu::DisplacementAsset  ~ DisplacementAsset's grid + TaylorPyramid
//                                 (displacement_asset.h:38-41, taylor_pyramid.h:92)
//   dmapgpu::ObjectIntersector  ~ ObjectIntersector (displaced_intersector.h:176-198):
//                                 the same intersect(o, d, t_min, t_max, options,
//                                 hit, triangle, stats) call, plus intersect_batch
//   dmapgpu::TraversalOptions, DisplacedHit, TraversalStats
//                               ~ the reference's structs of the same names
//                                 (traversal_options.h:30-38,
//                                 displaced_intersector.h:89-114)
//
// Header-only; link libdmap_b200.so. Vectors are std::array<double, 3>, so
// a caller converts from its own vector type at the call site. Errors throw
// dmapgpu::Error (the reference ASSERTs).
#pragma once
#include "dmap_b200.h"

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace dmapgpu
{

using vec2d = std::array<double, 2>;
using vec3d = std::array<double, 3>;

struct Error : std::runtime_error
{
    dmap_status status;
    Error(dmap_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

inline void check(dmap_status s, const dmap_context *ctx, const char *what)
{
    if (s != DMAP_OK)
        throw Error(s, std::string(what) + ": " + dmap_status_string(s) + (ctx ? std::string(": ") + dmap_last_error(ctx)
                                                                                : std::string()));
}

enum class BoundMode { Box = DMAP_BOUND_BOX, Slab = DMAP_BOUND_SLAB, Both = DMAP_BOUND_BOTH };
enum class LeafMode { Newton = DMAP_LEAF_NEWTON, TwoTriangle = DMAP_LEAF_TWO_TRIANGLE };

struct TraversalOptions
{
    BoundMode bound = BoundMode::Both;
    int slab_max_level = 1;
    LeafMode leaf = LeafMode::Newton;
    bool fp64 = false; // the reference's double arithmetic throughout (needs assets kept in FP64)
    // false: ObjectIntersector's flat loop, triangles in index order (the
    // drop-in default); true: nearest box entry first (DMAP_ORDER_NEAREST)
    bool nearest = false;
    // false: the reference's FP64 certified leaf, every hit the reference's
    // (the drop-in default); true: the FP32 leaf (hits within its tolerance)
    bool fp32_leaf = false;

    dmap_options c() const
    {
        dmap_options o;
        dmap_options_default(&o);
        o.bound = (int)bound;
        o.slab_max_level = slab_max_level;
        o.leaf = (int)leaf;
        o.precision = fp64 || leaf == LeafMode::TwoTriangle ? DMAP_PRECISION_F64 : DMAP_PRECISION_F32;
        o.order = nearest ? DMAP_ORDER_NEAREST : DMAP_ORDER_INDEX;
        o.leaf_precision = fp32_leaf ? DMAP_PRECISION_F32 : DMAP_PRECISION_F64;
        return o;
    }
};

struct DisplacedHit
{
    double t = 0.0;
    vec2d st{}, bary{};
    vec3d ng{};
    int64_t i = 0, j = 0;
};

struct TraversalStats
{
    int64_t triangle_tests = 0, node_tests = 0, leaf_tests = 0, sub_squares = 0, newton_iterations = 0;
    int64_t node_tests_after_hit = 0, leaf_tests_after_hit = 0;
};

// The base triangle as ObjectIntersector takes it: positions, vertex
// normals and texture coordinates (BaseTriangle's general chart).
struct BaseTriangleDesc
{
    vec3d p0, p1, p2, m0, m1, m2;
    vec2d t0, t1, t2;
};

class Context
{
  public:
    explicit Context(int device = 0) { check(dmap_create(device, &h_), nullptr, "dmap_create"); }
    ~Context() { dmap_destroy(h_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    dmap_context *get() const { return h_; }

  private:
    dmap_context *h_ = nullptr;
};

class DisplacementAsset
{
  public:
    // nodes x nodes values (row major, nodes = 2^L + 1), h = scale v + offset
    DisplacementAsset(Context &ctx, const float *values, int nodes, double scale = 1.0, double offset = 0.0,
                      bool repeat = false, bool keep_fp64 = false)
        : ctx_(&ctx)
    {
        check(dmap_asset_create(ctx.get(), values, DMAP_F32, nodes, scale, offset, repeat ? 1 : 0,
                                keep_fp64 ? DMAP_ASSET_KEEP_F64 : 0u, &h_),
              ctx.get(), "dmap_asset_create");
    }
    ~DisplacementAsset() { dmap_asset_destroy(h_); }
    DisplacementAsset(const DisplacementAsset &) = delete;
    DisplacementAsset &operator=(const DisplacementAsset &) = delete;
    dmap_asset *get() const { return h_; }
    int levels() const { return dmap_asset_levels(h_); }

  private:
    Context *ctx_;
    dmap_asset *h_ = nullptr;
};

class ObjectIntersector
{
  public:
    ObjectIntersector(Context &ctx, const std::vector<BaseTriangleDesc> &tris, DisplacementAsset &asset)
        : ctx_(&ctx)
    {
        std::vector<double> rec(24 * tris.size());
        for (size_t k = 0; k < tris.size(); ++k) {
            const BaseTriangleDesc &t = tris[k];
            double *r = &rec[24 * k];
            const vec3d *v[6] = {&t.p0, &t.p1, &t.p2, &t.m0, &t.m1, &t.m2};
            for (int q = 0; q < 6; ++q)
                for (int a = 0; a < 3; ++a)
                    r[3 * q + a] = (*v[q])[a];
            const vec2d *u[3] = {&t.t0, &t.t1, &t.t2};
            for (int q = 0; q < 3; ++q)
                for (int a = 0; a < 2; ++a)
                    r[18 + 2 * q + a] = (*u[q])[a];
        }
        std::vector<int> which(tris.size(), 0);
        dmap_asset *a = asset.get();
        check(dmap_scene_create(ctx.get(), &a, 1, which.data(), rec.data(), (int)tris.size(), &h_), ctx.get(),
              "dmap_scene_create");
    }
    ~ObjectIntersector() { dmap_scene_destroy(h_); }
    ObjectIntersector(const ObjectIntersector &) = delete;
    ObjectIntersector &operator=(const ObjectIntersector &) = delete;

    // ObjectIntersector::intersect (displaced_intersector.h:193-194)
    bool intersect(const vec3d &o, const vec3d &d, double t_min, double t_max, const TraversalOptions &options,
                   DisplacedHit &hit, int &triangle, TraversalStats *stats = nullptr) const
    {
        double ray[8] = {o[0], o[1], o[2], d[0], d[1], d[2], t_min, t_max};
        dmap_hit64 h;
        int64_t st[DMAP_ST_COUNT] = {};
        dmap_options opt = options.c();
        check(dmap_intersect_host(h_, ray, DMAP_F64, 1, &opt, &h, DMAP_F64, stats ? st : nullptr), ctx_->get(),
              "dmap_intersect_host");
        if (stats) {
            stats->triangle_tests += st[DMAP_ST_TRIANGLE_TESTS];
            stats->node_tests += st[DMAP_ST_NODE_TESTS];
            stats->leaf_tests += st[DMAP_ST_LEAF_TESTS];
            stats->sub_squares += st[DMAP_ST_SUB_SQUARES];
            stats->newton_iterations += st[DMAP_ST_NEWTON_ITERS];
            stats->node_tests_after_hit += st[DMAP_ST_NODE_AFTER_HIT];
            stats->leaf_tests_after_hit += st[DMAP_ST_LEAF_AFTER_HIT];
        }
        triangle = h.tri;
        if (h.tri < 0)
            return false;
        hit.t = h.t;
        hit.st = {h.st[0], h.st[1]};
        hit.bary = {h.bary[0], h.bary[1]};
        hit.ng = {h.ng[0], h.ng[1], h.ng[2]};
        hit.i = h.i;
        hit.j = h.j;
        return true;
    }

    // Throughput form: n rays of 8 doubles (o, d, t_min, t_max) in one query.
    void intersect_batch(const double *rays, int64_t n, const TraversalOptions &options, dmap_hit64 *hits,
                         bool occluded = false) const
    {
        dmap_options opt = options.c();
        opt.mode = occluded ? DMAP_MODE_OCCLUDED : DMAP_MODE_CLOSEST;
        check(dmap_intersect_host(h_, rays, DMAP_F64, n, &opt, hits, DMAP_F64, nullptr), ctx_->get(),
              "dmap_intersect_host");
    }

    dmap_scene *get() const { return h_; }

  private:
    Context *ctx_;
    dmap_scene *h_ = nullptr;
};

} // namespace dmapgpu
