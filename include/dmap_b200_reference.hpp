// dmap_b200 behind the reference's own intersector types.
//
// A C++ host built against the reference's headers includes this file after
// displaced_intersector.h (code/cpp/src) and replaces
//     dmap::ObjectIntersector obj(triangles, pyramid, field);
//     obj.intersect(o, d, t_min, t_max, options, hit, triangle, &stats);
// (displaced_intersector.h:183-197) with
//     dmap::GpuObjectIntersector obj(triangles, pyramid, field);
//     obj.intersect(o, d, t_min, t_max, options, hit, triangle, &stats);
// with no other change at its call sites (traversal_test_util.cpp:13-19,
// test_traversal_cost.cpp:246-249, DisplacedAreaLight::pdf). The triangles
// go to the device as the BaseTriangles the caller built (their chart
// fields verbatim, dmap_scene_create_charts), the height grid as the
// HeightGrid's own doubles, and the pyramid is rebuilt on the device with
// the caller's PyramidBuild; the device's FP64 pyramid and walk equal the
// reference's bit for bit, and its FP32 walk (the default here) returns the
// same hits.
//
// Errors follow the reference's convention: an ASSERT (ks/assertion.h)
// stops the program, since ObjectIntersector has no error channel.
#pragma once

#include "dmap_b200.h"
#include "ks/assertion.h"

#include <cstdint>
#include <vector>

namespace dmap
{

struct GpuObjectIntersector
{
    dmap_context *ctx = nullptr;
    dmap_asset *asset = nullptr;
    dmap_scene *scene = nullptr;
    int n_tri = 0;

    // ObjectIntersector(const std::vector<BaseTriangle> &, const TaylorPyramid &, const HeightGrid &)
    // (displaced_intersector.h:183-184). `device` picks the GPU.
    GpuObjectIntersector(const std::vector<BaseTriangle> &tris, const TaylorPyramid &pyramid, const HeightGrid &field,
                         int device = 0)
    {
        ASSERT(field.W == field.H, "the device pyramid needs a square node grid, got %d x %d", field.W, field.H);
        check(dmap_create(device, &ctx), "dmap_create");
        unsigned flags = DMAP_ASSET_KEEP_F64 | (pyramid.build == PyramidBuild::Direct ? DMAP_ASSET_BUILD_DIRECT : 0u);
        check(dmap_asset_create(ctx, field.values, DMAP_F64, field.W, field.scale, field.offset, field.repeat ? 1 : 0,
                                flags, &asset),
              "dmap_asset_create");
        n_tri = (int)tris.size();
        std::vector<double> rec(37 * tris.size());
        std::vector<int> which(tris.size(), 0);
        for (size_t k = 0; k < tris.size(); ++k) {
            const BaseTriangle &t = tris[k];
            double *r = &rec[37 * k];
            const ks::vec3d *v3[] = {&t.p0, &t.p1, &t.p2, &t.q0, &t.e1, &t.e2};
            for (int q = 0; q < 6; ++q)
                for (int a = 0; a < 3; ++a)
                    r[3 * q + a] = (*v3[q])[a];
            const ks::vec2d *uv[] = {&t.t0, &t.t1, &t.t2};
            for (int q = 0; q < 3; ++q) {
                r[18 + 2 * q] = (*uv[q])[0];
                r[19 + 2 * q] = (*uv[q])[1];
            }
            const ks::vec3d *m[] = {&t.m0, &t.Mu, &t.Mv};
            for (int q = 0; q < 3; ++q)
                for (int a = 0; a < 3; ++a)
                    r[24 + 3 * q + a] = (*m[q])[a];
            r[33] = t.J(0, 0);
            r[34] = t.J(0, 1);
            r[35] = t.J(1, 0);
            r[36] = t.J(1, 1);
        }
        check(dmap_scene_create_charts(ctx, &asset, 1, which.data(), rec.data(), n_tri, &scene),
              "dmap_scene_create_charts");
    }
    ~GpuObjectIntersector()
    {
        dmap_scene_destroy(scene);
        dmap_asset_destroy(asset);
        dmap_destroy(ctx);
    }
    // embree-free, but the reference's object is not copyable either
    GpuObjectIntersector(const GpuObjectIntersector &) = delete;
    GpuObjectIntersector &operator=(const GpuObjectIntersector &) = delete;

    // ObjectIntersector::intersect (displaced_intersector.h:193-194): the
    // flat loop's triangle order, one ray, one launch.
    bool intersect(const ks::vec3d &o, const ks::vec3d &d, double t_min, double t_max, const TraversalOptions &options,
                   DisplacedHit &hit, int &triangle, TraversalStats *stats = nullptr) const
    {
        double ray[8] = {o[0], o[1], o[2], d[0], d[1], d[2], t_min, t_max};
        dmap_options opt = to_c(options);
        opt.schedule = DMAP_SCHEDULE_SIMPLE; // one ray: one thread, one launch
        dmap_hit64 h;
        int64_t st[DMAP_ST_COUNT] = {};
        check(dmap_intersect_host(scene, ray, DMAP_F64, 1, &opt, &h, DMAP_F64, stats ? st : nullptr),
              "dmap_intersect_host");
        if (stats) {
            stats->triangle_tests += st[DMAP_ST_TRIANGLE_TESTS];
            stats->node_tests += st[DMAP_ST_NODE_TESTS];
            stats->leaf_tests += st[DMAP_ST_LEAF_TESTS];
            stats->sub_squares += st[DMAP_ST_SUB_SQUARES];
            stats->node_tests_after_hit += st[DMAP_ST_NODE_AFTER_HIT];
            stats->leaf_tests_after_hit += st[DMAP_ST_LEAF_AFTER_HIT];
        }
        triangle = h.tri;
        if (h.tri < 0)
            return false;
        copy_hit(h, hit);
        return true;
    }

    // Throughput form: n rays of 8 doubles (o, d, t_min, t_max) answered in
    // one batched device query; triangle[k] is -1 for a miss.
    void intersect_batch(const double *rays, int64_t n, const TraversalOptions &options, DisplacedHit *hits,
                         int *triangle) const
    {
        std::vector<dmap_hit64> h((size_t)n);
        dmap_options opt = to_c(options);
        check(dmap_intersect_host(scene, rays, DMAP_F64, n, &opt, h.data(), DMAP_F64, nullptr), "dmap_intersect_host");
        for (int64_t k = 0; k < n; ++k) {
            triangle[k] = h[k].tri;
            if (h[k].tri >= 0)
                copy_hit(h[k], hits[k]);
        }
    }

    static void copy_hit(const dmap_hit64 &h, DisplacedHit &hit)
    {
        hit.t = h.t;
        hit.st = ks::vec2d(h.st[0], h.st[1]);
        hit.bary = ks::vec2d(h.bary[0], h.bary[1]);
        hit.ng = ks::vec3d(h.ng[0], h.ng[1], h.ng[2]);
        hit.i = h.i;
        hit.j = h.j;
    }

    // TraversalOptions (traversal_options.h:30-38) in the C ABI's terms: the
    // FP32 walk with the FP64 leaf (whose hits equal the FP64 walk's) for the
    // Newton leaf, the FP64 path for the two-triangle leaf, the flat loop's
    // triangle order.
    static dmap_options to_c(const TraversalOptions &o)
    {
        dmap_options c;
        dmap_options_default(&c);
        c.bound = o.bound == BoundMode::Box ? DMAP_BOUND_BOX : o.bound == BoundMode::Slab ? DMAP_BOUND_SLAB
                                                                                           : DMAP_BOUND_BOTH;
        c.slab_max_level = o.slab_max_level;
        c.leaf = o.leaf == LeafMode::Newton ? DMAP_LEAF_NEWTON : DMAP_LEAF_TWO_TRIANGLE;
        c.precision = o.leaf == LeafMode::Newton ? DMAP_PRECISION_F32 : DMAP_PRECISION_F64;
        c.order = DMAP_ORDER_INDEX;
        c.leaf_precision = DMAP_PRECISION_F64;
        return c;
    }

    static void check(dmap_status s, const char *what)
    {
        ASSERT(s == DMAP_OK, "dmap_b200: %s: %s", what, dmap_status_string(s));
    }
};

} // namespace dmap
