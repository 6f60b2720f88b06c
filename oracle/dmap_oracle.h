/*
 * CPU oracle of the ray vs displaced-surface query. TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, double-precision restatement of the reference's hot path
 * (MangoSister/dmap, code/cpp/src): the Taylor bound pyramid, the per-triangle
 * setup, the stackless quadtree walk with its node tests, and the certified
 * Newton leaf. Every function cites the reference file:line it follows and
 * keeps the reference's operation order, so that results agree bit for bit
 * with the reference compiled here (oracle/_ref) and with the FP64 GPU path.
 *
 * Only the tests, the smoke check and the CPU-baseline leg of bench.py use
 * this library, and only as the checker; the product never links it.
 *
 * Operation order conventions shared by this file, the reference shim
 * (oracle/ref_shim/ks/maths.h) and the FP64 device code:
 *   dot(a, b)   = (a0*b0 + a1*b1) + a2*b2
 *   cross(a, b) = (a1*b2 - a2*b1, a2*b0 - a0*b2, a0*b1 - a1*b0)
 *   norm(a)     = sqrt(dot(a, a));  normalized(a) = a / norm(a) per component
 *   M * v       = row i: (M_i0*v0 + M_i1*v1) + M_i2*v2
 *   std::min(a, b) = b < a ? b : a;  std::max(a, b) = a < b ? b : a
 * No fused multiply-add: build with -ffp-contract=off.
 */
#ifndef DMAP_ORACLE_H
#define DMAP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct o_pyramid o_pyramid;
typedef struct o_scene o_scene;

/* Pyramid build modes (taylor_pyramid.h:41-45). */
enum { O_BUILD_FOLD = 0, O_BUILD_DIRECT = 1 };
/* Traversal options (traversal_options.h:17-38). */
enum { O_BOUND_BOX = 0, O_BOUND_SLAB = 1, O_BOUND_BOTH = 2 };
enum { O_LEAF_NEWTON = 0, O_LEAF_TWO_TRIANGLE = 1 };
/* Triangle order of a scene query: the reference's flat loop, or nearest box
 * entry first (the library's DMAP_ORDER_NEAREST). */
enum { O_ORDER_INDEX = 0, O_ORDER_NEAREST = 1 };

/* Per-ray statistics (TraversalStats, displaced_intersector.h:89-105), plus a
 * Newton-iteration counter that the reference does not keep. */
enum {
    O_ST_TRIANGLE_TESTS = 0,
    O_ST_NODE_TESTS = 1,
    O_ST_LEAF_TESTS = 2,
    O_ST_SUB_SQUARES = 3,
    O_ST_NEWTON_ITERS = 4,
    O_ST_NODE_AFTER_HIT = 5,
    O_ST_LEAF_AFTER_HIT = 6,
    O_ST_COUNT = 8
};

/* Hit record, 12 doubles per ray: t, st[2], bary[2], ng[3], i, j,
 * triangle (scene-global index, -1 on a miss), object. */
enum { O_HIT_DOUBLES = 12 };

/* TaylorPyramid(values, nodes, scale, build, offset), taylor_pyramid.cpp:215-251. */
o_pyramid *o_pyramid_build(const double *values, int nodes, double scale, double offset, int build);
void o_pyramid_free(o_pyramid *p);
int o_pyramid_levels(const o_pyramid *p);
int o_pyramid_n_leaf(const o_pyramid *p);
/* Level l as 8 channel planes (h0, gu, gv, r, ru, rv, h_min, h_max), each m*m, [j*m + i]. */
void o_pyramid_level(const o_pyramid *p, int level, double *out);
/* TaylorPyramid::node (taylor_pyramid.cpp:259-274), 8 doubles. */
void o_pyramid_node(const o_pyramid *p, int level, int64_t i, int64_t j, double *out8);

/* A scene: objects in order, each an ObjectIntersector (displaced_intersector.cpp:466-479)
 * over triangles that share one height grid and its pyramid. */
o_scene *o_scene_create(void);
void o_scene_free(o_scene *s);
/* values: the (W x W) node grid; the pyramid is built from it with scale/offset.
 * tris: n_tri x 24 doubles (p0, p1, p2, m0, m1, m2 as xyz; t0, t1, t2 as uv).
 * Returns the object index, or -1 when a triangle is degenerate. */
int o_scene_add_object(o_scene *s, const double *values, int W, double scale, double offset, int repeat,
                       int build, const double *tris, int n_tri);
int o_scene_triangle_count(const o_scene *s);
/* Per triangle: root_level, n_roots, residual_tolerance, aabb lo[3], hi[3] (9 doubles),
 * and height range h_min, h_max (2 doubles): 11 doubles. */
void o_scene_triangle_info(const o_scene *s, int tri, double *out11);
/* Per triangle: tangent frame to_tangent (9, row major), ng (3). */
void o_scene_triangle_frame(const o_scene *s, int tri, double *out12);

/* rays: n x 8 doubles (o, d, t_min, t_max). hits: n x O_HIT_DOUBLES.
 * stats: n x O_ST_COUNT int64 (may be NULL); level_stats: 32 int64 summed (may be NULL).
 * Flat loop over every triangle of every object, the walk of
 * ObjectIntersector::intersect_flat (displaced_intersector.cpp:578-599)
 * (order O_ORDER_INDEX), or the same triangles nearest box entry first
 * (O_ORDER_NEAREST). threads <= 0 uses every host core. Returns the number
 * of hits. */
int64_t o_scene_intersect(const o_scene *s, const double *rays, int64_t n, int bound, int slab_max_level, int leaf,
                          double *hits, int64_t *stats, int64_t *level_stats, int threads, int order);

/* The opacity filter of dmap_scene_set_opacity for o_scene_intersect: an h x w
 * mask (0 transparent) over the crossings' texture coordinates; map5 = uv_scale
 * u, v, uv_offset u, v, flip_v (NULL identity); tri_flags n_tri bytes (NULL
 * every triangle). mask NULL removes it. Both buffers are copied. */
void o_scene_set_opacity(o_scene *s, const uint8_t *mask, int w, int h, const double *map5, const uint8_t *tri_flags);

/* Single-triangle entry points for validation. */
int o_triangle_intersect(const o_scene *s, int tri, const double *ray8, int bound, int slab_max_level, int leaf,
                         double *hit, int64_t *stats);
/* The node test record at (level, i, j): box lo/hi (6), m intervals (6), box pass,
 * slab pass, t0/t1 of node_interval (4 doubles) = 16 doubles. */
void o_node_bound(const o_scene *s, int tri, int level, int64_t i, int64_t j, const double *ray8, int bound,
                  int slab_max_level, double *out16);
/* displaced_position (displaced_surface.cpp:162-166) on triangle tri at (s, t). */
void o_displaced_position(const o_scene *s, int tri, double sp, double tp, double *out3);
/* BaseTriangle::param (displaced_surface.h:87). */
void o_triangle_param(const o_scene *s, int tri, double u, double v, double *out2);
/* DisplacedGeometry::surface_point (displaced_geometry.cpp:126-152) with the
 * object's uv map: out14 = p, ng, dpdu, dpdv, uv. */
void o_surface_point(const o_scene *s, int tri, double u, double v, const double *uv_scale, const double *uv_offset,
                     int flip_v, double *out14);

/* Oracle meshes (displaced_tessellation.cpp). Uniform barycentric grid at
 * subdivision n (tessellation_grid + append_displaced_triangle, :11-56):
 * (n+1)(n+2)/2 vertices (pos 3 floats, uv 2, normal 3) and n*n faces
 * (3 uint32 indices, relative to the triangle's first vertex). */
void o_tessellate_uniform(const o_scene *s, int tri, int n, float *pos, float *uv, float *nrm, uint32_t *idx);
/* Texel-aligned tessellation with m x m sub-cells per leaf cell
 * (append_texel_tessellation, :101-136): returns the face count and writes
 * the first cap faces, three unshared vertices each (pos 9 floats, uv 6,
 * normals 9), the TexelFace st (6 doubles) and its interior flag. */
int64_t o_tessellate_texel(const o_scene *s, int tri, int m, int64_t cap, float *pos, float *uv, float *nrm,
                           double *st6, int *interior);

/* Displaced-emitter sampling (descent_sampler.h:105-160, emission_tile.h):
 * the DescentSampler of scene triangle `tri` over its object's height grid
 * and pyramid, with an emission tile of n x n texels (n = the pyramid's
 * leaf count, the repeating tile layout), variant 0 AreaOnly, 1 Product,
 * 2 ProductGeometry, blend floor beta. NULL when n does not match. */
typedef struct o_emitter o_emitter;
o_emitter *o_emitter_create(const o_scene *s, int tri, const double *texels, int n, int variant, double beta,
                            int emitter_cosine);
void o_emitter_free(o_emitter *e);
/* root_level, root_i0, root_j0, total_area, total_mass, footprint nodes */
void o_emitter_info(const o_emitter *e, double *out6);
/* One sample drawing its random numbers from u[0..n_u) in order (0.5 past
 * the end); recv6 = receiver position and normal for ProductGeometry (or
 * NULL). out11 = u, v, p, n, sqrt_det, pdf_uv, pdf_area. Returns the number
 * of draws used. */
int o_emitter_sample(const o_emitter *e, const float *u, int n_u, const double *recv6, double *out11);
double o_emitter_pdf_uv(const o_emitter *e, double u, double v, const double *recv6);
double o_emitter_pdf_area(const o_emitter *e, double u, double v, const double *recv6);
double o_emitter_leaf_prob(const o_emitter *e, int64_t i, int64_t j, const double *recv6);
/* DisplacedEmitterLight (displaced_emitter_light.cpp:20-116) over the
 * emitter's sampler, seen from shade6 = (p, n): a sample as out16 = u, v,
 * y[3], n_y[3], wi[3], dist, pdf_area, pdf_omega, Le, ok (returned); the
 * solid-angle pdf from (u, v); and by the walk of the emitter's triangle
 * from p along wi3 (DisplacedAreaLight::pdf), uv_out = the crossing (NaN on
 * a miss). */
int o_emitter_light_sample(const o_emitter *e, const float *u, int n_u, const double *shade6, double *out16);
double o_emitter_light_pdf_uv(const o_emitter *e, const double *shade6, double u, double v);
double o_emitter_light_pdf_walk(const o_emitter *e, const double *shade6, const double *wi3, double *uv_out);

#ifdef __cplusplus
}
#endif
#endif
