/*
 * dmap_b200: the ray vs displaced-surface query of MangoSister/dmap on NVIDIA
 * B200 (sm_100a). Plain C ABI: opaque handles, plain pointers and sizes,
 * integer status codes (never abort), no CUDA or C++ types in signatures
 * (streams are passed as `void *` holding a cudaStream_t).
 *
 * Each entry point names the reference interface it replaces
 * (code/cpp/src in the reference, file:line).
 *
 * Threading: one context per device. Calls on one context are serialized by
 * the caller; different contexts may be used from different threads.
 * Buffers passed as "device" must be device memory of the context's GPU;
 * "host" buffers may be pageable or pinned.
 */
#ifndef DMAP_B200_H
#define DMAP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum dmap_status {
    DMAP_OK = 0,
    DMAP_ERR_INVALID = 1,     /* bad argument (the reference ASSERTs instead) */
    DMAP_ERR_CUDA = 2,        /* a CUDA call failed; dmap_last_error() has the text */
    DMAP_ERR_OOM = 3,         /* device allocation failed */
    DMAP_ERR_DEGENERATE = 4,  /* a base triangle is degenerate in texture space (displaced_surface.cpp:67) */
    DMAP_ERR_BUDGET = 5,      /* the request does not fit the server's memory budget */
    DMAP_ERR_LIMIT = 6,       /* an iteration cap ran out on the device; results are flagged */
    DMAP_ERR_NOT_READY = 7,   /* a served request has not finished */
    DMAP_ERR_UNSUPPORTED = 8, /* combination of options the build does not offer */
    DMAP_ERR_CANCELLED = 9    /* a served request was cancelled */
} dmap_status;

/* Ray and hit records are F32 or F64; height texels may also be F16 or BF16. */
typedef enum dmap_dtype { DMAP_F32 = 0, DMAP_F16 = 1, DMAP_F64 = 2, DMAP_BF16 = 3 } dmap_dtype;

typedef struct dmap_context dmap_context;
typedef struct dmap_asset dmap_asset;
typedef struct dmap_scene dmap_scene;
typedef struct dmap_server dmap_server;

/* ---- context ---------------------------------------------------------- */

/* Binds a device and creates the library's streams and pinned staging. */
dmap_status dmap_create(int device, dmap_context **out);
void dmap_destroy(dmap_context *ctx);
const char *dmap_status_string(dmap_status s);
/* Text of the last error on this context (empty when none). */
const char *dmap_last_error(const dmap_context *ctx);
/* Number of the library's kernels launched on this context so far. */
int64_t dmap_kernel_launches(const dmap_context *ctx);

/* ---- displacement assets: HeightGrid + TaylorPyramid ------------------- */

/* Asset flags. */
#define DMAP_ASSET_KEEP_F64 1u /* keep the FP64 pyramid resident (needed by DMAP_PRECISION_F64) */
/* build every level from the node grid (PyramidBuild::Direct, taylor_pyramid.cpp:151-202:
 * tighter r than the default fold, about twice the work) */
#define DMAP_ASSET_BUILD_DIRECT 2u

/*
 * Uploads a (nodes x nodes) node grid, nodes = 2^L + 1, row major with
 * values[j * nodes + i] at (u, v) = (i, j) / (nodes - 1), and builds its
 * Taylor bound pyramid on the device: h = scale * value + offset, texture
 * coordinates wrapping when `repeat`, clamping otherwise.
 * Replaces DisplacementAsset's grid + TaylorPyramid(const HeightGrid &, PyramidBuild::Fold)
 * (displacement_asset.cpp:16-35, taylor_pyramid.h:89-92, taylor_pyramid.cpp:215-257).
 * `values_host` is host memory of `dtype` (F32, F16, BF16 or F64).
 */
dmap_status dmap_asset_create(dmap_context *ctx, const void *values_host, dmap_dtype dtype, int nodes, double scale,
                              double offset, int repeat, unsigned flags, dmap_asset **out);
void dmap_asset_destroy(dmap_asset *asset);
int dmap_asset_levels(const dmap_asset *asset);
/* Device bytes the asset holds. */
size_t dmap_asset_bytes(const dmap_asset *asset);
/* CUDA-event time in ms of the asset's pyramid build kernels (no reference
 * counterpart: the measurement of the build, which the reference times on
 * the CPU around the TaylorPyramid constructor). */
double dmap_asset_build_ms(const dmap_asset *asset);
/*
 * Copies pyramid level `level` to the host as 8 channel planes (h0, gu, gv, r,
 * ru, rv, h_min, h_max), each m*m doubles with m = 2^L >> level, [j*m + i]
 * (the TaylorLevel layout, taylor_pyramid.h:52-61). precision selects the
 * FP64 pyramid (DMAP_PRECISION_F64, needs KEEP_F64) or the outward-rounded
 * FP32 one widened to double (DMAP_PRECISION_F32).
 */
dmap_status dmap_asset_pyramid_level(const dmap_asset *asset, int level, int precision, double *out_host);

/*
 * The pyramid build without any device allocation. No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc (a host
 * application that owns all device memory through its own pool, or that must
 * not allocate while frames are in flight), which dmap_asset_create cannot
 * serve because it allocates the node grid, the FP64 working levels and the
 * output.
 * The caller passes the node grid already on the device (`nodes` x `nodes`
 * values of `dtype`, rows `pitch` elements apart, pitch * element size a
 * multiple of 16 bytes, 16-byte aligned) and a device buffer for the FP32
 * pyramid: sum over levels l = 0..L of (2^L >> l)^2 cells of 8 floats, laid
 * out as the asset's FP32 pyramid (dmap_asset_pyramid_level, DMAP_PRECISION_F32).
 * The FP64 working levels live in a fixed device array of the library (22.4
 * MB per GPU that loads it, held until exit), so maps are limited to
 * 2^L <= 512 texels per side; larger ones return DMAP_ERR_INVALID. The first
 * call on each device (and the first after that device's context was
 * recreated) looks up the array's device address. Under lazy module loading
 * (CUDA's default) that look-up loads the library's device code and commits
 * the array, so that first call can itself take device memory: make it at
 * start-up, before any frame and before any stream capture (a call on a 3 x 3
 * node grid is enough). Later calls allocate nothing. Runs on `stream` (a
 * cudaStream_t, NULL = the legacy default stream) and returns when the
 * pyramid is written. Calls share the array, which keeps the last call's
 * contents: calls that overlap on the GPU race, so serialize them.
 */
dmap_status dmap_pyramid_build_noalloc(const void *nodes_dev, dmap_dtype dtype, int nodes, int pitch, double scale,
                                       double offset, int repeat, float *pyr32_dev, void *stream);

/* ---- scenes: ObjectIntersector over base triangles --------------------- */

/*
 * Per-triangle setup on the device: the base triangle and its chart, the
 * tangent frame, the footprint roots, the height range and the object-space
 * AABB. tris_host: n_tri x 24 doubles (p0, p1, p2, m0, m1, m2 as xyz; t0,
 * t1, t2 as texture uv), tri_asset[k] indexes `assets`.
 * Replaces ObjectIntersector(const std::vector<BaseTriangle> &, const TaylorPyramid &,
 * const HeightGrid &) (displaced_intersector.h:183-184, displaced_intersector.cpp:466-479)
 * with the BaseTriangle general-chart constructor (displaced_surface.h:79-81).
 * A scene borrows its assets: destroy the scene first.
 */
dmap_status dmap_scene_create(dmap_context *ctx, dmap_asset *const *assets, int n_assets, const int *tri_asset_host,
                              const double *tris_host, int n_tri, dmap_scene **out);
/*
 * The same scene from BaseTriangles the caller already built (the
 * reference's own objects, displaced_surface.h:63-95): n_tri x 37 doubles
 * per triangle, p0 p1 p2 (positions), q0 e1 e2 (the chart's P), t0 t1 t2
 * (texture uv), m0 Mu Mv (the chart's M), J (2 x 2, row major), taken as
 * they are instead of rebuilt from vertex normals, so a drop-in over
 * ObjectIntersector(const std::vector<BaseTriangle> &, ...) sees exactly
 * the triangles the reference walks. Replaces the same constructor as
 * dmap_scene_create (displaced_intersector.cpp:466-479).
 */
dmap_status dmap_scene_create_charts(dmap_context *ctx, dmap_asset *const *assets, int n_assets,
                                     const int *tri_asset_host, const double *charts_host, int n_tri,
                                     dmap_scene **out);
/*
 * Scene-level instancing: the reference's scene objects placed by their
 * to_world transforms as embree instances (displaced_scene.cpp:79-87,
 * Builder::add_instance). Objects are consecutive ranges of the base
 * triangles: object o holds triangles object_first[o] .. object_first[o+1]-1
 * of tris_host / tri_asset_host (n_objects + 1 offsets). Instance k places
 * object instance_object[k] by the row-major 3x4 matrix instance_to_world +
 * 12 k (linear part L, translation t). hit.tri counts through the
 * instances' triangles in instance order; the instances share the assets'
 * pyramids. When every L is a rotation (orthogonal within 1e-9, mirrors
 * included), the scene holds each instance's triangles moved to world
 * space (positions L p + t, vertex normals L m): a rigid motion moves the
 * displaced surface exactly, S = L (P + h N) + t = (L P + t) + h (L N).
 * Otherwise (a scale or shear, which would scale the heights if the base
 * triangles were moved) every instance keeps its object's triangles and a
 * ray meets them in object space, x = Linv (w - t) with t unchanged, as the
 * reference's embree instancing hands the instanced geometry its ray; hit
 * normals are returned in world space (sign(det L) Linv^T n, normalized),
 * dmap_surface_points moves points and tangents by L, and
 * dmap_tessellate_* refuse such a scene (DMAP_ERR_UNSUPPORTED). A singular
 * L is DMAP_ERR_INVALID.
 */
dmap_status dmap_scene_create_instanced(dmap_context *ctx, dmap_asset *const *assets, int n_assets,
                                        const int *tri_asset_host, const double *tris_host,
                                        const int *object_first, int n_objects, const int *instance_object,
                                        const double *instance_to_world, int n_instances, dmap_scene **out);
void dmap_scene_destroy(dmap_scene *scene);
int dmap_scene_triangle_count(const dmap_scene *scene);
/*
 * Per-triangle setup results (11 doubles: root_level, n_roots,
 * residual_tolerance, aabb lo xyz, aabb hi xyz, h_min, h_max), the fields
 * DisplacedIntersector's constructor and triangle_aabb produce
 * (displaced_intersector.cpp:135-151, node_bounds.cpp:238-269).
 */
dmap_status dmap_scene_triangle_info(const dmap_scene *scene, int tri, double *out11);

/* ---- queries ------------------------------------------------------------ */

/* TraversalOptions (traversal_options.h:30-38) plus the device choices. */
#define DMAP_BOUND_BOX 0
#define DMAP_BOUND_SLAB 1
#define DMAP_BOUND_BOTH 2
#define DMAP_LEAF_NEWTON 0
#define DMAP_LEAF_TWO_TRIANGLE 1
#define DMAP_PRECISION_F64 0 /* the reference's double arithmetic, operation for operation */
/* FP32 walk, bounds widened outward so it admits every cell the FP64 walk
 * admits; each leaf cell re-tested with the reference's FP64 node test, its
 * leaf run in the precision dmap_options.leaf_precision selects */
#define DMAP_PRECISION_F32 1
#define DMAP_MODE_CLOSEST 0  /* closest hit in (t_min, t_max): rtcIntersect1 / intersect_callback */
#define DMAP_MODE_OCCLUDED 1 /* any hit in (t_min, t_max): rtcOccluded1 / occluded_callback */

#define DMAP_SCHEDULE_WAVEFRONT 0 /* rounds of a persistent walk kernel and a leaf kernel (default) */
#define DMAP_SCHEDULE_SIMPLE 1    /* one thread per ray, one launch: the plain per-request kernel */

/*
 * The order in which a ray visits the triangles whose boxes it meets.
 * INDEX is ObjectIntersector::intersect's flat loop (displaced_intersector.cpp:
 * 578-599): triangles in index order, each walked with the t_max the ones
 * before it left. NEAREST visits them by box entry distance (the FP64 slab
 * entry max(t_min, max_a min(ta, tb)), ta = (lo_a - o_a) * (1 / d_a), ties
 * to the lower index), as a BVH over the embree callbacks
 * (displaced_geometry.cpp:49-106) does, and skips a triangle whose box lies
 * beyond the current hit: the walk starts with a tight t_max, so far
 * triangles cost a box test instead of a walk. Both find the nearest
 * certified root; the returned t may differ in the last bits where the walks
 * run with different t_max. Scenes of more than 256 triangles find their
 * candidates in either order through a tree over the triangles' boxes built
 * by dmap_scene_create (the reference's embree BVH over rtc_bounds,
 * displaced_intersector.cpp:454-464); the visiting order is the same as a
 * scan over every triangle.
 */
#define DMAP_ORDER_INDEX 0
#define DMAP_ORDER_NEAREST 1

typedef struct dmap_options {
    int bound;          /* DMAP_BOUND_*, default BOTH */
    int slab_max_level; /* default 1 */
    int leaf;           /* DMAP_LEAF_*, default NEWTON */
    int precision;      /* DMAP_PRECISION_*, default F32 */
    int mode;           /* DMAP_MODE_*, default CLOSEST */
    double polish_cond; /* FP32 leaf: roots whose Newton Jacobian has cond(J) above this are refined by the
                           reference's FP64 Newton (default 1e4) */
    int schedule;       /* DMAP_SCHEDULE_*, FP32 path only, default WAVEFRONT */
    int rounds;         /* wavefront: walk/leaf rounds before the last walk finishes the rest inline (0..32,
                           default 2; 0 = one walk with every leaf inline) */
    int blocks_per_sm;  /* wavefront: 128-thread walk blocks per SM (0..16; default 0 = the occupancy the walk
                           is compiled for: 4 on scenes of up to 256 triangles, 5 above, where the triangle
                           tree takes the candidates) */
    int order;          /* DMAP_ORDER_*, default NEAREST */
    int node_visit_cap; /* FP32 path: cells one triangle's walk may visit before it gives up (0 = the default,
                           2^26, far above any walk of a well-formed scene). A ray whose walk gives up keeps
                           what it found, its hit record gets DMAP_HIT_CAPPED, and the call reports
                           DMAP_ERR_LIMIT */
    int leaf_precision; /* FP32 path's certified leaf: DMAP_PRECISION_F32 (default: the leaf's search and
                           Newton in FP32 with outward-rounded sub-square bounds, FP64 Newton polish above
                           polish_cond; the same hit set, t within 1e-5 of the scene extent) or
                           DMAP_PRECISION_F64 (the reference's leaf in double: every hit equal to the FP64
                           path's bit for bit, as the drop-in adapters set it) */
    int graph;          /* dmap_intersect_host on the FP32 path: 1 replays the query's launches (3 x rounds + 1
                           kernels and their memsets) from a CUDA graph captured once per (scene, options,
                           batch-size class) on the context, the ray count read on the device; the records
                           equal those without it. 0 (default): launched one by one */
} dmap_options;

/* Fills the defaults above. */
void dmap_options_default(dmap_options *opt);

/*
 * Rays: n records of 8 values of `ray_dtype` (F32 or F64): o.xyz, d.xyz,
 * t_min, t_max. Hits: n records of `hit_dtype` (F32: struct dmap_hit32, F64:
 * struct dmap_hit64). Misses have tri = -1 and t = +inf. In OCCLUDED mode
 * only `tri` (>= 0 when occluded) and `t` of some occluder are meaningful.
 */
typedef struct dmap_hit32 {
    float t, st[2], bary[2], ng[3];
    int32_t tri, i, j, flags;
} dmap_hit32;
typedef struct dmap_hit64 {
    double t, st[2], bary[2], ng[3];
    int32_t tri, i, j, flags;
} dmap_hit64;
/* dmap_hit*.flags bits */
#define DMAP_HIT_FP64_LEAF 1 /* the root is an FP64 Newton root (the FP64 leaf, or an FP32 root polished in FP64) */
#define DMAP_HIT_CAPPED 2   /* a device iteration cap ran out for this ray */
#define DMAP_HIT_POLISHED 4 /* an FP32 leaf root refined by FP64 Newton (cond(J) > polish_cond) */

/* Per-ray counters (TraversalStats, displaced_intersector.h:89-105), 8 int64 per ray. */
#define DMAP_ST_TRIANGLE_TESTS 0
#define DMAP_ST_NODE_TESTS 1
#define DMAP_ST_LEAF_TESTS 2
#define DMAP_ST_SUB_SQUARES 3
#define DMAP_ST_NEWTON_ITERS 4
#define DMAP_ST_NODE_AFTER_HIT 5
#define DMAP_ST_LEAF_AFTER_HIT 6
#define DMAP_ST_COUNT 8

/*
 * Batched query on device buffers, asynchronous on `stream` (a
 * cudaStream_t, NULL = the context's stream). `stats_dev` may be NULL.
 * Replaces, per ray, ObjectIntersector::intersect (displaced_intersector.h:193-194)
 * and the embree callbacks intersect_callback / occluded_callback
 * (displaced_geometry.cpp:49-106) for a scene of displaced objects.
 */
dmap_status dmap_intersect(dmap_scene *scene, const void *rays_dev, dmap_dtype ray_dtype, int64_t n,
                           const dmap_options *opt, void *hits_dev, dmap_dtype hit_dtype, int64_t *stats_dev,
                           void *stream);

/*
 * The same query on host buffers: copies the rays in, runs, copies the hits
 * back, and returns when they are on the host (synchronous). This is the
 * drop-in call a CPU-side scene makes per batch, and the single-ray
 * ObjectIntersector::intersect when n = 1.
 */
dmap_status dmap_intersect_host(dmap_scene *scene, const void *rays_host, dmap_dtype ray_dtype, int64_t n,
                                const dmap_options *opt, void *hits_host, dmap_dtype hit_dtype, int64_t *stats_host);

/*
 * Hit records to surface points: DisplacedGeometry::surface_point
 * (displaced_geometry.cpp:126-152), the step from a hit to the shading
 * record, for every hit at once. Per hit (tri, bary = the base triangle's
 * barycentrics u, v) 14 doubles: the displaced position p, the geometric
 * normal ng (oriented along the base face's winding (p1 - p0) x (p2 - p0),
 * unit), dpdu and dpdv (the surface tangents along the chart, scaled by the
 * object's uv map), and the object uv (DisplacedObject::object_uv,
 * scene_spec.cpp:382-388). Misses (tri < 0) give zeros. map NULL = identity.
 */
typedef struct dmap_uv_map {
    double uv_scale[2], uv_offset[2]; /* tile coordinates = uv * uv_scale + uv_offset */
    int flip_v;                       /* v' = 1 - v */
} dmap_uv_map;
dmap_status dmap_surface_points(dmap_scene *scene, const void *hits_dev, dmap_dtype hit_dtype, int64_t n,
                                const dmap_uv_map *map, double *out_dev, void *stream);
/* The same on host buffers (synchronous). */
dmap_status dmap_surface_points_host(dmap_scene *scene, const void *hits_host, dmap_dtype hit_dtype, int64_t n,
                                     const dmap_uv_map *map, double *out_host);

/*
 * Hit filter: ks's opacity map behind embree's filter functions, as
 * DisplacedGeometry's intersect and occluded callbacks run them
 * (displaced_geometry.cpp:53-106). The crossing a triangle's walk returns
 * goes to the filter; a crossing it rejects is skipped and the triangle is
 * walked again from t_min = that crossing's t, at most 64 times
 * (max_filter_passes, displaced_geometry.h:64); an occlusion query takes
 * the nearest crossing of each triangle for the filter to judge. The
 * filter: the crossing's texture coordinate (compute_hit_texcoord,
 * displaced_geometry.cpp:189-193: the float barycentrics the filter sees,
 * BaseTriangle::param, the object uv of `map` (NULL = identity), rounded to
 * float) picks texel (floor(u w) mod w, floor(v h) mod h) of a w x h mask,
 * row-major with rows along v; 0 is transparent and rejects the crossing.
 * tri_flags_host (n_tri bytes, NULL = every triangle) marks the triangles
 * the map covers (the object whose material carries it); the others accept
 * every crossing. mask_host NULL removes the filter. The mask is copied.
 * FP32 queries on a filtered scene (dmap_intersect*, dmap_render and
 * the server alike) take the filter's passes on either schedule: the
 * wavefront answers without them and hands every ray that took a crossing
 * the filter rejects to the one-thread-per-ray schedule, whose triangle
 * walks take the passes. While a server holds requests on the scene
 * (queued or running), the filter cannot change: this call returns
 * DMAP_ERR_NOT_READY until they are done (dmap_server_drain); do not call it
 * concurrently with a submit on the same scene.
 */
dmap_status dmap_scene_set_opacity(dmap_scene *scene, const uint8_t *mask_host, int w, int h, const dmap_uv_map *map,
                                   const uint8_t *tri_flags_host);

/*
 * Oracle meshes (displaced_tessellation.h:17-53): the displaced surface of
 * every scene triangle as a float mesh, for mesh-based cross-checks.
 * Positions S = P + h N, texture coordinates (s, t) and unit vertex normals
 * are evaluated in double with the reference's operation order and rounded
 * to float, so both meshes are bit-identical to the reference's.
 *
 * dmap_tessellate_uniform replaces append_displaced_triangle
 * (displaced_tessellation.cpp:32-56) over the scene's triangles in order:
 * the uniform barycentric grid at subdivision n (tessellation_grid, :11-30),
 * (n+1)(n+2)/2 vertices and n*n faces per triangle; triangle k's vertices
 * start at k (n+1)(n+2)/2 and its faces at k n^2, with indices global (the
 * reference's `base + f`). Buffers: vertices and normals 3 floats per
 * vertex, texcoords 2, indices 3 uint32 per face; the MeshData padding of
 * finalize_mesh_data is the caller's. Fails when the vertex count exceeds
 * the uint32 index range.
 */
dmap_status dmap_tessellate_uniform(dmap_scene *scene, int n, float *vertices_dev, float *texcoords_dev,
                                    float *normals_dev, uint32_t *indices_dev, void *stream);
dmap_status dmap_tessellate_uniform_host(dmap_scene *scene, int n, float *vertices, float *texcoords,
                                         float *normals, uint32_t *indices);

/*
 * The texel-aligned tessellation (append_texel_tessellation,
 * displaced_tessellation.cpp:101-136) over the scene's triangles in order:
 * every leaf cell meeting a triangle's uv domain split into m x m sub-cells,
 * each inside sub-cell into two faces along the (1,0)-(0,1) diagonal and each
 * straddling one into the fan of its clipped polygon; faces keep the base
 * face's winding. Three unshared vertices per face (vertex 3f + q of face
 * f), as append_face writes them, so the index buffer is the identity and is
 * not returned. faces_dev gets the TexelFace records (triangle = scene
 * triangle index). Synchronous on `stream`: *n_faces returns the face count.
 * With vertices_dev NULL only the count is computed; otherwise a count above
 * capacity writes nothing and returns DMAP_ERR_INVALID (with *n_faces set).
 */
typedef struct dmap_texel_face {
    int32_t triangle;
    int32_t interior; /* 1: from a sub-cell inside the domain; 0: a fan face of a clipped sub-cell */
    double st[3][2];  /* tile coordinates of the three vertices */
} dmap_texel_face;
dmap_status dmap_tessellate_texel(dmap_scene *scene, int m, int64_t capacity, float *vertices_dev,
                                  float *texcoords_dev, float *normals_dev, dmap_texel_face *faces_dev,
                                  int64_t *n_faces, void *stream);
dmap_status dmap_tessellate_texel_host(dmap_scene *scene, int m, int64_t capacity, float *vertices,
                                       float *texcoords, float *normals, dmap_texel_face *faces, int64_t *n_faces);

/*
 * Displaced-emitter sampling: DescentSampler (descent_sampler.h:105-160,
 * descent_sampler.cpp:85-362) for every triangle of a scene, over an
 * EmissionTile per asset (emission_tile.h:40-88, the texture's own
 * repeating tile: texels_host[a] is the asset's n_leaf x n_leaf texel grid,
 * row major, or NULL for a uniform emission of 1). variant: AreaOnly,
 * Product or ProductGeometry (DescentWeight); beta: the uniform blend floor;
 * emitter_cosine: ProductGeometry's |emitter cosine| factor. The descent
 * weights read the FP64 pyramid, so the scene's assets need
 * DMAP_ASSET_KEEP_F64. Built once on the host (each triangle's footprint:
 * root block and straddling tree with exact clipped areas and masses) and
 * uploaded.
 */
#define DMAP_DESCENT_AREA 0
#define DMAP_DESCENT_PRODUCT 1
#define DMAP_DESCENT_PRODUCT_GEOMETRY 2
typedef struct dmap_emitter dmap_emitter;
dmap_status dmap_emitter_create(dmap_scene *scene, const double *const *texels_host, int variant, double beta,
                                int emitter_cosine, dmap_emitter **out);
/* An emitter borrows its scene for queries: destroy it before the scene's
 * context (destroying it after the scene is allowed). */
void dmap_emitter_destroy(dmap_emitter *emitter);
/* Footprint of one triangle: root_level, root_i0, root_j0, total clipped
 * area, total clipped mass, straddling nodes (6 doubles). */
dmap_status dmap_emitter_triangle_info(const dmap_emitter *emitter, int tri, double *out6);
/*
 * DescentSampler::sample for n samples: sample k on triangle tri_dev[k]
 * draws its random numbers, in the reference's order (one per descent level,
 * two per leaf try, three for the clipped-polygon fallback after 32 misses),
 * from uniforms_dev[k * uniforms_per_sample ...] (0.5 past the end; 2^L + 70
 * covers every path), and receivers_dev (6 doubles per sample: position,
 * unit normal; NULL = none) steers ProductGeometry. draws = the uniforms
 * used, -1 for a bad triangle or one without mass. Asynchronous on stream.
 */
typedef struct dmap_emitter_point {
    double u, v;     /* texture coordinates */
    double p[3];     /* S(u, v) */
    double n[3];     /* unit surface normal */
    double sqrt_det; /* pointwise sqrt(det G) */
    double pdf_uv;   /* per unit parameter area */
    double pdf_area; /* per unit surface area */
    int32_t tri, draws;
} dmap_emitter_point;
dmap_status dmap_emitter_sample(dmap_emitter *emitter, const int32_t *tri_dev, const float *uniforms_dev,
                                int uniforms_per_sample, const double *receivers_dev, int64_t n,
                                dmap_emitter_point *out_dev, void *stream);
/* DescentSampler::pdf_uv / pdf_area (descent_sampler.cpp:346-364) at n
 * points (uv_dev: 2 doubles each) of triangles tri_dev; pdf_area_dev may be
 * NULL. The re-walk equals the sampled pdf at sampled points. */
dmap_status dmap_emitter_pdf(dmap_emitter *emitter, const int32_t *tri_dev, const double *uv_dev,
                             const double *receivers_dev, int64_t n, double *pdf_uv_dev, double *pdf_area_dev,
                             void *stream);
/* The same two on host buffers (synchronous). */
dmap_status dmap_emitter_sample_host(dmap_emitter *emitter, const int32_t *tri, const float *uniforms,
                                     int uniforms_per_sample, const double *receivers, int64_t n,
                                     dmap_emitter_point *out);
dmap_status dmap_emitter_pdf_host(dmap_emitter *emitter, const int32_t *tri, const double *uv,
                                  const double *receivers, int64_t n, double *pdf_uv, double *pdf_area);

/*
 * The displaced emitter as a light seen from shading points
 * (DisplacedEmitterLight, displaced_emitter_light.cpp:20-116; the light of
 * an emitter created with variant AREA / PRODUCT / PRODUCT_GEOMETRY is the
 * reference's AreaDescent / ProductDescent / ReceiverDescent, the last with
 * emitter_cosine 0 as the reference's light sets it). shade: 6 doubles per
 * query, the shading point p and its unit normal n.
 *
 * dmap_emitter_light replaces DisplacedEmitterLight::sample (:58-90): it
 * turns the points dmap_emitter_sample drew (with receivers = shade, which
 * the receiver variant reads) into light samples: direction wi from p to
 * the point, distance, pdf_area, solid-angle pdf_omega = pdf_area dist^2 /
 * |n_y . wi|, the emission texel Le; ok = 0 for a draw below the reference's
 * min |n_y . wi| = 1e-7 (its pdfs and Le are then 0).
 *
 * dmap_emitter_light_pdf replaces DisplacedEmitterLight::pdf_omega_from_uv
 * (:103-117) at uv (2 doubles per query), or with uv NULL the pdf of a
 * direction by the walk (DisplacedAreaLight::pdf,
 * displaced_area_light.cpp:174-186, in object space): triangle tri walked
 * from p along wi (3 doubles per query) with the reference's FP64
 * DisplacedIntersector::intersect over (0, inf), the pdf at the crossing's
 * (s, t); 0 on a miss. uv_hit (2 doubles per query, may be NULL) receives
 * the (u, v) used, NaN on a miss. Asynchronous on stream.
 */
typedef struct dmap_emitter_light_sample {
    double u, v;
    double y[3], n_y[3]; /* the point and its unit normal */
    double wi[3];        /* unit direction from the shading point to y */
    double dist;
    double pdf_area, pdf_omega, Le;
    int32_t tri, ok;
} dmap_emitter_light_sample;
dmap_status dmap_emitter_light(dmap_emitter *emitter, const dmap_emitter_point *points_dev, const double *shade_dev,
                               int64_t n, dmap_emitter_light_sample *out_dev, void *stream);
dmap_status dmap_emitter_light_pdf(dmap_emitter *emitter, const int32_t *tri_dev, const double *shade_dev,
                                   const double *uv_dev, const double *wi_dev, int64_t n, double *pdf_omega_dev,
                                   double *uv_hit_dev, void *stream);
/* The same two on host buffers (synchronous). */
dmap_status dmap_emitter_light_host(dmap_emitter *emitter, const dmap_emitter_point *points, const double *shade,
                                    int64_t n, dmap_emitter_light_sample *out);
dmap_status dmap_emitter_light_pdf_host(dmap_emitter *emitter, const int32_t *tri, const double *shade,
                                        const double *uv, const double *wi, int64_t n, double *pdf_omega,
                                        double *uv_hit);

/*
 * Schedule autotuner (no counterpart in the reference). Times the wavefront
 * schedule's launch shapes (rounds x blocks_per_sm) with `base`'s other
 * options on the first min(n, 2^22) of the caller's device rays and returns
 * `base` with the fastest shape in `best` (and its time in best_ms). With a
 * cache_path, a result is looked up first and appended after tuning, one
 * line per scene and query shape ("key rounds blocks_per_sm ms").
 */
dmap_status dmap_autotune(dmap_scene *scene, const void *rays_dev, dmap_dtype ray_dtype, int64_t n,
                          const dmap_options *base, const char *cache_path, dmap_options *best, double *best_ms);

/* ---- batched path tracer ------------------------------------------------- */

/*
 * A wavefront path tracer over a scene of displaced triangles lit by one
 * rectangular area emitter, every ray query going through the FP32 query
 * path above: per bounce, one closest-hit query for the extension rays and
 * one occlusion query for the emitter-sampled shadow rays. It replaces, for
 * diffuse scenes, the render loop that issues those queries through the
 * embree callbacks: ks's SmallPT driven by path_trace_render
 * (path_trace.cpp:98-124), next-event estimation in direct_lighting
 * (direct_lighting.cpp:198-217: light sample, shadow ray shortened by
 * shadow_eps = 1e-4, spawn_ray<NextBounce> offsets) and the occlusion query
 * behind Scene::occlude1 (occluded_callback, displaced_geometry.cpp:78-106).
 *
 * Shading (ours; ks's SmallPT is not part of the reference sources): every
 * displaced surface is Lambertian with `albedo`; the emitter is the one-sided
 * rectangle p0 + a e1 + b e2 (a, b in [0, 1]) emitting `radiance` on the side
 * of e1 x e2 and sampled uniformly by area; camera rays that see the emitter
 * add its radiance, later bounces that reach it end (next-event estimation
 * only); missed rays see black. Paths have at most `max_depth` vertices and
 * Russian roulette from vertex `rr_depth` on. Sample-major path order: path
 * g is pixel g % (width * height) of sample g / (width * height); the random
 * numbers of a path are a hash of (seed, g, vertex, dimension), so an image
 * is the same for any batching.
 */
typedef struct dmap_camera {
    double eye[3], target[3], up[3];
    double fov_deg; /* vertical field of view */
    int width, height;
} dmap_camera;

typedef struct dmap_render_desc {
    dmap_camera camera;
    double emitter_p0[3], emitter_e1[3], emitter_e2[3], radiance[3];
    double albedo[3];
    int spp, max_depth, rr_depth;
    uint64_t seed;
    int64_t paths_per_batch; /* paths in flight per wave: whole samples of the image (0 = 4M) */
    int use_graph;           /* capture one batch's stages in a CUDA graph and replay it per batch */
} dmap_render_desc;

typedef struct dmap_render_stats {
    int64_t paths, extension_rays, shadow_rays; /* queries issued */
    int64_t batches, kernel_launches;
    double device_ms;                           /* CUDA-event time of the whole render */
} dmap_render_stats;

/*
 * Optional record of every query the render issues, in issue order within a
 * stage (for ray replay against a CPU intersector): rays as issued (8 floats:
 * o, d, t_min, t_max), kind (0 extension / closest hit, 1 shadow / occlusion),
 * and the answer: the hit triangle (-1 for a miss / not occluded) and, for
 * extension rays, t. `count` returns the number of queries issued; at most
 * `capacity` are written.
 */
typedef struct dmap_ray_record {
    int64_t capacity;
    float *rays;
    int32_t *kind;
    int32_t *tri;
    float *t;
    int64_t count;
} dmap_ray_record;

/* Renders into rgb_host (height x width x 3 floats, the mean over spp, rows
 * top to bottom). opt: the query options (FP32 precision; NULL = defaults);
 * stats and record may be NULL. Synchronous. */
dmap_status dmap_render(dmap_scene *scene, const dmap_render_desc *desc, const dmap_options *opt, float *rgb_host,
                        dmap_render_stats *stats, dmap_ray_record *record);

/* ---- serving: continuous batching over resident scenes -------------------- */

/*
 * No counterpart in the reference, whose renderer runs one task at a time.
 * A server owns a worker thread and `slots` launch slots (each a stream, a
 * batch of device ray and hit buffers of max_batch_rays, and the wavefront
 * scratch). Requests are queued on submit and admitted in arrival order
 * while fewer than max_inflight are active and the device bytes the server
 * holds (slots, render jobs, and the assets of every scene it has served)
 * stay within hbm_budget_bytes. Admitted ray requests are cut into pieces
 * and packed, with the pieces of every other admitted request of the same
 * scene and mode, into one query per slot, so small requests share launches
 * and a large one does not hold back the rest; render requests run one batch
 * of image samples per slot turn. While one slot's launch runs the worker
 * fills the next, so requests that arrive mid-launch join the next launch.
 * Each result equals the one the request would get alone (a ray's answer
 * does not depend on the rays it shares a launch with; a render's image
 * does not depend on its batching). Latency is submit to completion. The
 * server's calls (submit, poll, wait, cancel, pause, drain, stats) may come
 * from several threads at once: it is the entry point for concurrent
 * callers of one device.
 */
typedef struct dmap_server_config {
    size_t hbm_budget_bytes; /* device bytes the server may hold, scene assets included (0 = no limit) */
    int64_t max_batch_rays;  /* rays per launch (0 = 4M) */
    int max_inflight;        /* admitted requests at once (0 = 256) */
    int slots;               /* launch slots in flight (0 = 2) */
    dmap_options options;    /* query options of every request (FP32 path) */
    int policy;              /* which admitted request an idle slot serves first: DMAP_SERVE_* */
} dmap_server_config;

/* Slot-filling policies (no reference counterpart: the serving loop is this
 * library's). OLDEST serves admitted requests in arrival order; SHORTEST
 * serves the one with the fewest queries left to issue (the oldest of
 * equals), so small requests overtake large ones that are in progress.
 * Either way a launch packs every admitted ray request of the chosen one's
 * scene and mode, and admission stays in arrival order. */
#define DMAP_SERVE_OLDEST 0
#define DMAP_SERVE_SHORTEST 1

typedef struct dmap_server_stats {
    int64_t submitted, completed, failed, cancelled, queued, active;
    int64_t rays;              /* rays answered (render queries included) */
    int64_t launches;          /* slot launches (queries or render batches) */
    double p50_ms, p99_ms, mean_ms, max_ms; /* latency of completed requests */
    size_t held_bytes, peak_bytes;
    double busy_s, wall_s;     /* time with a launch in flight; since the first submit */
} dmap_server_stats;

dmap_status dmap_server_create(dmap_context *ctx, const dmap_server_config *cfg, dmap_server **out);
/* Cancels what is queued, waits for what runs, joins the worker. */
void dmap_server_destroy(dmap_server *srv);
/*
 * A batch of n rays (8 F32 each, host) answered into n dmap_hit32 (host);
 * mode DMAP_MODE_CLOSEST or DMAP_MODE_OCCLUDED. Both buffers are borrowed
 * until the request completes; pinned (cudaHostAlloc / registered) buffers
 * are copied asynchronously, others through the server's pinned staging.
 * DMAP_ERR_BUDGET when the request could never fit the budget.
 */
dmap_status dmap_server_submit_rays(dmap_server *srv, dmap_scene *scene, const float *rays_host, int64_t n, int mode,
                                    dmap_hit32 *hits_host, uint64_t *id);
/* A render (dmap_render's parameters; rgb_host borrowed until completion). */
dmap_status dmap_server_submit_render(dmap_server *srv, dmap_scene *scene, const dmap_render_desc *desc,
                                      float *rgb_host, uint64_t *id);
/* DMAP_OK once complete, DMAP_ERR_NOT_READY before, DMAP_ERR_CANCELLED, or the request's error. */
dmap_status dmap_server_poll(dmap_server *srv, uint64_t id);
/* Blocks until the request completes or timeout_s passes (< 0: no limit). */
dmap_status dmap_server_wait(dmap_server *srv, uint64_t id, double timeout_s);
/*
 * Holds (paused != 0) or resumes admission: while held, submitted requests
 * stay queued (cancellable) and admitted ones run to completion. A drain
 * while held waits for queued requests until its timeout. No reference
 * counterpart (serving).
 */
dmap_status dmap_server_pause(dmap_server *srv, int paused);
/* Cancels a request that is still queued (DMAP_ERR_NOT_READY once it runs). */
dmap_status dmap_server_cancel(dmap_server *srv, uint64_t id);
/* Latency in ms of a completed request (submit to completion). */
dmap_status dmap_server_latency(dmap_server *srv, uint64_t id, double *ms);
/* Blocks until every submitted request has completed (or timeout_s passes). */
dmap_status dmap_server_drain(dmap_server *srv, double timeout_s);
dmap_status dmap_server_get_stats(dmap_server *srv, dmap_server_stats *out);

#ifdef __cplusplus
}
#endif
#endif
