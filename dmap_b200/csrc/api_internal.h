// Internal to the library: the handle structs behind the C ABI's opaque
// types and the error helpers shared by the translation units of the host
// side (api.cu, render.cu, server.cu).
#pragma once
#include "dmap_b200.h"

#include "device_types.cuh"
#include "launch.h"

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using dmapdev::AssetDev;
using dmapdev::TriDev;
using dmapdev::TriDev32;

static_assert(sizeof(dmap_hit32) == sizeof(dmapdev::Hit32), "hit32 layout");
static_assert(sizeof(dmap_hit64) == sizeof(dmapdev::Hit64), "hit64 layout");
static_assert(DMAP_ST_COUNT == DMAP_ST_N, "stats layout");

struct dmap_context
{
    int device = 0;
    cudaStream_t stream = nullptr;
    unsigned *status_dev = nullptr; // device status word
    dmapk::WaveScratch wave; // the wavefront schedule's scratch, grown to the largest batch
    std::atomic<int64_t> launches{0};
    std::string error;
    // CUDA graphs of dmap_intersect_host's query launches (dmap_options.graph):
    // one per scene, options and power-of-two capacity, valid while the
    // staging buffers and the wavefront scratch they were captured on stay
    struct QueryGraph
    {
        const dmap_scene *scene;
        std::string key;
        int64_t capacity;
        const void *rays, *hits, *scratch;
        cudaGraphExec_t exec;
    };
    std::vector<QueryGraph> graphs;
    long long *n_dev = nullptr;  // the ray count a replayed graph reads
    long long *n_host = nullptr; // its pinned host staging
    // device staging for dmap_intersect_host
    void *rays_dev = nullptr, *hits_dev = nullptr;
    int64_t *stats_dev = nullptr;
    size_t rays_cap = 0, hits_cap = 0, stats_cap = 0;
};

struct dmap_asset
{
    dmap_context *ctx = nullptr;
    AssetDev dev{};
    void *nodes = nullptr;
    double *pyr64 = nullptr;
    float *pyr32 = nullptr;
    size_t bytes = 0;
    int64_t cells = 0;
    float build_ms = 0.0f; // CUDA-event time of the pyramid kernels
};

struct dmap_scene
{
    dmap_context *ctx = nullptr;
    int n_tri = 0;
    std::vector<dmap_asset *> assets;
    AssetDev *assets_dev = nullptr;
    TriDev *tris_dev = nullptr;
    TriDev32 *tris32_dev = nullptr;
    float *bvh_nodes_dev = nullptr; // more than 256 triangles: the triangle tree the candidate orders walk
    float *bvh_tri_dev = nullptr;
    int *bvh_range_dev = nullptr;
    double *inst_dev = nullptr; // non-rigid instances: their transforms (instance.cuh), else null
    int n_inst = 0;
    int bvh_n_nodes = 0;
    std::vector<TriDev> tris_host;
    bool all_f64 = true;
    // the opacity filter (dmap_scene_set_opacity); op_mask_dev null: none
    unsigned char *op_mask_dev = nullptr;
    unsigned char *op_tri_dev = nullptr;
    int op_w = 0, op_h = 0;
    dmap_uv_map op_map = {{1.0, 1.0}, {0.0, 0.0}, 0};
    // server requests on this scene not yet done (queued or running): the
    // filter may not change under them
    std::atomic<int> server_pending{0};
};

namespace dmapi
{

inline dmap_status fail(dmap_context *ctx, dmap_status s, const std::string &msg)
{
    if (ctx)
        ctx->error = msg;
    return s;
}

inline dmap_status cuda_fail(dmap_context *ctx, cudaError_t e, const char *what)
{
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation)
        return fail(ctx, DMAP_ERR_OOM, msg);
    return fail(ctx, DMAP_ERR_CUDA, msg);
}

#define DMAP_CUDA(ctx, call)                                                                                         \
    do {                                                                                                              \
        cudaError_t e_ = (call);                                                                                      \
        if (e_ != cudaSuccess)                                                                                        \
            return cuda_fail(ctx, e_, #call);                                                                         \
    } while (0)

inline size_t dtype_size(dmap_dtype t) { return t == DMAP_F64 ? 8 : (t == DMAP_F16 || t == DMAP_BF16) ? 2 : 4; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// A scene's opacity filter in a query's options: the mask, the triangles it
// covers and the uv map. The one-thread-per-ray schedule takes the filter's
// passes in its triangle walks; the wavefront answers without them and
// hands every ray that took a crossing the filter rejects to that schedule
// (walk32.cuh).
inline void apply_filter(const dmap_scene *s, dmapk::QueryOpts &q)
{
    if (!s->op_mask_dev)
        return;
    q.op_mask = s->op_mask_dev;
    q.op_tri = s->op_tri_dev;
    q.op_w = s->op_w;
    q.op_h = s->op_h;
    q.op_flip = s->op_map.flip_v;
    q.op_scale[0] = s->op_map.uv_scale[0];
    q.op_scale[1] = s->op_map.uv_scale[1];
    q.op_offset[0] = s->op_map.uv_offset[0];
    q.op_offset[1] = s->op_map.uv_offset[1];
}

inline dmap_status sync_and_check(dmap_context *ctx, const char *what)
{
    DMAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned st = 0;
    DMAP_CUDA(ctx, cudaMemcpy(&st, ctx->status_dev, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st) {
        DMAP_CUDA(ctx, cudaMemset(ctx->status_dev, 0, sizeof(unsigned)));
        if (st & dmapdev::kStatusBadInput)
            return fail(ctx, DMAP_ERR_DEGENERATE, std::string(what) + ": degenerate input");
        return fail(ctx, DMAP_ERR_LIMIT, std::string(what) + ": a device iteration cap ran out");
    }
    return DMAP_OK;
}

template <typename T>
dmap_status grow(dmap_context *ctx, T **p, size_t *cap, size_t bytes)
{
    if (*cap >= bytes)
        return DMAP_OK;
    if (*p)
        cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    DMAP_CUDA(ctx, cudaMalloc((void **)p, bytes));
    *cap = bytes;
    return DMAP_OK;
}

inline void wave_release(dmapk::WaveScratch &w)
{
    cudaFree(w.state);
    cudaFree(w.queue[0]);
    cudaFree(w.queue[1]);
    cudaFree(w.leaves);
    cudaFree(w.counters);
    cudaFree(w.rerun);
    w = dmapk::WaveScratch{};
}

// Grows a wavefront scratch to n rays. The caller makes sure that no kernel
// using the old one is in flight.
inline dmap_status wave_reserve(dmap_context *ctx, dmapk::WaveScratch &w, int64_t n)
{
    if (n <= w.capacity)
        return DMAP_OK;
    wave_release(w);
    cudaError_t e;
    if ((e = cudaMalloc(&w.state, dmapk::wave_state_bytes() * n)) != cudaSuccess ||
        (e = cudaMalloc((void **)&w.queue[0], sizeof(int) * n)) != cudaSuccess ||
        (e = cudaMalloc((void **)&w.queue[1], sizeof(int) * n)) != cudaSuccess ||
        (e = cudaMalloc(&w.leaves, dmapk::wave_leaf_bytes() * n)) != cudaSuccess ||
        (e = cudaMalloc((void **)&w.counters, sizeof(unsigned long long) * dmapk::kWaveCounters)) != cudaSuccess ||
        (e = cudaMalloc((void **)&w.rerun, sizeof(int) * n)) != cudaSuccess) {
        wave_release(w);
        return cuda_fail(ctx, e, "wavefront scratch");
    }
    w.capacity = n;
    return DMAP_OK;
}

// Device bytes of a wavefront scratch for n rays.
inline size_t wave_bytes(int64_t n)
{
    return (dmapk::wave_state_bytes() + 3 * sizeof(int) + dmapk::wave_leaf_bytes()) * (size_t)n +
           sizeof(unsigned long long) * dmapk::kWaveCounters;
}

// Validates dmap_options into the kernels' QueryOpts (api.cu).
dmap_status check_query(dmap_scene *s, dmap_dtype ray_dtype, int64_t n, const dmap_options *opt,
                        dmap_dtype hit_dtype, dmapk::QueryOpts &q);

// A path-tracer render as a resumable job (render.cu): begin allocates its
// device buffers stream-ordered on `stream` and, with use_graph, captures
// one batch's stages there; each enqueue_batch runs the next batch of whole
// image samples on the stream given; end (once the job's work is done)
// copies the image, the counts and the record out. dmap_render is begin,
// every batch, end.
struct RenderJob;
size_t render_device_bytes(const dmap_render_desc *desc, int64_t record_capacity);
dmap_status render_begin(dmap_scene *s, const dmap_render_desc *desc, const dmap_options *opt,
                         const dmap_ray_record *record, cudaStream_t stream, RenderJob **out);
int render_batches(const RenderJob *job);
int render_enqueued(const RenderJob *job);
size_t render_bytes(const RenderJob *job);
cudaError_t render_enqueue_batch(RenderJob *job, cudaStream_t stream);
dmap_status render_end(RenderJob *job, float *rgb_host, dmap_render_stats *stats, dmap_ray_record *record,
                       double device_ms);
void render_free(RenderJob *job, cudaStream_t stream); // stream-ordered free

} // namespace dmapi

