// The C ABI of include/dmap_b200.h: contexts, assets (node grid + device
// pyramid), scenes (per-triangle setup) and the query entry points. Host
// C++ over the CUDA runtime; kernels live in pyramid.cu, setup.cu,
// walk64.cu and walk32.cu.
#include "api_internal.h"
#include "instance.cuh"

#include <algorithm>

using namespace dmapi;

extern "C" {

const char *dmap_status_string(dmap_status s)
{
    switch (s) {
    case DMAP_OK: return "ok";
    case DMAP_ERR_INVALID: return "invalid argument";
    case DMAP_ERR_CUDA: return "CUDA error";
    case DMAP_ERR_OOM: return "out of device memory";
    case DMAP_ERR_DEGENERATE: return "degenerate base triangle";
    case DMAP_ERR_BUDGET: return "over the memory budget";
    case DMAP_ERR_LIMIT: return "device iteration cap reached";
    case DMAP_ERR_NOT_READY: return "not ready";
    case DMAP_ERR_UNSUPPORTED: return "unsupported options";
    case DMAP_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

dmap_status dmap_create(int device, dmap_context **out)
{
    if (!out)
        return DMAP_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
        return DMAP_ERR_CUDA;
    auto *ctx = new dmap_context;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) ||
        cudaMalloc(&ctx->status_dev, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(ctx->status_dev, 0, sizeof(unsigned)) != cudaSuccess) {
        delete ctx;
        return DMAP_ERR_CUDA;
    }
    // stream-ordered allocations (render jobs, served requests) stay cached in
    // the device's default pool between calls instead of going back to the
    // driver at every synchronization
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = ctx;
    return DMAP_OK;
}

void dmap_destroy(dmap_context *ctx)
{
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->rays_dev);
    cudaFree(ctx->hits_dev);
    cudaFree(ctx->stats_dev);
    cudaFree(ctx->status_dev);
    for (auto &g : ctx->graphs)
        cudaGraphExecDestroy(g.exec);
    cudaFree(ctx->n_dev);
    cudaFreeHost(ctx->n_host);
    wave_release(ctx->wave);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *dmap_last_error(const dmap_context *ctx) { return ctx ? ctx->error.c_str() : ""; }
int64_t dmap_kernel_launches(const dmap_context *ctx) { return ctx ? ctx->launches.load() : 0; }

void dmap_options_default(dmap_options *opt)
{
    if (!opt)
        return;
    opt->bound = DMAP_BOUND_BOTH;
    opt->slab_max_level = 1;
    opt->leaf = DMAP_LEAF_NEWTON;
    opt->precision = DMAP_PRECISION_F32;
    opt->mode = DMAP_MODE_CLOSEST;
    opt->polish_cond = 1e4;
    opt->schedule = DMAP_SCHEDULE_WAVEFRONT;
    opt->rounds = 2;
    opt->blocks_per_sm = 0;
    opt->order = DMAP_ORDER_NEAREST;
    opt->node_visit_cap = 0;
    opt->leaf_precision = DMAP_PRECISION_F32;
    opt->graph = 0;
}

// ---- assets ---------------------------------------------------------------

dmap_status dmap_asset_create(dmap_context *ctx, const void *values_host, dmap_dtype dtype, int nodes, double scale,
                              double offset, int repeat, unsigned flags, dmap_asset **out)
{
    if (!ctx || !values_host || !out)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_asset_create: null argument");
    *out = nullptr;
    int n = nodes - 1;
    if (nodes < 2 || (n & (n - 1)) != 0 || n > (1 << 16))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_asset_create: the node grid must be (2^L + 1)^2 with 2^L <= 65536");
    if (dtype != DMAP_F32 && dtype != DMAP_F16 && dtype != DMAP_BF16 && dtype != DMAP_F64)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_asset_create: dtype must be F32, F16, BF16 or F64");
    if (!std::isfinite(scale) || !std::isfinite(offset))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_asset_create: scale and offset must be finite");
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    auto *a = new dmap_asset;
    a->ctx = ctx;
    size_t es = dtype_size(dtype);
    size_t per16 = 16 / es;
    int pitch = (int)(((size_t)nodes + per16 - 1) / per16 * per16);
    AssetDev &d = a->dev;
    d.dtype = dtype == DMAP_F32 ? 0 : dtype == DMAP_F16 ? 1 : dtype == DMAP_BF16 ? 3 : 2;
    d.W = nodes;
    d.pitch = pitch;
    d.n_leaf = n;
    d.n_levels = 1;
    while ((1 << d.n_levels) <= n)
        ++d.n_levels;
    d.repeat = repeat ? 1 : 0;
    d.scale = scale;
    d.offset = offset;
    int64_t cells = 0;
    for (int l = 0; l < d.n_levels; ++l) {
        d.level_off[l] = cells;
        int64_t m = n >> l;
        cells += m * m;
    }
    a->cells = cells;
    auto cleanup = [&](dmap_status s) {
        cudaFree(a->nodes);
        cudaFree(a->pyr64);
        cudaFree(a->pyr32);
        delete a;
        return s;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&a->nodes, (size_t)pitch * nodes * es)) != cudaSuccess ||
        (e = cudaMalloc((void **)&a->pyr64, (size_t)cells * 64)) != cudaSuccess ||
        (e = cudaMalloc((void **)&a->pyr32, (size_t)cells * 32)) != cudaSuccess)
        return cleanup(cuda_fail(ctx, e, "dmap_asset_create: cudaMalloc"));
    if ((e = cudaMemcpy2DAsync(a->nodes, (size_t)pitch * es, values_host, (size_t)nodes * es, (size_t)nodes * es,
                               nodes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return cleanup(cuda_fail(ctx, e, "dmap_asset_create: upload"));
    d.nodes = a->nodes;
    d.pyr64 = a->pyr64;
    d.pyr32 = a->pyr32;

    // TMA descriptor over the node grid: a (T+1) x box_w tile per CTA.
    EncodeTiledFn enc = encode_tiled();
    if (!enc)
        return cleanup(fail(ctx, DMAP_ERR_CUDA, "dmap_asset_create: cuTensorMapEncodeTiled unavailable"));
    int T = n < 16 ? n : 16;
    cuuint32_t box_w = (cuuint32_t)(((T + 1) * es + 15) / 16 * 16 / es);
    CUtensorMap tmap;
    cuuint64_t dims[2] = {(cuuint64_t)nodes, (cuuint64_t)nodes};
    cuuint64_t strides[1] = {(cuuint64_t)pitch * es};
    cuuint32_t box[2] = {box_w, (cuuint32_t)(T + 1)};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMapDataType tdt = dtype == DMAP_F32    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                              : dtype == DMAP_F16  ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                              : dtype == DMAP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUresult cr = enc(&tmap, tdt, 2, a->nodes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS)
        return cleanup(fail(ctx, DMAP_ERR_CUDA, "dmap_asset_create: cuTensorMapEncodeTiled failed"));
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaEventCreate(&ev[0]);
    cudaEventCreate(&ev[1]);
    const bool direct = (flags & DMAP_ASSET_BUILD_DIRECT) != 0;
    void *hull = nullptr; // the Direct build's slope hulls, 32 B per cell
    if (direct && (e = cudaMalloc(&hull, ((size_t)cells + 32768) * 32)) != cudaSuccess)
        return cleanup(cuda_fail(ctx, e, "dmap_asset_create: cudaMalloc"));
    cudaEventRecord(ev[0], ctx->stream);
    e = direct ? dmapk::launch_pyramid_direct(d, a->pyr64, a->pyr32, hull, ctx->stream,
                                              (flags & DMAP_ASSET_KEEP_F64) != 0)
               : dmapk::launch_pyramid(&tmap, d, T, a->pyr64, a->pyr32, ctx->status_dev, ctx->stream,
                                       (flags & DMAP_ASSET_KEEP_F64) != 0);
    cudaEventRecord(ev[1], ctx->stream);
    if (e != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        cudaStreamSynchronize(ctx->stream);
        cudaFree(hull);
        return cleanup(cuda_fail(ctx, e, "dmap_asset_create: pyramid launch"));
    }
    if (direct) {
        ctx->launches += dmapk::direct_launches(n);
    } else {
        // one leaf launch plus one fold launch per five levels above the tile
        int level = 0, t = T, launches = 1;
        while ((1 << level) * t < n) {
            level += __builtin_ctz((unsigned)t);
            int m = n >> level;
            t = m < 16 ? m : 16;
            ++launches;
        }
        ctx->launches += launches;
    }
    dmap_status s = sync_and_check(ctx, "dmap_asset_create");
    cudaEventElapsedTime(&a->build_ms, ev[0], ev[1]);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    cudaFree(hull);
    if (s != DMAP_OK)
        return cleanup(s);
    if (!(flags & DMAP_ASSET_KEEP_F64)) {
        cudaFree(a->pyr64);
        a->pyr64 = nullptr;
        d.pyr64 = nullptr;
    }
    a->bytes = (size_t)pitch * nodes * es + (size_t)cells * 32 + (a->pyr64 ? (size_t)cells * 64 : 0);
    *out = a;
    return DMAP_OK;
}

void dmap_asset_destroy(dmap_asset *a)
{
    if (!a)
        return;
    cudaSetDevice(a->ctx->device);
    cudaStreamSynchronize(a->ctx->stream);
    cudaFree(a->nodes);
    cudaFree(a->pyr64);
    cudaFree(a->pyr32);
    delete a;
}

int dmap_asset_levels(const dmap_asset *a) { return a ? a->dev.n_levels : 0; }
size_t dmap_asset_bytes(const dmap_asset *a) { return a ? a->bytes : 0; }
double dmap_asset_build_ms(const dmap_asset *a) { return a ? a->build_ms : 0.0; }

dmap_status dmap_asset_pyramid_level(const dmap_asset *a, int level, int precision, double *out)
{
    if (!a || !out || level < 0 || level >= a->dev.n_levels)
        return fail(a ? a->ctx : nullptr, DMAP_ERR_INVALID, "dmap_asset_pyramid_level: bad argument");
    dmap_context *ctx = a->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    int64_t m = a->dev.n_leaf >> level, cells = m * m;
    int64_t off = a->dev.level_off[level];
    std::vector<double> aos((size_t)cells * 8);
    if (precision == DMAP_PRECISION_F64) {
        if (!a->pyr64)
            return fail(ctx, DMAP_ERR_UNSUPPORTED, "dmap_asset_pyramid_level: the FP64 pyramid was not kept");
        DMAP_CUDA(ctx, cudaMemcpy(aos.data(), a->pyr64 + 8 * off, (size_t)cells * 64, cudaMemcpyDeviceToHost));
        if (a->dev.offset != 0.0)
            for (int64_t k = 0; k < cells; ++k) {
                aos[8 * k + 0] += a->dev.offset;
                aos[8 * k + 6] += a->dev.offset;
                aos[8 * k + 7] += a->dev.offset;
            }
    } else {
        std::vector<float> f((size_t)cells * 8);
        DMAP_CUDA(ctx, cudaMemcpy(f.data(), a->pyr32 + 8 * off, (size_t)cells * 32, cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < f.size(); ++k)
            aos[k] = f[k];
    }
    for (int c = 0; c < 8; ++c)
        for (int64_t k = 0; k < cells; ++k)
            out[c * cells + k] = aos[8 * k + c];
    return DMAP_OK;
}

// ---- scenes ----------------------------------------------------------------

// Non-rigid instances (dmap_scene_create_instanced): per triangle 1 + its
// instance (0: none), and the instance table (kInstDoubles each).
struct InstanceSpec
{
    const int *tri_inst = nullptr;
    std::vector<double> table;
};

// Moves the setup records of instanced triangles to world space where the
// walk reads them: the object AABB becomes the AABB of its 8 corners moved
// by the instance (widened by far more than their rounding), and the FP32
// tangent transform takes the world ray directly (A Linv, origin L q0 + T).
// The FP64 records stay in object space; the FP64 node test and the leaves
// move the ray (instance.cuh).
static void place_instances(std::vector<TriDev> &t64, std::vector<TriDev32> &t32, const InstanceSpec &spec)
{
    const int n_tri = (int)t64.size();
    for (int k = 0; k < n_tri; ++k) {
        const int inst = spec.tri_inst[k];
        if (inst <= 0)
            continue;
        const double *xf = spec.table.data() + dmapdev::kInstDoubles * (inst - 1);
        const double *L = xf, *Tr = xf + 9, *Li = xf + 12;
        TriDev &T = t64[k];
        TriDev32 &S = t32[k];
        T.inst = inst;
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int c = 0; c < 8; ++c) {
            const double p[3] = {(c & 1) ? T.box_hi[0] : T.box_lo[0], (c & 2) ? T.box_hi[1] : T.box_lo[1],
                                 (c & 4) ? T.box_hi[2] : T.box_lo[2]};
            for (int a = 0; a < 3; ++a) {
                const double w = ((L[3 * a] * p[0] + L[3 * a + 1] * p[1]) + L[3 * a + 2] * p[2]) + Tr[a];
                lo[a] = std::min(lo[a], w);
                hi[a] = std::max(hi[a], w);
            }
        }
        for (int a = 0; a < 3; ++a) {
            const double m = std::max(std::fabs(lo[a]), std::fabs(hi[a]));
            const double pad = 1e-12 * (1.0 + m);
            T.box_lo[a] = lo[a] - pad;
            T.box_hi[a] = hi[a] + pad;
            // the FP32 box as setup widens it (a few float ulps), rounded outward
            const double fpad = 4.0 * 1.1920928955078125e-7 * (1.0 + m);
            S.box_lo[a] = std::nextafter((float)(T.box_lo[a] - fpad), -INFINITY);
            S.box_hi[a] = std::nextafter((float)(T.box_hi[a] + fpad), INFINITY);
        }
        double A2[3][3], q2[3];
        for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 3; ++b)
                A2[a][b] = (T.A[a][0] * Li[b] + T.A[a][1] * Li[3 + b]) + T.A[a][2] * Li[6 + b];
            q2[a] = ((L[3 * a] * T.q0[0] + L[3 * a + 1] * T.q0[1]) + L[3 * a + 2] * T.q0[2]) + Tr[a];
        }
        for (int a = 0; a < 3; ++a) {
            S.q0[a] = q2[a];
            S.q0f[a] = (float)q2[a];
            for (int b = 0; b < 3; ++b) {
                S.A[a][b] = A2[a][b];
                S.Af[a][b] = (float)A2[a][b];
            }
        }
    }
}

static dmap_status scene_create(dmap_context *ctx, dmap_asset *const *assets, int n_assets, const int *tri_asset,
                                const double *tris, int stride, int n_tri, dmap_scene **out,
                                const InstanceSpec *inst = nullptr)
{
    if (!ctx || !assets || n_assets <= 0 || !tri_asset || !tris || n_tri <= 0 || !out)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create: bad argument");
    *out = nullptr;
    for (int k = 0; k < n_assets; ++k)
        if (!assets[k] || assets[k]->ctx != ctx)
            return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create: asset of another context");
    for (int k = 0; k < n_tri; ++k) {
        if (tri_asset[k] < 0 || tri_asset[k] >= n_assets)
            return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create: triangle asset index out of range");
        for (int q = 0; q < stride; ++q)
            if (!std::isfinite(tris[stride * (size_t)k + q]))
                return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create: non-finite triangle data");
    }
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    auto *s = new dmap_scene;
    s->ctx = ctx;
    s->n_tri = n_tri;
    s->assets.assign(assets, assets + n_assets);
    std::vector<AssetDev> ad(n_assets);
    for (int k = 0; k < n_assets; ++k) {
        ad[k] = assets[k]->dev;
        s->all_f64 = s->all_f64 && assets[k]->pyr64 != nullptr;
    }
    double *tris_dev = nullptr;
    int *ta_dev = nullptr;
    auto cleanup = [&](dmap_status st) {
        cudaFree(tris_dev);
        cudaFree(ta_dev);
        cudaFree(s->assets_dev);
        cudaFree(s->tris_dev);
        cudaFree(s->tris32_dev);
        cudaFree(s->bvh_nodes_dev);
        cudaFree(s->bvh_tri_dev);
        cudaFree(s->bvh_range_dev);
        cudaFree(s->inst_dev);
        delete s;
        return st;
    };
    cudaError_t e;
    if ((e = cudaMalloc((void **)&s->assets_dev, sizeof(AssetDev) * n_assets)) != cudaSuccess ||
        (e = cudaMalloc((void **)&s->tris_dev, sizeof(TriDev) * n_tri)) != cudaSuccess ||
        (e = cudaMalloc((void **)&s->tris32_dev, sizeof(TriDev32) * n_tri)) != cudaSuccess ||
        (e = cudaMalloc((void **)&tris_dev, sizeof(double) * stride * n_tri)) != cudaSuccess ||
        (e = cudaMalloc((void **)&ta_dev, sizeof(int) * n_tri)) != cudaSuccess)
        return cleanup(cuda_fail(ctx, e, "dmap_scene_create: cudaMalloc"));
    if ((e = cudaMemcpy(s->assets_dev, ad.data(), sizeof(AssetDev) * n_assets, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(tris_dev, tris, sizeof(double) * stride * n_tri, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(ta_dev, tri_asset, sizeof(int) * n_tri, cudaMemcpyHostToDevice)))
        return cleanup(cuda_fail(ctx, e, "dmap_scene_create: upload"));
    if ((e = dmapk::launch_setup(tris_dev, stride, ta_dev, s->assets_dev, n_tri, s->tris_dev, s->tris32_dev,
                                 ctx->status_dev, ctx->stream)) != cudaSuccess)
        return cleanup(cuda_fail(ctx, e, "dmap_scene_create: setup launch"));
    ctx->launches += 1;
    dmap_status st = sync_and_check(ctx, "dmap_scene_create");
    if (st != DMAP_OK)
        return cleanup(st);
    if (inst) {
        std::vector<TriDev> t64(n_tri);
        std::vector<TriDev32> t32(n_tri);
        if ((e = cudaMemcpy(t64.data(), s->tris_dev, sizeof(TriDev) * n_tri, cudaMemcpyDeviceToHost)) ||
            (e = cudaMemcpy(t32.data(), s->tris32_dev, sizeof(TriDev32) * n_tri, cudaMemcpyDeviceToHost)))
            return cleanup(cuda_fail(ctx, e, "dmap_scene_create_instanced: readback"));
        place_instances(t64, t32, *inst);
        if ((e = cudaMemcpy(s->tris_dev, t64.data(), sizeof(TriDev) * n_tri, cudaMemcpyHostToDevice)) ||
            (e = cudaMemcpy(s->tris32_dev, t32.data(), sizeof(TriDev32) * n_tri, cudaMemcpyHostToDevice)) ||
            (e = cudaMalloc((void **)&s->inst_dev, sizeof(double) * inst->table.size())) ||
            (e = cudaMemcpy(s->inst_dev, inst->table.data(), sizeof(double) * inst->table.size(),
                            cudaMemcpyHostToDevice)))
            return cleanup(cuda_fail(ctx, e, "dmap_scene_create_instanced: instances"));
        s->n_inst = (int)(inst->table.size() / dmapdev::kInstDoubles);
    }
    if (n_tri > 256) {
        // the triangle tree of the candidate orders (bvh.cu), over the
        // outward FP32 boxes the walk tests
        std::vector<TriDev32> t32(n_tri);
        if ((e = cudaMemcpy(t32.data(), s->tris32_dev, sizeof(TriDev32) * n_tri, cudaMemcpyDeviceToHost)))
            return cleanup(cuda_fail(ctx, e, "dmap_scene_create: readback"));
        std::vector<float> nodes, tri_box;
        std::vector<int> range;
        if (dmapk::build_bvh(t32.data(), n_tri, nodes, tri_box, range) < 0)
            return cleanup(fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create: triangle tree too deep"));
        auto upload = [&](void **dst, const void *src, size_t bytes, const char *what) -> dmap_status {
            cudaError_t er;
            if ((er = cudaMalloc(dst, bytes)) || (er = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice)))
                return cuda_fail(ctx, er, what);
            return DMAP_OK;
        };
        dmap_status us;
        if ((us = upload((void **)&s->bvh_nodes_dev, nodes.data(), sizeof(float) * nodes.size(),
                         "dmap_scene_create: triangle tree")) != DMAP_OK ||
            (us = upload((void **)&s->bvh_tri_dev, tri_box.data(), sizeof(float) * tri_box.size(),
                         "dmap_scene_create: triangle tree boxes")) != DMAP_OK ||
            (us = upload((void **)&s->bvh_range_dev, range.data(), sizeof(int) * range.size(),
                         "dmap_scene_create: triangle tree index ranges")) != DMAP_OK)
            return cleanup(us);
        s->bvh_n_nodes = (int)(nodes.size() / 16);
    }
    s->tris_host.resize(n_tri);
    if ((e = cudaMemcpy(s->tris_host.data(), s->tris_dev, sizeof(TriDev) * n_tri, cudaMemcpyDeviceToHost)))
        return cleanup(cuda_fail(ctx, e, "dmap_scene_create: readback"));
    cudaFree(tris_dev);
    cudaFree(ta_dev);
    tris_dev = nullptr;
    ta_dev = nullptr;
    *out = s;
    return DMAP_OK;
}

dmap_status dmap_scene_create(dmap_context *ctx, dmap_asset *const *assets, int n_assets, const int *tri_asset,
                              const double *tris, int n_tri, dmap_scene **out)
{
    return scene_create(ctx, assets, n_assets, tri_asset, tris, dmapk::kVertexRecord, n_tri, out);
}

dmap_status dmap_scene_create_charts(dmap_context *ctx, dmap_asset *const *assets, int n_assets,
                                     const int *tri_asset, const double *charts, int n_tri, dmap_scene **out)
{
    return scene_create(ctx, assets, n_assets, tri_asset, charts, dmapk::kChartRecord, n_tri, out);
}

dmap_status dmap_scene_create_instanced(dmap_context *ctx, dmap_asset *const *assets, int n_assets,
                                        const int *tri_asset, const double *tris, const int *object_first,
                                        int n_objects, const int *instance_object, const double *to_world,
                                        int n_instances, dmap_scene **out)
{
    if (!ctx || !tri_asset || !tris || !object_first || n_objects <= 0 || !instance_object || !to_world ||
        n_instances <= 0 || !out)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create_instanced: bad argument");
    for (int o = 0; o < n_objects; ++o)
        if (object_first[o] < 0 || object_first[o + 1] < object_first[o])
            return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create_instanced: object ranges must be ordered");
    bool rigid = true;
    for (int k = 0; k < n_instances; ++k) {
        const int o = instance_object[k];
        if (o < 0 || o >= n_objects)
            return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create_instanced: instance object out of range");
        const double *M = to_world + 12 * (size_t)k;
        for (int q = 0; q < 12; ++q)
            if (!std::isfinite(M[q]))
                return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create_instanced: non-finite transform");
        // rigid: the rotation part is orthogonal (R R^T = I within 1e-9)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                const double dot = (M[4 * a] * M[4 * b] + M[4 * a + 1] * M[4 * b + 1]) + M[4 * a + 2] * M[4 * b + 2];
                if (std::fabs(dot - (a == b ? 1.0 : 0.0)) > 1e-9)
                    rigid = false;
            }
    }
    std::vector<double> wt;
    std::vector<int> wa, wi;
    InstanceSpec spec;
    for (int k = 0; k < n_instances; ++k) {
        const int o = instance_object[k];
        const double *M = to_world + 12 * (size_t)k;
        if (!rigid) {
            // a scale or shear does not move the displaced surface with its
            // base triangles (the heights would scale): the instance keeps the
            // object's triangles and takes the rays to object space
            const double L[9] = {M[0], M[1], M[2], M[4], M[5], M[6], M[8], M[9], M[10]};
            const double c00 = L[4] * L[8] - L[5] * L[7], c01 = L[5] * L[6] - L[3] * L[8], c02 = L[3] * L[7] - L[4] * L[6];
            const double det = (L[0] * c00 + L[1] * c01) + L[2] * c02;
            double scale = 0.0;
            for (int q = 0; q < 9; ++q)
                scale = std::max(scale, std::fabs(L[q]));
            if (!(std::fabs(det) > 1e-12 * scale * scale * scale))
                return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create_instanced: singular transform");
            const double Li[9] = {c00 / det, (L[2] * L[7] - L[1] * L[8]) / det, (L[1] * L[5] - L[2] * L[4]) / det,
                                  c01 / det, (L[0] * L[8] - L[2] * L[6]) / det, (L[2] * L[3] - L[0] * L[5]) / det,
                                  c02 / det, (L[1] * L[6] - L[0] * L[7]) / det, (L[0] * L[4] - L[1] * L[3]) / det};
            spec.table.insert(spec.table.end(), L, L + 9);
            spec.table.insert(spec.table.end(), {M[3], M[7], M[11]});
            spec.table.insert(spec.table.end(), Li, Li + 9);
            spec.table.push_back(det > 0.0 ? 1.0 : -1.0);
        }
        auto point = [&](const double *p, double *q, bool translate) {
            for (int a = 0; a < 3; ++a)
                q[a] = ((M[4 * a] * p[0] + M[4 * a + 1] * p[1]) + M[4 * a + 2] * p[2]) + (translate ? M[4 * a + 3] : 0.0);
        };
        for (int t = object_first[o]; t < object_first[o + 1]; ++t) {
            const double *r = tris + 24 * (size_t)t;
            if (rigid) {
                double w[24];
                for (int v = 0; v < 3; ++v) {
                    point(r + 3 * v, w + 3 * v, true);      // p0, p1, p2
                    point(r + 9 + 3 * v, w + 9 + 3 * v, false); // m0, m1, m2
                }
                for (int q = 18; q < 24; ++q)
                    w[q] = r[q];
                wt.insert(wt.end(), w, w + 24);
            } else {
                wt.insert(wt.end(), r, r + 24);
                wi.push_back(k + 1);
            }
            wa.push_back(tri_asset[t]);
        }
    }
    if (wa.empty())
        return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_create_instanced: no triangles");
    if (rigid)
        return dmap_scene_create(ctx, assets, n_assets, wa.data(), wt.data(), (int)wa.size(), out);
    spec.tri_inst = wi.data();
    return scene_create(ctx, assets, n_assets, wa.data(), wt.data(), dmapk::kVertexRecord, (int)wa.size(), out,
                        &spec);
}

void dmap_scene_destroy(dmap_scene *s)
{
    if (!s)
        return;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    auto &gs = s->ctx->graphs;
    for (size_t k = 0; k < gs.size();) {
        if (gs[k].scene == s) {
            cudaGraphExecDestroy(gs[k].exec);
            gs.erase(gs.begin() + k);
        } else {
            ++k;
        }
    }
    cudaFree(s->assets_dev);
    cudaFree(s->tris_dev);
    cudaFree(s->tris32_dev);
    cudaFree(s->bvh_nodes_dev);
    cudaFree(s->bvh_tri_dev);
    cudaFree(s->bvh_range_dev);
    cudaFree(s->inst_dev);
    cudaFree(s->op_mask_dev);
    cudaFree(s->op_tri_dev);
    delete s;
}

dmap_status dmap_scene_set_opacity(dmap_scene *s, const uint8_t *mask_host, int w, int h, const dmap_uv_map *map,
                                   const uint8_t *tri_flags_host)
{
    if (!s)
        return DMAP_ERR_INVALID;
    dmap_context *ctx = s->ctx;
    if (mask_host && (w <= 0 || h <= 0 || (int64_t)w * h > (1ll << 30)))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_set_opacity: the mask needs 1 <= w h <= 2^30 texels");
    dmap_uv_map m = {{1.0, 1.0}, {0.0, 0.0}, 0};
    if (map)
        m = *map;
    if (mask_host && !(m.uv_scale[0] != 0.0 && m.uv_scale[1] != 0.0 && std::isfinite(m.uv_scale[0]) &&
                       std::isfinite(m.uv_scale[1]) && std::isfinite(m.uv_offset[0]) && std::isfinite(m.uv_offset[1])))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_scene_set_opacity: uv_scale must be finite and non-zero");
    // a server's queued or running requests on this scene were admitted
    // under the current filter, and its worker thread may be launching them
    if (s->server_pending.load() > 0)
        return fail(ctx, DMAP_ERR_NOT_READY,
                    "dmap_scene_set_opacity: a server still holds requests on this scene (drain it first)");
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    // queries in flight, on any stream, may read the old mask
    DMAP_CUDA(ctx, cudaDeviceSynchronize());
    cudaFree(s->op_mask_dev);
    cudaFree(s->op_tri_dev);
    s->op_mask_dev = s->op_tri_dev = nullptr;
    s->op_w = s->op_h = 0;
    if (!mask_host)
        return DMAP_OK;
    const size_t mb = (size_t)w * h, tb = tri_flags_host ? (size_t)s->n_tri : 0;
    unsigned char *md = nullptr, *td = nullptr;
    DMAP_CUDA(ctx, cudaMalloc(&md, mb));
    if (tb && cudaMalloc(&td, tb) != cudaSuccess) {
        cudaFree(md);
        return fail(ctx, DMAP_ERR_OOM, "dmap_scene_set_opacity: cudaMalloc");
    }
    if (cudaMemcpy(md, mask_host, mb, cudaMemcpyHostToDevice) != cudaSuccess ||
        (tb && cudaMemcpy(td, tri_flags_host, tb, cudaMemcpyHostToDevice) != cudaSuccess)) {
        cudaFree(md);
        cudaFree(td);
        return fail(ctx, DMAP_ERR_CUDA, "dmap_scene_set_opacity: copy");
    }
    s->op_mask_dev = md;
    s->op_tri_dev = td;
    s->op_w = w;
    s->op_h = h;
    s->op_map = m;
    return DMAP_OK;
}

int dmap_scene_triangle_count(const dmap_scene *s) { return s ? s->n_tri : 0; }

dmap_status dmap_scene_triangle_info(const dmap_scene *s, int tri, double *out)
{
    if (!s || !out || tri < 0 || tri >= s->n_tri)
        return DMAP_ERR_INVALID;
    const TriDev &T = s->tris_host[tri];
    double v[11] = {(double)T.root_level, (double)T.n_roots, T.residual_tol, T.box_lo[0], T.box_lo[1], T.box_lo[2],
                    T.box_hi[0], T.box_hi[1], T.box_hi[2], T.h_min, T.h_max};
    std::memcpy(out, v, sizeof(v));
    return DMAP_OK;
}

// ---- queries ---------------------------------------------------------------

} // extern "C"

dmap_status dmapi::check_query(dmap_scene *s, dmap_dtype ray_dtype, int64_t n, const dmap_options *opt,
                               dmap_dtype hit_dtype, dmapk::QueryOpts &q)
{
    dmap_options o;
    dmap_options_default(&o);
    if (opt)
        o = *opt;
    dmap_context *ctx = s->ctx;
    if (n < 0 || (ray_dtype != DMAP_F32 && ray_dtype != DMAP_F64) || (hit_dtype != DMAP_F32 && hit_dtype != DMAP_F64))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: rays and hits are F32 or F64");
    if (o.bound < 0 || o.bound > 2 || o.leaf < 0 || o.leaf > 1 || o.mode < 0 || o.mode > 1 || o.precision < 0 ||
        o.precision > 1)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: bad options");
    if (o.precision == DMAP_PRECISION_F64 && !s->all_f64)
        return fail(ctx, DMAP_ERR_UNSUPPORTED, "dmap_intersect: FP64 precision needs assets with DMAP_ASSET_KEEP_F64");
    if (o.precision == DMAP_PRECISION_F32 && o.leaf != DMAP_LEAF_NEWTON)
        return fail(ctx, DMAP_ERR_UNSUPPORTED, "dmap_intersect: the FP32 path has the Newton leaf only");
    q.bound = o.bound;
    q.slab_max_level = o.slab_max_level;
    q.leaf = o.leaf;
    q.mode = o.mode;
    q.polish_cond = o.polish_cond;
    q.ray_dtype = ray_dtype == DMAP_F64 ? 2 : 0;
    q.hit_dtype = hit_dtype == DMAP_F64 ? 2 : 0;
    q.precision = o.precision;
    if (o.schedule < 0 || o.schedule > 1 || o.rounds < 0 || o.rounds > dmapk::kMaxRounds || o.blocks_per_sm < 0 ||
        o.blocks_per_sm > 16)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: bad schedule options");
    if (o.order < 0 || o.order > 1)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: bad order");
    if (o.node_visit_cap < 0)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: node_visit_cap must be >= 0");
    q.order = o.order;
    q.guard_cap = o.node_visit_cap > 0 ? o.node_visit_cap : (1 << 26);
    if (o.leaf_precision != DMAP_PRECISION_F64 && o.leaf_precision != DMAP_PRECISION_F32)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: leaf_precision is DMAP_PRECISION_F64 or _F32");
    if (o.leaf_precision == DMAP_PRECISION_F32 && !(o.polish_cond >= 0.0))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_intersect: polish_cond must be >= 0");
    q.leaf_precision = o.precision == DMAP_PRECISION_F32 ? o.leaf_precision : DMAP_PRECISION_F64;
    q.schedule = o.schedule;
    q.rounds = o.rounds;
    q.blocks_per_sm = o.blocks_per_sm;
    q.bvh_nodes = reinterpret_cast<const float4 *>(s->bvh_nodes_dev);
    q.bvh_tri = reinterpret_cast<const float4 *>(s->bvh_tri_dev);
    q.bvh_range = reinterpret_cast<const int4 *>(s->bvh_range_dev);
    q.inst_xf = s->inst_dev;
    q.bvh_n_nodes = s->bvh_n_nodes;
    apply_filter(s, q);
    return DMAP_OK;
}

extern "C" {

static dmap_status run_query(dmap_scene *s, const void *rays, int64_t n, const dmapk::QueryOpts &q, void *hits,
                             int64_t *stats, cudaStream_t stream)
{
    dmap_context *ctx = s->ctx;
    cudaError_t e;
    if (q.precision == DMAP_PRECISION_F64) {
        e = dmapk::launch_walk64(s->tris_dev, s->n_tri, s->assets_dev, rays, n, q, hits, stats, ctx->status_dev,
                                 stream);
    } else {
        if (q.schedule == DMAP_SCHEDULE_WAVEFRONT && n > ctx->wave.capacity) {
            // grow the wavefront scratch to this batch (the previous one is idle
            // once the stream drains: calls on a context are serialized)
            DMAP_CUDA(ctx, cudaStreamSynchronize(stream));
            dmap_status ws = wave_reserve(ctx, ctx->wave, n);
            if (ws != DMAP_OK)
                return ws;
        }
        e = dmapk::launch_walk32(s->tris32_dev, s->tris_dev, s->n_tri, s->assets_dev, rays, n, q, hits, stats,
                                 ctx->status_dev, ctx->wave, stream);
    }
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "dmap_intersect: launch");
    if (n > 0)
        ctx->launches += q.precision == DMAP_PRECISION_F64 ? 1 : dmapk::walk32_launches(q);
    return DMAP_OK;
}

dmap_status dmap_intersect(dmap_scene *s, const void *rays_dev, dmap_dtype ray_dtype, int64_t n,
                           const dmap_options *opt, void *hits_dev, dmap_dtype hit_dtype, int64_t *stats_dev,
                           void *stream)
{
    if (!s || (n > 0 && (!rays_dev || !hits_dev)))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_intersect: null argument");
    dmapk::QueryOpts q;
    dmap_status st = check_query(s, ray_dtype, n, opt, hit_dtype, q);
    if (st != DMAP_OK)
        return st;
    DMAP_CUDA(s->ctx, cudaSetDevice(s->ctx->device));
    return run_query(s, rays_dev, n, q, hits_dev, stats_dev, stream ? (cudaStream_t)stream : s->ctx->stream);
}

// The query's launches for up to `cap` rays captured once (the count read
// from ctx->n_dev when a replay runs), or the cached graph of the same
// scene, options and capacity on the same buffers.
static dmap_status query_graph(dmap_scene *s, const dmapk::QueryOpts &q0, int64_t cap, cudaGraphExec_t *out)
{
    dmap_context *ctx = s->ctx;
    char key[256];
    snprintf(key, sizeof key, "b%d_s%d_l%d_m%d_p%.17g_r%d_h%d_sc%d_ro%d_bp%d_o%d_g%d_lp%d", q0.bound, q0.slab_max_level,
             q0.leaf, q0.mode, q0.polish_cond, q0.ray_dtype, q0.hit_dtype, q0.schedule, q0.rounds, q0.blocks_per_sm,
             q0.order, q0.guard_cap, q0.leaf_precision);
    for (auto &g : ctx->graphs)
        if (g.scene == s && g.capacity == cap && g.key == key && g.rays == ctx->rays_dev && g.hits == ctx->hits_dev &&
            g.scratch == ctx->wave.state) {
            *out = g.exec;
            return DMAP_OK;
        }
    if (!ctx->n_dev) {
        DMAP_CUDA(ctx, cudaMalloc(&ctx->n_dev, sizeof(long long)));
        DMAP_CUDA(ctx, cudaMallocHost(&ctx->n_host, sizeof(long long)));
    }
    dmapk::QueryOpts q = q0;
    q.n_dev = ctx->n_dev;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DMAP_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    const int64_t launches = ctx->launches.load();
    dmap_status st = run_query(s, ctx->rays_dev, cap, q, ctx->hits_dev, nullptr, ctx->stream);
    ctx->launches.store(launches); // counted per replay instead
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (st != DMAP_OK) {
        if (graph)
            cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "dmap_intersect_host: graph capture");
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "dmap_intersect_host: graph instantiate");
    // entries captured on buffers since replaced are dropped here
    auto &gs = ctx->graphs;
    for (size_t k = 0; k < gs.size();) {
        if (gs[k].rays != ctx->rays_dev || gs[k].hits != ctx->hits_dev || gs[k].scratch != ctx->wave.state) {
            cudaGraphExecDestroy(gs[k].exec);
            gs.erase(gs.begin() + k);
        } else {
            ++k;
        }
    }
    gs.push_back({s, key, cap, ctx->rays_dev, ctx->hits_dev, ctx->wave.state, exec});
    *out = exec;
    return DMAP_OK;
}

dmap_status dmap_intersect_host(dmap_scene *s, const void *rays_host, dmap_dtype ray_dtype, int64_t n,
                                const dmap_options *opt, void *hits_host, dmap_dtype hit_dtype, int64_t *stats_host)
{
    if (!s || (n > 0 && (!rays_host || !hits_host)))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_intersect_host: null argument");
    dmapk::QueryOpts q;
    dmap_status st = check_query(s, ray_dtype, n, opt, hit_dtype, q);
    if (st != DMAP_OK || n == 0)
        return st;
    dmap_context *ctx = s->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    // graph replay: FP32 path, no counters, no filter (whose mask may change)
    const bool graph = opt && opt->graph && q.precision == DMAP_PRECISION_F32 && !stats_host && !q.op_mask;
    int64_t cap = n;
    if (graph) {
        cap = 1024;
        while (cap < n)
            cap *= 2;
    }
    size_t rb = (size_t)n * 8 * dtype_size(ray_dtype);
    size_t hb = (size_t)n * (hit_dtype == DMAP_F64 ? sizeof(dmap_hit64) : sizeof(dmap_hit32));
    size_t sb = stats_host ? (size_t)n * DMAP_ST_COUNT * sizeof(int64_t) : 0;
    size_t rcap = (size_t)cap * 8 * dtype_size(ray_dtype);
    size_t hcap = (size_t)cap * (hit_dtype == DMAP_F64 ? sizeof(dmap_hit64) : sizeof(dmap_hit32));
    if ((st = grow(ctx, &ctx->rays_dev, &ctx->rays_cap, rcap)) != DMAP_OK ||
        (st = grow(ctx, &ctx->hits_dev, &ctx->hits_cap, hcap)) != DMAP_OK ||
        (sb && (st = grow(ctx, &ctx->stats_dev, &ctx->stats_cap, sb)) != DMAP_OK))
        return st;
    if (graph) {
        if (q.schedule == DMAP_SCHEDULE_WAVEFRONT && cap > ctx->wave.capacity) {
            // the scratch is captured into the graph: grow it before capture
            DMAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if ((st = wave_reserve(ctx, ctx->wave, cap)) != DMAP_OK)
                return st;
        }
        cudaGraphExec_t exec = nullptr;
        if ((st = query_graph(s, q, cap, &exec)) != DMAP_OK)
            return st;
        *ctx->n_host = (long long)n;
        DMAP_CUDA(ctx, cudaMemcpyAsync(ctx->n_dev, ctx->n_host, sizeof(long long), cudaMemcpyHostToDevice,
                                       ctx->stream));
        DMAP_CUDA(ctx, cudaMemcpyAsync(ctx->rays_dev, rays_host, rb, cudaMemcpyHostToDevice, ctx->stream));
        DMAP_CUDA(ctx, cudaGraphLaunch(exec, ctx->stream));
        ctx->launches += dmapk::walk32_launches(q);
    } else {
        DMAP_CUDA(ctx, cudaMemcpyAsync(ctx->rays_dev, rays_host, rb, cudaMemcpyHostToDevice, ctx->stream));
        if ((st = run_query(s, ctx->rays_dev, n, q, ctx->hits_dev, sb ? ctx->stats_dev : nullptr, ctx->stream)) !=
            DMAP_OK)
            return st;
    }
    DMAP_CUDA(ctx, cudaMemcpyAsync(hits_host, ctx->hits_dev, hb, cudaMemcpyDeviceToHost, ctx->stream));
    if (sb)
        DMAP_CUDA(ctx, cudaMemcpyAsync(stats_host, ctx->stats_dev, sb, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_and_check(ctx, "dmap_intersect_host");
}

} // extern "C"
