// Hit records to surface points (include/dmap_b200.h, dmap_surface_points):
// DisplacedGeometry::surface_point (displaced_geometry.cpp:126-152) on the
// device, one thread per hit, in double with the reference's operation
// order (compiled with -fmad=false): the displaced position, the geometric
// normal oriented along the base face's winding, the surface tangents scaled
// by the object's uv map, and the object's uv
// (DisplacedObject::object_uv, scene_spec.cpp:382-388).
#include "instance.cuh"
#include "api_internal.h"
#include "f64_math.cuh"

using namespace dmapi;

namespace
{
using namespace d64;

// Eigen's normalize(): a zero vector stays as it is.
__device__ __forceinline__ v3 eigen_normalized(v3 a)
{
    double z = dot3(a, a);
    return z > 0.0 ? div3(a, sqrt(z)) : a;
}

template <typename H>
__global__ void surface_points_kernel(const TriDev *__restrict__ tris, const AssetDev *__restrict__ assets,
                                      const H *__restrict__ hits, int64_t n, dmap_uv_map map, double *out,
                                      const double *__restrict__ inst_xf)
{
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const H h = hits[k];
    double *o = out + 14 * k;
    if (h.tri < 0) {
        for (int q = 0; q < 14; ++q)
            o[q] = 0.0;
        return;
    }
    const TriDev &T = tris[h.tri];
    const AssetDev &g = assets[T.asset];
    double u = (double)h.bary[0], v = (double)h.bary[1];
    // BaseTriangle::param (displaced_surface.h:87)
    v2 t0 = L2(T.t0), t1 = L2(T.t1), t2 = L2(T.t2);
    v2 st = add2(add2(t0, mul2(u, sub2(t1, t0))), mul2(v, sub2(t2, t0)));
    double s = st.x, t = st.y;
    nframe f = normal_frame_at(T, s, t);
    double hh;
    v2 gh;
    grid_h_grad(g, s, t, hh, gh);
    v3 Ss = add3(add3(L3(T.e1), mul3(gh.x, f.N)), mul3(hh, f.Nu));
    v3 St = add3(add3(L3(T.e2), mul3(gh.y, f.N)), mul3(hh, f.Nv));
    v3 p = add3(tri_P(T, s, t), mul3(hh, f.N));
    v3 wn = L3(T.wn);
    v3 ng = cross3(Ss, St);
    if (dot3(ng, wn) < 0.0)
        ng = V3(-ng.x, -ng.y, -ng.z);
    ng = eigen_normalized(ng);
    if (!(isfinite(ng.x) && isfinite(ng.y) && isfinite(ng.z)))
        ng = eigen_normalized(wn);
    double su = map.uv_scale[0], sv = map.flip_v ? -map.uv_scale[1] : map.uv_scale[1];
    v3 dpdu = mul3(su, Ss), dpdv = mul3(sv, St);
    if (T.inst) {
        // a non-rigid instance's point and tangents moved by its transform,
        // the normal as instance.cuh moves it
        const double *xf = inst_xf + dmapdev::kInstDoubles * (T.inst - 1), *L = xf, *Tr = xf + 9;
        auto lin = [&](v3 x) {
            return V3((L[0] * x.x + L[1] * x.y) + L[2] * x.z, (L[3] * x.x + L[4] * x.y) + L[5] * x.z,
                      (L[6] * x.x + L[7] * x.y) + L[8] * x.z);
        };
        p = add3(lin(p), V3(Tr[0], Tr[1], Tr[2]));
        dpdu = lin(dpdu);
        dpdv = lin(dpdv);
        dmapdev::world_normal(xf, ng);
    }
    double uvx = (s - map.uv_offset[0]) / map.uv_scale[0], uvy = (t - map.uv_offset[1]) / map.uv_scale[1];
    if (map.flip_v)
        uvy = 1.0 - uvy;
    double r[14] = {p.x, p.y, p.z, ng.x, ng.y, ng.z, dpdu.x, dpdu.y, dpdu.z, dpdv.x, dpdv.y, dpdv.z, uvx, uvy};
    for (int q = 0; q < 14; ++q)
        o[q] = r[q];
}

} // namespace

extern "C" {

dmap_status dmap_surface_points(dmap_scene *s, const void *hits_dev, dmap_dtype hit_dtype, int64_t n,
                                const dmap_uv_map *map, double *out_dev, void *stream)
{
    if (!s || n < 0 || (n > 0 && (!hits_dev || !out_dev)) || (hit_dtype != DMAP_F32 && hit_dtype != DMAP_F64))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_surface_points: bad argument");
    dmap_uv_map m = {{1.0, 1.0}, {0.0, 0.0}, 0};
    if (map)
        m = *map;
    if (!(m.uv_scale[0] != 0.0 && m.uv_scale[1] != 0.0))
        return fail(s->ctx, DMAP_ERR_INVALID, "dmap_surface_points: uv_scale must be non-zero");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = s->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    unsigned grid = (unsigned)((n + 127) / 128);
    if (hit_dtype == DMAP_F64)
        surface_points_kernel<dmapdev::Hit64><<<grid, 128, 0, st>>>(
            s->tris_dev, s->assets_dev, static_cast<const dmapdev::Hit64 *>(hits_dev), n, m, out_dev, s->inst_dev);
    else
        surface_points_kernel<dmapdev::Hit32><<<grid, 128, 0, st>>>(
            s->tris_dev, s->assets_dev, static_cast<const dmapdev::Hit32 *>(hits_dev), n, m, out_dev, s->inst_dev);
    DMAP_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return DMAP_OK;
}

dmap_status dmap_surface_points_host(dmap_scene *s, const void *hits_host, dmap_dtype hit_dtype, int64_t n,
                                     const dmap_uv_map *map, double *out_host)
{
    if (!s || n < 0 || (n > 0 && (!hits_host || !out_host)))
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_surface_points_host: null argument");
    if (n == 0)
        return DMAP_OK;
    dmap_context *ctx = s->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t hb = (size_t)n * (hit_dtype == DMAP_F64 ? sizeof(dmap_hit64) : sizeof(dmap_hit32));
    size_t ob = (size_t)n * 14 * sizeof(double);
    dmap_status st;
    if ((st = grow(ctx, &ctx->hits_dev, &ctx->hits_cap, hb)) != DMAP_OK ||
        (st = grow(ctx, &ctx->rays_dev, &ctx->rays_cap, ob)) != DMAP_OK)
        return st;
    DMAP_CUDA(ctx, cudaMemcpyAsync(ctx->hits_dev, hits_host, hb, cudaMemcpyHostToDevice, ctx->stream));
    if ((st = dmap_surface_points(s, ctx->hits_dev, hit_dtype, n, map, static_cast<double *>(ctx->rays_dev),
                                  ctx->stream)) != DMAP_OK)
        return st;
    DMAP_CUDA(ctx, cudaMemcpyAsync(out_host, ctx->rays_dev, ob, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_and_check(ctx, "dmap_surface_points_host");
}

} // extern "C"
