// The batched path tracer of include/dmap_b200.h (dmap_render): wavefront
// stages as kernels (camera rays; shading with next-event estimation and the
// diffuse bounce; shadow accumulation; per-pixel resolve) around the FP32
// query path, one batch of whole image samples at a time. Every count a
// stage produces stays on the device (the queries read theirs through
// QueryOpts::n_dev), so a batch's launches can be captured once in a CUDA
// graph and replayed for every batch.
#include "api_internal.h"

using namespace dmapi;

namespace
{

constexpr float kSpawnEps = 1e-4f;  // new rays start this far off the surface, along the normal
constexpr float kShadowEps = 1e-4f; // shadow rays end this far before the light sample (direct_lighting.cpp:50)
constexpr float kInvPi = 0.318309886183790671538f;
constexpr int kMaxDepth = 16;

struct RenderDev
{
    float eye[3], fwd[3], right[3], up[3];
    float tan_half, aspect;
    float ep0[3], ee1[3], ee2[3], en[3], Le[3], area, inv_e1, inv_e2;
    float albedo[3];
    int W, H, spp, max_depth, rr_depth, s_batch;
    long long P; // paths per batch: s_batch x W x H
    unsigned long long seed;
    const long long *p0; // first global path of the batch that runs (device)
};

// The path's random numbers: splitmix64 (Steele, Lea and Flood, "Fast
// splittable pseudorandom number generators", 2014) of the seed, the global
// path index, the vertex and the dimension.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ float rnd(const RenderDev &R, long long g, int vertex, int dim)
{
    unsigned long long z = mix64(R.seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(g + 1));
    z = mix64(z ^ (0x9E3779B97F4A7C15ull * (unsigned long long)(vertex * 16 + dim + 1)));
    return (float)(z >> 40) * 0x1.0p-24f;
}

__device__ __forceinline__ float dot3f(const float *a, const float *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__device__ __forceinline__ void put_ray(float *r, const float *o, const float *d, float t0, float t1)
{
    float4 *q = reinterpret_cast<float4 *>(r);
    q[0] = make_float4(o[0], o[1], o[2], d[0]);
    q[1] = make_float4(d[1], d[2], t0, t1);
}

__device__ __forceinline__ long long batch_paths(const RenderDev &R)
{
    long long total = (long long)R.W * R.H * R.spp, left = total - *R.p0;
    return left < R.P ? (left > 0 ? left : 0) : R.P;
}

// Depth-0 extension rays: a pinhole camera, jittered within the pixel.
__global__ void camera_kernel(RenderDev R, float *ray, int *path, float *beta, float *Lp, long long *cnt)
{
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long n = batch_paths(R);
    if (k == 0)
        cnt[0] = n;
    if (k >= n)
        return;
    long long g = *R.p0 + k;
    int pix = (int)(g % ((long long)R.W * R.H));
    int x = pix % R.W, y = pix / R.W;
    float sx = (2.0f * ((float)x + rnd(R, g, 0, 0)) / (float)R.W - 1.0f) * R.tan_half * R.aspect;
    float sy = (1.0f - 2.0f * ((float)y + rnd(R, g, 0, 1)) / (float)R.H) * R.tan_half;
    float d[3];
    for (int a = 0; a < 3; ++a)
        d[a] = R.fwd[a] + sx * R.right[a] + sy * R.up[a];
    float inv = rsqrtf(dot3f(d, d));
    for (int a = 0; a < 3; ++a)
        d[a] *= inv;
    put_ray(ray + 8 * k, R.eye, d, 0.0f, INFINITY);
    path[k] = (int)k;
    for (int c = 0; c < 3; ++c) {
        beta[3 * k + c] = 1.0f;
        Lp[3 * k + c] = 0.0f;
    }
}

// One path vertex per extension ray: the emitter seen directly, else the
// surface hit: a shadow ray toward a uniform sample of the emitter (its
// contribution held until the occlusion query answers) and the cosine-
// weighted bounce with Russian roulette.
__global__ void shade_kernel(RenderDev R, int v, const float *__restrict__ ray_in, const int *__restrict__ path_in,
                             const dmapdev::Hit32 *__restrict__ hit, long long *cnt, float *beta, float *Lp,
                             float *ray_out, int *path_out, float *srays, int *spath, float *scontrib)
{
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cnt[v])
        return;
    int p = path_in[k];
    long long g = *R.p0 + p;
    const float *r = ray_in + 8 * k;
    float o[3] = {r[0], r[1], r[2]}, d[3] = {r[3], r[4], r[5]};
    const dmapdev::Hit32 h = hit[k];
    float t = h.tri >= 0 ? h.t : INFINITY;
    float dn = dot3f(d, R.en);
    if (dn < 0.0f) {
        float w0[3] = {R.ep0[0] - o[0], R.ep0[1] - o[1], R.ep0[2] - o[2]};
        float te = dot3f(w0, R.en) / dn;
        if (te > 0.0f && te < t) {
            float q[3];
            for (int a = 0; a < 3; ++a)
                q[a] = o[a] + te * d[a] - R.ep0[a];
            float ua = dot3f(q, R.ee1) * R.inv_e1, ub = dot3f(q, R.ee2) * R.inv_e2;
            if (ua >= 0.0f && ua <= 1.0f && ub >= 0.0f && ub <= 1.0f) {
                if (v == 0)
                    for (int c = 0; c < 3; ++c)
                        Lp[3 * p + c] += beta[3 * p + c] * R.Le[c];
                return;
            }
        }
    }
    if (h.tri < 0)
        return;
    float n[3] = {h.ng[0], h.ng[1], h.ng[2]};
    if (dot3f(n, d) > 0.0f)
        for (int a = 0; a < 3; ++a)
            n[a] = -n[a];
    float xo[3];
    for (int a = 0; a < 3; ++a)
        xo[a] = o[a] + t * d[a] + kSpawnEps * n[a];
    float b[3] = {beta[3 * p], beta[3 * p + 1], beta[3 * p + 2]};

    // next-event estimation: one uniform point of the emitter
    float ua = rnd(R, g, v, 2), ub = rnd(R, g, v, 3), wv[3];
    for (int a = 0; a < 3; ++a)
        wv[a] = R.ep0[a] + ua * R.ee1[a] + ub * R.ee2[a] - xo[a];
    float d2 = dot3f(wv, wv), dist = sqrtf(d2), wi[3];
    for (int a = 0; a < 3; ++a)
        wi[a] = wv[a] / dist;
    float cs = dot3f(n, wi), cl = -dot3f(R.en, wi);
    if (cs > 0.0f && cl > 0.0f && dist > 2.0f * kShadowEps) {
        float f = cs * cl * R.area / d2 * kInvPi;
        unsigned long long slot = atomicAdd(reinterpret_cast<unsigned long long *>(cnt + R.max_depth + v), 1ull);
        put_ray(srays + 8 * slot, xo, wi, 0.0f, dist - kShadowEps);
        spath[slot] = p;
        for (int c = 0; c < 3; ++c)
            scontrib[3 * slot + c] = b[c] * R.albedo[c] * R.Le[c] * f;
    }

    // the diffuse bounce
    if (v + 1 >= R.max_depth)
        return;
    float nb[3] = {b[0] * R.albedo[0], b[1] * R.albedo[1], b[2] * R.albedo[2]};
    if (v + 1 >= R.rr_depth) {
        float q = fminf(fmaxf(fmaxf(nb[0], fmaxf(nb[1], nb[2])), 0.05f), 0.95f);
        if (rnd(R, g, v, 4) >= q)
            return;
        for (int c = 0; c < 3; ++c)
            nb[c] /= q;
    }
    float u1 = rnd(R, g, v, 5), u2 = rnd(R, g, v, 6);
    float rr = sqrtf(u1), phi = 6.283185307179586f * u2, sp, cp;
    sincosf(phi, &sp, &cp);
    float lz = sqrtf(fmaxf(0.0f, 1.0f - u1));
    float ax[3] = {fabsf(n[0]) < 0.9f ? 1.0f : 0.0f, fabsf(n[0]) < 0.9f ? 0.0f : 1.0f, 0.0f};
    float t1[3] = {ax[1] * n[2] - ax[2] * n[1], ax[2] * n[0] - ax[0] * n[2], ax[0] * n[1] - ax[1] * n[0]};
    float il = rsqrtf(dot3f(t1, t1));
    for (int a = 0; a < 3; ++a)
        t1[a] *= il;
    float t2[3] = {n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0]};
    float wo[3];
    for (int a = 0; a < 3; ++a)
        wo[a] = rr * cp * t1[a] + rr * sp * t2[a] + lz * n[a];
    for (int c = 0; c < 3; ++c)
        beta[3 * p + c] = nb[c];
    unsigned long long slot = atomicAdd(reinterpret_cast<unsigned long long *>(cnt + v + 1), 1ull);
    put_ray(ray_out + 8 * slot, xo, wo, 0.0f, INFINITY);
    path_out[slot] = p;
}

// Unoccluded shadow rays add their contribution (one shadow ray per path and
// vertex: no two threads touch a path).
__global__ void shadow_kernel(RenderDev R, int v, const long long *cnt, const dmapdev::Hit32 *__restrict__ shit,
                              const int *__restrict__ spath, const float *__restrict__ scontrib, float *Lp)
{
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cnt[R.max_depth + v] || shit[k].tri >= 0)
        return;
    int p = spath[k];
    for (int c = 0; c < 3; ++c)
        Lp[3 * p + c] += scontrib[3 * k + c];
}

// Per pixel, the batch's samples in sample order (the image does not depend
// on the batching or on the order queries finish in).
__global__ void resolve_kernel(RenderDev R, const float *__restrict__ Lp, float *accum)
{
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long wh = (long long)R.W * R.H;
    if (q >= wh)
        return;
    long long n = batch_paths(R);
    float s[3] = {accum[3 * q], accum[3 * q + 1], accum[3 * q + 2]};
    for (long long k = q; k < n; k += wh)
        for (int c = 0; c < 3; ++c)
            s[c] += Lp[3 * k + c];
    for (int c = 0; c < 3; ++c)
        accum[3 * q + c] = s[c];
}

// Batch totals of the queries issued, then the next batch's first path.
__global__ void advance_kernel(RenderDev R, const long long *cnt, long long *p0, unsigned long long *totals)
{
    long long n = batch_paths(R);
    unsigned long long e = 0, s = 0;
    for (int v = 0; v < R.max_depth; ++v) {
        e += (unsigned long long)cnt[v];
        s += (unsigned long long)cnt[R.max_depth + v];
    }
    totals[0] += (unsigned long long)n;
    totals[1] += e;
    totals[2] += s;
    *p0 += R.P;
}

// Appends a stage's queries and answers to the record.
__global__ void record_kernel(int kind, const long long *count, const float *__restrict__ rays,
                              const dmapdev::Hit32 *__restrict__ hits, unsigned long long *rec_n, long long cap,
                              float *rr, int *rk, int *rt, float *rtv)
{
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= *count)
        return;
    unsigned long long slot = atomicAdd(rec_n, 1ull);
    if ((long long)slot >= cap)
        return;
    for (int a = 0; a < 8; ++a)
        rr[8 * slot + a] = rays[8 * k + a];
    rk[slot] = kind;
    rt[slot] = hits[k].tri;
    rtv[slot] = hits[k].t;
}

void normalize3(double *v)
{
    double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int a = 0; a < 3; ++a)
        v[a] /= l;
}

void cross3(const double *a, const double *b, double *c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

bool finite_n(const double *v, int n)
{
    for (int k = 0; k < n; ++k)
        if (!std::isfinite(v[k]))
            return false;
    return true;
}

} // namespace

namespace dmapi
{

// One render in progress: its parameters, device buffers, the captured
// batch graph and the count of batches enqueued.
struct RenderJob
{
    dmap_context *ctx = nullptr;
    dmap_scene *scene = nullptr;
    dmapk::QueryOpts q{};
    RenderDev R{};
    int spp = 0, n_batches = 0, enqueued = 0;
    bool use_graph = false;
    long long P = 0, wh = 0, cap = 0;
    int64_t launches_per_batch = 0;
    size_t bytes = 0;
    // device buffers
    float *ray[2] = {nullptr, nullptr};
    int *path[2] = {nullptr, nullptr};
    dmapdev::Hit32 *hit = nullptr, *shit = nullptr;
    float *beta = nullptr, *Lp = nullptr, *srays = nullptr, *scontrib = nullptr, *accum = nullptr;
    int *spath = nullptr;
    long long *cnt = nullptr, *p0 = nullptr;
    unsigned long long *totals = nullptr, *rec_n = nullptr;
    float *rec_rays = nullptr, *rec_t = nullptr;
    int *rec_kind = nullptr, *rec_tri = nullptr;
    dmapk::WaveScratch wave;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    // Device memory is stream-ordered (cudaMallocAsync on the stream begin
    // was given, cudaFreeAsync here), so that jobs come and go while other
    // streams' kernels run; the caller makes sure none of the job's work is
    // still in flight.
    void release(cudaStream_t stream)
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        void *all[] = {ray[0], ray[1], path[0], path[1], hit, shit, beta, Lp, srays, scontrib, accum, spath,
                       cnt, p0, totals, rec_n, rec_rays, rec_t, rec_kind, rec_tri,
                       wave.state, wave.queue[0], wave.queue[1], wave.leaves, wave.counters, wave.rerun};
        for (void *p : all)
            if (p)
                cudaFreeAsync(p, stream);
        wave = dmapk::WaveScratch{};
    }

    // One batch's stages on `stream`.
    cudaError_t enqueue_stages(cudaStream_t stream)
    {
        cudaError_t err;
        int64_t lc = 0;
        const unsigned g = (unsigned)((P + 255) / 256);
        dmap_scene *s = scene;
        if ((err = cudaMemsetAsync(cnt, 0, sizeof(long long) * 2 * kMaxDepth, stream)) != cudaSuccess)
            return err;
        camera_kernel<<<g, 256, 0, stream>>>(R, ray[0], path[0], beta, Lp, cnt);
        ++lc;
        for (int v = 0; v < R.max_depth; ++v) {
            dmapk::QueryOpts qe = q, qs = q;
            qe.mode = DMAP_MODE_CLOSEST;
            qe.ray_dtype = qe.hit_dtype = 0;
            qe.n_dev = cnt + v;
            if ((err = dmapk::launch_walk32(s->tris32_dev, s->tris_dev, s->n_tri, s->assets_dev, ray[v & 1], P, qe,
                                            hit, nullptr, ctx->status_dev, wave, stream)) != cudaSuccess)
                return err;
            lc += dmapk::walk32_launches(qe);
            if (cap > 0) {
                record_kernel<<<g, 256, 0, stream>>>(0, cnt + v, ray[v & 1], hit, rec_n, cap, rec_rays, rec_kind,
                                                     rec_tri, rec_t);
                ++lc;
            }
            shade_kernel<<<g, 256, 0, stream>>>(R, v, ray[v & 1], path[v & 1], hit, cnt, beta, Lp, ray[(v + 1) & 1],
                                                path[(v + 1) & 1], srays, spath, scontrib);
            ++lc;
            qs.mode = DMAP_MODE_OCCLUDED;
            qs.ray_dtype = qs.hit_dtype = 0;
            qs.n_dev = cnt + R.max_depth + v;
            if ((err = dmapk::launch_walk32(s->tris32_dev, s->tris_dev, s->n_tri, s->assets_dev, srays, P, qs, shit,
                                            nullptr, ctx->status_dev, wave, stream)) != cudaSuccess)
                return err;
            lc += dmapk::walk32_launches(qs);
            if (cap > 0) {
                record_kernel<<<g, 256, 0, stream>>>(1, cnt + R.max_depth + v, srays, shit, rec_n, cap, rec_rays,
                                                     rec_kind, rec_tri, rec_t);
                ++lc;
            }
            shadow_kernel<<<g, 256, 0, stream>>>(R, v, cnt, shit, spath, scontrib, Lp);
            ++lc;
        }
        resolve_kernel<<<(unsigned)((wh + 255) / 256), 256, 0, stream>>>(R, Lp, accum);
        advance_kernel<<<1, 1, 0, stream>>>(R, cnt, p0, totals);
        lc += 2;
        launches_per_batch = lc;
        return cudaGetLastError();
    }
};

size_t render_device_bytes(const dmap_render_desc *desc, int64_t record_capacity)
{
    const dmap_camera &C = desc->camera;
    long long wh = (long long)C.width * C.height;
    long long ppb = desc->paths_per_batch > 0 ? desc->paths_per_batch : (4ll << 20);
    long long s_batch = std::max(1ll, std::min((long long)desc->spp, ppb / std::max(1ll, wh)));
    long long P = s_batch * wh;
    size_t per_path = 2 * (32 + 4) + 2 * sizeof(dmapdev::Hit32) + 12 + 12 + 32 + 12 + 4;
    return (size_t)P * per_path + wave_bytes(P) + (size_t)wh * 12 +
           (size_t)std::max<int64_t>(record_capacity, 0) * 44 + 4096;
}

dmap_status render_begin(dmap_scene *s, const dmap_render_desc *desc, const dmap_options *opt,
                         const dmap_ray_record *record, cudaStream_t stream, RenderJob **out)
{
    *out = nullptr;
    if (!s || !desc)
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_render: null argument");
    dmap_context *ctx = s->ctx;
    const dmap_render_desc &D = *desc;
    const dmap_camera &C = D.camera;
    if (C.width <= 0 || C.height <= 0 || (int64_t)C.width * C.height > (1ll << 28) || D.spp <= 0 ||
        D.max_depth < 1 || D.max_depth > kMaxDepth || D.rr_depth < 1 || !(C.fov_deg > 0.0 && C.fov_deg < 180.0) ||
        D.paths_per_batch < 0)
        return fail(ctx, DMAP_ERR_INVALID, "dmap_render: bad image, depth or camera parameters");
    if (!finite_n(C.eye, 3) || !finite_n(C.target, 3) || !finite_n(C.up, 3) || !finite_n(D.emitter_p0, 3) ||
        !finite_n(D.emitter_e1, 3) || !finite_n(D.emitter_e2, 3) || !finite_n(D.radiance, 3) || !finite_n(D.albedo, 3))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_render: non-finite camera, emitter or material");
    if (record && record->capacity > 0 && (!record->rays || !record->kind || !record->tri || !record->t))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_render: record buffers missing");
    dmapk::QueryOpts q;
    dmap_status st = check_query(s, DMAP_F32, 0, opt, DMAP_F32, q);
    if (st != DMAP_OK)
        return st;
    if (q.precision != DMAP_PRECISION_F32)
        return fail(ctx, DMAP_ERR_UNSUPPORTED, "dmap_render: the path tracer runs the FP32 query path");

    // camera frame and emitter
    RenderDev R{};
    double f[3] = {C.target[0] - C.eye[0], C.target[1] - C.eye[1], C.target[2] - C.eye[2]}, rt[3], up[3];
    normalize3(f);
    cross3(f, C.up, rt);
    normalize3(rt);
    cross3(rt, f, up);
    double en[3];
    cross3(D.emitter_e1, D.emitter_e2, en);
    double area = std::sqrt(en[0] * en[0] + en[1] * en[1] + en[2] * en[2]);
    double l1 = D.emitter_e1[0] * D.emitter_e1[0] + D.emitter_e1[1] * D.emitter_e1[1] + D.emitter_e1[2] * D.emitter_e1[2];
    double l2 = D.emitter_e2[0] * D.emitter_e2[0] + D.emitter_e2[1] * D.emitter_e2[1] + D.emitter_e2[2] * D.emitter_e2[2];
    if (!(area > 0.0) || !std::isfinite(f[0] + rt[0]))
        return fail(ctx, DMAP_ERR_INVALID, "dmap_render: degenerate camera or emitter");
    for (int a = 0; a < 3; ++a) {
        R.eye[a] = (float)C.eye[a];
        R.fwd[a] = (float)f[a];
        R.right[a] = (float)rt[a];
        R.up[a] = (float)up[a];
        R.ep0[a] = (float)D.emitter_p0[a];
        R.ee1[a] = (float)D.emitter_e1[a];
        R.ee2[a] = (float)D.emitter_e2[a];
        R.en[a] = (float)(en[a] / area);
        R.Le[a] = (float)D.radiance[a];
        R.albedo[a] = (float)D.albedo[a];
    }
    R.area = (float)area;
    R.inv_e1 = (float)(1.0 / l1);
    R.inv_e2 = (float)(1.0 / l2);
    R.tan_half = (float)std::tan(0.5 * C.fov_deg * 3.14159265358979323846 / 180.0);
    R.aspect = (float)C.width / (float)C.height;
    R.W = C.width;
    R.H = C.height;
    R.spp = D.spp;
    R.max_depth = D.max_depth;
    R.rr_depth = D.rr_depth;
    R.seed = D.seed;
    const long long wh = (long long)C.width * C.height;
    long long ppb = D.paths_per_batch > 0 ? D.paths_per_batch : (4ll << 20);
    R.s_batch = (int)std::max(1ll, std::min((long long)D.spp, ppb / wh));
    R.P = (long long)R.s_batch * wh;

    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    auto *J = new RenderJob;
    J->ctx = ctx;
    J->scene = s;
    J->q = q;
    J->spp = D.spp;
    J->P = R.P;
    J->wh = wh;
    J->n_batches = (D.spp + R.s_batch - 1) / R.s_batch;
    J->use_graph = D.use_graph != 0;
    J->cap = record ? std::max<int64_t>(record->capacity, 0) : 0;
    J->bytes = render_device_bytes(desc, J->cap);
    const long long P = R.P, cap = J->cap;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess)
            e = cudaMallocAsync(p, bytes, stream);
    };
    for (int k = 0; k < 2; ++k) {
        alloc((void **)&J->ray[k], sizeof(float) * 8 * P);
        alloc((void **)&J->path[k], sizeof(int) * P);
    }
    alloc((void **)&J->hit, sizeof(dmapdev::Hit32) * P);
    alloc((void **)&J->shit, sizeof(dmapdev::Hit32) * P);
    alloc((void **)&J->beta, sizeof(float) * 3 * P);
    alloc((void **)&J->Lp, sizeof(float) * 3 * P);
    alloc((void **)&J->srays, sizeof(float) * 8 * P);
    alloc((void **)&J->scontrib, sizeof(float) * 3 * P);
    alloc((void **)&J->spath, sizeof(int) * P);
    alloc((void **)&J->accum, sizeof(float) * 3 * wh);
    alloc((void **)&J->cnt, sizeof(long long) * 2 * kMaxDepth);
    alloc((void **)&J->p0, sizeof(long long));
    alloc((void **)&J->totals, sizeof(unsigned long long) * 4);
    if (cap > 0) {
        alloc((void **)&J->rec_n, sizeof(unsigned long long));
        alloc((void **)&J->rec_rays, sizeof(float) * 8 * cap);
        alloc((void **)&J->rec_t, sizeof(float) * cap);
        alloc((void **)&J->rec_kind, sizeof(int) * cap);
        alloc((void **)&J->rec_tri, sizeof(int) * cap);
    }
    alloc(&J->wave.state, dmapk::wave_state_bytes() * P);
    alloc((void **)&J->wave.queue[0], sizeof(int) * P);
    alloc((void **)&J->wave.queue[1], sizeof(int) * P);
    alloc(&J->wave.leaves, dmapk::wave_leaf_bytes() * P);
    alloc((void **)&J->wave.counters, sizeof(unsigned long long) * dmapk::kWaveCounters);
    alloc((void **)&J->wave.rerun, sizeof(int) * P);
    J->wave.capacity = P;
    if (e != cudaSuccess) {
        J->release(stream);
        delete J;
        return cuda_fail(ctx, e, "dmap_render: cudaMallocAsync");
    }
    R.p0 = J->p0;
    J->R = R;
    if ((e = cudaMemsetAsync(J->p0, 0, sizeof(long long), stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(J->accum, 0, sizeof(float) * 3 * wh, stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(J->totals, 0, sizeof(unsigned long long) * 4, stream)) != cudaSuccess ||
        (cap > 0 && (e = cudaMemsetAsync(J->rec_n, 0, sizeof(unsigned long long), stream)) != cudaSuccess)) {
        J->release(stream);
        delete J;
        return cuda_fail(ctx, e, "dmap_render: clear");
    }
    if (J->use_graph) {
        // capture one batch's stages once; each replay runs the next batch
        cudaError_t eq = cudaSuccess;
        if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed)) == cudaSuccess) {
            eq = J->enqueue_stages(stream);
            e = cudaStreamEndCapture(stream, &J->graph);
        }
        if (eq != cudaSuccess || e != cudaSuccess ||
            (e = cudaGraphInstantiate(&J->exec, J->graph, 0)) != cudaSuccess) {
            J->release(stream);
            delete J;
            return cuda_fail(ctx, eq != cudaSuccess ? eq : e, "dmap_render: graph capture");
        }
    } else {
        J->launches_per_batch = 0;
    }
    *out = J;
    return DMAP_OK;
}

int render_batches(const RenderJob *J) { return J->n_batches; }
int render_enqueued(const RenderJob *J) { return J->enqueued; }
size_t render_bytes(const RenderJob *J) { return J->bytes; }

cudaError_t render_enqueue_batch(RenderJob *J, cudaStream_t stream)
{
    if (J->enqueued >= J->n_batches)
        return cudaSuccess;
    cudaError_t e = J->use_graph ? cudaGraphLaunch(J->exec, stream) : J->enqueue_stages(stream);
    if (e == cudaSuccess) {
        ++J->enqueued;
        J->ctx->launches += J->launches_per_batch;
    }
    return e;
}

dmap_status render_end(RenderJob *J, float *rgb_host, dmap_render_stats *stats, dmap_ray_record *record,
                       double device_ms)
{
    dmap_context *ctx = J->ctx;
    std::vector<float> acc((size_t)3 * J->wh);
    unsigned long long tot[4] = {0, 0, 0, 0};
    DMAP_CUDA(ctx, cudaMemcpy(acc.data(), J->accum, sizeof(float) * 3 * J->wh, cudaMemcpyDeviceToHost));
    DMAP_CUDA(ctx, cudaMemcpy(tot, J->totals, sizeof(tot), cudaMemcpyDeviceToHost));
    const float inv_spp = 1.0f / (float)J->spp;
    if (rgb_host)
        for (size_t k = 0; k < acc.size(); ++k)
            rgb_host[k] = acc[k] * inv_spp;
    if (stats) {
        stats->paths = (int64_t)tot[0];
        stats->extension_rays = (int64_t)tot[1];
        stats->shadow_rays = (int64_t)tot[2];
        stats->batches = J->n_batches;
        stats->kernel_launches = J->launches_per_batch * J->n_batches;
        stats->device_ms = device_ms;
    }
    if (record) {
        record->count = (int64_t)(tot[1] + tot[2]);
        if (J->cap > 0) {
            unsigned long long rn = 0;
            DMAP_CUDA(ctx, cudaMemcpy(&rn, J->rec_n, sizeof(rn), cudaMemcpyDeviceToHost));
            record->count = (int64_t)rn;
            size_t m = (size_t)std::min<long long>((long long)rn, J->cap);
            DMAP_CUDA(ctx, cudaMemcpy(record->rays, J->rec_rays, sizeof(float) * 8 * m, cudaMemcpyDeviceToHost));
            DMAP_CUDA(ctx, cudaMemcpy(record->kind, J->rec_kind, sizeof(int) * m, cudaMemcpyDeviceToHost));
            DMAP_CUDA(ctx, cudaMemcpy(record->tri, J->rec_tri, sizeof(int) * m, cudaMemcpyDeviceToHost));
            DMAP_CUDA(ctx, cudaMemcpy(record->t, J->rec_t, sizeof(float) * m, cudaMemcpyDeviceToHost));
        }
    }
    return DMAP_OK;
}

void render_free(RenderJob *J, cudaStream_t stream)
{
    J->release(stream);
    delete J;
}

} // namespace dmapi

extern "C" dmap_status dmap_render(dmap_scene *s, const dmap_render_desc *desc, const dmap_options *opt,
                                   float *rgb_host, dmap_render_stats *stats, dmap_ray_record *record)
{
    if (!s || !desc || !rgb_host)
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_render: null argument");
    dmap_context *ctx = s->ctx;
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t stream = ctx->stream;
    RenderJob *J = nullptr;
    dmap_status st = render_begin(s, desc, opt, record, stream, &J);
    if (st != DMAP_OK)
        return st;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaError_t e;
    if ((e = cudaEventCreate(&ev0)) != cudaSuccess || (e = cudaEventCreate(&ev1)) != cudaSuccess) {
        render_free(J, stream);
        return cuda_fail(ctx, e, "dmap_render: events");
    }
    cudaEventRecord(ev0, stream);
    for (int b = 0; b < J->n_batches && e == cudaSuccess; ++b)
        e = render_enqueue_batch(J, stream);
    cudaEventRecord(ev1, stream);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(stream);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        render_free(J, stream);
        return cuda_fail(ctx, e, "dmap_render: batch launch");
    }
    st = sync_and_check(ctx, "dmap_render");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (st == DMAP_OK)
        st = render_end(J, rgb_host, stats, record, ms);
    render_free(J, stream);
    cudaStreamSynchronize(stream);
    return st;
}
