// The schedule autotuner of include/dmap_b200.h (dmap_autotune): times the
// wavefront schedule's launch shapes on a sample of the caller's own rays
// and keeps the fastest, optionally remembered in a text cache keyed by the
// scene and query shape.
#include "api_internal.h"

#include <algorithm>
#include <fstream>
#include <iomanip>
#include <sstream>

using namespace dmapi;

namespace
{

// The scene and query shape a tuning result applies to.
std::string tune_key(const dmap_scene *s, const dmapk::QueryOpts &q, int64_t n)
{
    int64_t texels = 0;
    int dtypes = 0;
    for (const dmap_asset *a : s->assets) {
        texels += (int64_t)a->dev.n_leaf * a->dev.n_leaf;
        dtypes |= 1 << a->dev.dtype;
    }
    int log2n = 0;
    while ((int64_t(1) << (log2n + 1)) <= n)
        ++log2n;
    std::ostringstream k;
    k << "tri" << s->n_tri << "_assets" << s->assets.size() << "_texels" << texels << "_dt" << dtypes << "_mode"
      << q.mode << "_bound" << q.bound << "_slab" << q.slab_max_level << "_order" << q.order << "_leaf"
      << q.leaf_precision << "_n2^" << log2n;
    return k.str();
}

bool cache_lookup(const char *path, const std::string &key, int &rounds, int &bps, double &ms)
{
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) { // the last entry of a key wins
        std::istringstream in(line);
        std::string k;
        int r, b;
        double t;
        if (in >> k >> r >> b >> t && k == key) {
            rounds = r;
            bps = b;
            ms = t;
            found = true;
        }
    }
    return found;
}

} // namespace

extern "C" dmap_status dmap_autotune(dmap_scene *s, const void *rays_dev, dmap_dtype ray_dtype, int64_t n,
                                     const dmap_options *base, const char *cache_path, dmap_options *best,
                                     double *best_ms)
{
    if (!s || !rays_dev || n <= 0 || !best)
        return fail(s ? s->ctx : nullptr, DMAP_ERR_INVALID, "dmap_autotune: bad argument");
    dmap_context *ctx = s->ctx;
    dmap_options o;
    dmap_options_default(&o);
    if (base)
        o = *base;
    o.schedule = DMAP_SCHEDULE_WAVEFRONT;
    dmapk::QueryOpts q;
    dmap_status st = check_query(s, ray_dtype, n, &o, DMAP_F32, q);
    if (st != DMAP_OK)
        return st;
    if (q.precision != DMAP_PRECISION_F32)
        return fail(ctx, DMAP_ERR_UNSUPPORTED, "dmap_autotune: the wavefront schedule is on the FP32 path");
    // the sample: the first rays, the whole batch up to 4M (the best shape
    // depends on how many rays are in flight, so a small prefix of a large
    // batch misleads)
    const int64_t m = std::min<int64_t>(n, 4 << 20);
    const std::string key = tune_key(s, q, m);
    int r_best = o.rounds, b_best = o.blocks_per_sm;
    double t_best = 0.0;
    if (cache_path && cache_lookup(cache_path, key, r_best, b_best, t_best)) {
        *best = o;
        best->rounds = r_best;
        best->blocks_per_sm = b_best;
        if (best_ms)
            *best_ms = t_best;
        return DMAP_OK;
    }
    DMAP_CUDA(ctx, cudaSetDevice(ctx->device));
    void *hits = nullptr;
    DMAP_CUDA(ctx, cudaMalloc(&hits, sizeof(dmap_hit32) * m));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // rounds: how long rays park at leaves before the inline drain takes the
    // rest; blocks per SM: resident walk warps (the walk rounds are compiled
    // for 4 CTAs of 128 threads per SM over the candidate mask, 5 over the
    // triangle tree; more than that wait for a resident CTA to finish)
    const int rounds_c[] = {2, 3, 4, 6, 8, 12};
    const int bps_c[] = {3, 4, 5};
    t_best = 1e30;
    for (int r : rounds_c)
        for (int b : bps_c) {
            dmap_options c = o;
            c.rounds = r;
            c.blocks_per_sm = b;
            double t = 1e30;
            for (int rep = 0; rep < 3 && st == DMAP_OK; ++rep) {
                cudaEventRecord(e0, ctx->stream);
                st = dmap_intersect(s, rays_dev, ray_dtype, m, &c, hits, DMAP_F32, nullptr, ctx->stream);
                cudaEventRecord(e1, ctx->stream);
                if (st == DMAP_OK && cudaEventSynchronize(e1) == cudaSuccess) {
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0) // the first run warms caches and grows scratch
                        t = std::min(t, (double)ms);
                }
            }
            if (st != DMAP_OK)
                break;
            if (t < t_best) {
                t_best = t;
                r_best = r;
                b_best = b;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(hits);
    if (st != DMAP_OK)
        return st;
    *best = o;
    best->rounds = r_best;
    best->blocks_per_sm = b_best;
    if (best_ms)
        *best_ms = t_best;
    if (cache_path) {
        std::ofstream f(cache_path, std::ios::app);
        f << std::setprecision(17) << key << " " << r_best << " " << b_best << " " << t_best << "\n";
    }
    return DMAP_OK;
}
