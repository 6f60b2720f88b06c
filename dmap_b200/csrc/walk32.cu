// The FP32 query's schedule and its contracted launches (compiled with FMA
// contraction): the walk rounds, whose arithmetic is conservative by its
// error bounds, and whose rounding never reaches a result (every leaf cell
// the walk reaches is re-tested in FP64 before its leaf runs). The launches
// that must round the same way wherever they run are in walk32_exact.cu.
#include "walk32.cuh"

namespace dmapk
{
namespace w32
{

template <typename R, typename H, typename Fp>
cudaError_t walk_round(const Args &a, const int *q_in, int round, cudaStream_t stream)
{
    // scenes of more than 256 triangles take the triangle tree; each
    // candidate mode and each triangle order has its own instances, so every
    // kernel carries one order's candidate code, and scenes of up to 256
    // triangles keep the smaller kernel
    const bool nearest = a.opt.order == 1, tree = a.n_tri > 32 * kMaskWords;
    const R *rr = static_cast<const R *>(a.rays);
    H *hh = static_cast<H *>(a.hits);
    RayState *states = static_cast<RayState *>(a.states);
    LeafJob *leaves = static_cast<LeafJob *>(a.leaves);
#define DMAP_ROUND(ST_, TR_, NR_)                                                                                   \
    wave_walk<ST_, false, TR_, NR_, R, H, Fp><<<a.grid, 128, 0, stream>>>(a.t32, a.t64, a.n_tri, a.assets, rr, a.n, \
                                                                          a.opt, hh, ST_ ? a.stats : nullptr,      \
                                                                          states, q_in, round, leaves, a.counters, \
                                                                          a.status, a.rerun)
#define DMAP_ROUND_MODE(ST_)                                                                                        \
    (tree ? (nearest ? DMAP_ROUND(ST_, true, true) : DMAP_ROUND(ST_, true, false))                                  \
          : (nearest ? DMAP_ROUND(ST_, false, true) : DMAP_ROUND(ST_, false, false)))
    if (a.stats)
        DMAP_ROUND_MODE(true);
    else
        DMAP_ROUND_MODE(false);
#undef DMAP_ROUND_MODE
#undef DMAP_ROUND
    return cudaGetLastError();
}

// One query: the simple schedule's single launch, or the wavefront's rounds
// of (walk, FP64 re-test of the parked cells, leaves) and the last walk with
// its leaves inline; on a filtered scene then the filter's schedule over the
// rays that took a crossing the filter rejects.
template <typename R, typename H, typename Fp>
cudaError_t launch(Args a, const WaveScratch &ws, cudaStream_t stream)
{
    if (a.opt.schedule == 1)
        return simple<R, H, Fp>(a, stream);
    if (ws.capacity < a.n)
        return cudaErrorInvalidValue;
    if (a.n_tri > 32 * kMaskWords && !a.opt.bvh_nodes)
        return cudaErrorInvalidValue; // a scene without its triangle tree (every such scene has one)
    cudaError_t e;
    if (a.stats && (e = cudaMemsetAsync(a.stats, 0, sizeof(int64_t) * DMAP_ST_N * a.n, stream)) != cudaSuccess)
        return e;
    // rounds = 0: a single walk that runs every leaf inline
    int rounds = a.opt.rounds > 0 ? a.opt.rounds : 0;
    if (rounds > kMaxRounds)
        rounds = kMaxRounds;
    if ((e = cudaMemsetAsync(ws.counters, 0, sizeof(unsigned long long) * kWaveCounters, stream)) != cudaSuccess)
        return e;
    // blocks_per_sm 0: the occupancy the scene's walk is compiled for
    const int bps = a.opt.blocks_per_sm > 0              ? a.opt.blocks_per_sm
                    : a.n_tri > 32 * kMaskWords ? DMAP_WALK_TREE_MIN_BLOCKS
                                                         : DMAP_WALK_MIN_BLOCKS;
    const int64_t need = (a.n + 127) / 128;
    a.grid = sm_count() * bps;
    if (need < a.grid)
        a.grid = (int)need;
    a.states = ws.state;
    a.leaves = ws.leaves;
    a.counters = ws.counters;
    a.rerun = ws.rerun;
    for (int rd = 0; rd <= rounds; ++rd) {
        const int *q_in = ws.queue[(rd + 1) & 1];
        int *q_out = ws.queue[rd & 1];
        if (rd == rounds) {
            if ((e = walk_drain<R, H, Fp>(a, q_in, rd, stream)) != cudaSuccess || !a.opt.op_mask)
                return e;
            return simple_rerun<R, H, Fp>(a, stream);
        }
        if ((e = walk_round<R, H, Fp>(a, q_in, rd, stream)) != cudaSuccess ||
            (e = filter<R>(a, rd, stream)) != cudaSuccess)
            return e;
        e = a.opt.leaf_precision == 1 ? leaf32<R, H, Fp>(a, rd, q_out, stream) // the FP32 certified leaf
                                      : leaf64<R, H, Fp>(a, rd, q_out, stream);
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

} // namespace w32

size_t wave_state_bytes() { return sizeof(RayState); }
size_t wave_leaf_bytes() { return sizeof(LeafJob); }

int walk32_launches(const QueryOpts &opt)
{
    if (opt.schedule == 1)
        return 1;
    int rounds = opt.rounds > 0 ? opt.rounds : 0;
    if (rounds > kMaxRounds)
        rounds = kMaxRounds;
    // per round: walk, cell filter, leaves; then the inline walk (and on a
    // filtered scene the filter's schedule over the rays it lists)
    return 3 * rounds + 1 + (opt.op_mask ? 1 : 0);
}

cudaError_t launch_walk32(const dmapdev::TriDev32 *t32, const dmapdev::TriDev *t64, int n_tri,
                          const dmapdev::AssetDev *assets, const void *rays, int64_t n, const QueryOpts &opt,
                          void *hits, int64_t *stats, unsigned *status, const WaveScratch &ws, cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    const w32::Args a = {t32, t64, n_tri, assets, rays, n, opt, hits, stats, status, nullptr, nullptr, nullptr,
                         nullptr, 0};
    const bool r64 = opt.ray_dtype == 2, h64 = opt.hit_dtype == 2;
    if (r64 && h64)
        return w32::launch<double, dmapdev::Hit64, double>(a, ws, stream);
    if (r64)
        return w32::launch<double, dmapdev::Hit32, float>(a, ws, stream);
    if (h64)
        return w32::launch<float, dmapdev::Hit64, double>(a, ws, stream);
    return w32::launch<float, dmapdev::Hit32, float>(a, ws, stream);
}

} // namespace dmapk
