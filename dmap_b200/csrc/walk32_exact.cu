// The FP32 query's launches that must round like the reference, or the same
// way wherever they run (compiled with -fmad=false): the simple schedule, the
// last walk with its leaves inline, the FP64 re-test of parked cells, and the
// leaf rounds of both leaves (the FP32 leaf also runs inline in the last
// walk, so both places round alike and a ray's answer does not depend on the
// round it finishes in).
#include "walk32.cuh"

namespace dmapk
{
namespace w32
{

template <typename R, typename H, typename Fp>
cudaError_t simple(const Args &a, cudaStream_t stream)
{
    const int threads = 128;
    const int64_t blocks = (a.n + threads - 1) / threads;
    walk32_simple<R, H, Fp><<<(unsigned)blocks, threads, 0, stream>>>(
        a.t32, a.t64, a.n_tri, a.assets, static_cast<const R *>(a.rays), a.n, a.opt, static_cast<H *>(a.hits),
        a.stats, a.status);
    return cudaGetLastError();
}

template <typename R, typename H, typename Fp>
cudaError_t simple_rerun(const Args &a, cudaStream_t stream)
{
    const int threads = 128;
    const int64_t blocks = (a.n + threads - 1) / threads;
    walk32_simple<R, H, Fp><<<(unsigned)blocks, threads, 0, stream>>>(
        a.t32, a.t64, a.n_tri, a.assets, static_cast<const R *>(a.rays), a.n, a.opt, static_cast<H *>(a.hits),
        a.stats, a.status, a.rerun, a.counters + 4 * (kMaxRounds + 1));
    return cudaGetLastError();
}

template <typename R, typename H, typename Fp>
cudaError_t walk_drain(const Args &a, const int *q_in, int round, cudaStream_t stream)
{
    const bool nearest = a.opt.order == 1, tree = a.n_tri > 32 * kMaskWords;
    const R *rr = static_cast<const R *>(a.rays);
    H *hh = static_cast<H *>(a.hits);
    RayState *states = static_cast<RayState *>(a.states);
    LeafJob *leaves = static_cast<LeafJob *>(a.leaves);
#define DMAP_DRAIN(ST_, TR_, NR_)                                                                                   \
    wave_walk<ST_, true, TR_, NR_, R, H, Fp><<<a.grid, 128, 0, stream>>>(a.t32, a.t64, a.n_tri, a.assets, rr, a.n,  \
                                                                         a.opt, hh, ST_ ? a.stats : nullptr,       \
                                                                         states, q_in, round, leaves, a.counters,  \
                                                                         a.status, a.rerun)
#define DMAP_DRAIN_MODE(ST_)                                                                                        \
    (tree ? (nearest ? DMAP_DRAIN(ST_, true, true) : DMAP_DRAIN(ST_, true, false))                                  \
          : (nearest ? DMAP_DRAIN(ST_, false, true) : DMAP_DRAIN(ST_, false, false)))
    if (a.stats)
        DMAP_DRAIN_MODE(true);
    else
        DMAP_DRAIN_MODE(false);
#undef DMAP_DRAIN_MODE
#undef DMAP_DRAIN
    return cudaGetLastError();
}

template <typename R>
cudaError_t filter(const Args &a, int round, cudaStream_t stream)
{
    wave_filter<R><<<sm_count() * 4, 128, 0, stream>>>(a.t64, a.assets, static_cast<const R *>(a.rays), a.opt,
                                                       static_cast<RayState *>(a.states),
                                                       static_cast<LeafJob *>(a.leaves), round, a.counters);
    return cudaGetLastError();
}

template <typename R, typename H, typename Fp>
cudaError_t leaf64(const Args &a, int round, int *q_out, cudaStream_t stream)
{
    const int lgrid = sm_count() * 4;
    const R *rr = static_cast<const R *>(a.rays);
    H *hh = static_cast<H *>(a.hits);
    RayState *states = static_cast<RayState *>(a.states);
    LeafJob *leaves = static_cast<LeafJob *>(a.leaves);
    if (a.stats)
        wave_leaf<true, R, H, Fp><<<lgrid, 128, 0, stream>>>(a.t64, a.assets, rr, a.opt, hh, a.stats, states, leaves,
                                                            round, q_out, a.counters, a.rerun);
    else
        wave_leaf<false, R, H, Fp><<<lgrid, 128, 0, stream>>>(a.t64, a.assets, rr, a.opt, hh, nullptr, states,
                                                             leaves, round, q_out, a.counters, a.rerun);
    return cudaGetLastError();
}

template <typename R, typename H, typename Fp>
cudaError_t leaf32(const Args &a, int round, int *q_out, cudaStream_t stream)
{
    const int lgrid = sm_count() * 4;
    const R *rr = static_cast<const R *>(a.rays);
    H *hh = static_cast<H *>(a.hits);
    RayState *states = static_cast<RayState *>(a.states);
    LeafJob *leaves = static_cast<LeafJob *>(a.leaves);
    if (a.stats)
        wave_leaf32<true, R, H, Fp><<<lgrid, 128, 0, stream>>>(a.t32, a.t64, a.assets, rr, a.opt, hh, a.stats, states,
                                                              leaves, round, q_out, a.counters, a.rerun);
    else
        wave_leaf32<false, R, H, Fp><<<lgrid, 128, 0, stream>>>(a.t32, a.t64, a.assets, rr, a.opt, hh, nullptr,
                                                               states, leaves, round, q_out, a.counters, a.rerun);
    return cudaGetLastError();
}

#define DMAP_W32_EXACT(R, H, Fp)                                                                                    \
    template cudaError_t simple<R, H, Fp>(const Args &, cudaStream_t);                                              \
    template cudaError_t simple_rerun<R, H, Fp>(const Args &, cudaStream_t);                                        \
    template cudaError_t walk_drain<R, H, Fp>(const Args &, const int *, int, cudaStream_t);                        \
    template cudaError_t leaf64<R, H, Fp>(const Args &, int, int *, cudaStream_t);                                  \
    template cudaError_t leaf32<R, H, Fp>(const Args &, int, int *, cudaStream_t);
DMAP_W32_EXACT(float, dmapdev::Hit32, float)
DMAP_W32_EXACT(float, dmapdev::Hit64, double)
DMAP_W32_EXACT(double, dmapdev::Hit32, float)
DMAP_W32_EXACT(double, dmapdev::Hit64, double)
#undef DMAP_W32_EXACT
template cudaError_t filter<float>(const Args &, int, cudaStream_t);
template cudaError_t filter<double>(const Args &, int, cudaStream_t);

} // namespace w32
} // namespace dmapk
