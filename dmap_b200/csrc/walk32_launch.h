// The FP32 query's launches, split between the two translation units that
// instantiate walk32.cuh: walk32.cu (contracted FP32 arithmetic: the walk
// rounds, and the schedule that orders the launches) and walk32_exact.cu
// (-fmad=false: the simple schedule, the last walk with its leaves inline,
// the FP64 re-test of parked cells and the leaf rounds of both leaves). Each entry is instantiated for the ray / hit record types
// (R, H, Fp) = (float | double, Hit32 | Hit64, float | double).
#pragma once
#include "launch.h"

namespace dmapk
{
namespace w32
{

// One query's arguments as every launch of it sees them.
struct Args
{
    const dmapdev::TriDev32 *t32;
    const dmapdev::TriDev *t64;
    int n_tri;
    const dmapdev::AssetDev *assets;
    const void *rays;
    int64_t n;
    QueryOpts opt;
    void *hits;
    int64_t *stats;
    unsigned *status;
    void *states;                 // wavefront: the parked walk states
    void *leaves;                 // wavefront: the leaf jobs
    unsigned long long *counters; // wavefront: kWaveCounters
    int *rerun;                   // wavefront, filtered scene: rays the filter's schedule answers again
    int grid;                     // wavefront: walk CTAs
};

// walk32_exact.cu
template <typename R, typename H, typename Fp>
cudaError_t simple(const Args &a, cudaStream_t stream);
// the filter's schedule over the rays a filtered wavefront query listed
template <typename R, typename H, typename Fp>
cudaError_t simple_rerun(const Args &a, cudaStream_t stream);
template <typename R, typename H, typename Fp>
cudaError_t walk_drain(const Args &a, const int *q_in, int round, cudaStream_t stream);
template <typename R>
cudaError_t filter(const Args &a, int round, cudaStream_t stream);
template <typename R, typename H, typename Fp>
cudaError_t leaf64(const Args &a, int round, int *q_out, cudaStream_t stream);
template <typename R, typename H, typename Fp>
cudaError_t leaf32(const Args &a, int round, int *q_out, cudaStream_t stream);

// walk32.cu
template <typename R, typename H, typename Fp>
cudaError_t walk_round(const Args &a, const int *q_in, int round, cudaStream_t stream);

} // namespace w32
} // namespace dmapk
