// Stand-in for the reference's missing `ks/rng.h`: the random source the
// descent sampler draws from. It replays a caller-given array of uniforms
// in [0, 1) in order (0.5 once the array is used up), so the oracle build
// of the reference's sampler and the restatements under test consume the
// same numbers in the same order.
#pragma once
namespace ks
{
struct RNG
{
    const float *u = nullptr;
    int n = 0, k = 0;
    float next() { return k < n ? u[k++] : 0.5f; }
};
} // namespace ks
