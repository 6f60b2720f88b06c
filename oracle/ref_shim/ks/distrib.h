// Stand-in for the reference's missing `ks/distrib.h`: the tabulated
// distributions that descent_sampler.cpp's texel-table baseline uses. The
// oracle build compiles that baseline but never constructs or samples it, so
// every member that would compute something stops the program.
#pragma once
#include "maths.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

namespace ks
{
struct DistribTable
{
    std::vector<float> cdf;
};

struct DistribTable2D
{
    DistribTable margin;
    std::vector<DistribTable> cond;

    DistribTable2D() = default;
    DistribTable2D(const float *, int, int) { unavailable(); }
    vec2 sample_linear(const vec2 &, float &, vec2i *) const { unavailable(); return vec2(); }
    float pdf(const vec2 &) const { unavailable(); return 0.0f; }

  private:
    [[noreturn]] static void unavailable()
    {
        std::fprintf(stderr, "ks::DistribTable2D is not part of the oracle build\n");
        std::abort();
    }
};
} // namespace ks
