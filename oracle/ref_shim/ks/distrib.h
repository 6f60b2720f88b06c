// Stand-in for the reference's missing `ks/distrib.h`. The hot path only
// includes descent_sampler.h for footprint_roots; the tabulated sampler that
// names this type is never constructed in the oracle build.
#pragma once
namespace ks
{
struct DistribTable2D
{};
} // namespace ks
