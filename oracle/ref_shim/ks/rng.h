// Stand-in for the reference's missing `ks/rng.h`: the sampler declarations
// in descent_sampler.h name the type by reference only.
#pragma once
namespace ks
{
struct RNG;
}
