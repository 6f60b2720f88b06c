// TFDM's find_roots as the reference states it (descent_sampler.cpp:66-83):
// the coarsest level at which the domain's bounding box spans at most two
// cells per axis, and the lowest cell of that 2 x 2 block.
#include "descent_sampler.h" // the reference header, which declares it
#include <cmath>

namespace dmap
{
void footprint_roots(const UvTriangle &domain, int n_leaf, int &level, int64_t &i0, int64_t &j0)
{
    level = 0;
    while (true) {
        double w = std::ldexp(1.0, level) / n_leaf;
        int64_t ilo = (int64_t)std::floor(domain.lo[0] / w), ihi = (int64_t)std::ceil(domain.hi[0] / w) - 1;
        int64_t jlo = (int64_t)std::floor(domain.lo[1] / w), jhi = (int64_t)std::ceil(domain.hi[1] / w) - 1;
        if (ihi - ilo <= 1 && jhi - jlo <= 1) {
            i0 = ilo;
            j0 = jlo;
            return;
        }
        ++level;
    }
}
} // namespace dmap
