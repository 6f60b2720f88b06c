// Placeholder until the FP32 path lands.
#include "launch.h"
namespace dmapk
{
cudaError_t launch_walk32(const dmapdev::TriDev32 *, const dmapdev::TriDev *, int, const dmapdev::AssetDev *,
                          const void *, int64_t, const QueryOpts &, void *, int64_t *, unsigned *, cudaStream_t)
{
    return cudaErrorNotSupported;
}
} // namespace dmapk
