// Conservative FP32 slab tests of object boxes against the float ray (rounded
// from the caller's double ray), shared by the FP32 walk's candidate code and
// the top-level tree (bvh.cuh).
#pragma once
#include "f32_node.cuh"

namespace d32
{

// The slabs of a box, widened, against the float ray: where the exact ray is
// inside the box, |t d| <= |o| + |box|, so the float ray is within
// u (2|o| + |box|) of it; the widening is more than that and more than the
// float rounding of the slab products. t0 / t1 enter as the ray's range and
// leave as the entry / exit bounds: t0 is a lower bound of the exact entry
// of any box inside this one, t1 an upper bound of its exit. False when an
// axis the ray does not move along misses the box.
__device__ __forceinline__ bool box_slabs(const float *box_lo, const float *box_hi, const float *of, const float *df,
                                          const float *invf, float &t0, float &t1)
{
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float bmag = fmaxf(fabsf(box_lo[a]), fabsf(box_hi[a]));
        float pad = ru_mul(2.0f * G, ru_add(ru_fma(2.0f, fabsf(of[a]), bmag), 1.0f));
        float lo = __fsub_rd(box_lo[a], pad), hi = __fadd_ru(box_hi[a], pad);
        if (df[a] != 0.0f) {
            float ta = (lo - of[a]) * invf[a], tb = (hi - of[a]) * invf[a];
            t0 = fmaxf(t0, fminf(ta, tb));
            t1 = fminf(t1, fmaxf(ta, tb));
        } else if (of[a] < lo || of[a] > hi) {
            ok = false;
        }
    }
    return ok;
}

// The triangle-level test: the box passes when its slab range is not empty
// beyond the FP32 tolerance. On a pass t1 is the exit parameter (rounded up).
__device__ __forceinline__ bool box_range(const float *box_lo, const float *box_hi, const float *of, const float *df,
                                          const float *invf, float &t0, float &t1)
{
    const bool ok = box_slabs(box_lo, box_hi, of, df, invf, t0, t1);
    return ok && !(t0 > t1 + tol32(fmaxf(fabsf(t0), fabsf(t1))));
}

__device__ __forceinline__ bool box_pass(const float *box_lo, const float *box_hi, const float *of, const float *df,
                                         const float *invf, float t0, float &t1)
{
    return box_range(box_lo, box_hi, of, df, invf, t0, t1);
}

__device__ __forceinline__ bool object_box(const TriDev32 &T, const float *of, const float *df, const float *invf,
                                           float t0, float &t1)
{
    return box_pass(T.box_lo, T.box_hi, of, df, invf, t0, t1);
}

// The test of a box that encloses triangle boxes (a tree node): it passes
// whenever box_range passes for some box inside it. The slab range of the
// enclosing box contains the inner one's (float rounding is monotone and the
// widening grows with the box), and the tolerance is taken at twice the
// magnitude bound that covers the inner box's own (its range lies within
// [t_lo, t1] of this one, both bounded by max(|t0|, |t1|, |t_lo|)).
__device__ __forceinline__ bool node_range(const float *box_lo, const float *box_hi, const float *of,
                                           const float *df, const float *invf, float t_lo, float &t0, float &t1)
{
    const bool ok = box_slabs(box_lo, box_hi, of, df, invf, t0, t1);
    const float m = fmaxf(fmaxf(fabsf(t0), fabsf(t1)), fabsf(t_lo));
    return ok && !(t0 > t1 + 2.0f * tol32(m));
}

} // namespace d32
