// The nearest-first candidate order (DMAP_ORDER_NEAREST, include/dmap_b200.h)
// shared by the FP64 and FP32 walks. A ray's candidates are the triangles
// whose boxes it meets; each has a fixed key, the FP64 slab entry distance
// of its object box, and the walks visit them in increasing (key, index)
// with a cursor: the next triangle is the smallest (key, index) above the
// last one among the candidates the ray still reaches with its current
// t_max. The keys use IEEE products with 1 / d (no FMA in the translation
// units that include this), so the C oracle computes the same order.
#pragma once
#include "f64_math.cuh"

namespace d64
{

// 1 / d per axis (0 where d is 0, which the key then ignores).
__device__ __forceinline__ void ray_inverse(const double *d, double *inv)
{
    for (int a = 0; a < 3; ++a)
        inv[a] = d[a] != 0.0 ? 1.0 / d[a] : 0.0;
}

// max(t_min, max over axes with d != 0 of min(ta, tb)), ta = (lo - o) / d
// and tb = (hi - o) / d as products with 1 / d, over the box lo .. hi.
__device__ __forceinline__ double entry_key(const double *lo, const double *hi, const double *o, const double *d,
                                            const double *inv, double t_min)
{
    double key = t_min;
    for (int a = 0; a < 3; ++a)
        if (d[a] != 0.0) {
            const double ta = (lo[a] - o[a]) * inv[a], tb = (hi[a] - o[a]) * inv[a];
            key = dmax(key, dmin(ta, tb));
        }
    return key;
}

// The key of a triangle's object box.
__device__ __forceinline__ double entry_key(const TriDev &T, const double *o, const double *d, const double *inv,
                                            double t_min)
{
    return entry_key(T.box_lo, T.box_hi, o, d, inv, t_min);
}

// (key, t) comes after the cursor (ck, ct)
__device__ __forceinline__ bool after_cursor(double key, int t, double ck, int ct)
{
    return key > ck || (key == ck && t > ct);
}

// (key, t) comes before the best so far (bk, bt); bt < 0: none yet
__device__ __forceinline__ bool before_best(double key, int t, double bk, int bt)
{
    return bt < 0 || key < bk || (key == bk && t < bt);
}

} // namespace d64
