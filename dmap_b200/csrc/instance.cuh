// Instances placed by an affine to_world transform that is not rigid
// (dmap_scene_create_instanced). Their triangles keep the object's records;
// a ray meets an instance's triangle in object space: the world ray moved by
// the inverse transform, its parameter t unchanged (the reference's
// instancing, displaced_scene.cpp:79-87, hands the instanced geometry the
// ray in the instance's space). The FP32 walk takes the move folded into
// each triangle's tangent transform (set up on the host); the FP64 node test
// and both leaves move the ray here, and a hit's geometric normal goes back
// to world space.
//
// The instance table holds kInstDoubles per instance: L (3 x 3, row major),
// T (3), Linv (3 x 3, row major), sign(det L); to_world(x) = L x + T. Every
// double operation is an explicitly rounded intrinsic, so the moved ray is
// the same in any translation unit, contracted or not.
#pragma once
#include "f64_math.cuh"

namespace dmapdev
{

constexpr int kInstDoubles = 22;

// o, d (world) -> oo = Linv (o - T), od = Linv d.
__device__ __forceinline__ void object_ray(const double *xf, const double *o, const double *d, double *oo,
                                           double *od)
{
    const double *T = xf + 9, *Li = xf + 12;
    const double u0 = __dsub_rn(o[0], T[0]), u1 = __dsub_rn(o[1], T[1]), u2 = __dsub_rn(o[2], T[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        oo[a] = __dadd_rn(__dadd_rn(__dmul_rn(Li[3 * a], u0), __dmul_rn(Li[3 * a + 1], u1)),
                          __dmul_rn(Li[3 * a + 2], u2));
        od[a] = __dadd_rn(__dadd_rn(__dmul_rn(Li[3 * a], d[0]), __dmul_rn(Li[3 * a + 1], d[1])),
                          __dmul_rn(Li[3 * a + 2], d[2]));
    }
}

// A hit's unit geometric normal from object to world space:
// sign(det L) Linv^T n, normalized (the cross product of the surface's two
// tangents, both moved by L, is det(L) Linv^T times theirs).
__device__ __forceinline__ void world_normal(const double *xf, d64::v3 &n)
{
    const double *Li = xf + 12;
    double m[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        m[a] = __dadd_rn(__dadd_rn(__dmul_rn(Li[a], n.x), __dmul_rn(Li[3 + a], n.y)), __dmul_rn(Li[6 + a], n.z));
    const double len2 = __dadd_rn(__dadd_rn(__dmul_rn(m[0], m[0]), __dmul_rn(m[1], m[1])), __dmul_rn(m[2], m[2]));
    const double s = __ddiv_rn(xf[21], __dsqrt_rn(len2));
    n = d64::V3(__dmul_rn(m[0], s), __dmul_rn(m[1], s), __dmul_rn(m[2], s));
}

// The ray of instanced triangle T in its object space, else the ray itself.
__device__ __forceinline__ void ray_for(const double *table, int inst, const double *o, const double *d,
                                        double *oo, double *od)
{
    if (inst > 0) {
        object_ray(table + kInstDoubles * (inst - 1), o, d, oo, od);
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            oo[a] = o[a];
            od[a] = d[a];
        }
    }
}

} // namespace dmapdev
