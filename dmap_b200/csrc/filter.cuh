// The opacity filter behind embree's filter functions, as DisplacedGeometry's
// intersect and occluded callbacks run it (displaced_geometry.cpp:53-106):
// the triangle's nearest crossing past t_lo goes to the filter; a crossing it
// rejects raises t_lo to the crossing's t and the triangle is walked again,
// at most max_filter_passes times (displaced_geometry.h:64). The filter is
// ks's opacity map reduced to a binary texel mask over the object's texture
// coordinates. Every double operation is an explicitly rounded intrinsic, so
// the texture coordinate is the reference's to the bit in any translation
// unit, contracted or not.
#pragma once
#include "device_types.cuh"
#include "launch.h"

namespace dmapdev
{

constexpr int kFilterPasses = 64; // DisplacedGeometry::max_filter_passes

// True when the filter accepts the crossing of triangle `tri` at the base
// triangle's barycentrics (bu, bv); triangles the mask does not cover accept.
__device__ inline bool crossing_opaque(const dmapk::QueryOpts &q, const TriDev &T, int tri, double bu, double bv)
{
    if (!q.op_mask || (q.op_tri && !q.op_tri[tri]))
        return true;
    // potential_hit hands the filter float barycentrics (displaced_geometry.cpp:21-34);
    // compute_hit_texcoord (:189-193): BaseTriangle::param (displaced_surface.h:87)
    // and DisplacedObject::object_uv (scene_spec.cpp:382-388), rounded to float
    const double u = (double)(float)bu, v = (double)(float)bv;
    const double s = __dadd_rn(__dadd_rn(T.t0[0], __dmul_rn(u, __dsub_rn(T.t1[0], T.t0[0]))),
                               __dmul_rn(v, __dsub_rn(T.t2[0], T.t0[0])));
    const double t = __dadd_rn(__dadd_rn(T.t0[1], __dmul_rn(u, __dsub_rn(T.t1[1], T.t0[1]))),
                               __dmul_rn(v, __dsub_rn(T.t2[1], T.t0[1])));
    double x = __ddiv_rn(__dsub_rn(s, q.op_offset[0]), q.op_scale[0]);
    double y = __ddiv_rn(__dsub_rn(t, q.op_offset[1]), q.op_scale[1]);
    if (q.op_flip)
        y = __dsub_rn(1.0, y);
    // the texel under the float texture coordinate, repeated outside [0, 1)
    const double fx = __dmul_rn((double)(float)x, (double)q.op_w), fy = __dmul_rn((double)(float)y, (double)q.op_h);
    if (!(fabs(fx) < 1e15 && fabs(fy) < 1e15))
        return true;
    long long i = (long long)floor(fx) % q.op_w, j = (long long)floor(fy) % q.op_h;
    if (i < 0)
        i += q.op_w;
    if (j < 0)
        j += q.op_h;
    return q.op_mask[j * q.op_w + i] != 0;
}

} // namespace dmapdev
