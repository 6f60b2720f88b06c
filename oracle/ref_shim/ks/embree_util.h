// Stand-in for the reference's missing `ks/embree_util.h`: the one helper
// displaced_intersector.cpp names, on the embree type stub.
#pragma once
#include "ks/maths.h"
#include <embree3/rtcore.h>

namespace ks
{
inline RTCRayHit spawn_rtcrayhit(const vec3 &o, const vec3 &d, float tnear, float tfar)
{
    RTCRayHit rh{};
    rh.ray.org_x = o[0];
    rh.ray.org_y = o[1];
    rh.ray.org_z = o[2];
    rh.ray.dir_x = d[0];
    rh.ray.dir_y = d[1];
    rh.ray.dir_z = d[2];
    rh.ray.tnear = tnear;
    rh.ray.tfar = tfar;
    return rh;
}
} // namespace ks
