// Type-only stand-in for Embree 3's <embree3/rtcore.h>, enough for the
// reference's displaced_intersector.cpp to compile. The oracle build never
// builds a BVH, so ObjectIntersector::intersect takes its flat loop; every
// function here aborts if called.
#pragma once
#include <cstdio>
#include <cstdlib>

#define RTC_MAX_INSTANCE_LEVEL_COUNT 1

typedef struct RTCDeviceTy *RTCDevice;
typedef struct RTCSceneTy *RTCScene;
typedef struct RTCGeometryTy *RTCGeometry;

enum RTCGeometryType { RTC_GEOMETRY_TYPE_USER = 120 };
enum RTCSceneFlags { RTC_SCENE_FLAG_NONE = 0, RTC_SCENE_FLAG_ROBUST = 4 };

struct RTCBounds {
    float lower_x, lower_y, lower_z, align0;
    float upper_x, upper_y, upper_z, align1;
};
struct RTCIntersectContext {
    unsigned flags;
    void *filter;
    unsigned instID[RTC_MAX_INSTANCE_LEVEL_COUNT];
};
struct RTCRay {
    float org_x, org_y, org_z, tnear;
    float dir_x, dir_y, dir_z, time;
    float tfar;
    unsigned mask, id, flags;
};
struct RTCHit {
    float Ng_x, Ng_y, Ng_z;
    float u, v;
    unsigned primID, geomID;
    unsigned instID[RTC_MAX_INSTANCE_LEVEL_COUNT];
};
struct RTCRayHit {
    RTCRay ray;
    RTCHit hit;
};
struct RTCRayN;
struct RTCHitN;
struct RTCBoundsFunctionArguments {
    void *geometryUserPtr;
    unsigned primID, timeStep;
    RTCBounds *bounds_o;
};
struct RTCIntersectFunctionNArguments {
    int *valid;
    void *geometryUserPtr;
    unsigned primID;
    RTCIntersectContext *context;
    RTCRayHit *rayhit;
    unsigned N, geomID;
};
typedef void (*RTCBoundsFunction)(const RTCBoundsFunctionArguments *);
typedef void (*RTCIntersectFunctionN)(const RTCIntersectFunctionNArguments *);

[[noreturn]] inline void rtc_stub_abort(const char *f)
{
    std::fprintf(stderr, "embree stub: %s is not available in the oracle build\n", f);
    std::abort();
}
inline RTCGeometry rtcNewGeometry(RTCDevice, RTCGeometryType) { rtc_stub_abort("rtcNewGeometry"); }
inline void rtcSetGeometryUserPrimitiveCount(RTCGeometry, unsigned) { rtc_stub_abort("rtcSetGeometryUserPrimitiveCount"); }
inline void rtcSetGeometryUserData(RTCGeometry, void *) { rtc_stub_abort("rtcSetGeometryUserData"); }
inline void rtcSetGeometryBoundsFunction(RTCGeometry, RTCBoundsFunction, void *) { rtc_stub_abort("rtcSetGeometryBoundsFunction"); }
inline void rtcSetGeometryIntersectFunction(RTCGeometry, RTCIntersectFunctionN) { rtc_stub_abort("rtcSetGeometryIntersectFunction"); }
inline void rtcCommitGeometry(RTCGeometry) { rtc_stub_abort("rtcCommitGeometry"); }
inline RTCScene rtcNewScene(RTCDevice) { rtc_stub_abort("rtcNewScene"); }
inline void rtcSetSceneFlags(RTCScene, RTCSceneFlags) { rtc_stub_abort("rtcSetSceneFlags"); }
inline unsigned rtcAttachGeometry(RTCScene, RTCGeometry) { rtc_stub_abort("rtcAttachGeometry"); }
inline void rtcReleaseGeometry(RTCGeometry) { rtc_stub_abort("rtcReleaseGeometry"); }
inline void rtcCommitScene(RTCScene) { rtc_stub_abort("rtcCommitScene"); }
inline void rtcReleaseScene(RTCScene) { rtc_stub_abort("rtcReleaseScene"); }
inline void rtcInitIntersectContext(RTCIntersectContext *) { rtc_stub_abort("rtcInitIntersectContext"); }
inline void rtcIntersect1(RTCScene, RTCIntersectContext *, RTCRayHit *) { rtc_stub_abort("rtcIntersect1"); }
