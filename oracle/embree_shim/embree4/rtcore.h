/* embree4/rtcore.h - TEST INFRASTRUCTURE ONLY: the subset of the Intel Embree 4 ray-tracing API
 * that the reference's shadow ray tracer calls (src/raytracer/shadow_maker.c:127-196 and
 * :252-268), declared from Embree's public API so that the reference's own shadow_maker.c
 * compiles here without Embree (a CMake dependency, `find_package(embree 4 REQUIRED)` in the
 * reference's CMakeLists.txt, not installed in this image). The implementation
 * (oracle/embree_shim/rtcore_shim.c) answers occlusion queries by testing every triangle; it is
 * used only by the oracle build in oracle/_ref/. */
#ifndef ORACLE_EMBREE_SHIM_RTCORE_H
#define ORACLE_EMBREE_SHIM_RTCORE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct RTCDeviceTy *RTCDevice;
typedef struct RTCSceneTy *RTCScene;
typedef struct RTCGeometryTy *RTCGeometry;

enum RTCSceneFlags { RTC_SCENE_FLAG_NONE = 0, RTC_SCENE_FLAG_DYNAMIC = 1,
                     RTC_SCENE_FLAG_COMPACT = 2, RTC_SCENE_FLAG_ROBUST = 4 };
enum RTCBuildQuality { RTC_BUILD_QUALITY_LOW = 0, RTC_BUILD_QUALITY_MEDIUM = 1,
                       RTC_BUILD_QUALITY_HIGH = 2 };
enum RTCGeometryType { RTC_GEOMETRY_TYPE_TRIANGLE = 0 };
enum RTCBufferType { RTC_BUFFER_TYPE_INDEX = 0, RTC_BUFFER_TYPE_VERTEX = 1 };
enum RTCFormat { RTC_FORMAT_UNDEFINED = 0, RTC_FORMAT_UINT3 = 0x5003, RTC_FORMAT_FLOAT3 = 0x9003 };

/* One ray: origin, the start of the valid interval, direction, time, the end of the interval
 * (set to -inf by rtcOccluded1 when something blocks the ray), mask, id and flags. */
struct RTCRay {
    float org_x, org_y, org_z;
    float tnear;
    float dir_x, dir_y, dir_z;
    float time;
    float tfar;
    unsigned int mask;
    unsigned int id;
    unsigned int flags;
};

struct RTCOccludedArguments {
    unsigned int flags;
    unsigned int feature_mask;
    void *context;
    void *filter;
    void *intersect;
};

RTCDevice rtcNewDevice(const char *config);
void rtcReleaseDevice(RTCDevice device);
RTCScene rtcNewScene(RTCDevice device);
void rtcSetSceneFlags(RTCScene scene, enum RTCSceneFlags flags);
void rtcSetSceneBuildQuality(RTCScene scene, enum RTCBuildQuality quality);
void rtcCommitScene(RTCScene scene);
void rtcReleaseScene(RTCScene scene);
RTCGeometry rtcNewGeometry(RTCDevice device, enum RTCGeometryType type);
void *rtcSetNewGeometryBuffer(RTCGeometry geometry, enum RTCBufferType type, unsigned int slot,
                              enum RTCFormat format, size_t byte_stride, size_t item_count);
void rtcCommitGeometry(RTCGeometry geometry);
unsigned int rtcAttachGeometry(RTCScene scene, RTCGeometry geometry);
void rtcReleaseGeometry(RTCGeometry geometry);
void rtcInitOccludedArguments(struct RTCOccludedArguments *args);
void rtcOccluded1(RTCScene scene, struct RTCRay *ray, struct RTCOccludedArguments *args);

#ifdef __cplusplus
}
#endif
#endif /* ORACLE_EMBREE_SHIM_RTCORE_H */
