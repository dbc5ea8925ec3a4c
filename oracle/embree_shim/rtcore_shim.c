/* rtcore_shim.c - TEST INFRASTRUCTURE ONLY: a brute-force stand-in for the Embree calls of the
 * reference's shadow ray tracer (declarations in oracle/embree_shim/embree4/rtcore.h).
 *
 * A scene holds one triangle geometry (FP32 vertices, unsigned index triples, the buffers the
 * reference fills through rtcSetNewGeometryBuffer). rtcCommitScene turns the triangles into
 * (v0, e1, e2) FP32 triples; rtcOccluded1 tests every triangle with the Moller-Trumbore algorithm
 * in FP32 over [tnear, tfar] and sets tfar to -inf on the first hit, which is how Embree reports
 * occlusion (shadow_maker.c:193). This is the same occlusion test as oracle/raytrace_oracle.c and
 * the GPU kernel's leaves; Embree's own intersector can differ from it only for rays that graze a
 * triangle edge. Scenes are read-only after the commit, so concurrent queries are safe. */
#include <embree4/rtcore.h>

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct RTCDeviceTy { int unused; };

struct RTCGeometryTy {
    float *verts;
    unsigned int *index;
    size_t nvert, ntri;
    int refs;
};

struct RTCSceneTy {
    RTCGeometry geom;
    float *tri;          /* [ntri][9]: v0, e1 = v1 - v0, e2 = v2 - v0 */
    size_t ntri;
};

RTCDevice rtcNewDevice(const char *config)
{
    (void)config;
    return calloc(1, sizeof(struct RTCDeviceTy));
}

void rtcReleaseDevice(RTCDevice device) { free(device); }

RTCScene rtcNewScene(RTCDevice device)
{
    (void)device;
    return calloc(1, sizeof(struct RTCSceneTy));
}

void rtcSetSceneFlags(RTCScene scene, enum RTCSceneFlags flags) { (void)scene; (void)flags; }

void rtcSetSceneBuildQuality(RTCScene scene, enum RTCBuildQuality quality)
{
    (void)scene;
    (void)quality;
}

static void geometry_release(RTCGeometry g)
{
    if (g && --g->refs == 0) {
        free(g->verts);
        free(g->index);
        free(g);
    }
}

RTCGeometry rtcNewGeometry(RTCDevice device, enum RTCGeometryType type)
{
    (void)device;
    if (type != RTC_GEOMETRY_TYPE_TRIANGLE) return NULL;
    RTCGeometry g = calloc(1, sizeof(struct RTCGeometryTy));
    if (g) g->refs = 1;
    return g;
}

void *rtcSetNewGeometryBuffer(RTCGeometry g, enum RTCBufferType type, unsigned int slot,
                              enum RTCFormat format, size_t byte_stride, size_t item_count)
{
    if (!g || slot != 0) return NULL;
    if (type == RTC_BUFFER_TYPE_VERTEX && format == RTC_FORMAT_FLOAT3 && byte_stride == 3 * sizeof(float)) {
        free(g->verts);
        g->verts = calloc(3 * item_count + 1, sizeof(float));
        g->nvert = item_count;
        return g->verts;
    }
    if (type == RTC_BUFFER_TYPE_INDEX && format == RTC_FORMAT_UINT3 && byte_stride == 3 * sizeof(unsigned)) {
        free(g->index);
        g->index = calloc(3 * item_count + 1, sizeof(unsigned));
        g->ntri = item_count;
        return g->index;
    }
    return NULL;
}

void rtcCommitGeometry(RTCGeometry geometry) { (void)geometry; }

unsigned int rtcAttachGeometry(RTCScene scene, RTCGeometry g)
{
    if (scene && g && !scene->geom) {
        g->refs++;
        scene->geom = g;
    }
    return 0;
}

void rtcReleaseGeometry(RTCGeometry geometry) { geometry_release(geometry); }

void rtcCommitScene(RTCScene scene)
{
    if (!scene || !scene->geom) return;
    const RTCGeometry g = scene->geom;
    free(scene->tri);
    scene->tri = malloc(sizeof(float) * 9 * (g->ntri ? g->ntri : 1));
    scene->ntri = scene->tri ? g->ntri : 0;
    for (size_t f = 0; f < scene->ntri; f++) {
        const float *v[3];
        for (int j = 0; j < 3; j++) {
            const unsigned k = g->index[3 * f + j];
            v[j] = g->verts + 3 * (k < g->nvert ? k : 0);
        }
        for (int k = 0; k < 3; k++) {
            scene->tri[9 * f + k] = v[0][k];
            scene->tri[9 * f + 3 + k] = v[1][k] - v[0][k];
            scene->tri[9 * f + 6 + k] = v[2][k] - v[0][k];
        }
    }
}

void rtcReleaseScene(RTCScene scene)
{
    if (!scene) return;
    geometry_release(scene->geom);
    free(scene->tri);
    free(scene);
}

void rtcInitOccludedArguments(struct RTCOccludedArguments *args)
{
    if (args) memset(args, 0, sizeof(*args));
}

/* Moller-Trumbore in FP32; hit when the distance lies in [t0, t1]. */
static int hit(const float o[3], const float d[3], const float *tri, float t0, float t1)
{
    const float *v0 = tri, *e1 = tri + 3, *e2 = tri + 6;
    const float px = d[1] * e2[2] - d[2] * e2[1], py = d[2] * e2[0] - d[0] * e2[2],
                pz = d[0] * e2[1] - d[1] * e2[0];
    const float det = e1[0] * px + e1[1] * py + e1[2] * pz;
    if (det == 0.0f) return 0;
    const float inv = 1.0f / det;
    const float sx = o[0] - v0[0], sy = o[1] - v0[1], sz = o[2] - v0[2];
    const float u = (sx * px + sy * py + sz * pz) * inv;
    if (u < 0.0f || u > 1.0f) return 0;
    const float qx = sy * e1[2] - sz * e1[1], qy = sz * e1[0] - sx * e1[2], qz = sx * e1[1] - sy * e1[0];
    const float v = (d[0] * qx + d[1] * qy + d[2] * qz) * inv;
    if (v < 0.0f || u + v > 1.0f) return 0;
    const float t = (e2[0] * qx + e2[1] * qy + e2[2] * qz) * inv;
    return t >= t0 && t <= t1;
}

void rtcOccluded1(RTCScene scene, struct RTCRay *ray, struct RTCOccludedArguments *args)
{
    (void)args;
    if (!scene || !ray) return;
    const float o[3] = {ray->org_x, ray->org_y, ray->org_z};
    const float d[3] = {ray->dir_x, ray->dir_y, ray->dir_z};
    for (size_t f = 0; f < scene->ntri; f++)
        if (hit(o, d, scene->tri + 9 * f, ray->tnear, ray->tfar)) {
            ray->tfar = -INFINITY;
            return;
        }
}
