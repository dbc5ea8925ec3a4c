/* raytrace_oracle.c - CPU oracle of the Monte Carlo shadow flux - TEST INFRASTRUCTURE ONLY.
 *
 * Checker for dsmc_shadow_flux_host; nothing in the product links it. Restates the flux loop of
 * the reference's ray tracer (rubby0605/dsmc_suite, src/raytracer/shadow_maker.c:198-238): sun
 * direction (cos(-za) sin(phi), cos(-za) cos(phi), sin(-za)) with phi = 2 pi (t + 1/2) / tt + pi;
 * zero flux where s . n < 0; Nmonte points per face from glibc rand_r seeded t * nface + f + 42
 * (r1 = sqrt(u1), r2 = u2, point (1 - r1) a + r1 (1 - r2) b + r1 r2 c, :120-128); FP32 rays from
 * the point lifted 1e-3 (a float) along n toward s, t in [0, 1e30] (:171-196).
 *
 * The reference finds hits with Intel Embree, which is not installed here, so parity of the
 * occlusion test with Embree itself is unpinned: this oracle tests every triangle of the mesh
 * (no acceleration structure) with the Moller-Trumbore algorithm in FP32, the test the GPU runs
 * inside its BVH leaves; the sampling and flux arithmetic follow the reference exactly.
 */
#include "dsmc_oracle.h"

#include <math.h>
#include <stdlib.h>

static int mt_hit(const float o[3], const float d[3], const float v0[3], const float e1[3],
                  const float e2[3])
{
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
    return t >= 0.0f && t <= 1e30f;
}

int or_shadow_flux(int npoint, const double *spot, int nface, const int32_t *facet,
                   const double *normal, double za, int tt, int nmonte, double *F, int nthreads)
{
    if (npoint < 3 || nface < 1 || tt < 1 || nmonte < 1 || !spot || !facet || !normal || !F)
        return -1;
    float *tri = malloc(sizeof(float) * 9 * (size_t)nface);   /* v0, e1, e2 per face */
    if (!tri) return -2;
    for (int f = 0; f < nface; f++) {
        float v[3][3];
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) v[j][k] = (float)spot[3 * facet[3 * f + j] + k];
        for (int k = 0; k < 3; k++) {
            tri[9 * f + k] = v[0][k];
            tri[9 * f + 3 + k] = v[1][k] - v[0][k];
            tri[9 * f + 6 + k] = v[2][k] - v[0][k];
        }
    }
    #pragma omp parallel for collapse(2) num_threads(nthreads) schedule(dynamic)
    for (int t = 0; t < tt; t++) {
        for (int f = 0; f < nface; f++) {
            const double phi = ((t + 0.5) / tt) * 2.0 * M_PI + M_PI;
            const double s[3] = {cos(-za) * sin(phi), cos(-za) * cos(phi), sin(-za)};
            const double *n = normal + 3 * f;
            const double c6 = s[0] * n[0] + s[1] * n[1] + s[2] * n[2];
            if (c6 < 0) { F[(size_t)f * tt + t] = 0.0; continue; }
            const double *a = spot + 3 * facet[3 * f], *b = spot + 3 * facet[3 * f + 1],
                         *c = spot + 3 * facet[3 * f + 2];
            const float d[3] = {(float)s[0], (float)s[1], (float)s[2]};
            const float lift = 1e-3f;
            unsigned int seed = (unsigned int)(t * nface + f + 42);
            int dark = 0;
            for (int m = 0; m < nmonte; m++) {
                const double r1 = sqrt((double)rand_r(&seed) / RAND_MAX);
                const double r2 = (double)rand_r(&seed) / RAND_MAX;
                float o[3];
                for (int k = 0; k < 3; k++) {
                    const double p = a[k] * (1.0 - r1) + b[k] * (r1 * (1.0 - r2)) + c[k] * (r1 * r2);
                    o[k] = (float)(p + lift * n[k]);
                }
                int hit = 0;
                for (int g = 0; g < nface && !hit; g++)
                    hit = mt_hit(o, d, tri + 9 * g, tri + 9 * g + 3, tri + 9 * g + 6);
                dark += hit;
            }
            F[(size_t)f * tt + t] = (1.0 - (double)dark / nmonte) * c6;
        }
    }
    free(tri);
    return 0;
}
