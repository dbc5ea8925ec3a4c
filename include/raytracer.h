/* raytracer.h - Monte Carlo shadow flux of a body mesh (the step before the thermal model).
 *
 * Kept interface of the reference (include/raytracer.h of rubby0605/dsmc_suite): same names and
 * signatures, so code written against the reference links against this library. The reference
 * traces its shadow rays with Intel Embree on the CPU; here run_raytracer traces them on the GPU
 * through a BVH of the mesh (dsmc_shadow_flux_host in dsmc_cuda.h). nthreads is accepted and
 * ignored.
 */
#ifndef RAYTRACER_H
#define RAYTRACER_H

#include "types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Body mesh from a vertex file (npoint lines "x y z") and a face file (nface lines "i j k",
 * 1-based vertex indices). */
Mesh *mesh_load(const char *vertex_file, const char *face_file, int npoint, int nface);
void mesh_free(Mesh *m);

/* Face centroids, areas, outward unit normals and normal directions (latitude, longitude). */
void mesh_compute_normals(Mesh *m);

/* Point of triangle (a, b, c) from two rand_r draws: (1 - r1) a + r1 (1 - r2) b + r1 r2 c with
 * r1 = sqrt(u1), r2 = u2. */
Vec3 random_point_on_triangle(Vec3 a, Vec3 b, Vec3 c, unsigned int *seed);

/* Flux factor of every face at tt rotation phases (sun at declination -za_deg), each the cosine
 * of the solar incidence times the unshadowed fraction of Nmonte random points of the face;
 * written as a flux file (nface, tt, then nface x tt values). */
void run_raytracer(const char *mesh_vertex_file, const char *mesh_face_file, int npoint, int nface,
                   double za_deg, int tt, int Nmonte, const char *output_file, int nthreads);

#ifdef __cplusplus
}
#endif
#endif /* RAYTRACER_H */
