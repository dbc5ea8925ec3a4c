/* Test infrastructure: link stub for the reference build in oracle/_ref.
 *
 * The reference's MC shadow ray tracer (src/raytracer/shadow_maker.c) needs Embree 4, which is
 * not installed, and it is not on the DSMC path. Its one entry point, declared in
 * include/raytracer.h:19-21, is replaced by this stub so that src/main.c links. */
#include <stdio.h>

void run_raytracer(const char *vertex_file, const char *face_file, int npoint, int nface,
                   double za_deg, int tt, int nmonte, const char *flux_file, int nthreads)
{
    (void)vertex_file; (void)face_file; (void)npoint; (void)nface;
    (void)za_deg; (void)tt; (void)nmonte; (void)flux_file; (void)nthreads;
    fprintf(stderr, "raytrace: not built (needs Embree)\n");
}
