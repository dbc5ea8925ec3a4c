/* host_raytrace.c - drop-in mesh_load / mesh_free / mesh_compute_normals /
 * random_point_on_triangle / run_raytracer (signatures of the reference's include/raytracer.h)
 * on top of the C ABI: the shadow rays are traced on the GPU (dsmc_shadow_flux_host); mesh I/O,
 * normals and the flux file contract are the reference's (src/raytracer/shadow_maker.c:23-118,
 * 242-271; src/common/fileio.c:188-203). nthreads is accepted for the signature. */
#include "dsmc_cuda.h"
#include "fileio.h"
#include "raytracer.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

Mesh *mesh_load(const char *vertex_file, const char *face_file, int npoint, int nface)
{
    Mesh *m = calloc(1, sizeof *m);
    if (!m) return NULL;
    m->npoint = npoint;
    m->nface = nface;
    m->spot = calloc((size_t)npoint, sizeof *m->spot);
    m->facet = calloc((size_t)nface, sizeof *m->facet);
    m->face_normal = calloc((size_t)nface, sizeof *m->face_normal);
    m->face_area = calloc((size_t)nface, sizeof *m->face_area);
    m->loc_xyz = calloc((size_t)nface, sizeof *m->loc_xyz);
    m->dir = calloc((size_t)nface, sizeof *m->dir);
    FILE *fp = fopen(vertex_file, "r");
    if (!fp) { fprintf(stderr, "Cannot open %s\n", vertex_file); return m; }
    for (int i = 0; i < npoint; i++)
        if (fscanf(fp, "%lf %lf %lf", &m->spot[i][0], &m->spot[i][1], &m->spot[i][2]) != 3) break;
    fclose(fp);
    fp = fopen(face_file, "r");
    if (!fp) { fprintf(stderr, "Cannot open %s\n", face_file); return m; }
    for (int i = 0; i < nface; i++) {
        if (fscanf(fp, "%d %d %d", &m->facet[i][0], &m->facet[i][1], &m->facet[i][2]) != 3) break;
        for (int j = 0; j < 3; j++) m->facet[i][j]--;   /* files are 1-based */
    }
    fclose(fp);
    return m;
}

void mesh_free(Mesh *m)
{
    if (!m) return;
    free(m->spot);
    free(m->facet);
    free(m->face_normal);
    free(m->face_area);
    free(m->loc_xyz);
    free(m->dir);
    free(m);
}

static Vec3 vertex(const Mesh *m, int f, int j)
{
    const double *p = m->spot[m->facet[f][j]];
    Vec3 v = {p[0], p[1], p[2]};
    return v;
}

void mesh_compute_normals(Mesh *m)
{
    for (int f = 0; f < m->nface; f++) {
        const Vec3 a = vertex(m, f, 0), b = vertex(m, f, 1), c = vertex(m, f, 2);
        m->loc_xyz[f][0] = (a.x + b.x + c.x) / 3.0;
        m->loc_xyz[f][1] = (a.y + b.y + c.y) / 3.0;
        m->loc_xyz[f][2] = (a.z + b.z + c.z) / 3.0;
        const Vec3 ab = vec3_sub(b, a), ac = vec3_sub(c, a);
        m->face_area[f] = vec3_len(vec3_cross(ab, ac)) / 2.0;
        /* unit normal from the normalised edges, turned away from the body centre */
        Vec3 n = vec3_normalize(vec3_cross(vec3_normalize(ac), vec3_normalize(ab)));
        const Vec3 centroid = {m->loc_xyz[f][0], m->loc_xyz[f][1], m->loc_xyz[f][2]};
        if (vec3_dot(n, centroid) < 0) n = vec3_scale(n, -1.0);
        m->face_normal[f][0] = n.x;
        m->face_normal[f][1] = n.y;
        m->face_normal[f][2] = n.z;
        double lon = atan2(n.x, n.y);
        if (lon < 0) lon += 2.0 * M_PI;
        m->dir[f][0] = asin(n.z);
        m->dir[f][1] = lon;
    }
}

Vec3 random_point_on_triangle(Vec3 a, Vec3 b, Vec3 c, unsigned int *seed)
{
    const double r1 = sqrt((double)rand_r(seed) / RAND_MAX);
    const double r2 = (double)rand_r(seed) / RAND_MAX;
    return vec3_add(vec3_add(vec3_scale(a, 1.0 - r1), vec3_scale(b, r1 * (1.0 - r2))),
                    vec3_scale(c, r1 * r2));
}

void run_raytracer(const char *mesh_vertex_file, const char *mesh_face_file, int npoint, int nface,
                   double za_deg, int tt, int Nmonte, const char *output_file, int nthreads)
{
    (void)nthreads;
    printf("Loading mesh: %d vertices, %d faces\n", npoint, nface);
    Mesh *m = mesh_load(mesh_vertex_file, mesh_face_file, npoint, nface);
    if (!m) { fprintf(stderr, "out of host memory\n"); return; }
    mesh_compute_normals(m);
    dsmc_ctx *ctx = NULL;
    const char *dev = getenv("DSMC_DEVICE");
    int rc = dsmc_ctx_create(dev && *dev ? atoi(dev) : 0, &ctx);
    double *F = calloc((size_t)nface * (size_t)(tt > 0 ? tt : 1), sizeof(double));
    if (rc != DSMC_OK || !F) {
        fprintf(stderr, "dsmc_ctx_create failed: %s (%s)\n", dsmc_status_string(rc), dsmc_last_error(NULL));
        free(F);
        if (ctx) dsmc_ctx_destroy(ctx);
        mesh_free(m);
        return;
    }
    printf("Computing flux with %d MC samples (GPU BVH)...\n", Nmonte);
    rc = dsmc_shadow_flux_host(ctx, npoint, &m->spot[0][0], nface, &m->facet[0][0],
                               &m->face_normal[0][0], za_deg / 180.0 * M_PI, tt, Nmonte, F);
    if (rc != DSMC_OK) {
        fprintf(stderr, "dsmc_shadow_flux_host failed: %s (%s)\n", dsmc_status_string(rc),
                dsmc_last_error(ctx));
    } else if (write_flux_dat(output_file, F, nface, tt) == 0) {
        printf("Flux written to %s\n", output_file);
    }
    free(F);
    dsmc_ctx_destroy(ctx);
    mesh_free(m);
}
