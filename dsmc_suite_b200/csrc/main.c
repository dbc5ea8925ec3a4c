/* main.c - the dsmc_suite command line (flags and subcommands of the reference's
 * src/main.c:52-213). dsmc, dsmc-adv and thermal run on the GPU through the drop-in runners and
 * thermal_solve, raytrace through run_raytracer (shadow rays on the GPU instead of Embree);
 * pipeline chains raytrace (when a mesh is given) -> thermal -> dsmc -> dsmc-adv through the same
 * files as the reference (main.c:153-205). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dsmc_runners.h"
#include "grid.h"
#include "raytracer.h"
#include "thermal.h"

/* thermal model on the 36 x 72 grid, written as <prefix>_temperature.dat (main.c:118-143) */
static int run_thermal(const char *output_prefix, const double *za_deg, int nthreads, char *t_file,
                       size_t t_len)
{
    const int ftd = 36, ffd = 72;
    SphericalGrid *grid = grid_create(ftd, ffd, 1);
    if (!grid) { fprintf(stderr, "out of host memory\n"); return 1; }
    ThermalParams tp;
    thermal_params_default(&tp);
    if (za_deg) tp.z_angle = *za_deg / 180.0 * M_PI;
    thermal_solve(grid, &tp, NULL, nthreads);
    if (isnan(grid->temperature[0])) { grid_free(grid); return 1; }   /* the solve failed */
    snprintf(t_file, t_len, "%s_temperature.dat", output_prefix);
    FILE *fp = fopen(t_file, "w");
    if (!fp) { fprintf(stderr, "cannot write %s\n", t_file); grid_free(grid); return 1; }
    fprintf(fp, "%d\n%d\n", ftd, ffd);
    for (int k = 0; k < ftd * ffd; k++) fprintf(fp, "%8.6f\n", grid->temperature[k]);
    fclose(fp);
    grid_free(grid);
    return 0;
}

static void print_usage(const char *prog)
{
    printf("DSMC Suite - Planetary Atmosphere Simulation (CUDA, sm_100a)\n\n");
    printf("Usage: %s <command> [options]\n\n", prog);
    printf("Commands:\n");
    printf("  dsmc      - Basic ballistic DSMC (no collisions)\n");
    printf("  dsmc-adv  - Advanced DSMC with collisions\n");
    printf("  raytrace  - MC shadow flux of a mesh (GPU BVH)\n");
    printf("  thermal   - 1D spherical thermal diffusion model (GPU)\n");
    printf("  pipeline  - thermal, then dsmc, then dsmc-adv\n\n");
    printf("Options:\n");
    printf("  -n <particles>     Number of test particles (default: 10000)\n");
    printf("  -t <threads>       Accepted for compatibility (the solve runs on one GPU)\n");
    printf("  -T <temp_file>     Temperature input file\n");
    printf("  -d <den_file>      Density input file (for dsmc-adv)\n");
    printf("  -v <v_record_file> Velocity record file (for dsmc-adv)\n");
    printf("  -o <output_prefix> Output file prefix (default: output)\n");
    printf("  --bin              Also write <prefix>_grids.bin (exact grids, FP64 rows)\n");
    printf("  --ndensity <Q>     Also write <prefix>_ndensity.dat: FP64 number density [m^-3]\n");
    printf("                     for a production rate of Q molecules/s\n");
    printf("Environment: DSMC_DEVICE, DSMC_PATH (plain|fast32|fast64), DSMC_SEED, DSMC_SIDECAR,\n");
    printf("             DSMC_NDENSITY_RATE\n");
}

int main(int argc, char *argv[])
{
    if (argc < 2) { print_usage(argv[0]); return 1; }
    const char *command = argv[1];
    int totaln = 10000, nthreads = 1;
    const char *temp_file = "Ceres_T_VP.dat", *den_file = NULL, *v_record_file = NULL;
    const char *output_prefix = "output";
    double za_deg = 12.3;
    const char *vertex_file = NULL, *face_file = NULL;
    int npoint = 0, nface_mesh = 0, tt = 24, nmonte = 50;
    for (int i = 2; i < argc; i++) {
        const int more = i + 1 < argc;
        if (!strcmp(argv[i], "-n") && more) totaln = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-t") && more) nthreads = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-T") && more) temp_file = argv[++i];
        else if (!strcmp(argv[i], "-d") && more) den_file = argv[++i];
        else if (!strcmp(argv[i], "-v") && more) v_record_file = argv[++i];
        else if (!strcmp(argv[i], "-o") && more) output_prefix = argv[++i];
        else if (!strcmp(argv[i], "--za") && more) za_deg = atof(argv[++i]);
        else if (!strcmp(argv[i], "-m") && more) vertex_file = argv[++i];
        else if (!strcmp(argv[i], "-f") && more) face_file = argv[++i];
        else if (!strcmp(argv[i], "--npoint") && more) npoint = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--nface") && more) nface_mesh = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--tt") && more) tt = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--nmonte") && more) nmonte = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--bin")) setenv("DSMC_SIDECAR", "1", 1);
        else if (!strcmp(argv[i], "--ndensity") && more) setenv("DSMC_NDENSITY_RATE", argv[++i], 1);
    }
    if (!strcmp(command, "dsmc")) {
        run_ballistic(totaln, temp_file, output_prefix, nthreads);
    } else if (!strcmp(command, "dsmc-adv")) {
        run_advanced(totaln, temp_file, den_file, v_record_file, output_prefix, nthreads);
    } else if (!strcmp(command, "thermal")) {
        char t_file[1100];
        if (run_thermal(output_prefix, &za_deg, nthreads, t_file, sizeof t_file)) return 1;
    } else if (!strcmp(command, "pipeline")) {
        char t_file[1100], p1[1024], p2[1024], den[1100], vr[1100];
        printf("=== FULL PIPELINE ===\n\n");
        if (vertex_file && face_file && npoint > 0 && nface_mesh > 0) {
            char flux_file[1100];
            snprintf(flux_file, sizeof flux_file, "%s_flux.dat", output_prefix);
            printf("--- Step 1: Ray Tracing ---\n");
            run_raytracer(vertex_file, face_file, npoint, nface_mesh, za_deg, tt, nmonte, flux_file,
                          nthreads);
        } else {
            printf("--- Step 1: Skipped (no mesh provided) ---\n");
        }
        printf("\n--- Step 2: Thermal Model ---\n");
        if (run_thermal(output_prefix, NULL, nthreads, t_file, sizeof t_file)) return 1;
        snprintf(p1, sizeof p1, "%s_phase1", output_prefix);
        snprintf(p2, sizeof p2, "%s_phase2", output_prefix);
        snprintf(den, sizeof den, "%s_den.dat", p1);
        snprintf(vr, sizeof vr, "%s_v_record.dat", p1);
        printf("\n--- Step 3: Basic DSMC ---\n");
        run_ballistic(totaln, t_file, p1, nthreads);
        printf("\n--- Step 4: Advanced DSMC ---\n");
        run_advanced(totaln, t_file, den, vr, p2, nthreads);
        printf("\n=== PIPELINE COMPLETE ===\n");
    } else if (!strcmp(command, "raytrace")) {
        if (!vertex_file || !face_file || npoint <= 0 || nface_mesh <= 0) {
            fprintf(stderr, "raytrace requires -m <vertex_file> -f <face_file> --npoint <n> --nface <n>\n");
            return 1;
        }
        char flux_file[1100];
        snprintf(flux_file, sizeof flux_file, "%s_flux.dat", output_prefix);
        run_raytracer(vertex_file, face_file, npoint, nface_mesh, za_deg, tt, nmonte, flux_file,
                      nthreads);
    } else {
        fprintf(stderr, "Unknown command: %s\n", command);
        print_usage(argv[0]);
        return 1;
    }
    return 0;
}
