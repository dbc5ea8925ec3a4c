/* main.c - the dsmc_suite command line (flags and subcommands of the reference's
 * src/main.c:52-213). dsmc and dsmc-adv run on the GPU through the drop-in runners; pipeline
 * chains them through the same files as the reference (main.c:153-205). The thermal model and
 * the Embree ray tracer are not part of this build: thermal and raytrace report that and exit 1,
 * and pipeline needs an existing temperature file (-T). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dsmc_runners.h"

static void print_usage(const char *prog)
{
    printf("DSMC Suite - Planetary Atmosphere Simulation (CUDA, sm_100a)\n\n");
    printf("Usage: %s <command> [options]\n\n", prog);
    printf("Commands:\n");
    printf("  dsmc      - Basic ballistic DSMC (no collisions)\n");
    printf("  dsmc-adv  - Advanced DSMC with collisions\n");
    printf("  pipeline  - dsmc then dsmc-adv on the same temperature file\n\n");
    printf("Options:\n");
    printf("  -n <particles>     Number of test particles (default: 10000)\n");
    printf("  -t <threads>       Accepted for compatibility (the solve runs on one GPU)\n");
    printf("  -T <temp_file>     Temperature input file\n");
    printf("  -d <den_file>      Density input file (for dsmc-adv)\n");
    printf("  -v <v_record_file> Velocity record file (for dsmc-adv)\n");
    printf("  -o <output_prefix> Output file prefix (default: output)\n");
    printf("Environment: DSMC_DEVICE, DSMC_PATH (plain|fast32|fast64), DSMC_SEED\n");
}

int main(int argc, char *argv[])
{
    if (argc < 2) { print_usage(argv[0]); return 1; }
    const char *command = argv[1];
    int totaln = 10000, nthreads = 1;
    const char *temp_file = "Ceres_T_VP.dat", *den_file = NULL, *v_record_file = NULL;
    const char *output_prefix = "output";
    for (int i = 2; i < argc; i++) {
        const int more = i + 1 < argc;
        if (!strcmp(argv[i], "-n") && more) totaln = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-t") && more) nthreads = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-T") && more) temp_file = argv[++i];
        else if (!strcmp(argv[i], "-d") && more) den_file = argv[++i];
        else if (!strcmp(argv[i], "-v") && more) v_record_file = argv[++i];
        else if (!strcmp(argv[i], "-o") && more) output_prefix = argv[++i];
        else if ((!strcmp(argv[i], "-m") || !strcmp(argv[i], "-f") || !strcmp(argv[i], "--npoint") ||
                  !strcmp(argv[i], "--nface") || !strcmp(argv[i], "--za") ||
                  !strcmp(argv[i], "--tt") || !strcmp(argv[i], "--nmonte")) && more)
            ++i;   /* ray-tracer and thermal flags: accepted and ignored */
    }
    if (!strcmp(command, "dsmc")) {
        run_ballistic(totaln, temp_file, output_prefix, nthreads);
    } else if (!strcmp(command, "dsmc-adv")) {
        run_advanced(totaln, temp_file, den_file, v_record_file, output_prefix, nthreads);
    } else if (!strcmp(command, "pipeline")) {
        char p1[1024], p2[1024], den[1100], vr[1100];
        snprintf(p1, sizeof p1, "%s_phase1", output_prefix);
        snprintf(p2, sizeof p2, "%s_phase2", output_prefix);
        snprintf(den, sizeof den, "%s_den.dat", p1);
        snprintf(vr, sizeof vr, "%s_v_record.dat", p1);
        printf("=== PIPELINE (phases 3-4) ===\n\n--- Basic DSMC ---\n");
        run_ballistic(totaln, temp_file, p1, nthreads);
        printf("\n--- Advanced DSMC ---\n");
        run_advanced(totaln, temp_file, den, vr, p2, nthreads);
        printf("\n=== PIPELINE COMPLETE ===\n");
    } else if (!strcmp(command, "thermal") || !strcmp(command, "raytrace")) {
        fprintf(stderr, "%s: not part of this build (the DSMC hot path only)\n", command);
        return 1;
    } else {
        fprintf(stderr, "Unknown command: %s\n", command);
        print_usage(argv[0]);
        return 1;
    }
    return 0;
}
