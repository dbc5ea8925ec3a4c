/* host_thermal.c - drop-in thermal_params_default / thermal_solve (signatures of the reference's
 * include/thermal.h:23-30) on top of the C ABI: the column model runs on the GPU
 * (dsmc_thermal_solve_host); the console lines and the output contract are the reference's
 * (src/thermal/thermal_model.c:126, 184, 281). nthreads is accepted for the signature. */
#include "constants.h"
#include "dsmc_cuda.h"
#include "thermal.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

void thermal_params_default(ThermalParams *tp)
{
    /* Ceres regolith and the H2O Antoine / latent-heat coefficients
     * (src/thermal/thermal_model.c:22-48) */
    const ThermalParams d = {
        .density = 730.0, .conductivity = 6e-4, .Cp = 1300.0, .albedo = 0.02,
        .distance_AU = 2.6, .depth = 0.05, .n_substep = 5, .z_angle = 12.3 / 180.0 * M_PI,
        .p_mat = {-2445.5646, -6.757169, -0.01677006, 1.20514e-5, 8.2312},
        .LH_mat = {0.0, 12420.0, -4.8, 0.0, 0.0},
        .tran_unit_p = 133.32237, .tran_unit_LH = 4.2,
    };
    *tp = d;
}

void thermal_solve(SphericalGrid *grid, const ThermalParams *tp, const double *flux, int nthreads)
{
    (void)nthreads;
    if (!grid || !tp || !grid->temperature) {
        fprintf(stderr, "thermal_solve: grid with a temperature array and parameters required\n");
        return;
    }
    const double dt = CONST_P_CERES / grid->ffd / tp->n_substep;
    const double dr = sqrt(0.1 * 2.0 * dt * tp->conductivity / tp->density / tp->Cp);
    /* the reference's interface has no status: a failed solve leaves NaN temperatures */
    for (int k = 0; k < grid->ftd * grid->ffd; k++) grid->temperature[k] = NAN;
    dsmc_ctx *ctx = NULL;
    const char *dev = getenv("DSMC_DEVICE");
    int rc = dsmc_ctx_create(dev && *dev ? atoi(dev) : 0, &ctx);
    if (rc != DSMC_OK) {
        fprintf(stderr, "dsmc_ctx_create failed: %s (%s)\n", dsmc_status_string(rc), dsmc_last_error(NULL));
        return;
    }
    int h = 0;
    const int h_est = (int)ceil(tp->depth / dr);
    printf("Thermal model: dr=%.6f m, depth points=%d\n", dr, h_est < 3 ? 3 : h_est);
    printf("Running thermal diffusion...\n");
    rc = dsmc_thermal_solve_host(ctx, grid->ftd, grid->ffd, tp, flux, grid->temperature, &h);
    if (rc != DSMC_OK) {
        fprintf(stderr, "dsmc_thermal_solve_host failed: %s (%s)\n", dsmc_status_string(rc),
                dsmc_last_error(ctx));
        for (int k = 0; k < grid->ftd * grid->ffd; k++) grid->temperature[k] = NAN;
    } else
        printf("Thermal model done.\n");
    dsmc_ctx_destroy(ctx);
}
