/* host_density.c - FP64 normalisation of the deposited grids into number density.
 *
 * The reference's runners write raw weight sums per cell (src/dsmc/ballistic.c:235-236,
 * src/dsmc/advanced.c:401-402) and never divide by the cell volumes they compute
 * (src/common/grid.c:41-84). Here the fixed-point sums the kernels return become molecules per
 * m^3 in FP64 on the host: each of the n test particles stands for production_rate / n
 * molecules/s, one deposited weight-step is dt seconds of residence, so
 *     n_den = (fx / 2^24) * (production_rate / n) * dt / V_cell.
 * Two cell-volume conventions: the physical spherical-shell volume (r_o^3 - r^3) / 3 * dphi *
 * |sin b_o - sin b| (shell radii r_j = R + j unih, or R + unih ((1 + a2)^j - 1) / a2 for the
 * exponential grid), or the reference's own grid_compute_volume_uniform / _exp formula, which
 * adds the cubes (grid.c:41-84) - kept for callers that compare with tools built on it. */
#include "dsmc_cuda.h"
#include "grid.h"

#include <math.h>
#include <stdlib.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static int check_grid(const dsmc_params *p)
{
    if (!p || p->ftd < 1 || p->ffd < 1 || p->hd < 1 || !(p->Radii > 0.0) || !(p->unih > 0.0))
        return DSMC_ERR_INVALID;
    if (p->use_exp_grid && !(p->alpha2 > 0.0)) return DSMC_ERR_INVALID;
    return DSMC_OK;
}

int dsmc_cell_volumes(const dsmc_params *p, int volume_mode, double *vol)
{
    if (check_grid(p) != DSMC_OK || !vol) return DSMC_ERR_INVALID;
    const int ftd = p->ftd, ffd = p->ffd, hd = p->hd;
    if (volume_mode == DSMC_VOLUME_REFERENCE) {
        SphericalGrid g = {ftd, ffd, hd, NULL, NULL, vol, NULL};
        if (p->use_exp_grid) grid_compute_volume_exp(&g, p->Radii, p->unih, p->alpha2);
        else grid_compute_volume_uniform(&g, p->Radii, p->unih);
        return DSMC_OK;
    }
    if (volume_mode != DSMC_VOLUME_PHYSICAL) return DSMC_ERR_INVALID;
    const double dphi = 2.0 * M_PI / ffd;
    for (int ht = 0; ht < hd; ht++) {
        const double r0 = p->use_exp_grid
                              ? p->Radii + p->unih * (pow(1.0 + p->alpha2, ht) - 1.0) / p->alpha2
                              : p->Radii + ht * p->unih;
        const double r1 = p->use_exp_grid
                              ? p->Radii + p->unih * (pow(1.0 + p->alpha2, ht + 1) - 1.0) / p->alpha2
                              : p->Radii + (ht + 1) * p->unih;
        const double dr3 = (r1 * r1 * r1 - r0 * r0 * r0) / 3.0;
        for (int td = 0; td < ftd; td++) {
            const double b0 = (double)td / ftd * M_PI - M_PI / 2.0;
            const double b1 = (double)(td + 1) / ftd * M_PI - M_PI / 2.0;
            const double v = dr3 * fabs(sin(b1) - sin(b0)) * dphi;
            for (int fd = 0; fd < ffd; fd++) vol[((long)ht * ftd + td) * ffd + fd] = v;
        }
    }
    return DSMC_OK;
}

int dsmc_number_density_host(const dsmc_params *p, const uint64_t *density_fx, int64_t n,
                             double production_rate, int volume_mode, double *nden)
{
    if (check_grid(p) != DSMC_OK || !density_fx || !nden || n <= 0 ||
        !(production_rate >= 0.0) || !(p->dt_step > 0.0))
        return DSMC_ERR_INVALID;
    const long ncell = (long)p->hd * p->ftd * p->ffd;
    int rc = dsmc_cell_volumes(p, volume_mode, nden);
    if (rc != DSMC_OK) return rc;
    const double per_weight_step = production_rate / (double)n * p->dt_step / DSMC_FIXED_SCALE;
    for (long i = 0; i < ncell; i++) nden[i] = (double)density_fx[i] * per_weight_step / nden[i];
    return DSMC_OK;
}
