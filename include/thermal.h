/* thermal.h - the thermal model that produces the surface temperature map of the DSMC phases.
 *
 * Kept interface of the reference (include/thermal.h:6-30 of rubby0605/dsmc_suite): same struct
 * layout, same function names and signatures, so code written against the reference links
 * against this library. Here thermal_solve runs every surface column on the GPU
 * (dsmc_thermal_solve_host in dsmc_cuda.h); nthreads is accepted and ignored.
 */
#ifndef THERMAL_H
#define THERMAL_H

#include "types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Regolith, orbit and sublimation parameters of the 1-D column model. */
typedef struct {
    double density;       /* regolith bulk density [kg/m^3] */
    double conductivity;  /* thermal conductivity [W/m/K] */
    double Cp;            /* specific heat [J/kg/K] */
    double albedo;        /* Bond albedo */
    double distance_AU;   /* heliocentric distance [AU] */
    double depth;         /* depth of the column [m] */
    int n_substep;        /* time steps per rotation step (P / ffd) */
    double z_angle;       /* obliquity [rad] (carried, not used by the column model) */
    double p_mat[5];      /* H2O vapour pressure: log10 p[Torr] = p0/T + p1 + p2 T + p3 T^2 + p4 log10 T */
    double LH_mat[5];     /* latent heat [cal/mol-like units], same form as p_mat */
    double tran_unit_p;   /* Torr -> Pa */
    double tran_unit_LH;  /* cal -> J */
} ThermalParams;

/* Ceres defaults of the reference (src/thermal/thermal_model.c:22-48). */
void thermal_params_default(ThermalParams *tp);

/* Surface temperature of every (td, fd) cell into grid->temperature [ftd][ffd]. flux [ftd][ffd]
 * is the absorbed solar flux per cell [W/m^2]; NULL uses the reference's analytic flux (sub-solar
 * longitude pi/2, night side for longitudes >= pi). */
void thermal_solve(SphericalGrid *grid, const ThermalParams *tp, const double *flux, int nthreads);

#ifdef __cplusplus
}
#endif
#endif /* THERMAL_H */
