/* thermal_oracle.c - CPU oracle of the thermal column model - TEST INFRASTRUCTURE ONLY.
 *
 * Checker for dsmc_thermal_solve_host; nothing in the product links it. Restates the column
 * model of the reference's thermal_solve (rubby0605/dsmc_suite, src/thermal/thermal_model.c):
 *   - scalars dt = P / ffd / n_sub, dr = sqrt(0.2 dt k / rho / Cp), depth points
 *     max(3, ceil(depth / dr)), R = k dt / rho / 2 / Cp / dr^2 (:110-127);
 *   - absorbed flux: given, or dF cos(lat) sin(lon) on longitudes below pi, 0 beyond (:130-148);
 *   - initial profile (|F| / sigma)^(1/4), or 100 K where |F| = 0 (:172-181);
 *   - per column and step: bisection of the surface energy balance on [50, 300] K with the upper
 *     end growing x5 while both ends have one sign, bracket <= 0.01 K, at most 30 passes
 *     (:196-221, balance :50-77); then one implicit step: identity first row, CN interior rows
 *     -R, 1 + 2R, -R against R T_(i-1) + (1 - 2R) T_i + R T_(i+1), bottom row (-1/dr, 1/dr) = 0
 *     (:223-246), solved by the Thomas algorithm (:80-103).
 * Same FP64 operation order, glibc math; pinned bit for bit against the reference's own
 * thermal_solve built in oracle/_ref (tests/test_oracle_golden.py).
 */
#include "dsmc_oracle.h"

#include <math.h>
#include <stdlib.h>

#include "../include/constants.h"

static double vapour_pressure(const ThermalParams *tp, double T)
{
    const double e = tp->p_mat[0] / T + tp->p_mat[1] + tp->p_mat[2] * T + tp->p_mat[3] * T * T +
                     tp->p_mat[4] * log10(T);
    return tp->tran_unit_p * pow(10.0, e);
}

static double latent(const ThermalParams *tp, double T)
{
    const double e = tp->LH_mat[0] / T + tp->LH_mat[1] + tp->LH_mat[2] * T +
                     tp->LH_mat[3] * T * T + tp->LH_mat[4] * log10(T);
    return tp->tran_unit_LH * e;
}

static double balance(const ThermalParams *tp, double T, double F, double kdr, double T_below)
{
    const double mm = CONST_MMOL_H2O;
    const double loss = latent(tp, T) * sqrt(mm / (2.0 * M_PI * CONST_K_B * T)) *
                        vapour_pressure(tp, T);
    return F + kdr * T_below - kdr * T - CONST_SIGMA * T * T * T * T - loss;
}

int or_thermal_solve(int ftd, int ffd, const ThermalParams *tp, const double *flux,
                     double *T_out, int *h_depth)
{
    if (ftd < 1 || ffd < 1 || !tp || !T_out || tp->n_substep < 1) return -1;
    const double dt = CONST_P_CERES / ffd / tp->n_substep;
    const double dr = sqrt(0.1 * 2.0 * dt * tp->conductivity / tp->density / tp->Cp);
    int h = (int)ceil(tp->depth / dr);
    if (h < 3) h = 3;
    if (h_depth) *h_depth = h;
    const double R = tp->conductivity * dt / tp->density / 2.0 / tp->Cp / (dr * dr);
    const double kdr = tp->conductivity / dr;
    const double dF = CONST_SOLAR_1AU * (1.0 / tp->distance_AU) * (1.0 / tp->distance_AU) *
                      (1.0 - tp->albedo);
    double *col = malloc(sizeof(double) * (size_t)h * 4);
    if (!col) return -2;
    double *x = col, *rhs = col + h, *cp = col + 2 * h, *dp = col + 3 * h;
    for (int td = 0; td < ftd; td++) {
        for (int fd = 0; fd < ffd; fd++) {
            double F;
            if (flux) {
                F = fabs(flux[td * ffd + fd]);
            } else {
                const double lat = (td + 0.5) / ftd * M_PI - M_PI / 2.0;
                const double lon = (fd + 0.5) / ffd * 2.0 * M_PI;
                F = fabs(lon >= M_PI ? 0.0 : dF * cos(lat) * sin(lon));
            }
            const double T_init = F > 0 ? pow(F / CONST_SIGMA, 0.25) : 100.0;
            for (int d = 0; d < h; d++) x[d] = T_init;
            for (int step = 0; step < tp->n_substep; step++) {
                const double below = x[1];
                double lo = 50.0, hi = 300.0;
                double flo = balance(tp, lo, F, kdr, below), fhi = balance(tp, hi, F, kdr, below);
                for (int pass = 0; pass < 30 && hi < 10000.0; pass++) {
                    if (flo * fhi > 0) {          /* no sign change yet: widen upwards */
                        hi *= 5.0;
                        fhi = balance(tp, hi, F, kdr, below);
                        continue;
                    }
                    const double mid = (lo + hi) / 2.0, fmid = balance(tp, mid, F, kdr, below);
                    if (flo * fmid <= 0) { hi = mid; fhi = fmid; }
                    else { lo = mid; flo = fmid; }
                    if (fabs(lo - hi) <= 0.01) break;
                }
                x[0] = (lo + hi) / 2.0;
                rhs[0] = x[0];
                for (int i = 1; i < h - 1; i++)
                    rhs[i] = R * x[i - 1] + (1.0 - 2.0 * R) * x[i] + R * x[i + 1];
                rhs[h - 1] = 0.0;
                /* Thomas: rows (a_i, b_i, c_i) = (0, 1, 0), (-R, 1 + 2R, -R)..., (-1/dr, 1/dr, 0) */
                cp[0] = 0.0 / 1.0;
                dp[0] = rhs[0] / 1.0;
                for (int i = 1; i < h; i++) {
                    const int last = i == h - 1;
                    const double a = last ? -1.0 / dr : -R, b = last ? 1.0 / dr : 1.0 + 2.0 * R;
                    const double c = last ? 0.0 : -R;
                    const double piv = b - a * cp[i - 1];
                    cp[i] = c / piv;
                    dp[i] = (rhs[i] - a * dp[i - 1]) / piv;
                }
                x[h - 1] = dp[h - 1];
                for (int i = h - 2; i >= 0; i--) x[i] = dp[i] - cp[i] * x[i + 1];
            }
            T_out[td * ffd + fd] = x[0];
        }
    }
    free(col);
    return 0;
}
