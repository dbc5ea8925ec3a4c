// kernel_thermal.cu - the thermal model that feeds the DSMC phases (src/thermal/thermal_model.c
// of the reference), one GPU thread per surface column. Compiled with -fmad=false: the column
// arithmetic follows the reference's FP64 operation order, so the Crank-Nicolson steps and the
// Thomas sweeps are bit-identical to the CPU's; only CUDA's log10 / pow / sqrt inside the surface
// energy balance may round differently in the last place from glibc's.
//
// Per column (td, fd), each of n_sub time steps (thermal_model.c:196-254):
//   1. surface temperature by bisection of the energy balance
//        F + k/dr T_1 - k/dr T - sigma T^4 - L(T) sqrt(m / (2 pi k_B T)) p(T) = 0
//      on [50, 300] K, the upper end growing x5 while both ends have one sign, until the bracket
//      is within 0.01 K (at most 30 iterations);
//   2. one implicit (Crank-Nicolson) diffusion step with the surface fixed and a zero-flux
//      bottom, by the Thomas algorithm.
// Layout: the depth profiles are [depth][column] in device memory, so the threads of a warp
// (adjacent columns) read and write each depth level together. The coefficients of the
// tridiagonal system are the same for every column and step, so the forward-sweep terms that
// depend on them alone (c'_i and the pivots) come from the host.
#include "dsmc_kernels.h"

#include <cmath>

namespace dsmc {
namespace {

struct ThermalArgs {
    int ncol, h, n_sub;
    double R, k_over_dr, a_last;     // CN weight, k/dr, lower coefficient of the bottom row
    double p[5], LH[5], tran_p, tran_LH, mmol;
    const double *flux;              // [ncol] absorbed flux |F|
    const double *T_init;            // [ncol] initial column temperature
    const double *cp, *piv;          // [h] forward-sweep c'_i and pivots b_i - a_i c'_(i-1)
    double *qT, *dp;                 // [h][ncol] profiles and forward-sweep d'_i
    double *T_surface;               // [ncol]
};

__device__ double surface_balance(const ThermalArgs &a, double T, double F, double oT) {
    const double log10_p = a.p[0] / T + a.p[1] + a.p[2] * T + a.p[3] * T * T + a.p[4] * log10(T);
    const double pres = a.tran_p * pow(10.0, log10_p);
    const double LH = a.tran_LH * (a.LH[0] / T + a.LH[1] + a.LH[2] * T + a.LH[3] * T * T +
                                   a.LH[4] * log10(T));
    constexpr double kSigma = 5.6704e-8, kKB = 1.38e-23, kPi = 3.14159265358979323846;
    const double sublim = LH * sqrt(a.mmol / (2.0 * kPi * kKB * T)) * pres;
    return F + a.k_over_dr * oT - a.k_over_dr * T - kSigma * T * T * T * T - sublim;
}

__global__ void thermal_column_kernel(const ThermalArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.ncol) return;
    const int h = a.h;
    const long long n = a.ncol;
    double *qT = a.qT + c, *dp = a.dp + c;   // element d at [d * n]
    const double F = a.flux[c];
    const double R = a.R, w0 = 1.0 - 2.0 * R;
    const double T_init = a.T_init[c];
    for (int d = 0; d < h; d++) qT[d * n] = T_init;
    for (int step = 0; step < a.n_sub; step++) {
        const double oT = qT[1 * n];
        double T0 = 50.0, T1 = 300.0;
        double f0 = surface_balance(a, T0, F, oT), f1 = surface_balance(a, T1, F, oT);
        for (int m = 0; m < 30; m++) {
            if (T1 >= 10000.0) break;
            if (f0 * f1 > 0) {
                T1 *= 5.0;
                f1 = surface_balance(a, T1, F, oT);
                continue;
            }
            const double T2 = (T0 + T1) / 2.0;
            const double f2 = surface_balance(a, T2, F, oT);
            if (f0 * f2 <= 0) { T1 = T2; f1 = f2; }
            else { T0 = T2; f0 = f2; }
            if (fabs(T0 - T1) <= 0.01) break;
        }
        const double Ts = (T0 + T1) / 2.0;
        // forward sweep with the right-hand side built on the fly from the old profile:
        // d_0 = Ts (row 0 is the identity), d_i = R T_(i-1) + (1 - 2R) T_i + R T_(i+1), d_(h-1) = 0
        double prev_old = Ts, cur_old = qT[1 * n];   // the old T_0 is replaced by Ts first
        double dprev = Ts;                          // d'_0 = d_0 / b_0 with b_0 = 1
        dp[0] = dprev;
        for (int i = 1; i < h - 1; i++) {
            const double next_old = qT[(i + 1) * n];
            const double d = R * prev_old + w0 * cur_old + R * next_old;
            dprev = (d - (-R) * dprev) / a.piv[i];
            dp[i * n] = dprev;
            prev_old = cur_old;
            cur_old = next_old;
        }
        dprev = (0.0 - a.a_last * dprev) / a.piv[h - 1];
        // back substitution, overwriting the profile
        double x = dprev;
        qT[(h - 1) * n] = x;
        for (int i = h - 2; i >= 0; i--) {
            x = dp[i * n] - a.cp[i] * x;
            qT[i * n] = x;
        }
    }
    a.T_surface[c] = qT[0];
}

}  // namespace

cudaError_t launch_thermal(const ThermalSetup &s, const double *flux, const double *T_init,
                           const double *cp, const double *piv, double *qT, double *dp,
                           double *T_surface, cudaStream_t stream) {
    ThermalArgs a{};
    a.ncol = s.ncol;
    a.h = s.h;
    a.n_sub = s.n_sub;
    a.R = s.R;
    a.k_over_dr = s.k_over_dr;
    a.a_last = s.a_last;
    for (int k = 0; k < 5; k++) {
        a.p[k] = s.p[k];
        a.LH[k] = s.LH[k];
    }
    a.tran_p = s.tran_p;
    a.tran_LH = s.tran_LH;
    a.mmol = s.mmol;
    a.flux = flux;
    a.T_init = T_init;
    a.cp = cp;
    a.piv = piv;
    a.qT = qT;
    a.dp = dp;
    a.T_surface = T_surface;
    const int block = 32;   // one warp per block: the 81 warps of a 36 x 72 grid spread over 81 SMs
    thermal_column_kernel<<<(s.ncol + block - 1) / block, block, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace dsmc
