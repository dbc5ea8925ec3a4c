// dsmc_kernels.h - host-side launchers of the DSMC kernels (internal to the library).
#pragma once

#include "dsmc_device.cuh"

namespace dsmc {

// Plain FP64 path: one thread per particle for its whole life (kernel_plain.cu).
cudaError_t launch_plain_fp64(const dsmc_params &p, const DevTables &t, long long pid_begin,
                              long long n, int num_sms, cudaStream_t stream);

// Velocity-record replay of particles [pid_begin, pid_begin + n): count pass, per-bucket scan
// (filled[b] holds the records each bucket already has and is advanced), record pass.
cudaError_t launch_plain_record(const dsmc_params &p, const DevTables &t, long long pid_begin,
                                long long n, const RecordArgs &ra, int *filled, int num_sms,
                                cudaStream_t stream);

// Fed-state pushes (n particles, up to nsteps steps each; pos/vel [n][3] in place).
cudaError_t launch_push_fp64(const dsmc_params &p, long long n, int nsteps, double *pos,
                             double *vel, int *status, int *taken, cudaStream_t stream);
cudaError_t launch_push_fp32(const dsmc_params &p, long long n, int nsteps, double *pos,
                             double *vel, int *status, int *taken, cudaStream_t stream);

// FMA-throughput probe (kernel_peak.cu); scratch holds `blocks` elements.
cudaError_t launch_fma_peak(bool fp64, void *scratch, int blocks, int iters, cudaStream_t stream);

// Per-cell FP64 CDF fits (kernel_fit.cu).
cudaError_t launch_fit_samples(int ncell, int max_per_cell, const double *speeds,
                               const int *counts, int degree, double *coef, double *box,
                               double *total, int *valid, cudaStream_t stream);
cudaError_t launch_fit_hist(int ncell, int nbins, double bin_width, const unsigned long long *hist,
                            int degree, double *coef, double *box, double *total, int *valid,
                            cudaStream_t stream);

// Thermal column model (kernel_thermal.cu): scalars of one solve, formed on the host in the
// reference's operation order.
struct ThermalSetup {
    int ncol, h, n_sub;
    double R, k_over_dr, a_last;
    double p[5], LH[5], tran_p, tran_LH, mmol;
};
// flux, T_init [ncol] = |F| and the initial (uniform) column temperature; cp, piv [h]; qT, dp
// [h][ncol] scratch (qT ends with the final profiles); T_surface [ncol].
cudaError_t launch_thermal(const ThermalSetup &s, const double *flux, const double *T_init,
                           const double *cp, const double *piv, double *qT, double *dp,
                           double *T_surface, cudaStream_t stream);

// Monte Carlo shadow flux (kernel_raytrace.cu): builds the BVH of the mesh on the host, traces
// on `stream` and copies F [nface][tt] back (synchronous). *overflows counts traversal-stack
// overflows (0 for meshes below 2^24 faces).
cudaError_t shadow_flux(int npoint, const double *spot, int nface, const int *facet,
                        const double *normal, double za, int tt, int nmonte, double *F_host,
                        cudaStream_t stream, long long *overflows, double *kernel_ms);

}  // namespace dsmc
