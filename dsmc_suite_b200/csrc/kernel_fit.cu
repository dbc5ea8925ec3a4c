// kernel_fit.cu - FP64 least-squares fits of the per-cell collision-partner speed CDFs.
//
// One thread per grid cell. Compiled with -fmad=false: the sums, the elimination and the back
// substitution round each operation as the reference's src/common/polyfit.c:10-101 does on
// x86-64, so fits of identical inputs are bit-identical to the reference's.
#include "dsmc_device.cuh"
#include "dsmc_kernels.h"

namespace dsmc {
namespace {

constexpr int kMaxPoints = 64;

// Normal equations + Gaussian elimination with partial pivoting (polyfit.c:10-101).
// Coefficients highest power first. Returns false when singular.
__device__ bool polyfit_dev(const double *x, const double *y, int n, int degree, double *coef) {
    const int m = degree + 1;
    if (n < m || degree > DSMC_CDF_MAX_DEGREE) return false;
    double S[2 * DSMC_CDF_MAX_DEGREE + 1], b[DSMC_CDF_MAX_DEGREE + 1], a[DSMC_CDF_MAX_DEGREE + 1];
    for (int k = 0; k <= 2 * degree; k++) S[k] = 0.0;
    for (int j = 0; j < m; j++) b[j] = 0.0;
    for (int i = 0; i < n; i++) {
        double xp = 1.0;
        for (int k = 0; k <= 2 * degree; k++) { S[k] += xp; xp *= x[i]; }
    }
    for (int i = 0; i < n; i++) {
        double xp = 1.0;
        for (int j = 0; j < m; j++) { b[j] += xp * y[i]; xp *= x[i]; }
    }
    double A[DSMC_CDF_MAX_DEGREE + 1][DSMC_CDF_MAX_DEGREE + 2];
    for (int r = 0; r < m; r++) {
        for (int c = 0; c < m; c++) A[r][c] = S[r + c];
        A[r][m] = b[r];
    }
    for (int col = 0; col < m; col++) {
        int piv = col;
        double best = fabs(A[col][col]);
        for (int r = col + 1; r < m; r++)
            if (fabs(A[r][col]) > best) { best = fabs(A[r][col]); piv = r; }
        if (best < 1e-30) return false;
        if (piv != col)
            for (int k = 0; k <= m; k++) { double t = A[col][k]; A[col][k] = A[piv][k]; A[piv][k] = t; }
        for (int r = col + 1; r < m; r++) {
            const double f = A[r][col] / A[col][col];
            for (int k = col; k <= m; k++) A[r][k] -= f * A[col][k];
        }
    }
    for (int r = m - 1; r >= 0; r--) {
        a[r] = A[r][m];
        for (int c = r + 1; c < m; c++) a[r] -= A[r][c] * a[c];
        a[r] /= A[r][r];
    }
    for (int i = 0; i < m; i++) coef[i] = a[degree - i];
    return true;
}

// build_poly_fits for one cell, src/dsmc/advanced.c:44-108: sort the nn speeds, histogram them
// into max(4, (nn+1)/2) bins between min and max, fit the reverse-cumulative counts.
__global__ void fit_samples_kernel(int ncell, int max_per_cell, const double *__restrict__ speeds,
                                   const int *__restrict__ counts, int degree, double *coef,
                                   double *box, double *total, int *valid) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const int nn = counts[c];
    double *cf = coef + static_cast<long long>(DSMC_CDF_STRIDE) * c;
    for (int i = 0; i < DSMC_CDF_STRIDE; i++) cf[i] = 0.0;
    valid[c] = 0;
    if (nn <= 8 || nn > max_per_cell || nn > kMaxPoints) return;
    double v[kMaxPoints];
    const double *src = speeds + static_cast<long long>(max_per_cell) * c;
    for (int i = 0; i < nn; i++) v[i] = src[i];
    for (int i = 1; i < nn; i++) {           // insertion sort, ascending
        const double key = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > key) { v[j + 1] = v[j]; j--; }
        v[j + 1] = key;
    }
    const double min_v = v[0], max_v = v[nn - 1];
    int nbins = (nn + 1) / 2;
    if (nbins < 4) nbins = 4;
    double xx[kMaxPoints], yy[kMaxPoints];
    const double dv = (max_v - min_v) / nbins;
    for (int i = 0; i < nbins; i++) { xx[i] = min_v + (i + 0.5) * dv; yy[i] = 0.0; }
    for (int i = 0; i < nn; i++) {
        int bin = static_cast<int>((v[i] - min_v) / dv);
        bin = bin >= nbins ? nbins - 1 : (bin < 0 ? 0 : bin);
        yy[bin] += 1.0;
    }
    // reverse-cumulative counts, summed from each bin to the last as advanced.c:90-95 does
    double y2[kMaxPoints];
    for (int i = 0; i < nbins; i++) {
        double s = 0.0;
        for (int j = i; j < nbins; j++) s += yy[j];
        y2[i] = s;
    }
    double cc[DSMC_CDF_MAX_DEGREE + 1];
    if (!polyfit_dev(xx, y2, nbins, degree, cc)) return;
    for (int i = 0; i <= degree; i++) cf[i] = cc[i];
    double *bx = box + 4ll * c;
    bx[0] = min_v; bx[1] = max_v; bx[2] = 0.0; bx[3] = 1.0;
    total[c] = static_cast<double>(nn);
    valid[c] = 1;
}

// Config-model fit from a per-cell speed histogram: the reverse-cumulative fraction over the
// occupied bin range, speeds mapped to t in [-1, 1] so degree 6 stays well conditioned.
__global__ void fit_hist_kernel(int ncell, int nbins, double bin_width,
                                const unsigned long long *__restrict__ hist, int degree,
                                double *coef, double *box, double *total, int *valid) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const unsigned long long *h = hist + static_cast<long long>(nbins) * c;
    double *cf = coef + static_cast<long long>(DSMC_CDF_STRIDE) * c;
    for (int i = 0; i < DSMC_CDF_STRIDE; i++) cf[i] = 0.0;
    valid[c] = 0;
    int lo = -1, hi = -1;
    unsigned long long nn = 0;
    for (int i = 0; i < nbins; i++)
        if (h[i]) { if (lo < 0) lo = i; hi = i; nn += h[i]; }
    if (lo < 0) return;
    const int m = hi - lo + 1;
    if (m < degree + 2 || nn <= 8 || m > kMaxPoints) return;
    const double min_v = lo * bin_width, max_v = (hi + 1) * bin_width;
    const double xc = 0.5 * (min_v + max_v), xs = 0.5 * (max_v - min_v);
    double t[kMaxPoints], y[kMaxPoints];
    double acc = 0.0;
    const double inv = 1.0 / static_cast<double>(nn);
    for (int i = hi; i >= lo; i--) {
        acc += static_cast<double>(h[i]);
        t[i - lo] = ((lo + (i - lo) + 0.5) * bin_width - xc) / xs;
        y[i - lo] = acc * inv;
    }
    double cc[DSMC_CDF_MAX_DEGREE + 1];
    if (!polyfit_dev(t, y, m, degree, cc)) return;
    for (int i = 0; i <= degree; i++) cf[i] = cc[i];
    double *bx = box + 4ll * c;
    bx[0] = min_v; bx[1] = max_v; bx[2] = xc; bx[3] = xs;
    total[c] = 1.0;
    valid[c] = 1;
}

}  // namespace

cudaError_t launch_fit_samples(int ncell, int max_per_cell, const double *speeds,
                               const int *counts, int degree, double *coef, double *box,
                               double *total, int *valid, cudaStream_t stream) {
    if (ncell <= 0) return cudaSuccess;
    fit_samples_kernel<<<(ncell + 127) / 128, 128, 0, stream>>>(ncell, max_per_cell, speeds, counts,
                                                                degree, coef, box, total, valid);
    return cudaGetLastError();
}

cudaError_t launch_fit_hist(int ncell, int nbins, double bin_width, const unsigned long long *hist,
                            int degree, double *coef, double *box, double *total, int *valid,
                            cudaStream_t stream) {
    if (ncell <= 0) return cudaSuccess;
    fit_hist_kernel<<<(ncell + 127) / 128, 128, 0, stream>>>(ncell, nbins, bin_width, hist, degree,
                                                             coef, box, total, valid);
    return cudaGetLastError();
}

}  // namespace dsmc
