// kernel_peak.cu - FMA-throughput probe used as the roofline denominator of the push kernels.
//
// Each thread runs 8 independent FMA chains for `iters` rounds, so the FP32 (or FP64) pipe is
// the only limit. The caller times the launch; flops = 2 * 8 * iters * threads.
#include "dsmc_device.cuh"
#include "dsmc_kernels.h"

namespace dsmc {
namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *out, int iters, T a, T b) {
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = static_cast<T>(threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == static_cast<T>(-1.2345)) out[blockIdx.x] = s;   // keeps the chains live
}

}  // namespace

cudaError_t launch_fma_peak(bool fp64, void *scratch, int blocks, int iters, cudaStream_t stream) {
    if (fp64)
        fma_peak_kernel<double><<<blocks, 256, 0, stream>>>(static_cast<double *>(scratch), iters,
                                                            0.999999, 1e-7);
    else
        fma_peak_kernel<float><<<blocks, 256, 0, stream>>>(static_cast<float *>(scratch), iters,
                                                           0.999999f, 1e-7f);
    return cudaGetLastError();
}

}  // namespace dsmc
