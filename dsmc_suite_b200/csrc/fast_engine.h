// fast_engine.h - resident-slot engine of the FAST paths (internal to the library).
#pragma once

#include "dsmc_device.cuh"

namespace dsmc {

class FastEngine {
public:
    FastEngine() = default;
    ~FastEngine();
    FastEngine(const FastEngine &) = delete;
    FastEngine &operator=(const FastEngine &) = delete;

    // Solve particles [pid_begin, pid_begin + n) to the end of their lives.
    cudaError_t run(const dsmc_params &p, const DevTables &t, bool fp64, long long pid_begin,
                    long long n, int num_sms, cudaStream_t stream);
};

}  // namespace dsmc
