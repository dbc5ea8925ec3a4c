// fast_engine.cu - resident-slot engine (placeholder until the FP32 path lands).
#include "fast_engine.h"

namespace dsmc {

FastEngine::~FastEngine() = default;

cudaError_t FastEngine::run(const dsmc_params &, const DevTables &, bool, long long, long long,
                            int, cudaStream_t) {
    return cudaErrorNotSupported;
}

}  // namespace dsmc
