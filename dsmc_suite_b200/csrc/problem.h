// problem.h - device copy of one DSMC problem (internal to the library): its tables, grids and
// the DevTables view the kernels read. Shared by dsmc_setup (one problem per context) and the
// server (one problem per request).
#pragma once

#include <cstddef>
#include <vector>

#include "dsmc_cuda.h"
#include "dsmc_device.cuh"

namespace dsmc {

struct Problem {
    dsmc_params p{};
    DevTables t{};
    std::vector<void *> owned;     // device allocations of this problem
    long long ncell = 0, nhcell = 0, nhist = 0;
    size_t bytes = 0;              // device bytes held by the problem
    bool async_alloc = false;      // owned buffers are stream-ordered allocations on `stream`
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;  // pool of the stream-ordered allocations (nullptr: default)

    Problem() = default;
    Problem(const Problem &) = delete;
    Problem &operator=(const Problem &) = delete;
    ~Problem() { release(); }
    void release();
};

// Device bytes a problem with these inputs would hold (grids, tables, histograms).
size_t problem_bytes(const dsmc_params *p, const dsmc_surface *s, const dsmc_collision *col);

// Validates the inputs; DSMC_OK or DSMC_ERR_INVALID with a message in err.
int problem_check(const dsmc_params *p, const dsmc_surface *s, const dsmc_collision *col,
                  char *err, size_t errlen);

// Uploads the tables and allocates zeroed grids on `stream` (stream-ordered allocations from
// `pool`, or the device's default pool when it is nullptr, when async_alloc). `stats` is the
// statistics buffer the kernels add into (owned by the caller).
int problem_build(Problem &pr, const dsmc_params *p, const dsmc_surface *s,
                  const dsmc_collision *col, unsigned long long *stats, cudaStream_t stream,
                  bool async_alloc, char *err, size_t errlen, cudaMemPool_t pool = nullptr);

}  // namespace dsmc
