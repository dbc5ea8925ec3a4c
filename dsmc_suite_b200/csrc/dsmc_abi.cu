// dsmc_abi.cu - implementation of the C ABI in include/dsmc_cuda.h: contexts, uploads,
// launches and result copies. Everything here is host code; the kernels live in kernel_*.cu.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "dsmc_cuda.h"
#include "dsmc_kernels.h"
#include "fast_engine.h"
#include "problem.h"

extern "C" {
#include "constants.h"
#include "types.h"
#include "velocity.h"
}

using dsmc::DevTables;

struct dsmc_ctx {
    int device = -1;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    bool ready = false;
    dsmc_params params{};
    DevTables t{};
    long long ncell = 0, nhcell = 0, nhist = 0;
    dsmc::Problem prob;             // tables and grids of the current problem
    void *outputs[3] = {nullptr, nullptr, nullptr};  // ttime, fate, steps
    unsigned long long *stats = nullptr;
    dsmc::FastEngine *fast = nullptr;
    long long last_launches = 0;
    double last_kernel_ms = 0.0;     // device time of the last thermal / shadow-flux kernel
    void *scratch = nullptr;          // grow-only device scratch of the thermal solve
    size_t scratch_bytes = 0;
    char err[512] = {0};
};

namespace {

thread_local char g_create_err[512];

int fail(dsmc_ctx *c, int status, const char *fmt, ...) {
    char *buf = c ? c->err : g_create_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    return status;
}

#define DSMC_CUDA_TRY(ctx, call)                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail((ctx), e_ == cudaErrorMemoryAllocation ? DSMC_ERR_NO_MEMORY     \
                                                               : DSMC_ERR_CUDA,         \
                        "%s: %s", #call, cudaGetErrorString(e_));                       \
    } while (0)

int set_device(dsmc_ctx *c) {
    DSMC_CUDA_TRY(c, cudaSetDevice(c->device));
    return DSMC_OK;
}

void free_tables(dsmc_ctx *c) {
    c->prob.release();
    c->ready = false;
}

void free_outputs(dsmc_ctx *c) {
    for (void *&p : c->outputs) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    c->t.ttime = nullptr;
    c->t.fate = nullptr;
    c->t.steps = nullptr;
    c->t.out_cap = 0;
    c->t.out_base = 0;
}

}  // namespace

extern "C" {

const char *dsmc_status_string(int status) {
    switch (status) {
        case DSMC_OK: return "ok";
        case DSMC_ERR_INVALID: return "invalid argument";
        case DSMC_ERR_CUDA: return "CUDA error";
        case DSMC_ERR_NO_DEVICE: return "no CUDA device";
        case DSMC_ERR_NO_MEMORY: return "out of memory";
        case DSMC_ERR_STATE: return "call out of order";
        case DSMC_ERR_BUDGET: return "memory budget exceeded";
        case DSMC_ERR_IO: return "file I/O error";
        default: return "unknown status";
    }
}

const char *dsmc_last_error(const dsmc_ctx *ctx) { return ctx ? ctx->err : g_create_err; }

int dsmc_ctx_create(int device, dsmc_ctx **out) {
    if (!out) return fail(nullptr, DSMC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(nullptr, DSMC_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n)
        return fail(nullptr, DSMC_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, n);
    dsmc_ctx *c = new (std::nothrow) dsmc_ctx();
    if (!c) return fail(nullptr, DSMC_ERR_NO_MEMORY, "host allocation failed");
    c->device = device;
    int rc = set_device(c);
    if (rc == DSMC_OK) {
        e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaMalloc(&c->stats, dsmc::kStatCount * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemset(c->stats, 0, dsmc::kStatCount * sizeof(unsigned long long));
        if (e != cudaSuccess) rc = fail(nullptr, DSMC_ERR_CUDA, "context set-up: %s", cudaGetErrorString(e));
    } else {
        snprintf(g_create_err, sizeof g_create_err, "%s", c->err);
    }
    if (rc != DSMC_OK) {
        if (c->stats) cudaFree(c->stats);
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        delete c;
        return rc;
    }
    c->stream = c->own_stream;
    *out = c;
    return DSMC_OK;
}

int dsmc_ctx_destroy(dsmc_ctx *c) {
    if (!c) return DSMC_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    delete c->fast;
    free_tables(c);
    free_outputs(c);
    if (c->stats) cudaFree(c->stats);
    if (c->scratch) cudaFree(c->scratch);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return DSMC_OK;
}

int dsmc_ctx_set_stream(dsmc_ctx *c, void *stream) {
    if (!c) return DSMC_ERR_INVALID;
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return DSMC_OK;
}

int dsmc_setup(dsmc_ctx *c, const dsmc_params *p, const dsmc_surface *s,
               const dsmc_collision *col) {
    if (!c) return DSMC_ERR_INVALID;
    int rc = dsmc::problem_check(p, s, col, c->err, sizeof c->err);
    if (rc != DSMC_OK) return rc;
    if ((rc = set_device(c)) != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    free_tables(c);
    rc = dsmc::problem_build(c->prob, p, s, col, c->stats, c->stream, false, c->err, sizeof c->err);
    if (rc != DSMC_OK) {
        free_tables(c);
        return rc;
    }
    // keep the per-particle output buffers of dsmc_enable_particle_outputs
    DevTables &t = c->t;
    const DevTables old = t;
    t = c->prob.t;
    t.ttime = old.ttime;
    t.fate = old.fate;
    t.steps = old.steps;
    t.out_cap = old.out_cap;
    c->params = *p;
    c->ncell = c->prob.ncell;
    c->nhcell = c->prob.nhcell;
    c->nhist = c->prob.nhist;
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->stats, 0, dsmc::kStatCount * sizeof(unsigned long long), c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->ready = true;
    return DSMC_OK;
}

int dsmc_enable_particle_outputs(dsmc_ctx *c, int64_t n) {
    if (!c || n < 0) return DSMC_ERR_INVALID;
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    free_outputs(c);
    if (n == 0) return DSMC_OK;
    DSMC_CUDA_TRY(c, cudaMalloc(&c->outputs[0], static_cast<size_t>(n) * 9 * sizeof(double)));
    DSMC_CUDA_TRY(c, cudaMalloc(&c->outputs[1], static_cast<size_t>(n) * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMalloc(&c->outputs[2], static_cast<size_t>(n) * sizeof(long long)));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->outputs[0], 0, static_cast<size_t>(n) * 9 * sizeof(double), c->stream));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->outputs[1], 0, static_cast<size_t>(n) * sizeof(int), c->stream));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->outputs[2], 0, static_cast<size_t>(n) * sizeof(long long), c->stream));
    c->t.ttime = static_cast<double *>(c->outputs[0]);
    c->t.fate = static_cast<int *>(c->outputs[1]);
    c->t.steps = static_cast<long long *>(c->outputs[2]);
    c->t.out_cap = n;
    return DSMC_OK;
}

int dsmc_zero(dsmc_ctx *c) {
    if (!c) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "dsmc_zero before dsmc_setup");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->t.density, 0, c->ncell * sizeof(unsigned long long), c->stream));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->t.horizon, 0, c->nhcell * sizeof(unsigned long long), c->stream));
    if (c->t.speed_hist)
        DSMC_CUDA_TRY(c, cudaMemsetAsync(c->t.speed_hist, 0, c->nhist * sizeof(unsigned long long), c->stream));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(c->stats, 0, dsmc::kStatCount * sizeof(unsigned long long), c->stream));
    if (c->t.out_cap > 0) {
        DSMC_CUDA_TRY(c, cudaMemsetAsync(c->t.ttime, 0, c->t.out_cap * 9 * sizeof(double), c->stream));
        DSMC_CUDA_TRY(c, cudaMemsetAsync(c->t.fate, 0, c->t.out_cap * sizeof(int), c->stream));
        DSMC_CUDA_TRY(c, cudaMemsetAsync(c->t.steps, 0, c->t.out_cap * sizeof(long long), c->stream));
    }
    return DSMC_OK;
}

int dsmc_run(dsmc_ctx *c, int path, int64_t pid_begin, int64_t n) {
    if (!c) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "dsmc_run before dsmc_setup");
    if (n < 0 || pid_begin < 0 || pid_begin + n > (int64_t(1) << 32))
        return fail(c, DSMC_ERR_INVALID, "particle ids must lie in [0, 2^32)");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    c->t.out_base = pid_begin;
    switch (path) {
        case DSMC_PATH_PLAIN_FP64:
            DSMC_CUDA_TRY(c, dsmc::launch_plain_fp64(c->params, c->t, pid_begin, n, c->num_sms, c->stream));
            c->last_launches = n > 0 ? 1 : 0;
            return DSMC_OK;
        case DSMC_PATH_FAST_FP64:
        case DSMC_PATH_FAST_FP32: {
            if (!c->fast) {
                c->fast = new (std::nothrow) dsmc::FastEngine();
                if (!c->fast) return fail(c, DSMC_ERR_NO_MEMORY, "host allocation failed");
            }
            if (path == DSMC_PATH_FAST_FP64 && c->fast->block != 128)
                return fail(c, DSMC_ERR_INVALID, "FAST_FP64 runs 128-thread blocks (launch shape has %d)",
                            c->fast->block);
            cudaError_t e = c->fast->run(c->params, c->t, path == DSMC_PATH_FAST_FP64, pid_begin, n,
                                         c->num_sms, c->stream);
            c->last_launches = c->fast->launches;
            if (e != cudaSuccess)
                return fail(c, e == cudaErrorMemoryAllocation ? DSMC_ERR_NO_MEMORY : DSMC_ERR_CUDA,
                            "fast path: %s", cudaGetErrorString(e));
            return DSMC_OK;
        }
        default:
            return fail(c, DSMC_ERR_INVALID, "unknown path %d", path);
    }
}

int dsmc_set_launch_shape(dsmc_ctx *c, int block, int blocks_per_sm, int steps_per_launch,
                          int launches_per_graph) {
    if (!c) return DSMC_ERR_INVALID;
    if (block < 32 || block > 1024 || block % 32 || blocks_per_sm < 0 || blocks_per_sm > 64 ||
        steps_per_launch < 1 || steps_per_launch > (1 << 24) || launches_per_graph < 1 ||
        launches_per_graph > 4096)
        return fail(c, DSMC_ERR_INVALID, "launch shape out of range");
    if (!c->fast) {
        c->fast = new (std::nothrow) dsmc::FastEngine();
        if (!c->fast) return fail(c, DSMC_ERR_NO_MEMORY, "host allocation failed");
    }
    c->fast->set_shape(block, blocks_per_sm, steps_per_launch, launches_per_graph);
    return DSMC_OK;
}

int dsmc_measure_fma_peak(dsmc_ctx *c, int fp64, double *tflops) {
    if (!c || !tflops) return DSMC_ERR_INVALID;
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    const int blocks = c->num_sms * 8, iters = fp64 ? 20000 : 40000;
    void *scratch = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DSMC_CUDA_TRY(c, cudaMalloc(&scratch, blocks * sizeof(double)));
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best_ms = 0.0f;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
        e = cudaEventRecord(e0, c->stream);
        if (e == cudaSuccess) e = dsmc::launch_fma_peak(fp64 != 0, scratch, blocks, iters, c->stream);
        if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(scratch);
    if (e != cudaSuccess) return fail(c, DSMC_ERR_CUDA, "fma peak: %s", cudaGetErrorString(e));
    const double flops = 2.0 * 8.0 * iters * 256.0 * blocks;
    *tflops = flops / (best_ms * 1e-3) / 1e12;
    return DSMC_OK;
}

int dsmc_get_launch_info(dsmc_ctx *c, int64_t *launches, int64_t *nslots) {
    if (!c || !launches || !nslots) return DSMC_ERR_INVALID;
    *launches = c->last_launches;
    *nslots = c->fast ? c->fast->slot_count() : 0;
    return DSMC_OK;
}

int dsmc_sync(dsmc_ctx *c) {
    if (!c) return DSMC_ERR_INVALID;
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_get_density(dsmc_ctx *c, uint64_t *out) {
    if (!c || !out) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "no problem set up");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(out, c->t.density, c->ncell * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_get_horizon(dsmc_ctx *c, uint64_t *out) {
    if (!c || !out) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "no problem set up");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(out, c->t.horizon, c->nhcell * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_get_speed_hist(dsmc_ctx *c, uint64_t *out) {
    if (!c || !out) return DSMC_ERR_INVALID;
    if (!c->ready || !c->t.speed_hist) return fail(c, DSMC_ERR_STATE, "no speed histogram");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(out, c->t.speed_hist, c->nhist * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_get_stats(dsmc_ctx *c, dsmc_stats *out) {
    if (!c || !out) return DSMC_ERR_INVALID;
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    unsigned long long s[dsmc::kStatCount];
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(s, c->stats, sizeof s, cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    out->total_steps = static_cast<int64_t>(s[dsmc::kStatSteps]);
    out->n_escaped = static_cast<int64_t>(s[dsmc::kStatEscaped]);
    out->n_collisions = static_cast<int64_t>(s[dsmc::kStatCollisions]);
    out->n_bound_launch = static_cast<int64_t>(s[dsmc::kStatBound]);
    out->n_finished = static_cast<int64_t>(s[dsmc::kStatFinished]);
    out->n_drift_flagged = static_cast<int64_t>(s[dsmc::kStatDrift]);
    return DSMC_OK;
}

int dsmc_get_particle_outputs(dsmc_ctx *c, int64_t n, double *ttime, int32_t *fate,
                              int64_t *steps) {
    if (!c || n < 0) return DSMC_ERR_INVALID;
    if (n > c->t.out_cap) return fail(c, DSMC_ERR_INVALID, "n exceeds the per-particle capacity");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    if (n == 0) return DSMC_OK;
    if (ttime)
        for (int r = 0; r < 9; r++)
            DSMC_CUDA_TRY(c, cudaMemcpyAsync(ttime + r * n, c->t.ttime + r * c->t.out_cap, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (fate) DSMC_CUDA_TRY(c, cudaMemcpyAsync(fate, c->t.fate, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    if (steps) DSMC_CUDA_TRY(c, cudaMemcpyAsync(steps, c->t.steps, n * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_copy_grids_device(dsmc_ctx *c, uint64_t *density_dst, uint64_t *horizon_dst) {
    if (!c) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "no problem set up");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    if (density_dst)
        DSMC_CUDA_TRY(c, cudaMemcpyAsync(density_dst, c->t.density, c->ncell * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
    if (horizon_dst)
        DSMC_CUDA_TRY(c, cudaMemcpyAsync(horizon_dst, c->t.horizon, c->nhcell * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->stream));
    return DSMC_OK;
}

int dsmc_density_device(dsmc_ctx *c, uint64_t **dev_ptr, int64_t *ncell) {
    if (!c || !dev_ptr || !ncell) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "no problem set up");
    *dev_ptr = reinterpret_cast<uint64_t *>(c->t.density);
    *ncell = c->ncell;
    return DSMC_OK;
}

int dsmc_horizon_device(dsmc_ctx *c, uint64_t **dev_ptr, int64_t *ncell) {
    if (!c || !dev_ptr || !ncell) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "no problem set up");
    *dev_ptr = reinterpret_cast<uint64_t *>(c->t.horizon);
    *ncell = c->nhcell;
    return DSMC_OK;
}

namespace {

// Temporary device buffers of one fit call, freed on every exit path.
struct FitBuffers {
    void *p[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    ~FitBuffers() { for (void *q : p) if (q) cudaFree(q); }
};

int fit_common(dsmc_ctx *c, FitBuffers &b, int64_t ncell, size_t in_bytes, const void *in_host,
               const int32_t *counts) {
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[0], in_bytes));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(b.p[0], in_host, in_bytes, cudaMemcpyHostToDevice, c->stream));
    if (counts) {
        DSMC_CUDA_TRY(c, cudaMalloc(&b.p[1], ncell * sizeof(int)));
        DSMC_CUDA_TRY(c, cudaMemcpyAsync(b.p[1], counts, ncell * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    }
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[2], ncell * DSMC_CDF_STRIDE * sizeof(double)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[3], ncell * 4 * sizeof(double)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[4], ncell * sizeof(double)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[5], ncell * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(b.p[3], 0, ncell * 4 * sizeof(double), c->stream));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(b.p[4], 0, ncell * sizeof(double), c->stream));
    return DSMC_OK;
}

int fit_finish(dsmc_ctx *c, FitBuffers &b, int64_t ncell, double *coef, double *box,
               double *total, int32_t *valid) {
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(coef, b.p[2], ncell * DSMC_CDF_STRIDE * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(box, b.p[3], ncell * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(total, b.p[4], ncell * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(valid, b.p[5], ncell * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

}  // namespace

int dsmc_fit_cdf_samples_host(dsmc_ctx *c, int64_t ncell, int max_per_cell, const double *speeds,
                              const int32_t *counts, int degree, double *coef, double *box,
                              double *total, int32_t *valid) {
    if (!c || !speeds || !counts || !coef || !box || !total || !valid) return DSMC_ERR_INVALID;
    if (ncell <= 0 || ncell > (1 << 30) || max_per_cell < 1 || max_per_cell > 64 || degree < 0 ||
        degree > DSMC_CDF_MAX_DEGREE)
        return fail(c, DSMC_ERR_INVALID, "fit: bad sizes");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    FitBuffers b;
    if ((rc = fit_common(c, b, ncell, ncell * max_per_cell * sizeof(double), speeds, counts)) != DSMC_OK)
        return rc;
    DSMC_CUDA_TRY(c, dsmc::launch_fit_samples(static_cast<int>(ncell), max_per_cell,
                                              static_cast<const double *>(b.p[0]),
                                              static_cast<const int *>(b.p[1]), degree,
                                              static_cast<double *>(b.p[2]), static_cast<double *>(b.p[3]),
                                              static_cast<double *>(b.p[4]), static_cast<int *>(b.p[5]),
                                              c->stream));
    return fit_finish(c, b, ncell, coef, box, total, valid);
}

int dsmc_fit_cdf_hist_host(dsmc_ctx *c, int64_t ncell, int nbins, double bin_width,
                           const uint64_t *hist, int degree, double *coef, double *box,
                           double *total, int32_t *valid) {
    if (!c || !hist || !coef || !box || !total || !valid) return DSMC_ERR_INVALID;
    if (ncell <= 0 || ncell > (1 << 30) || nbins < 1 || nbins > 64 || !(bin_width > 0.0) ||
        degree < 0 || degree > DSMC_CDF_MAX_DEGREE)
        return fail(c, DSMC_ERR_INVALID, "fit: bad sizes");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    FitBuffers b;
    if ((rc = fit_common(c, b, ncell, ncell * nbins * sizeof(uint64_t), hist, nullptr)) != DSMC_OK)
        return rc;
    DSMC_CUDA_TRY(c, dsmc::launch_fit_hist(static_cast<int>(ncell), nbins, bin_width,
                                           static_cast<const unsigned long long *>(b.p[0]), degree,
                                           static_cast<double *>(b.p[2]), static_cast<double *>(b.p[3]),
                                           static_cast<double *>(b.p[4]), static_cast<int *>(b.p[5]),
                                           c->stream));
    return fit_finish(c, b, ncell, coef, box, total, valid);
}

int dsmc_push_host(dsmc_ctx *c, int path, int64_t n, int nsteps, double *pos, double *vel,
                   int32_t *status, int32_t *steps_taken) {
    if (!c || !pos || !vel || !status || n < 0 || nsteps < 0) return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "dsmc_push_host before dsmc_setup");
    if (path != DSMC_PATH_PLAIN_FP64 && path != DSMC_PATH_FAST_FP32 && path != DSMC_PATH_FAST_FP64)
        return fail(c, DSMC_ERR_INVALID, "unknown path %d", path);
    int rc = set_device(c);
    if (rc != DSMC_OK || n == 0) return rc;
    struct Bufs {
        void *p[4] = {nullptr, nullptr, nullptr, nullptr};
        ~Bufs() { for (void *q : p) if (q) cudaFree(q); }
    } b;
    const size_t vb = static_cast<size_t>(n) * 3 * sizeof(double);
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[0], vb));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[1], vb));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[2], n * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[3], n * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(b.p[0], pos, vb, cudaMemcpyHostToDevice, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(b.p[1], vel, vb, cudaMemcpyHostToDevice, c->stream));
    double *dp = static_cast<double *>(b.p[0]), *dv = static_cast<double *>(b.p[1]);
    int *ds = static_cast<int *>(b.p[2]), *dt = static_cast<int *>(b.p[3]);
    if (path == DSMC_PATH_FAST_FP32)
        DSMC_CUDA_TRY(c, dsmc::launch_push_fp32(c->params, n, nsteps, dp, dv, ds, dt, c->stream));
    else
        DSMC_CUDA_TRY(c, dsmc::launch_push_fp64(c->params, n, nsteps, dp, dv, ds, dt, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(pos, dp, vb, cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(vel, dv, vb, cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(status, ds, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    if (steps_taken)
        DSMC_CUDA_TRY(c, cudaMemcpyAsync(steps_taken, dt, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return DSMC_OK;
}

int dsmc_thermal_solve_host(dsmc_ctx *c, int ftd, int ffd, const ThermalParams *tp,
                            const double *flux, double *T_surface, int *h_depth) {
    if (!c || !tp || !T_surface || ftd < 1 || ffd < 1 || ftd > 4096 || ffd > 4096)
        return DSMC_ERR_INVALID;
    if (tp->n_substep < 1 || !(tp->density > 0.0) || !(tp->conductivity > 0.0) || !(tp->Cp > 0.0) ||
        !(tp->depth > 0.0) || !(tp->distance_AU > 0.0))
        return fail(c, DSMC_ERR_INVALID, "thermal parameters must be positive");
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    // scalars of the column model in the reference's operation order (thermal_model.c:110-127)
    const double P = CONST_P_CERES;
    const int n_sub = tp->n_substep;
    const double dt = P / ffd / n_sub;
    const double kk = tp->conductivity, rho = tp->density, Cp = tp->Cp;
    const double dr = sqrt(0.1 * 2.0 * dt * kk / rho / Cp);
    const double hd_real = ceil(tp->depth / dr);
    if (!(hd_real < 1e6)) return fail(c, DSMC_ERR_INVALID, "thermal column of more than 1e6 points");
    const int h = hd_real < 3.0 ? 3 : static_cast<int>(hd_real);
    if (h_depth) *h_depth = h;
    dsmc::ThermalSetup st{};
    st.ncol = ftd * ffd;
    st.h = h;
    st.n_sub = n_sub;
    st.R = kk * dt / rho / 2.0 / Cp / (dr * dr);
    st.k_over_dr = kk / dr;
    st.a_last = -1.0 / dr;
    for (int k = 0; k < 5; k++) {
        st.p[k] = tp->p_mat[k];
        st.LH[k] = tp->LH_mat[k];
    }
    st.tran_p = tp->tran_unit_p;
    st.tran_LH = tp->tran_unit_LH;
    st.mmol = CONST_MMOL_H2O;
    // absorbed flux (the reference's analytic one when none is given, thermal_model.c:130-148),
    // the initial profile from radiative balance (:172-181), and the coefficients of the
    // tridiagonal system shared by every column (:230-244, forward sweep of :80-103)
    // one host block [|F| | initial T | c'_i | pivots] and one device block for everything
    const size_t ncol = static_cast<size_t>(st.ncol), hh = static_cast<size_t>(h);
    std::vector<double> in(2 * ncol + 2 * hh);
    double *F = in.data(), *T_init = F + ncol, *cpv = T_init + ncol, *piv = cpv + hh;
    const double Si = CONST_SOLAR_1AU * (1.0 / tp->distance_AU) * (1.0 / tp->distance_AU);
    const double dF = Si * (1.0 - tp->albedo);
    for (int td = 0; td < ftd; td++)
        for (int fd = 0; fd < ffd; fd++) {
            double f;
            if (flux) {
                f = flux[td * ffd + fd];
            } else {
                const double thi = (td + 0.5) / ftd * M_PI - M_PI / 2.0;
                const double fi = (fd + 0.5) / ffd * 2.0 * M_PI;
                f = fi >= M_PI ? 0.0 : dF * cos(thi) * sin(fi);
            }
            F[td * ffd + fd] = fabs(f);
        }
    for (size_t k = 0; k < ncol; k++) T_init[k] = F[k] > 0 ? pow(F[k] / CONST_SIGMA, 0.25) : 100.0;
    cpv[0] = 0.0 / 1.0;
    piv[0] = 1.0;
    for (int i = 1; i < h; i++) {
        const double ai = i < h - 1 ? -st.R : st.a_last;
        const double bi = i < h - 1 ? 1.0 + 2.0 * st.R : 1.0 / dr;
        const double ci = i < h - 1 ? -st.R : 0.0;
        piv[i] = bi - ai * cpv[i - 1];
        cpv[i] = ci / piv[i];
    }
    const size_t words = in.size() + 2 * ncol * hh + ncol;
    if (words > (size_t(1) << 30)) return fail(c, DSMC_ERR_INVALID, "thermal grid too large (%zu doubles)", words);
    if (c->scratch_bytes < words * sizeof(double)) {
        DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        if (c->scratch) cudaFree(c->scratch);
        c->scratch = nullptr;
        c->scratch_bytes = 0;
        DSMC_CUDA_TRY(c, cudaMalloc(&c->scratch, words * sizeof(double)));
        c->scratch_bytes = words * sizeof(double);
    }
    double *d_in = static_cast<double *>(c->scratch);
    double *dq = d_in + in.size(), *ddp = dq + ncol * hh, *dT = ddp + ncol * hh;
    cudaError_t e = cudaMemcpyAsync(d_in, in.data(), in.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (e == cudaSuccess) e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], c->stream);
    if (e == cudaSuccess)
        e = dsmc::launch_thermal(st, d_in, d_in + ncol, d_in + 2 * ncol, d_in + 2 * ncol + hh, dq, ddp, dT,
                                 c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[1], c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(T_surface, dT, ncol * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    float ms = 0.f;
    if (e == cudaSuccess && cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) c->last_kernel_ms = ms;
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    if (e != cudaSuccess) return fail(c, DSMC_ERR_CUDA, "thermal solve: %s", cudaGetErrorString(e));
    return DSMC_OK;
}

int dsmc_last_kernel_ms(const dsmc_ctx *c, double *ms) {
    if (!c || !ms) return DSMC_ERR_INVALID;
    *ms = c->last_kernel_ms;
    return DSMC_OK;
}

int dsmc_shadow_flux_host(dsmc_ctx *c, int npoint, const double *spot, int nface,
                          const int32_t *facet, const double *face_normal, double za, int tt,
                          int nmonte, double *F) {
    if (!c || !spot || !facet || !face_normal || !F || npoint < 3 || nface < 1 || tt < 1 ||
        nmonte < 1 || static_cast<long long>(nface) * tt > (1ll << 31))
        return DSMC_ERR_INVALID;
    for (long long k = 0; k < 3ll * nface; k++)
        if (facet[k] < 0 || facet[k] >= npoint)
            return fail(c, DSMC_ERR_INVALID, "face %lld names vertex %d of %d", k / 3, facet[k], npoint);
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    long long overflows = 0;
    DSMC_CUDA_TRY(c, dsmc::shadow_flux(npoint, spot, nface, facet, face_normal, za, tt, nmonte, F,
                                       c->stream, &overflows, &c->last_kernel_ms));
    if (overflows) return fail(c, DSMC_ERR_INVALID, "BVH deeper than the traversal stack");
    return DSMC_OK;
}

int dsmc_velocity_record(dsmc_ctx *c, int64_t n, int per_bucket, int64_t total_cap,
                         double *v_out, int32_t *td, int32_t *fd, int32_t *ht, int64_t *n_out) {
    if (!c || !v_out || !td || !fd || !ht || !n_out || n < 0 || per_bucket < 1 || total_cap < 0)
        return DSMC_ERR_INVALID;
    if (!c->ready) return fail(c, DSMC_ERR_STATE, "dsmc_velocity_record before dsmc_setup");
    if (c->params.runner != DSMC_RUNNER_BALLISTIC)
        return fail(c, DSMC_ERR_INVALID, "the velocity record belongs to the ballistic runner");
    if (n > (int64_t(1) << 32)) return fail(c, DSMC_ERR_INVALID, "particle ids must lie in [0, 2^32)");
    *n_out = 0;
    int rc = set_device(c);
    if (rc != DSMC_OK) return rc;
    const int hd = c->params.hd;
    const long long nb = static_cast<long long>(c->params.ftd) * hd;
    // Chunk of particles whose per-bucket counter rows fit in ~64 MB.
    long long chunk = (64ll << 20) / (4 * nb);
    chunk = chunk < 256 ? 256 : chunk;
    if (chunk > n) chunk = n > 0 ? n : 1;
    struct Bufs {
        void *p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
        ~Bufs() { for (void *q : p) if (q) cudaFree(q); }
    } b;
    const long long slots = nb * per_bucket;
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[0], chunk * nb * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[1], nb * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[2], slots * 3 * sizeof(double)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[3], slots * sizeof(int)));
    DSMC_CUDA_TRY(c, cudaMalloc(&b.p[4], slots * sizeof(unsigned long long)));
    DSMC_CUDA_TRY(c, cudaMemsetAsync(b.p[1], 0, nb * sizeof(int), c->stream));
    dsmc::RecordArgs ra{};
    ra.rows = static_cast<int *>(b.p[0]);
    ra.cap = per_bucket;
    ra.rec_v = static_cast<double *>(b.p[2]);
    ra.rec_fd = static_cast<int *>(b.p[3]);
    ra.rec_key = static_cast<unsigned long long *>(b.p[4]);
    std::vector<int> filled(static_cast<size_t>(nb), 0);
    for (long long p0 = 0; p0 < n; p0 += chunk) {
        const long long kc = n - p0 < chunk ? n - p0 : chunk;
        ra.row_base = p0;
        DSMC_CUDA_TRY(c, cudaMemsetAsync(ra.rows, 0, kc * nb * sizeof(int), c->stream));
        DSMC_CUDA_TRY(c, dsmc::launch_plain_record(c->params, c->t, p0, kc, ra,
                                                   static_cast<int *>(b.p[1]), c->num_sms, c->stream));
        DSMC_CUDA_TRY(c, cudaMemcpyAsync(filled.data(), b.p[1], nb * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        long long have = 0;
        bool all_full = true;
        for (long long k = 0; k < nb; k++) {
            have += filled[k] < per_bucket ? filled[k] : per_bucket;
            all_full = all_full && filled[k] >= per_bucket;
        }
        if (all_full || have >= total_cap) break;
    }
    std::vector<double> hv(static_cast<size_t>(slots) * 3);
    std::vector<int> hfd(static_cast<size_t>(slots));
    std::vector<unsigned long long> hkey(static_cast<size_t>(slots));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(hv.data(), b.p[2], slots * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(hfd.data(), b.p[3], slots * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaMemcpyAsync(hkey.data(), b.p[4], slots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    DSMC_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    // Records in global (pid, step) order, as the reference's single-thread run appends them.
    std::vector<std::pair<unsigned long long, long long>> order;
    for (long long k = 0; k < nb; k++) {
        const int m = filled[k] < per_bucket ? filled[k] : per_bucket;
        for (int j = 0; j < m; j++) order.emplace_back(hkey[k * per_bucket + j], k * per_bucket + j);
    }
    std::sort(order.begin(), order.end());
    const long long nrec = static_cast<long long>(order.size()) < total_cap
                               ? static_cast<long long>(order.size()) : total_cap;
    for (long long i = 0; i < nrec; i++) {
        const long long s = order[i].second, bucket = s / per_bucket;
        v_out[3 * i] = hv[3 * s];
        v_out[3 * i + 1] = hv[3 * s + 1];
        v_out[3 * i + 2] = hv[3 * s + 2];
        td[i] = static_cast<int32_t>(bucket / hd);
        ht[i] = static_cast<int32_t>(bucket % hd);
        fd[i] = hfd[s];
    }
    *n_out = nrec;
    return DSMC_OK;
}

int dsmc_solve_host(dsmc_ctx *c, int path, const dsmc_params *p, const dsmc_surface *s,
                    const dsmc_collision *col, int64_t n, uint64_t *density_fx,
                    uint64_t *horizon_fx, dsmc_stats *stats) {
    int rc = dsmc_setup(c, p, s, col);
    if (rc == DSMC_OK) rc = dsmc_run(c, path, 0, n);
    if (rc == DSMC_OK && density_fx) rc = dsmc_get_density(c, density_fx);
    if (rc == DSMC_OK && horizon_fx) rc = dsmc_get_horizon(c, horizon_fx);
    if (rc == DSMC_OK && stats) rc = dsmc_get_stats(c, stats);
    if (rc == DSMC_OK) rc = dsmc_sync(c);
    return rc;
}

}  // extern "C"
