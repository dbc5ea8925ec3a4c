// server.cu - batched and served solves: the dsmc_server_* entry points of include/dsmc_cuda.h.
//
// One server owns one GPU's FAST_FP32 engine in serving mode: a fixed set of resident particle
// slots fed from one device work queue that grows while it drains. A request is a whole
// problem; admission uploads its tables and zeroed grids (stream-ordered allocation on the
// upload stream, charged against the memory budget), and the next poll appends its particles
// to the queue behind the queued ones. Polling keeps two rounds (graph replays of the engine's
// launches) in flight on the compute stream; each round ends with a copy of the queue counters
// and of the per-request statistic rows into pinned memory, and a request is complete when its
// finished count reaches its particle count. Appends write on the upload stream while the rounds
// run, and publish the larger queue on the compute stream in stream order.
//
// The requests admitted since the last poll join the queue grouped by their hop length, longest
// first (ties in admission order): a warp whose lanes hold particles of short-hop and long-hop
// problems runs the event-gathering loop for all of them, so grouping keeps warps uniform. On the
// 64-exosphere batch (three bodies in random order) the grouped queue ran 1.555e11
// particle-steps/s against 1.503e11 in submission order. Each particle's trajectory, random
// stream and deposits are its own, so the order changes no result.
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <new>
#include <vector>

#include "dsmc_cuda.h"
#include "fast_engine.h"
#include "problem.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kSnapHead = 4;   // words of FastCounters at the start of a snapshot

struct Request {
    long long n = 0;
    int inst = -1;                          // engine instance index (current queue epoch)
    std::unique_ptr<dsmc::Problem> prob;
    size_t bytes = 0;                       // charged against the budget
    unsigned long long stats[dsmc::kStatCount] = {};
    double t_submit = 0.0, t_done = 0.0;
    int mode = 0;                           // engine loop it needs (0 general, 1 lean, 2 lean+col)
    enum State { kActive, kDone, kFetched } state = kActive;
};

struct Round {
    cudaEvent_t start = nullptr, end = nullptr;
    unsigned long long *snap = nullptr;     // pinned: counters, then stat rows [lo, hi)
    int lo = 0, hi = 0;
};

}  // namespace

struct dsmc_server {
    int device = -1;
    int num_sms = 0;
    int max_requests = 0;
    cudaStream_t compute = nullptr, upload = nullptr;
    cudaMemPool_t pool = nullptr;                   // requests' device memory
    size_t budget = 0, engine_bytes = 0, in_use = 0;
    dsmc::FastEngine engine;
    std::vector<std::unique_ptr<Request>> reqs;     // by ticket
    std::vector<long long> active;                  // tickets still running, in queue order
    std::vector<long long> pending;                 // admitted, joining the queue at the next poll
    std::deque<long long> done_queue;               // completed, not yet reported by a poll
    Round rounds[2];
    int head = 0, inflight = 0;
    Clock::time_point t0;
    long long submitted = 0, completed = 0, fetched = 0, rejected = 0, nrounds = 0, nlaunches = 0;
    long long total_steps = 0;
    double busy_ms = 0.0;
    unsigned long long last_finished = 0;
    long long stalled = 0;
    long long general_active = 0;                   // active requests only the general loop runs
    long long collide_active = 0;                   // active requests needing the collision loop
    char err[512] = {0};
};

namespace {

thread_local char g_server_err[512];

int fail(dsmc_server *s, int status, const char *fmt, ...) {
    char *buf = s ? s->err : g_server_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    return status;
}

int cuda_fail(dsmc_server *s, const char *what, cudaError_t e) {
    return fail(s, e == cudaErrorMemoryAllocation ? DSMC_ERR_NO_MEMORY : DSMC_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

double now_s(const dsmc_server *s) {
    return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

// Empty queue of max_requests instances; the engine's slots are (re)allocated for its shape.
int open_queue(dsmc_server *s) {
    cudaError_t e = s->engine.serve_open(s->num_sms, s->max_requests, s->compute);
    if (e != cudaSuccess) return cuda_fail(s, "opening the work queue", e);
    s->engine_bytes = s->engine.serve_fixed_bytes(s->max_requests);
    s->last_finished = 0;
    s->stalled = 0;
    return DSMC_OK;
}

size_t recount(const dsmc_server *s) {
    size_t b = s->engine_bytes;
    for (const auto &r : s->reqs)
        if (r && r->state != Request::kFetched) b += r->bytes;
    return b;
}

int launch_round(dsmc_server *s) {
    Round &R = s->rounds[(s->head + s->inflight) % 2];
    R.lo = s->reqs[static_cast<size_t>(s->active.front())]->inst;
    R.hi = s->engine.serve_instances();
    cudaError_t e = cudaEventRecord(R.start, s->compute);
    // Rounds run the leanest loop every queued request qualifies for (same results, fewer
    // registers and branches); a request published after this launch is not seen by it.
    const int mode = s->general_active ? 0 : s->collide_active ? 2 : 1;
    if (e == cudaSuccess) e = s->engine.serve_launch(s->compute, mode);
    if (e == cudaSuccess) s->nlaunches += std::max(1, s->engine.launches_per_graph);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(R.snap, s->engine.serve_counters(), sizeof(dsmc::FastCounters),
                            cudaMemcpyDeviceToHost, s->compute);
    if (e == cudaSuccess && R.hi > R.lo)
        e = cudaMemcpyAsync(R.snap + kSnapHead,
                            s->engine.serve_stats_rows() + static_cast<size_t>(R.lo) * dsmc::kStatCount,
                            static_cast<size_t>(R.hi - R.lo) * dsmc::kStatCount * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s->compute);
    if (e == cudaSuccess) e = cudaEventRecord(R.end, s->compute);
    if (e != cudaSuccess) return cuda_fail(s, "launching a round", e);
    s->inflight++;
    return DSMC_OK;
}

// Waits for the oldest round in flight and retires the requests it shows complete.
int retire_round(dsmc_server *s) {
    Round &R = s->rounds[s->head];
    cudaError_t e = cudaEventSynchronize(R.end);
    if (e != cudaSuccess) return cuda_fail(s, "waiting for a round", e);
    s->head = (s->head + 1) % 2;
    s->inflight--;
    s->nrounds++;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, R.start, R.end) == cudaSuccess) s->busy_ms += ms;
    const double t = now_s(s);
    size_t keep = 0;
    for (size_t k = 0; k < s->active.size(); k++) {
        const long long tk = s->active[k];
        Request &q = *s->reqs[static_cast<size_t>(tk)];
        bool done = false;
        if (q.inst >= R.lo && q.inst < R.hi) {
            const unsigned long long *row =
                R.snap + kSnapHead + static_cast<size_t>(q.inst - R.lo) * dsmc::kStatCount;
            if (row[dsmc::kStatFinished] >= static_cast<unsigned long long>(q.n)) {
                std::memcpy(q.stats, row, sizeof q.stats);
                done = true;
            }
        }
        if (done) {
            q.state = Request::kDone;
            q.t_done = t;
            if (q.mode == 0) s->general_active--;
            if (q.mode == 2) s->collide_active--;
            s->completed++;
            s->total_steps += static_cast<long long>(q.stats[dsmc::kStatSteps]);
            s->done_queue.push_back(tk);
            s->engine.serve_release(q.inst, s->upload);
        } else {
            s->active[keep++] = tk;
        }
    }
    s->active.resize(keep);
    // Every round advances each live particle or ends it, and every life is bounded by its step
    // caps; a queue in which no particle ends for 4096 rounds means a logic error.
    const unsigned long long fin = R.snap[1];
    s->stalled = (fin == s->last_finished && !s->active.empty()) ? s->stalled + 1 : 0;
    s->last_finished = fin;
    if (s->stalled > 4096) return fail(s, DSMC_ERR_CUDA, "no particle finished in 4096 rounds");
    return DSMC_OK;
}

// Appends the requests admitted since the last poll to the work queue, longest hops first.
int publish_pending(dsmc_server *s) {
    if (s->pending.empty()) return DSMC_OK;
    std::vector<std::pair<double, long long>> order;
    order.reserve(s->pending.size());
    for (long long tk : s->pending)
        order.emplace_back(-dsmc::fast_hop_steps(s->reqs[static_cast<size_t>(tk)]->prob->p), tk);
    std::stable_sort(order.begin(), order.end(),
                     [](const auto &a, const auto &b) { return a.first < b.first; });
    for (size_t k = 0; k < order.size(); k++) {
        Request &q = *s->reqs[static_cast<size_t>(order[k].second)];
        const cudaError_t e = s->engine.serve_append(q.prob->p, q.prob->t, q.n, &q.inst, s->upload, s->compute);
        if (e != cudaSuccess) {
            // the requests not yet in the queue stay pending, in their queue order
            s->pending.clear();
            for (size_t j = k; j < order.size(); j++) s->pending.push_back(order[j].second);
            return cuda_fail(s, "appending to the work queue", e);
        }
        s->active.push_back(order[k].second);
        if (q.mode == 0) s->general_active++;
        if (q.mode == 2) s->collide_active++;
    }
    s->pending.clear();
    return DSMC_OK;
}

int drain_rounds(dsmc_server *s) {
    while (s->inflight > 0) {
        const int rc = retire_round(s);
        if (rc != DSMC_OK) return rc;
    }
    return DSMC_OK;
}

void free_server(dsmc_server *s) {
    if (s->compute) cudaStreamSynchronize(s->compute);
    if (s->upload) cudaStreamSynchronize(s->upload);
    s->reqs.clear();   // Problem destructors free on the upload stream
    if (s->upload) cudaStreamSynchronize(s->upload);
    for (Round &R : s->rounds) {
        if (R.start) cudaEventDestroy(R.start);
        if (R.end) cudaEventDestroy(R.end);
        if (R.snap) cudaFreeHost(R.snap);
        R = Round{};
    }
    if (s->compute) s->engine.serve_close(s->compute);
    s->engine.serve_set_pool(nullptr);
    if (s->compute) cudaStreamSynchronize(s->compute);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    s->pool = nullptr;
    if (s->compute) cudaStreamDestroy(s->compute);
    if (s->upload) cudaStreamDestroy(s->upload);
    s->compute = s->upload = nullptr;
}

}  // namespace

extern "C" {

const char *dsmc_server_last_error(const dsmc_server *s) { return s ? s->err : g_server_err; }

int dsmc_server_create(int device, int64_t hbm_budget, int max_requests, dsmc_server **out) {
    if (!out) return fail(nullptr, DSMC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (hbm_budget <= 0 || max_requests < 1 || max_requests > (1 << 22))
        return fail(nullptr, DSMC_ERR_INVALID, "hbm_budget must be > 0 and max_requests in [1, 2^22]");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return fail(nullptr, DSMC_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n)
        return fail(nullptr, DSMC_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, n);
    dsmc_server *s = new (std::nothrow) dsmc_server();
    if (!s) return fail(nullptr, DSMC_ERR_NO_MEMORY, "host allocation failed");
    s->device = device;
    s->max_requests = max_requests;
    s->budget = static_cast<size_t>(hbm_budget);
    s->t0 = Clock::now();
    // serving defaults: 5 blocks of 128 per SM (20 warps at 96 registers: the lean and collision
    // loops that serve config-model requests run fastest there, 8 % above 4 blocks of 128 on a
    // 200 req/s stream), short rounds, so that completions are seen within a few milliseconds.
    // A round is 8192 steps per slot; two launches of 4096 rather than four of 2048 pay the end
    // of a launch (its slowest warp) half as often: 200 req/s for 15 s ran 1.0545e11
    // particle-steps/s (device rate 1.079e11) against 1.035e11 (1.042e11), p99 latency 51.5 s
    // against 52.7 s
    s->engine.set_shape(128, 5, 4096, 2);
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->compute, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // a pool of its own: admitted requests allocate and free without returning memory to
        // the driver between polls, and nothing else in the process shares it
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&s->pool, &props);
        if (e == cudaSuccess) {
            unsigned long long keep = static_cast<unsigned long long>(hbm_budget);
            e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        if (e == cudaSuccess) s->engine.serve_set_pool(s->pool);
    }
    const size_t snap_words = kSnapHead + static_cast<size_t>(max_requests) * dsmc::kStatCount;
    for (Round &R : s->rounds) {
        if (e == cudaSuccess) e = cudaEventCreate(&R.start);
        if (e == cudaSuccess) e = cudaEventCreate(&R.end);
        if (e == cudaSuccess) e = cudaMallocHost(&R.snap, snap_words * sizeof(unsigned long long));
    }
    int rc = e == cudaSuccess ? DSMC_OK : cuda_fail(s, "server set-up", e);
    if (rc == DSMC_OK) rc = open_queue(s);
    if (rc == DSMC_OK && s->engine_bytes > s->budget)
        rc = fail(s, DSMC_ERR_BUDGET, "the engine alone needs %zu bytes, over the budget of %zu",
                  s->engine_bytes, s->budget);
    if (rc != DSMC_OK) {
        std::snprintf(g_server_err, sizeof g_server_err, "%s", s->err);
        free_server(s);
        delete s;
        return rc;
    }
    s->in_use = s->engine_bytes;
    *out = s;
    return DSMC_OK;
}

int dsmc_server_destroy(dsmc_server *s) {
    if (!s) return DSMC_OK;
    cudaSetDevice(s->device);
    free_server(s);
    delete s;
    return DSMC_OK;
}

int dsmc_server_set_shape(dsmc_server *s, int block, int blocks_per_sm, int steps_per_launch,
                          int launches_per_graph) {
    if (!s) return DSMC_ERR_INVALID;
    if (block < 32 || block > 1024 || (block & 31) || blocks_per_sm < 0 || blocks_per_sm > 32 ||
        steps_per_launch < 1 || launches_per_graph < 1 || launches_per_graph > 1024)
        return fail(s, DSMC_ERR_INVALID, "bad launch shape");
    if (!s->active.empty())
        return fail(s, DSMC_ERR_STATE, "the launch shape changes only while no request is active");
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_fail(s, "cudaSetDevice", e);
    int rc = drain_rounds(s);
    if (rc != DSMC_OK) return rc;
    s->engine.set_shape(block, blocks_per_sm, steps_per_launch, launches_per_graph);
    rc = open_queue(s);
    if (rc != DSMC_OK) return rc;
    s->in_use = recount(s);
    return DSMC_OK;
}

int dsmc_server_submit(dsmc_server *s, const dsmc_params *p, const dsmc_surface *surf,
                       const dsmc_collision *col, int64_t n, int64_t *ticket) {
    if (!s || !ticket) return DSMC_ERR_INVALID;
    *ticket = -1;
    if (n < 0 || n > (int64_t(1) << 32)) return fail(s, DSMC_ERR_INVALID, "particle count out of [0, 2^32]");
    int rc = dsmc::problem_check(p, surf, col, s->err, sizeof s->err);
    if (rc != DSMC_OK) return rc;
    if (p->ftd > 255 || p->ffd > 255 || p->hd > 32767)
        return fail(s, DSMC_ERR_INVALID, "served grids need ftd, ffd <= 255 and hd <= 32767");
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_fail(s, "cudaSetDevice", e);
    const int queued = s->engine.serve_instances() + static_cast<int>(s->pending.size());
    if (n > 0 && queued >= s->engine.serve_capacity()) {
        if (!s->active.empty() || static_cast<int>(s->pending.size()) >= s->engine.serve_capacity()) {
            s->rejected++;
            return fail(s, DSMC_ERR_BUDGET, "request queue full (%d requests); poll and retry", s->max_requests);
        }
        // every request has completed: retire the (empty) rounds still in flight, then restart
        if ((rc = drain_rounds(s)) != DSMC_OK) return rc;
        if ((rc = open_queue(s)) != DSMC_OK) return rc;
    }
    const size_t tab = dsmc::FastEngine::serve_table_floats(
                           *p, p->model == DSMC_MODEL_CONFIG ? surf->nlevel : -1) * sizeof(float);
    const size_t est = dsmc::problem_bytes(p, surf, col) + tab;
    if (s->in_use + est > s->budget) {
        s->rejected++;
        return fail(s, DSMC_ERR_BUDGET, "request needs %zu bytes; %zu of %zu in use", est, s->in_use, s->budget);
    }
    auto q = std::make_unique<Request>();
    q->n = n;
    q->prob = std::make_unique<dsmc::Problem>();
    rc = dsmc::problem_build(*q->prob, p, surf, col, nullptr, s->upload, true, s->err, sizeof s->err,
                             s->pool);
    if (rc != DSMC_OK) return rc;
    q->bytes = q->prob->bytes + (n > 0 ? tab : 0);
    q->t_submit = now_s(s);
    const long long tk = static_cast<long long>(s->reqs.size());
    if (n > 0) {
        q->mode = dsmc::FastEngine::loop_mode(*p, q->prob->t);
        s->pending.push_back(tk);
    } else {
        q->state = Request::kDone;
        q->t_done = q->t_submit;
        s->completed++;
        s->done_queue.push_back(tk);
    }
    s->in_use += q->bytes;
    s->reqs.push_back(std::move(q));
    s->submitted++;
    *ticket = tk;
    return DSMC_OK;
}

int dsmc_server_poll(dsmc_server *s, int64_t *done, int cap, int *ndone) {
    if (!s || !ndone || cap < 0 || (cap > 0 && !done)) return DSMC_ERR_INVALID;
    *ndone = 0;
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_fail(s, "cudaSetDevice", e);
    int rc = publish_pending(s);
    if (rc != DSMC_OK) return rc;
    if (!s->active.empty())
        while (s->inflight < 2 && (rc = launch_round(s)) == DSMC_OK) {}
    if (rc != DSMC_OK) {
        drain_rounds(s);
        return rc;
    }
    if (s->inflight > 0 && (rc = retire_round(s)) != DSMC_OK) return rc;
    while (*ndone < cap && !s->done_queue.empty()) {
        done[(*ndone)++] = s->done_queue.front();
        s->done_queue.pop_front();
    }
    return DSMC_OK;
}

int dsmc_server_fetch(dsmc_server *s, int64_t ticket, uint64_t *density, uint64_t *horizon,
                      dsmc_stats *stats, dsmc_request_info *info) {
    if (!s) return DSMC_ERR_INVALID;
    if (ticket < 0 || ticket >= static_cast<int64_t>(s->reqs.size()))
        return fail(s, DSMC_ERR_INVALID, "unknown ticket %lld", static_cast<long long>(ticket));
    Request &q = *s->reqs[static_cast<size_t>(ticket)];
    if (q.state == Request::kActive) return fail(s, DSMC_ERR_STATE, "request %lld is still running", static_cast<long long>(ticket));
    if (q.state == Request::kFetched) return fail(s, DSMC_ERR_INVALID, "request %lld was already fetched", static_cast<long long>(ticket));
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_fail(s, "cudaSetDevice", e);
    const dsmc::Problem &pr = *q.prob;
    // The request's kernels have all ended: its grids are read on the upload stream, beside the
    // rounds still running for other requests.
    if (density)
        e = cudaMemcpyAsync(density, pr.t.density, static_cast<size_t>(pr.ncell) * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, s->upload);
    if (e == cudaSuccess && horizon)
        e = cudaMemcpyAsync(horizon, pr.t.horizon, static_cast<size_t>(pr.nhcell) * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, s->upload);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->upload);
    if (e != cudaSuccess) return cuda_fail(s, "reading results", e);
    if (stats) {
        stats->total_steps = static_cast<int64_t>(q.stats[dsmc::kStatSteps]);
        stats->n_escaped = static_cast<int64_t>(q.stats[dsmc::kStatEscaped]);
        stats->n_collisions = static_cast<int64_t>(q.stats[dsmc::kStatCollisions]);
        stats->n_bound_launch = static_cast<int64_t>(q.stats[dsmc::kStatBound]);
        stats->n_finished = static_cast<int64_t>(q.stats[dsmc::kStatFinished]);
        stats->n_drift_flagged = static_cast<int64_t>(q.stats[dsmc::kStatDrift]);
    }
    if (info) {
        info->n = q.n;
        info->ncell = pr.ncell;
        info->nhcell = pr.nhcell;
        info->t_submit = q.t_submit;
        info->t_done = q.t_done;
    }
    q.prob.reset();
    q.state = Request::kFetched;
    s->in_use -= std::min(s->in_use, q.bytes);
    s->fetched++;
    return DSMC_OK;
}

int dsmc_server_info_get(const dsmc_server *s, dsmc_server_info *info) {
    if (!s || !info) return DSMC_ERR_INVALID;
    info->submitted = s->submitted;
    info->completed = s->completed;
    info->fetched = s->fetched;
    info->rejected = s->rejected;
    info->active = static_cast<int64_t>(s->active.size() + s->pending.size());
    info->bytes_in_use = static_cast<int64_t>(s->in_use);
    info->bytes_budget = static_cast<int64_t>(s->budget);
    info->slots = s->engine.slot_count();
    info->rounds = s->nrounds;
    info->launches = s->nlaunches;
    info->total_steps = s->total_steps;
    info->busy_ms = s->busy_ms;
    return DSMC_OK;
}

double dsmc_server_now(const dsmc_server *s) { return s ? now_s(s) : 0.0; }

}  // extern "C"
