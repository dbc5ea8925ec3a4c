// fast_engine.h - resident-slot engine of the FAST paths (internal to the library).
//
// A fixed set of particle slots (one per resident thread) lives in HBM as structure-of-arrays.
// Each launch advances every slot by up to K Verlet steps; a slot whose particle ends takes the
// next particle from a device work queue that spans one or many problem instances. The launch
// loop is captured once as a CUDA graph of G launches and replayed until the queue is drained.
#pragma once

#include <vector>

#include "dsmc_device.cuh"

namespace dsmc {

// One problem instance as the fast kernel sees it.
struct FastInst {
    dsmc_params p;
    DevTables t;
    const float *rb2;        // [hd+1] squared shell boundaries, rb2[0] = R^2, rb2[hd] = r_top^2
    const float *sbs;        // [ftd+1] sin(b)|sin(b)| of latitude boundaries b_k
    const float2 *lonb;      // [ffd+1] (sin, cos) of longitude boundaries phi_k = 2 pi k / ffd
    // the same boundary tables in FP64 (FAST_FP64 solves; nullptr elsewhere)
    const double *rb2d, *sbsd;
    const double2 *lonbd;
    long long work_base;     // first work index of this instance in the queue
    long long n;             // particles
    long long pid_begin;     // particle id of the first particle
    float c_day;             // h / lifetime / ln 2 (W = W0 * 2^(-c_day * n_day))
    float r_land2, r_esc2;   // Radii^2, max_height^2
    double c_day_d;          // c_day in FP64
    int gather;              // lane-chunks a stopped lane may idle before its warp runs the events
                             // it gathered (0: no gathering), from the hop length (gather_chunks)
    double drift_abs;        // drift_tol * GM / Radii: the energy-drift guard's bound (0 = off)
    const float4 *face_f;    // FP32 icosphere tables (config model), or nullptr: FP64 descent
};

// FP32 icosphere tables of an instance (floats; 0 when the problem has no icosphere) and their
// construction on the device from the problem's FP64 tables.
size_t face_floats_for(int nlevel);
size_t face_table_floats(const dsmc_params &p, const DevTables &t);
cudaError_t build_face_tables(const DevTables &t, float4 *out, cudaStream_t stream);

// Structure-of-arrays particle slots of an engine computing in R: float (the FAST_FP32 path:
// position and velocity as two-sum (hi, lo) pairs) or double (FAST_FP64: the lo arrays are
// carved but unused).
template <typename R>
struct SlotsT {
    int *inst;               // instance index, -1 = empty
    unsigned *pid;           // particle id within its instance
    unsigned *evt;           // Philox event counter
    R *sh, *sl, *vh, *vl, *oa;   // [3][S] each: position hi/lo, velocity hi/lo, old accel
                                 // (times dt in the FP32 engine)
    R *w0;                   // weight factor outside photolysis
    int *nday;               // day-side steps (photolysis exponent)
    int *steps;              // steps in the particle's life
    int *hop;                // steps in the current hop
    int *cell;               // packed (ht << 16) | (td << 8) | fd
    int *run_cell;           // cell of the register deposit run, -1 = none
    R *run_w;                // weight-steps in run_cell not yet flushed (8-byte slot reserved)
    int *hist_key;           // (cell * nbins + bin) of the speed-histogram run, -1 = none
    int *hist_cnt;
    R *pcol, *pthr;          // accumulated collision probability and its threshold
    int *ncol;
    float *rest;             // freeze waiting time (reference model)
    R *wcur;                 // running weight (the hot loop's W between launches)
    int *face;               // icosphere face of the last launch point (config model), -1 = none
    float *e0;               // orbital energy at the hop's launch or last collision (drift guard)
};
using Slots = SlotsT<float>;

// Bytes of one slot in the structure-of-arrays block: run_w (an 8-byte slot), the 4-byte fields
// (inst pid evt nday steps hop cell run_cell hist_key hist_cnt ncol rest face e0) and the R fields
// (15 vector components, w0, pcol, pthr, wcur). carve_slots lays the arrays out over slot memory
// of fast_slot_bytes(nslots) bytes; nslots a multiple of 128 keeps every array 512-byte aligned.
template <typename R>
constexpr size_t slot_bytes_per_slot() { return 8 + 14 * 4 + 19 * sizeof(R); }
constexpr size_t kSlotBytesPerSlot = slot_bytes_per_slot<float>();
template <typename R>
SlotsT<R> carve_slots(void *mem, long long nslots);

// Device-side queue state. `total` and `ninst` live here rather than in the kernel arguments so
// that the host can append instances between launches of an already captured graph.
struct FastCounters {
    unsigned long long next;      // next work index
    unsigned long long finished;  // particles whose life ended
    unsigned long long total;     // work items in the queue (sum of the instances' particles)
    long long ninst;              // instances in the queue
};

// Pieces of the engine for callers that supply every buffer themselves (no allocation here):
// bytes of the slot arrays for nslots slots, of one instance descriptor and of the counters;
// fast_fill_instance builds one descriptor and its boundary tables in host memory (tab_host,
// tab_floats entries; d_tab is where the caller will copy them); fast_drain_external runs the
// launch loop without graphs on caller memory until the queue of `total` particles is empty, and
// gives up (cudaErrorLaunchTimeout) after stall_launches launches in a row in which no particle
// finished.
size_t fast_slot_bytes(long long nslots, bool fp64 = false);
size_t fast_inst_bytes();
size_t fast_counter_bytes();
// Expected steps of a typical hop: the ballistic flight time 2 v / g of a molecule launched at
// the thermal speed sqrt(k_B T / m) of a 235 K surface, over the time step.
double fast_hop_steps(const dsmc_params &p);
// Event gathering of an instance from its typical hop (see fast_kernel): 16 lane-chunks below
// 300 steps per hop, 4 below 600, none above.
int gather_chunks(const dsmc_params &p);
cudaError_t fast_fill_instance(const dsmc_params &p, const DevTables &t, long long pid_begin,
                               long long n, float *d_tab, size_t tab_floats, void *inst_host,
                               float *tab_host);
cudaError_t fast_drain_external(const void *d_inst, void *slot_mem, long long nslots, void *d_ctr,
                                long long total, int steps_per_launch, int block,
                                long long stall_launches, cudaStream_t stream,
                                long long *launches);

class FastEngine {
public:
    FastEngine() = default;
    ~FastEngine();
    FastEngine(const FastEngine &) = delete;
    FastEngine &operator=(const FastEngine &) = delete;

    // Solve particles [pid_begin, pid_begin + n) of one instance to the end of their lives, in
    // FP32 with two-sum compensation (fp64 false) or in FP64 (the FAST_FP64 path: the same
    // slots, queue, cell tracking and register deposits on double state and FP64 tables).
    cudaError_t run(const dsmc_params &p, const DevTables &t, bool fp64, long long pid_begin,
                    long long n, int num_sms, cudaStream_t stream);

    void set_shape(int blk, int per_sm, int k, int g) {
        if (blk != block || per_sm != blocks_per_sm) nslots_want_changed_ = true;
        block = blk;
        blocks_per_sm = per_sm;
        steps_per_launch = k;
        launches_per_graph = g;
    }
    long long slot_count() const { return nslots_; }

    // Launch shape (autotuned or set by the caller).
    int block = 128;          // threads per block
    int blocks_per_sm = 0;    // resident blocks per SM (0 = as many as fit)
    int steps_per_launch = 8192;
    int launches_per_graph = 8;
    long long launches = 0;   // launches issued by the last run

private:
    cudaError_t ensure_slots(int num_sms);
    cudaError_t upload_instances(const std::vector<dsmc_params> &ps,
                                 const std::vector<DevTables> &ts,
                                 const std::vector<long long> &counts,
                                 const std::vector<long long> &pid_begins, cudaStream_t stream);
    cudaError_t drain(long long total, cudaStream_t stream);
    cudaError_t prepare_graph(cudaStream_t stream);
    cudaError_t capture(cudaStream_t stream, int mode, cudaGraphExec_t *out);
    cudaError_t round(cudaStream_t stream);
    void launch_kernel(cudaStream_t stream, int mode, unsigned grid);   // one launch, fp64_ state

public:
    // Serving: an open queue that grows while it drains. serve_open resets the engine to an
    // empty queue with room for max_instances instances. serve_append adds one instance: its
    // boundary tables and descriptor are written on `upload` (which it synchronises), and the
    // larger queue is published on `compute` in stream order, so kernels already in flight are
    // not waited for; its statistics go to the engine's per-instance row `index`. serve_launch
    // enqueues one round (the captured graph, or one launch) without waiting. serve_release
    // frees an instance's boundary tables once all its particles have finished.
    cudaError_t serve_open(int num_sms, int max_instances, cudaStream_t stream);
    cudaError_t serve_append(const dsmc_params &p, const DevTables &t, long long n, int *index,
                             cudaStream_t upload, cudaStream_t compute);
    cudaError_t serve_launch(cudaStream_t stream, int mode);
    // Loop an instance may run in: 1 lean (config model, ballistic, no speed histogram, hop cap
    // not below the life cap), 2 lean with collisions (the same, collisional), 0 general only.
    // Every loop that can run an instance gives it identical results.
    static int loop_mode(const dsmc_params &p, const DevTables &t);
    void serve_release(int index, cudaStream_t stream);
    const FastCounters *serve_counters() const { return d_ctr_; }
    const unsigned long long *serve_stats_rows() const { return d_stats_; }
    int serve_instances() const { return ninst_; }
    int serve_capacity() const { return ninst_cap_; }
    // floats of an instance's table block: boundary tables, plus the FP32 icosphere tables of a
    // config-model problem with an icosphere of nlevel levels (nlevel < 0: none)
    static size_t serve_table_floats(const dsmc_params &p, int nlevel);
    void serve_set_pool(cudaMemPool_t pool) { pool_ = pool; }
    void serve_close(cudaStream_t stream);   // frees every instance's boundary tables
    size_t serve_fixed_bytes(int max_instances) const;

private:
    unsigned long long *d_stats_ = nullptr;   // [max_instances][kStatCount] (serving)
    int stats_cap_ = 0;
    cudaMemPool_t pool_ = nullptr;            // stream-ordered allocations (serving)
    std::vector<void *> inst_tabs_;           // boundary tables per instance (serving)
    unsigned long long serve_total_ = 0;
    void free_all();

    Slots slots_{};
    SlotsT<double> slots64_{};                // the same memory carved for FP64 state
    void *slot_mem_ = nullptr;
    bool fp64_ = false;                       // precision of run launches
    bool slot_fp64_ = false;                  // precision the slot memory is carved for
    long long nslots_ = 0;
    FastInst *d_inst_ = nullptr;
    int ninst_cap_ = 0;
    int ninst_ = 0;
    float *d_tab_ = nullptr;
    size_t tab_cap_ = 0;
    FastCounters *d_ctr_ = nullptr;
    FastCounters *h_ctr_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    cudaGraphExec_t graph_mode_[3] = {nullptr, nullptr, nullptr};   // serving: lean loops 1, 2
    cudaStream_t graph_stream_ = nullptr;
    int graph_key_[4] = {0, 0, 0, 0};
    bool nslots_want_changed_ = false;
    int variant_ = 2;
    int mode_ = 0;   // loop of run launches (see fast_kernel)
};

}  // namespace dsmc
