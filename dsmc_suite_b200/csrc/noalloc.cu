// noalloc.cu - dsmc_solve_fast_noalloc: the FAST_FP32 solve for callers that cannot allocate
// device memory.
//
// Some callers can't call cudaMalloc: code running inside a host framework that owns all device
// memory through its own pool (and forbids driver allocations that would fragment it or escape
// its accounting), code launched between captured graph segments of a larger application, or a
// plugin loaded into a process whose allocation calls are intercepted or budgeted. They can
// still pass device buffers they already hold. This entry point therefore allocates nothing: the
// scratch the fast kernel needs (the resident particle slots, the instance descriptor, the cell
// boundary tables, the work-queue counters, the reference-model speed table and the FP32
// icosphere tables) lives in one
// file-scope device array of fixed size, which every GPU that loads the library holds until the
// process exits.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "dsmc_cuda.h"
#include "fast_engine.h"

extern "C" {
#include "types.h"
#include "velocity.h"
}

namespace {

constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Stated maximum sizes of the no-allocation path.
constexpr long long kSlots = 32768;        // resident particle slots (threads)
constexpr int kBlock = 128;                // threads per block: 256 blocks of 128
constexpr int kStepsPerLaunch = 8192;      // Verlet steps per slot per launch (the engine's)
constexpr size_t kTabFloats = 4096;        // (hd+1) + (ftd+1) + 2 (ffd+1) + 1 floats at most

constexpr size_t kSlotOff = 0;
constexpr size_t kSlotBytes = round_up(static_cast<size_t>(kSlots) * dsmc::kSlotBytesPerSlot + 256);
constexpr size_t kInstOff = kSlotOff + kSlotBytes;
constexpr size_t kInstBytes = round_up(sizeof(dsmc::FastInst));
constexpr size_t kTabOff = kInstOff + kInstBytes;
constexpr size_t kTabBytes = round_up(kTabFloats * sizeof(float));
constexpr size_t kCtrOff = kTabOff + kTabBytes;
constexpr size_t kCtrBytes = round_up(sizeof(dsmc::FastCounters));
constexpr size_t kVtOff = kCtrOff + kCtrBytes;
constexpr size_t kVtBytes = round_up(23 * 1000 * sizeof(double));
constexpr size_t kCntOff = kVtOff + kVtBytes;
constexpr size_t kCntBytes = round_up(23 * sizeof(int));
constexpr size_t kFaceOff = kCntOff + kCntBytes;       // FP32 icosphere tables, up to 6 levels
constexpr size_t kFaceBytes = round_up(4 * (20 + 3 * 27300 + 3 * 81920) * sizeof(float));
constexpr size_t kScratchBytes = kFaceOff + kFaceBytes;   // about 10.0 MB

// The scratch itself. In host code `g_scratch` names a host-side stand-in, not the device
// memory: its device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;                         // one call at a time in this process
unsigned char *g_scratch_dev[kMaxDevices]; // device address of g_scratch on each device
thread_local char g_err[512];

int fail(int status, const char *msg) {
    std::snprintf(g_err, sizeof g_err, "%s", msg);
    return status;
}

int fail_cuda(const char *what, cudaError_t e) {
    std::snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DSMC_ERR_NO_MEMORY : DSMC_ERR_CUDA;
}

const VelocityTable &speed_table() {
    static VelocityTable vt;
    static std::once_flag once;
    std::call_once(once, [] { velocity_table_init(&vt, 18e-3, 6.02e23, 1.38e-23); });
    return vt;
}

}  // namespace

extern "C" const char *dsmc_noalloc_last_error(void) { return g_err; }

extern "C" int dsmc_solve_fast_noalloc(const dsmc_params *p, const dsmc_surface *surf,
                                       int64_t pid_begin, int64_t n, uint64_t *density,
                                       uint64_t *horizon, uint64_t *stats, void *stream_ptr) {
    if (!p || !surf || !density || !horizon || !stats)
        return fail(DSMC_ERR_INVALID, "params, surface, density, horizon and stats are required");
    constexpr int64_t kIds = int64_t(1) << 32;
    if (n < 0 || pid_begin < 0 || n > kIds || pid_begin > kIds - n)
        return fail(DSMC_ERR_INVALID, "particle ids must lie in [0, 2^32)");
    if (p->model != DSMC_MODEL_REFERENCE && p->model != DSMC_MODEL_CONFIG)
        return fail(DSMC_ERR_INVALID, "unknown physics model");
    if (p->runner != DSMC_RUNNER_BALLISTIC)
        return fail(DSMC_ERR_INVALID, "the no-allocation path solves the ballistic runner only");
    if (p->ftd < 1 || p->ffd < 2 || p->hd < 1 || p->ftd > 255 || p->ffd > 255 ||
        static_cast<size_t>(p->hd + 1) + (p->ftd + 1) + 1 + 2 * static_cast<size_t>(p->ffd + 1) > kTabFloats)
        return fail(DSMC_ERR_INVALID,
                    "grid too large for the no-allocation path: ftd, ffd <= 255 and "
                    "(hd+1) + (ftd+1) + 2 (ffd+1) + 1 <= 4096");
    if (!(p->dt_step > 0.0) || !(p->Radii > 0.0) || !(p->GM > 0.0) || !(p->max_height > p->Radii) ||
        p->hop_step_cap < 1)
        return fail(DSMC_ERR_INVALID, "dt, Radii, GM and max_height must be positive");
    const bool ref = p->model == DSMC_MODEL_REFERENCE;
    if (ref ? !surf->T_map
            : (!surf->face_verts || !surf->face_T || !surf->base_centroid || !surf->split_planes ||
               surf->nlevel < 0 || surf->nlevel > 6 || surf->nface != (20 << (2 * surf->nlevel))))
        return fail(DSMC_ERR_INVALID, "incomplete surface (device pointers)");

    std::lock_guard<std::mutex> guard(g_lock);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda("cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return fail(DSMC_ERR_NO_DEVICE, "device index out of range");
    if (!g_scratch_dev[dev]) {
        // set-up on the first call on this device, with the device current
        void *addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_scratch);
        if (e != cudaSuccess) return fail_cuda("cudaGetSymbolAddress", e);
        g_scratch_dev[dev] = static_cast<unsigned char *>(addr);
    }
    unsigned char *base = g_scratch_dev[dev];
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);

    dsmc::DevTables t{};
    if (ref) {
        const VelocityTable &vt = speed_table();
        e = cudaMemcpyAsync(base + kVtOff, &vt.speeds[0][0], 23 * 1000 * sizeof(double),
                            cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(base + kCntOff, vt.count, 23 * sizeof(int), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return fail_cuda("speed table copy", e);
        t.T_map = surf->T_map;
        t.vt_speeds = reinterpret_cast<const double *>(base + kVtOff);
        t.vt_count = reinterpret_cast<const int *>(base + kCntOff);
    } else {
        t.face_verts = surf->face_verts;
        t.face_T = surf->face_T;
        t.face_cdf = surf->face_cdf;
        t.base_centroid = surf->base_centroid;
        t.split_planes = surf->split_planes;
        t.nface = surf->nface;
        t.nlevel = surf->nlevel;
    }
    t.density = reinterpret_cast<unsigned long long *>(density);
    t.horizon = reinterpret_cast<unsigned long long *>(horizon);
    t.stats = reinterpret_cast<unsigned long long *>(stats);
    t.out_base = pid_begin;

    // instance descriptor and boundary tables, built on the host and copied into the scratch
    unsigned char inst_host[sizeof(dsmc::FastInst)];
    float tab_host[kTabFloats];
    e = dsmc::fast_fill_instance(*p, t, pid_begin, n, reinterpret_cast<float *>(base + kTabOff),
                                 kTabFloats, inst_host, tab_host);
    if (e != cudaSuccess) return fail_cuda("instance tables", e);
    if (!ref) {
        // the FP32 copies of the icosphere tables the fast kernel descends (same as the engine)
        float4 *face = reinterpret_cast<float4 *>(base + kFaceOff);
        reinterpret_cast<dsmc::FastInst *>(inst_host)->face_f = face;
        e = dsmc::build_face_tables(t, face, stream);
        if (e != cudaSuccess) return fail_cuda("icosphere tables", e);
    }
    e = cudaMemcpyAsync(base + kInstOff, inst_host, sizeof inst_host, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + kTabOff, tab_host, sizeof tab_host, cudaMemcpyHostToDevice, stream);
    // the statistics start at zero; density and horizon are added into
    if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, dsmc::kStatCount * sizeof(uint64_t), stream);
    if (e != cudaSuccess) return fail_cuda("scratch set-up", e);
    // The drain gives up when no particle has finished for stall_launches launches in a row.
    // A legal solve can go that long only while its last particles fly: at most one hop of
    // hop_step_cap steps ends without a finish, and a life ends by its cap; the limit allows
    // twice the longest hop plus the life cap, and never fewer than 2^28 steps.
    const double hop = static_cast<double>(p->hop_step_cap);
    const double life = p->life_step_cap > 0 ? static_cast<double>(p->life_step_cap) : 0.0;
    const double quiet_steps = hop * 2.0 + life > 268435456.0 ? hop * 2.0 + life : 268435456.0;
    const long long stall_launches = static_cast<long long>(quiet_steps / kStepsPerLaunch) + 1;
    long long launches = 0;
    e = dsmc::fast_drain_external(base + kInstOff, base + kSlotOff, kSlots, base + kCtrOff, n,
                                  kStepsPerLaunch, kBlock, stall_launches, stream, &launches);
    if (e != cudaSuccess) return fail_cuda("fast solve", e);
    return DSMC_OK;
}
