// dsmc_device.cuh - device-side definitions shared by the DSMC kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "dsmc_params.h"

namespace dsmc {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwo32 = 4294967296.0;

// Statistics slots, accumulated with one atomic per warp at kernel end.
enum StatSlot { kStatSteps = 0, kStatEscaped, kStatCollisions, kStatBound, kStatFinished,
                kStatDrift, kStatCount };

// Device copies of every table a solve reads, plus the output buffers it writes.
struct DevTables {
    // reference model
    const double *T_map;          // [ftd][ffd]
    const double *vt_speeds;      // [23][1000], velocity table of src/common/velocity.c:6-47
    const int *vt_count;          // [23]
    // config model
    const double *face_verts;     // [nface][9]
    const double *face_T;         // [nface]
    const double *face_cdf;       // [nface] or nullptr (uniform face choice)
    const double *base_centroid;  // [20][3]
    const double *split_planes;   // [nnode][9]
    int nface, nlevel;
    // collisions
    const double *n_bg;
    long long n_bg_len;
    const double *cdf_coef;       // [ncell][DSMC_CDF_STRIDE]
    const double *cdf_box;        // [ncell][4]
    const double *cdf_total;      // [ncell]
    const int *cdf_valid;         // [ncell]
    int cdf_degree;
    // outputs
    unsigned long long *density;  // [hd][ftd][ffd] fixed point
    unsigned long long *horizon;  // [ftd][ffd] fixed point
    unsigned long long *speed_hist;  // [hd*ftd*ffd][n_speed_bins] or nullptr
    double *ttime;                // [9][out_cap] or nullptr
    int *fate;                    // [out_cap] or nullptr
    long long *steps;             // [out_cap] or nullptr
    long long out_base, out_cap;
    unsigned long long *stats;    // [kStatCount]
};

// Buffers of the velocity-record replay (ballistic runner): one row of per-bucket counters per
// particle of the chunk, and cap record slots per (td, ht) bucket.
struct RecordArgs {
    int *rows;                    // [chunk][ftd*hd]
    long long row_base;           // pid of row 0
    int cap;                      // records per bucket (200 in the reference)
    double *rec_v;                // [ftd*hd][cap][3]
    int *rec_fd;                  // [ftd*hd][cap]
    unsigned long long *rec_key;  // [ftd*hd][cap], (pid << 32) | step within the life
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds, two 32x32 multiplies each,
// Weyl-sequence key bumps between rounds. Counter (pid, event, instance, 0), key = seed.
struct Philox {
    uint32_t k0, k1, pid, inst, event;
    uint32_t w[4];

    __device__ __forceinline__ void init(uint64_t seed, uint32_t instance, uint32_t p) {
        k0 = static_cast<uint32_t>(seed);
        k1 = static_cast<uint32_t>(seed >> 32);
        inst = instance;
        pid = p;
        event = 0;
    }
    __device__ __forceinline__ void next() {
        uint32_t c0 = pid, c1 = event, c2 = inst, c3 = 0u, a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; r++) {
            const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
            const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
            c0 = hi1 ^ c1 ^ a;
            c1 = lo1;
            c2 = hi0 ^ c3 ^ b;
            c3 = lo0;
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        w[0] = c0; w[1] = c1; w[2] = c2; w[3] = c3;
        event++;
    }
    __device__ __forceinline__ double raw(int i) const { return static_cast<double>(w[i]); }
};

__device__ __forceinline__ unsigned long long to_fixed(double W) {
    return __double2ull_rn(W * DSMC_FIXED_SCALE);
}

// Face of the icosphere containing unit direction p: nearest base-face centroid (exact for
// the regular icosahedron), then one corner-cut test triple per subdivision level.
__device__ __forceinline__ int locate_face(const DevTables &t, const double p[3]) {
    int node = 0;
    double best = -2.0;
    for (int f = 0; f < 20; f++) {
        const double *c = t.base_centroid + 3 * f;
        double d = c[0] * p[0] + c[1] * p[1] + c[2] * p[2];
        if (d > best) { best = d; node = f; }
    }
    int offset = 0, width = 20;
    for (int level = 0; level < t.nlevel; level++) {
        const double *pl = t.split_planes + 9 * (offset + node);
        int child = (pl[0] * p[0] + pl[1] * p[1] + pl[2] * p[2] > 0.0) ? 0
                  : (pl[3] * p[0] + pl[4] * p[1] + pl[5] * p[2] > 0.0) ? 1
                  : (pl[6] * p[0] + pl[7] * p[1] + pl[8] * p[2] > 0.0) ? 2 : 3;
        node = node * 4 + child;
        offset += width;
        width *= 4;
    }
    return node;
}

// Launch face: uniform, or by binary search of the cumulative source weights.
__device__ __forceinline__ int pick_face(const DevTables &t, double u) {
    if (!t.face_cdf) {
        int f = static_cast<int>(u * t.nface);
        return f < t.nface ? f : t.nface - 1;
    }
    int lo = 0, hi = t.nface - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (t.face_cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// Warp-level sum of a 64-bit counter followed by one atomic from lane 0. Every lane of the warp
// must call it.
__device__ __forceinline__ void warp_add_stat(unsigned long long *slot, unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(slot, v);
}

}  // namespace dsmc
