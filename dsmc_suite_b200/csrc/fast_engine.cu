// fast_engine.cu - the FAST paths: resident particle slots, a device work queue, cell tracking by
// comparisons against register-cached cell bounds, and per-cell register accumulation of the
// fixed-point deposits. Two precisions share this code: FAST_FP32 pushes in FP32 with two-sum
// compensated position and velocity; FAST_FP64 runs the same loop on double state and FP64
// boundary tables without compensation, so the pair isolates what the precision buys.
//
// Per step the hot loop does one gravity evaluation (one rsqrt), the reference's Verlet variant
// (src/common/integrator.c:21-44) with the position and velocity sums kept as (hi, lo) float
// pairs (FP32) or doubles (FP64), an in-cell test against the eight bounds of the current cell
// held in registers (no asin, atan2, log or table load), photolysis as a running product
// re-anchored to W0 * 2^(-c * n_day) (one ex2), and the deposit into the register accumulator of
// the current cell, flushed with one 64-bit atomic when the particle leaves the cell. Rare events
// (cell change, launch, landing, collision, end of life) leave the loop for code that reads the
// boundary tables and the cold per-particle fields.
#include "fast_engine.h"
#include "dsmc_kernels.h"

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

namespace dsmc {
namespace {

constexpr float kPiF = 3.14159265358979f;

template <typename R>
constexpr bool is_f64() { return std::is_same<R, double>::value; }

// Compensated accumulation hi + lo += b (Dekker's fast two-sum): exact when |hi| >= |b|, which
// holds for position and velocity components except in the few steps where a component passes
// through zero, whose error is then at most ulp(b) (< 1e-4 m or 1e-7 m/s here). In FP64 the sum
// is a plain addition (lo stays zero).
__device__ __forceinline__ void accumulate(float &hi, float &lo, float b) {
    const float t = hi + b;
    lo += b - (t - hi);
    hi = t;
}

__device__ __forceinline__ void accumulate(double &hi, double &, double b) { hi += b; }

// Philox4x32-10 block of the generator's current counter, with the ten rounds kept as a loop: the
// same words as Philox::next in a fraction of its code. The collision loop takes it in its event
// paths (launch, start, collision), which run on single lanes: there it cuts ptxas' spill stores
// from 416 B to 188 B and measured 7 % faster on the 1e7-particle collisional
// phase 2; the lean and general loops measured
// 1-3 % slower with it and keep the unrolled rounds.
__device__ __forceinline__ void philox_next_rolled(Philox &r) {
    uint32_t c0 = r.pid, c1 = r.event, c2 = r.inst, c3 = 0u, a = r.k0, b = r.k1;
#pragma unroll 1
    for (int k = 0; k < 10; k++) {
        const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        c0 = hi1 ^ c1 ^ a;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ b;
        c3 = lo0;
        a += 0x9E3779B9u;
        b += 0xBB67AE85u;
    }
    r.w[0] = c0; r.w[1] = c1; r.w[2] = c2; r.w[3] = c3;
    r.event++;
}

// kRoll: the collision loop's choice of the rolled rounds (same random words either way).
template <bool kRoll>
__device__ __forceinline__ void philox_next(Philox &r) {
    if (kRoll) philox_next_rolled(r);
    else r.next();
}

// u in (0, 1): 24 random bits plus half an ulp, so 1 - u and u are never 0.
__device__ __forceinline__ float unit_open(uint32_t w) {
    return (static_cast<float>(w >> 8) + 0.5f) * (1.0f / 16777216.0f);
}

// Kernel arguments; the queue's size (total work items, instances) is read from the counters.
template <typename R>
struct FastArgsT {
    const FastInst *inst;
    SlotsT<R> s;
    long long nslots;
    FastCounters *ctr;
    int K;
};
using FastArgs = FastArgsT<float>;

// Register-resident state of the particle a thread pushes. The cold fields (particle id, Philox
// event counter, collision count, freeze waiting time) stay in the slot arrays.
template <typename R>
struct HotT {
    R sh[3], sl[3], vh[3], vl[3], oa[3];
    R w0, pcol, pthr, nsig;
    int nday, steps, hop;
    int cell;                  // packed (ht << 16) | (td << 8) | fd
    int ci;                    // (ht * ftd + td) * ffd + fd, -1 = none
    R run_w;                   // weight-steps deposited in cell ci, not yet flushed
    R W;                       // current weight: exact W0 2^(-c n_day) at cell changes and
                               // events, times 2^(-c) per day-side step in between
    int hist_key, hist_cnt;
    int inst;                  // -1 = empty slot
};
using Hot = HotT<float>;

// Bounds of the current cell: r^2 in (r2lo, r2hi], z|z| in (r^2 zlo, r^2 zhi], longitude between
// the directions (s0, c0) and (s1, c1).
template <typename R>
struct BoundsT {
    R r2lo, r2hi, zlo, zhi, s0, c0, s1, c1;
};

// The boundary tables of an instance in the engine's precision.
template <typename R> struct Tables;
template <> struct Tables<float> {
    using V2 = float2;
    __device__ static const float *rb2(const FastInst &I) { return I.rb2; }
    __device__ static const float *sbs(const FastInst &I) { return I.sbs; }
    __device__ static const float2 *lonb(const FastInst &I) { return I.lonb; }
};
template <> struct Tables<double> {
    using V2 = double2;
    __device__ static const double *rb2(const FastInst &I) { return I.rb2d; }
    __device__ static const double *sbs(const FastInst &I) { return I.sbsd; }
    __device__ static const double2 *lonb(const FastInst &I) { return I.lonbd; }
};

template <typename R>
__device__ __forceinline__ void load_hot(const SlotsT<R> &s, long long i, long long S, HotT<R> &h) {
    h.inst = s.inst[i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        h.sh[k] = s.sh[k * S + i];
        h.vh[k] = s.vh[k * S + i];
        h.oa[k] = s.oa[k * S + i];
        if constexpr (is_f64<R>()) {
            h.sl[k] = 0.0;
            h.vl[k] = 0.0;
        } else {
            h.sl[k] = s.sl[k * S + i];
            h.vl[k] = s.vl[k * S + i];
        }
    }
    h.w0 = s.w0[i];
    h.nday = s.nday[i];
    h.steps = s.steps[i];
    h.hop = s.hop[i];
    h.cell = s.cell[i];
    h.ci = s.run_cell[i];
    h.run_w = s.run_w[i];
    h.W = s.wcur[i];
    h.hist_key = s.hist_key[i];
    h.hist_cnt = s.hist_cnt[i];
    h.pcol = s.pcol[i];
    h.pthr = s.pthr[i];
    h.nsig = 0.0f;
}

template <typename R>
__device__ __forceinline__ void store_hot(const SlotsT<R> &s, long long i, long long S,
                                          const HotT<R> &h) {
    s.inst[i] = h.inst;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        s.sh[k * S + i] = h.sh[k];
        s.vh[k * S + i] = h.vh[k];
        s.oa[k * S + i] = h.oa[k];
        if constexpr (!is_f64<R>()) {
            s.sl[k * S + i] = h.sl[k];
            s.vl[k * S + i] = h.vl[k];
        }
    }
    s.w0[i] = h.w0;
    s.nday[i] = h.nday;
    s.steps[i] = h.steps;
    s.hop[i] = h.hop;
    s.cell[i] = h.cell;
    s.run_cell[i] = h.ci;
    s.run_w[i] = h.run_w;
    s.wcur[i] = h.W;
    s.hist_key[i] = h.hist_key;
    s.hist_cnt[i] = h.hist_cnt;
    s.pcol[i] = h.pcol;
    s.pthr[i] = h.pthr;
}

template <typename R>
__device__ __forceinline__ void set_pos(HotT<R> &h, const double s[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        h.sh[k] = static_cast<R>(s[k]);
        h.sl[k] = static_cast<R>(s[k] - static_cast<double>(h.sh[k]));
    }
}

template <typename R>
__device__ __forceinline__ void set_vel(HotT<R> &h, const double v[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        h.vh[k] = static_cast<R>(v[k]);
        h.vl[k] = static_cast<R>(v[k] - static_cast<double>(h.vh[k]));
    }
}

template <typename R>
__device__ __forceinline__ void get_pos(const HotT<R> &h, double s[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if constexpr (is_f64<R>()) s[k] = h.sh[k];
        else s[k] = static_cast<double>(h.sh[k]) + static_cast<double>(h.sl[k]);
    }
}

template <typename R>
__device__ __forceinline__ void get_vel(const HotT<R> &h, double v[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if constexpr (is_f64<R>()) v[k] = h.vh[k];
        else v[k] = static_cast<double>(h.vh[k]) + static_cast<double>(h.vl[k]);
    }
}

// Position component k in the engine's precision (hi + lo in FP32, the double in FP64).
template <typename R>
__device__ __forceinline__ R pos(const HotT<R> &h, int k) {
    if constexpr (is_f64<R>()) return h.sh[k];
    else return h.sh[k] + h.sl[k];
}

__device__ __forceinline__ int pack_cell(int ht, int td, int fd) { return (ht << 16) | (td << 8) | fd; }

__device__ __forceinline__ float fma_r(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }

// Latitude row and longitude column of position (x, y, z) with r2 = |s|^2, moved from the
// current (td, fd) by boundary comparisons. Row td covers latitudes (b_td, b_td+1] and column fd
// longitudes (phi_fd, phi_fd+1], the upper-inclusive cells of grid_spherical_to_index
// (src/common/grid.c:28-39).
template <typename R>
__device__ void track_angles(const FastInst &I, R x, R y, R z, R r2, int &td, int &fd) {
    const int ftd = I.p.ftd, ffd = I.p.ffd;
    const R *sbs = Tables<R>::sbs(I);
    const typename Tables<R>::V2 *lonb = Tables<R>::lonb(I);
    const R zz = z * fabs(z);
    for (int it = 0; it < 64 && td + 1 < ftd && zz > r2 * __ldg(sbs + td + 1); it++) td++;
    for (int it = 0; it < 64 && td > 0 && zz <= r2 * __ldg(sbs + td); it++) td--;
    for (int it = 0; it < 2 * 256; it++) {
        const auto hi = __ldg(lonb + fd + 1);
        if (x * hi.y - y * hi.x > R(0)) { fd = fd + 1 == ffd ? 0 : fd + 1; continue; }
        const auto lo = __ldg(lonb + fd);
        if (x * lo.y - y * lo.x <= R(0) && !(fd == 0 && x >= R(0) && y > R(0))) {
            fd = fd == 0 ? ffd - 1 : fd - 1;
            continue;
        }
        break;
    }
}

template <typename R>
__device__ void track_shell(const FastInst &I, R r2, int &ht) {
    const int hd = I.p.hd;
    const R *rb2 = Tables<R>::rb2(I);
    for (int it = 0; it < 64 && ht + 1 < hd && r2 > __ldg(rb2 + ht + 1); it++) ht++;
    for (int it = 0; it < 64 && ht > 0 && r2 <= __ldg(rb2 + ht); it++) ht--;
}

// Cell of a position from scratch: an estimate from the angles, then the comparison fix-up.
template <typename R>
__device__ int cell_from_scratch(const FastInst &I, const R x, const R y, const R z) {
    const R r2 = x * x + y * y + z * z;
    const float xf = static_cast<float>(x), yf = static_cast<float>(y), zf = static_cast<float>(z);
    const float r = sqrtf(static_cast<float>(r2));
    const float th = asinf(fminf(1.0f, fmaxf(-1.0f, zf / r)));
    float ph = atan2f(xf, yf);
    if (ph < 0.0f) ph += 2.0f * kPiF;
    int td = static_cast<int>((th + 0.5f * kPiF) / kPiF * I.p.ftd);
    int fd = static_cast<int>(ph / (2.0f * kPiF) * I.p.ffd);
    td = min(max(td, 0), I.p.ftd - 1);
    fd = min(max(fd, 0), I.p.ffd - 1);
    track_angles<R>(I, x, y, z, r2, td, fd);
    int ht;
    if (I.p.use_exp_grid) {
        // FP32 estimate; track_shell below settles the exact shell
        const float arg = static_cast<float>(I.p.alpha2 / I.p.unih) * (r - static_cast<float>(I.p.Radii)) + 1.0f;
        ht = arg <= 1.0f ? 0 : static_cast<int>(logf(arg) * static_cast<float>(1.0 / I.p.log1p_alpha2));
    } else {
        ht = static_cast<int>((static_cast<double>(r) - I.p.Radii) / I.p.unih);
    }
    ht = min(max(ht, 0), I.p.hd - 1);
    track_shell<R>(I, r2, ht);
    return pack_cell(ht, td, fd);
}

// Fixed-point deposit of a weight sum: W x 2^24 rounded once.
__device__ __forceinline__ unsigned long long fixed_of(float w) { return __float2ull_rn(w * 16777216.0f); }
__device__ __forceinline__ unsigned long long fixed_of(double w) { return __double2ull_rn(w * 16777216.0); }

// Flushes the weight-steps of the current cell as one 64-bit fixed-point atomic (W x 2^24
// summed over the steps spent in the cell, rounded once). The sum of a run is a function of the
// particle's own trajectory only, so the grid stays independent of thread order.
template <typename R>
__device__ __forceinline__ void flush_cell(const FastInst &I, HotT<R> &h) {
    if (h.ci >= 0 && h.run_w > R(0)) atomicAdd(&I.t.density[h.ci], fixed_of(h.run_w));
    h.run_w = R(0);
}

template <typename R>
__device__ __forceinline__ void flush_hist(const FastInst &I, HotT<R> &h) {
    if (h.hist_key >= 0 && h.hist_cnt)
        atomicAdd(&I.t.speed_hist[h.hist_key], static_cast<unsigned long long>(h.hist_cnt));
    h.hist_key = -1;
    h.hist_cnt = 0;
}

// Makes `cell` the current cell: flushes the previous cell's deposits, loads the eight bounds
// and the collision rate n * sigma of the new cell.
template <typename R>
__device__ void enter_cell(const FastInst &I, HotT<R> &h, BoundsT<R> &b, int cell) {
    flush_cell(I, h);
    const int ht = cell >> 16, td = (cell >> 8) & 0xff, fd = cell & 0xff;
    h.cell = cell;
    h.ci = (ht * I.p.ftd + td) * I.p.ffd + fd;
    const R *rb2 = Tables<R>::rb2(I);
    const R *sbs = Tables<R>::sbs(I);
    const typename Tables<R>::V2 *lonb = Tables<R>::lonb(I);
    b.r2lo = __ldg(rb2 + ht);
    b.r2hi = __ldg(rb2 + ht + 1);
    b.zlo = __ldg(sbs + td);
    b.zhi = __ldg(sbs + td + 1);
    const auto lo = __ldg(lonb + fd), hi = __ldg(lonb + fd + 1);
    b.s0 = lo.x;
    b.c0 = lo.y;
    b.s1 = hi.x;
    b.c1 = hi.y;
    h.nsig = R(0);
    if (I.t.n_bg && I.p.runner == DSMC_RUNNER_ADVANCED && ht < I.p.collide_ht_max &&
        h.ci < I.t.n_bg_len)
        h.nsig = static_cast<R>(__ldg(I.t.n_bg + h.ci) * I.p.cross_section);
}

template <typename R>
__device__ __forceinline__ R exp2_r(R x) {
    if constexpr (is_f64<R>()) return exp2(x);
    else return exp2f(x);
}

// FP32 engines keep the day constant in FP32, FP64 engines in FP64.
template <typename R>
__device__ __forceinline__ R c_day_of(const FastInst &I) {
    if constexpr (is_f64<R>()) return I.c_day_d;
    else return I.c_day;
}

// The particle left its cell: walk to the new cell one boundary at a time. Each move keeps the
// shared boundary from the registers and loads only the next one, so a typical crossing costs
// one table load. Same cells as track_shell / track_angles. in_r, in_t, in_f are the step's own
// inside tests per coordinate; only the coordinates that failed are walked (7 % faster on
// the 1e8-particle Ceres-like workload than walking all three, identical cells).
template <bool kNoBg, typename R>
__device__ __forceinline__ void move_cell(const FastInst &I, HotT<R> &h, BoundsT<R> &b, R x, R y,
                                          R r2, R zz, bool in_r, bool in_t, bool in_f) {
    int ht = h.cell >> 16, td = (h.cell >> 8) & 0xff, fd = h.cell & 0xff;
    // the three walks are independent (shells by r^2, rows by z|z| / r^2, columns by the
    // longitude tests), so a coordinate still inside its two bounds needs no walk. Each walk
    // goes one way only: after a move up the old upper bound is the new lower one, which the
    // particle is above, so the downward test cannot pass (and the other way round); the
    // walks test one bound per move (same cells as testing both).
    if (!in_r) {
        const int hd = I.p.hd;
        const R *rb2 = Tables<R>::rb2(I);
        if (r2 > b.r2hi) {
            for (int it = 0; it < 64 && r2 > b.r2hi && ht + 1 < hd; it++) {
                ht++;
                b.r2lo = b.r2hi;
                b.r2hi = __ldg(rb2 + ht + 1);
            }
        } else {
            for (int it = 0; it < 64 && r2 <= b.r2lo && ht > 0; it++) {
                ht--;
                b.r2hi = b.r2lo;
                b.r2lo = __ldg(rb2 + ht);
            }
        }
    }
    if (!in_t) {
        const int ftd = I.p.ftd;
        const R *sbs = Tables<R>::sbs(I);
        if (zz > r2 * b.zhi) {
            for (int it = 0; it < 64 && zz > r2 * b.zhi && td + 1 < ftd; it++) {
                td++;
                b.zlo = b.zhi;
                b.zhi = __ldg(sbs + td + 1);
            }
        } else {
            for (int it = 0; it < 64 && zz <= r2 * b.zlo && td > 0; it++) {
                td--;
                b.zhi = b.zlo;
                b.zlo = __ldg(sbs + td);
            }
        }
    }
    if (!in_f) {
        const int ffd = I.p.ffd;
        const typename Tables<R>::V2 *lonb = Tables<R>::lonb(I);
        if (x * b.c1 - y * b.s1 > R(0)) {
            for (int it = 0; it < 512 && x * b.c1 - y * b.s1 > R(0); it++) {
                fd = fd + 1 == ffd ? 0 : fd + 1;
                b.s0 = b.s1;
                b.c0 = b.c1;
                const auto q = __ldg(lonb + fd + 1);
                b.s1 = q.x;
                b.c1 = q.y;
            }
        } else {
            for (int it = 0; it < 512 && x * b.c0 - y * b.s0 <= R(0) && !(fd == 0 && x >= R(0) && y > R(0));
                 it++) {
                fd = fd == 0 ? ffd - 1 : fd - 1;
                b.s1 = b.s0;
                b.c1 = b.c0;
                const auto q = __ldg(lonb + fd);
                b.s0 = q.x;
                b.c0 = q.y;
            }
        }
    }
    const int cell = pack_cell(ht, td, fd);
    if (cell == h.cell) return;
    // the run of a flying particle has a cell and no negative weight: flushed without the tests
    // of flush_cell (a run of zero adds zero)
    atomicAdd(&I.t.density[h.ci], fixed_of(h.run_w));
    h.run_w = R(0);
    h.cell = cell;
    h.ci = (ht * I.p.ftd + td) * I.p.ffd + fd;
    h.W = h.w0 * exp2_r<R>(-c_day_of<R>(I) * static_cast<R>(h.nday));   // re-anchor the running weight
    if (!kNoBg && I.t.n_bg) {
        h.nsig = R(0);
        if (I.p.runner == DSMC_RUNNER_ADVANCED && ht < I.p.collide_ht_max && h.ci < I.t.n_bg_len)
            h.nsig = static_cast<R>(__ldg(I.t.n_bg + h.ci) * I.p.cross_section);
    }
}

__device__ __forceinline__ double cdf_eval(const double *coef, const double *box, int degree,
                                           double x) {
    const double t = (x - box[2]) / box[3];
    double r = 0.0;
    for (int i = 0; i <= degree; i++) r = r * t + coef[i];
    return r;
}

// Bisection of the fitted reverse-cumulative speed distribution (collision.c:43-101).
__device__ double cdf_sample(const double *coef, const double *box, double total, int degree,
                             double u) {
    const double at_max = cdf_eval(coef, box, degree, box[1]);
    const double ranking = u * (total - at_max) + at_max;
    double v0 = box[0], v1 = box[1];
    for (int iter = 0; iter < 100; iter++) {
        const double vm = (v0 + v1) * 0.5;
        const double fm = cdf_eval(coef, box, degree, vm) - ranking;
        const double f1 = cdf_eval(coef, box, degree, v1) - ranking;
        if (fm * f1 < 0) v0 = vm;
        else v1 = vm;
        if (fabs(v1 - v0) < 0.01) break;
    }
    return (v0 + v1) * 0.5;
}

__device__ __forceinline__ void unit_sphere_f(float zu, float pu, float o[3]) {
    const float z = 2.0f * zu - 1.0f;
    const float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float sn, cs;
    sincosf(2.0f * kPiF * pu, &sn, &cs);
    o[0] = rr * cs;
    o[1] = rr * sn;
    o[2] = z;
}

// The FP64 path's unit vector: the plain FP64 kernel's map of two uniforms.
__device__ __forceinline__ void unit_sphere_d(double zu, double pu, double o[3]) {
    const double z = 2.0 * zu - 1.0;
    const double rr = sqrt(fmax(0.0, 1.0 - z * z));
    double sn, cs;
    sincos(2.0 * kPi * pu, &sn, &cs);
    o[0] = rr * cs;
    o[1] = rr * sn;
    o[2] = z;
}

struct StatAcc {
    unsigned steps = 0, escaped = 0, collisions = 0, bound = 0, finished = 0, drift = 0;
    int inst = -1;
};

// Adds the thread's statistics into its instance's counters: lanes of one instance are summed
// with one warp reduction and one atomic per counter. Every lane of the warp must call it.
template <typename A>
__device__ void flush_stats(const A &a, StatAcc &st) {
    const unsigned full = 0xffffffffu;
    const int key = st.inst;
    const unsigned group = __match_any_sync(full, key);
    const unsigned v[6] = {st.steps, st.escaped, st.collisions, st.bound, st.finished, st.drift};
    const int slot_of[6] = {kStatSteps, kStatEscaped, kStatCollisions, kStatBound, kStatFinished,
                            kStatDrift};
    const bool leader = (threadIdx.x & 31) == (__ffs(group) - 1);
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const unsigned sum = __reduce_add_sync(group, v[k]);
        if (leader && key >= 0 && sum)
            atomicAdd(&a.inst[key].t.stats[slot_of[k]], static_cast<unsigned long long>(sum));
    }
    st = StatAcc{};
}

// The previous instance's share of the counters, lane by lane (an instance switch inside a
// launch happens at most once per particle and is rare).
template <typename A>
__device__ void flush_stats_lane(const A &a, StatAcc &st) {
    if (st.inst >= 0) {
        unsigned long long *dst = a.inst[st.inst].t.stats;
        if (st.steps) atomicAdd(dst + kStatSteps, static_cast<unsigned long long>(st.steps));
        if (st.escaped) atomicAdd(dst + kStatEscaped, static_cast<unsigned long long>(st.escaped));
        if (st.collisions) atomicAdd(dst + kStatCollisions, static_cast<unsigned long long>(st.collisions));
        if (st.bound) atomicAdd(dst + kStatBound, static_cast<unsigned long long>(st.bound));
        if (st.drift) atomicAdd(dst + kStatDrift, static_cast<unsigned long long>(st.drift));
        if (st.finished) {
            atomicAdd(dst + kStatFinished, static_cast<unsigned long long>(st.finished));
            atomicAdd(&a.ctr->finished, static_cast<unsigned long long>(st.finished));
        }
    }
    st = StatAcc{};
}

template <typename R>
__device__ __forceinline__ R weight(const FastInst &I, const HotT<R> &h) {
    return h.w0 * exp2_r<R>(-c_day_of<R>(I) * static_cast<R>(h.nday));
}

// Row and column of the reference model's angles (grid_spherical_to_index, grid.c:28-39).
__device__ __forceinline__ void ref_index(float thi, float fi, int ftd, int ffd, int &td, int &fd) {
    td = static_cast<int>(ceilf((thi + 0.5f * kPiF) / kPiF * ftd)) - 1;
    fd = static_cast<int>(ceilf(fi / (2.0f * kPiF) * ffd)) - 1;
    td = min(max(td, 0), ftd - 1);
    fd = min(max(fd, 0), ffd - 1);
}

__device__ __forceinline__ void ref_index(double thi, double fi, int ftd, int ffd, int &td, int &fd) {
    td = static_cast<int>(ceil((thi + kPi / 2.0) / kPi * ftd)) - 1;
    fd = static_cast<int>(ceil(fi / (2.0 * kPi) * ffd)) - 1;
    td = min(max(td, 0), ftd - 1);
    fd = min(max(fd, 0), ffd - 1);
}

// Latitude and longitude of the current position, computed in FP64 (pos_to_angles,
// ballistic.c:29-33) and returned in the engine's precision.
template <typename R>
__device__ __forceinline__ void angles_of(const HotT<R> &h, R &thi, R &fi) {
    double s[3];
    get_pos(h, s);
    const double Ri = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    thi = static_cast<R>(asin(s[2] / Ri));
    double f = atan2(s[0], s[1]);
    if (f < 0) f += 2.0 * kPi;
    fi = static_cast<R>(f);
}

// Orbital energy per unit mass |v|^2 / 2 - GM / |s| of the current state in FP64, for the
// per-hop energy-drift guard: 1 / |s| from the FP32 reciprocal square root and one Newton step in
// FP64 (relative error ~1e-14), so the event path takes no FP64 square root or division.
template <typename R>
__device__ __forceinline__ double orbital_energy(const FastInst &I, const HotT<R> &h) {
    double s[3], v[3];
    get_pos(h, s);
    get_vel(h, v);
    const double r2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    double ir = rsqrtf(static_cast<float>(r2));
    ir = ir * (1.5 - 0.5 * r2 * ir * ir);
    return 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - I.p.GM * ir;
}

// The hop's energy baseline: taken at every launch and after every collision.
template <typename R>
__device__ __forceinline__ void drift_start(const FastArgsT<R> &a, long long i, const FastInst &I,
                                            const HotT<R> &h) {
    if (I.drift_abs > 0.0) a.s.e0[i] = static_cast<float>(orbital_energy(I, h));
}

// The hop ended (landing, escape radius, hop or life cap): counts it when the energy moved by
// more than the guard's bound since the baseline.
template <typename R>
__device__ __forceinline__ void drift_check(const FastArgsT<R> &a, long long i, const FastInst &I,
                                            const HotT<R> &h, StatAcc &st) {
    if (I.drift_abs > 0.0 &&
        fabs(orbital_energy(I, h) - static_cast<double>(a.s.e0[i])) > I.drift_abs)
        st.drift++;
}

__device__ __forceinline__ void horizon_add(const FastInst &I, int td, int fd, float W) {
    atomicAdd(&I.t.horizon[td * I.p.ffd + fd], __float2ull_rn(W * 16777216.0f));
}

__device__ __forceinline__ void horizon_add(const FastInst &I, int td, int fd, double W) {
    atomicAdd(&I.t.horizon[td * I.p.ffd + fd], __double2ull_rn(W * DSMC_FIXED_SCALE));
}

// Old acceleration GM s / r^3 of a launch point (ballistic.c:176-181; the FP32 engine keeps it
// times dt) and the hop's start. The energy baseline of the drift guard comes from e_launch when
// the launch already formed it.
template <typename R>
__device__ __forceinline__ void start_hop_state(const FastArgsT<R> &a, long long i,
                                                const FastInst &I, HotT<R> &h,
                                                const double *e_launch) {
    if constexpr (is_f64<R>()) {
        const double sx = h.sh[0], sy = h.sh[1], sz = h.sh[2];
        const double ir = rsqrt(sx * sx + sy * sy + sz * sz);
        const double g = I.p.GM * (ir * ir * ir);
        h.oa[0] = g * sx;
        h.oa[1] = g * sy;
        h.oa[2] = g * sz;
    } else {
        const float sx = h.sh[0] + h.sl[0], sy = h.sh[1] + h.sl[1], sz = h.sh[2] + h.sl[2];
        const float ir = rsqrtf(fmaf(sx, sx, fmaf(sy, sy, sz * sz)));
        const float g = static_cast<float>(I.p.GM * I.p.dt_step) * (ir * ir * ir);
        h.oa[0] = g * sx;
        h.oa[1] = g * sy;
        h.oa[2] = g * sz;
    }
    h.hop = 0;
    if (!e_launch) drift_start(a, i, I, h);
    else if (I.drift_abs > 0.0) a.s.e0[i] = static_cast<float>(*e_launch);
}

// Orbital energy of a launch from the |v|^2 and |s|^2 its bound test formed: 1 / |s| as in
// orbital_energy, so the baseline equals orbital_energy of the launched state.
__device__ __forceinline__ double launch_energy(const FastInst &I, double v2, double r2) {
    double ir = rsqrtf(static_cast<float>(r2));
    ir = ir * (1.5 - 0.5 * r2 * ir * ir);
    return 0.5 * v2 - I.p.GM * ir;
}

// Launch from the current surface position (ballistic.c:156-181; config: flux-weighted
// Maxwell-Boltzmann). Returns false when the reference's launch-speed escape test fires.
// kCfg: every instance of the launch is a config-model problem, so the reference-model branches
// of the event code are compiled out (shorter code on the path that high-gravity bodies take every
// few hundred steps). The FP32 engine maps the random words in FP32 with reciprocal square roots;
// the FP64 engine takes the plain FP64 kernel's maps.
template <bool kCfg, bool kRoll, typename R>
__device__ bool launch(const FastArgsT<R> &a, long long i, const FastInst &I, HotT<R> &h,
                       StatAcc &st, R local_T, R thi, R fi) {
    const dsmc_params &p = I.p;
    Philox rng;
    rng.init(p.seed, p.instance, a.s.pid[i]);
    rng.event = a.s.evt[i];
    philox_next<kRoll>(rng);
    a.s.evt[i] = rng.event;
    double s[3];
    get_pos(h, s);
    double vd[3];
    double e_launch = 0.0;
    bool have_e = false;
    if constexpr (is_f64<R>()) {
        if (!kCfg && p.model == DSMC_MODEL_REFERENCE) {
            // velocity_sample / velocity_sticking (velocity.c:49-73), ballistic.c:156-173
            const double KF = 2.0 * kPi * p.Radii * fabs(cos(thi)) / p.P;
            int idx = local_T >= 220.0 ? 20 : static_cast<int>(ceil(local_T / 10.0)) - 2;
            idx = idx < 0 ? 0 : (idx >= 23 ? 22 : idx);
            const double vr = I.t.vt_speeds[idx * 1000 + rng.w[0] % static_cast<uint32_t>(I.t.vt_count[idx])];
            double v_old[3];
            get_vel(h, v_old);
            const double vold2 = v_old[0] * v_old[0] + v_old[1] * v_old[1] + v_old[2] * v_old[2];
            const double vout = sqrt(p.alpha * vr * vr + (1.0 - p.alpha) * vold2);
            const double flyd = rng.raw(1) / kTwo32 * kPi + thi - kPi / 2.0;
            const double xi = rng.raw(2) / kTwo32 * kPi + fi - kPi / 2.0;
            vd[0] = cos(flyd) * sin(xi) * vout + KF * sin(fi + kPi / 2.0);
            vd[1] = cos(flyd) * cos(xi) * vout + KF * cos(fi + kPi / 2.0);
            vd[2] = sin(flyd) * vout;
            if (sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]) >= p.ve) return false;
        } else {
            const double sigma = sqrt(p.kB_over_m * local_T);
            const double vn = sigma * sqrt(-2.0 * log(1.0 - rng.raw(0) / kTwo32));
            const double rho = sqrt(-2.0 * log(1.0 - rng.raw(1) / kTwo32));
            double sa, ca;
            sincos(2.0 * kPi * (rng.raw(2) / kTwo32), &sa, &ca);
            const double t1 = rho * ca, t2 = rho * sa;
            const double ir = rsqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
            const double n[3] = {s[0] * ir, s[1] * ir, s[2] * ir};
            double e[3] = {-n[1], n[0], 0.0};
            const double le2 = e[0] * e[0] + e[1] * e[1];
            if (le2 < 1e-24) { e[0] = 1.0; e[1] = 0.0; }
            else { const double il = rsqrt(le2); e[0] *= il; e[1] *= il; }
            const double nt[3] = {n[1] * e[2] - n[2] * e[1], n[2] * e[0] - n[0] * e[2], n[0] * e[1] - n[1] * e[0]};
            const double omega = p.P > 0.0 ? 2.0 * kPi / p.P : 0.0;
            const double rot[3] = {omega * s[1], -omega * s[0], 0.0};
#pragma unroll
            for (int k = 0; k < 3; k++) vd[k] = vn * n[k] + (sigma * t1) * e[k] + (sigma * t2) * nt[k] + rot[k];
            // FP64 escape/bound classification: E < 0 exactly when (v^2)^2 r^2 < (2 GM)^2
            const double v2 = vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2];
            const double rr = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
            if (v2 * v2 * rr < 4.0 * p.GM * p.GM) st.bound++;
            e_launch = launch_energy(I, v2, rr);
            have_e = true;
        }
    } else {
        float v[3];
        if (!kCfg && p.model == DSMC_MODEL_REFERENCE) {
            const float KF = 2.0f * kPiF * static_cast<float>(p.Radii) * fabsf(cosf(thi)) / static_cast<float>(p.P);
            int idx = local_T >= 220.0f ? 20 : static_cast<int>(ceilf(local_T / 10.0f)) - 2;
            idx = idx < 0 ? 0 : (idx >= 23 ? 22 : idx);
            const float vr = static_cast<float>(I.t.vt_speeds[idx * 1000 + rng.w[0] % static_cast<uint32_t>(I.t.vt_count[idx])]);
            float vold2 = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; k++) vold2 += h.vh[k] * h.vh[k];
            const float alpha = static_cast<float>(p.alpha);
            const float vout = sqrtf(alpha * vr * vr + (1.0f - alpha) * vold2);
            const float flyd = static_cast<float>(rng.w[1]) * (kPiF / 4294967296.0f) + thi - 0.5f * kPiF;
            const float xi = static_cast<float>(rng.w[2]) * (kPiF / 4294967296.0f) + fi - 0.5f * kPiF;
            float sf, cf, sx, cx, sr, cr;
            sincosf(flyd, &sf, &cf);
            sincosf(xi, &sx, &cx);
            sincosf(fi + 0.5f * kPiF, &sr, &cr);
            v[0] = cf * sx * vout + KF * sr;
            v[1] = cf * cx * vout + KF * cr;
            v[2] = sf * vout;
            if (sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) >= static_cast<float>(p.ve)) return false;
        } else {
            // the same maps of the random words as the FP64 path: log(1 - u) and angle 2 pi u
            const float sigma = sqrtf(static_cast<float>(p.kB_over_m) * local_T);
            const float vn = sigma * sqrtf(-2.0f * logf(1.0f - unit_open(rng.w[0])));
            const float rho = sqrtf(-2.0f * logf(1.0f - unit_open(rng.w[1])));
            float sa, ca;
            __sincosf(2.0f * kPiF * unit_open(rng.w[2]), &sa, &ca);   // argument in [0, 2 pi)
            const float t1 = rho * ca, t2 = rho * sa;
            // the event path stays short (no divisions, no FP64 square roots): unit normal and
            // east vector by reciprocal square roots
            const float px = h.sh[0] + h.sl[0], py = h.sh[1] + h.sl[1], pz = h.sh[2] + h.sl[2];
            const float ir = rsqrtf(fmaf(px, px, fmaf(py, py, pz * pz)));
            const float n[3] = {px * ir, py * ir, pz * ir};
            float e[3] = {-n[1], n[0], 0.0f};
            const float le2 = fmaf(e[0], e[0], e[1] * e[1]);
            if (le2 < 1e-12f) { e[0] = 1.0f; e[1] = 0.0f; }
            else { const float il = rsqrtf(le2); e[0] *= il; e[1] *= il; }
            const float nt[3] = {n[1] * e[2] - n[2] * e[1], n[2] * e[0] - n[0] * e[2], n[0] * e[1] - n[1] * e[0]};
            const float omega = p.P > 0.0 ? static_cast<float>(2.0 * kPi / p.P) : 0.0f;
            const float rot[3] = {omega * static_cast<float>(s[1]), -omega * static_cast<float>(s[0]), 0.0f};
#pragma unroll
            for (int k = 0; k < 3; k++) v[k] = vn * n[k] + (sigma * t1) * e[k] + (sigma * t2) * nt[k] + rot[k];
            // FP64 escape/bound classification of the launch: E = v^2/2 - GM/r < 0 exactly when
            // (v^2)^2 r^2 < (2 GM)^2, which needs no square root or division
            const double v2 = static_cast<double>(v[0]) * v[0] + static_cast<double>(v[1]) * v[1] +
                              static_cast<double>(v[2]) * v[2];
            const double rr = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
            if (v2 * v2 * rr < 4.0 * p.GM * p.GM) st.bound++;
            e_launch = launch_energy(I, v2, rr);
            have_e = true;
        }
        vd[0] = v[0];
        vd[1] = v[1];
        vd[2] = v[2];
    }
    set_vel(h, vd);
    start_hop_state(a, i, I, h, have_e ? &e_launch : nullptr);
    return true;
}

// Cell of a launch point from the latitude and longitude the particle had when it landed,
// starting in the lowest shell, moved by the comparison walks (no asin, atan2 or log).
template <typename R>
__device__ void enter_cell_near(const FastInst &I, HotT<R> &h, BoundsT<R> &b) {
    const R x = pos(h, 0), y = pos(h, 1), z = pos(h, 2);
    const R r2 = fma_r(x, x, fma_r(y, y, z * z));
    int ht = 0, td = (h.cell >> 8) & 0xff, fd = h.cell & 0xff;
    track_shell<R>(I, r2, ht);
    track_angles<R>(I, x, y, z, r2, td, fd);
    enter_cell(I, h, b, pack_cell(ht, td, fd));
}

// Longitude of the centre of column fd (the reference's freeze scan, ballistic.c:140).
template <typename R>
__device__ __forceinline__ R column_centre(int fd, int ffd) {
    if constexpr (is_f64<R>()) return (fd + 0.5) / ffd * 2.0 * kPi;
    else return (fd + 0.5f) / ffd * 2.0f * kPiF;
}

// Start of a hop (ballistic.c:124-181, advanced.c:271-333): weight and life checks, the
// reference freeze scan, the launch and the starting cell. Returns 0 when the particle flies,
// else its fate.
template <bool kCfg, bool kRoll, typename R>
__device__ int hop_top(const FastArgsT<R> &a, long long i, const FastInst &I, HotT<R> &h,
                       BoundsT<R> &b, StatAcc &st, R thi, R fi, R local_T, bool first) {
    const dsmc_params &p = I.p;
    const R W = weight(I, h);
    if (W < static_cast<R>(p.w_min)) return DSMC_FATE_PHOTOLYSED;
    if (p.life_step_cap > 0 && h.steps >= p.life_step_cap) return DSMC_FATE_STEP_CAP;
    if (!kCfg && p.model == DSMC_MODEL_REFERENCE) {
        const int ftd = p.ftd, ffd = p.ffd;
        int td, fd;
        ref_index(thi, fi, ftd, ffd, td, fd);
        const double *T = I.t.T_map;
        local_T = static_cast<R>(T[td * ffd + fd]);
        if (local_T < static_cast<R>(p.freeze_T)) {
            bool found = false;
            float rest = a.s.rest[i];
            if (p.runner == DSMC_RUNNER_BALLISTIC) {
                for (int add = 0; add < ffd; add++) {
                    rest += static_cast<float>(p.dt_rot);
                    const int check = (fd + add + 1) % ffd;
                    if (T[td * ffd + check] >= p.freeze_T) {
                        fd = check;
                        fi = column_centre<R>(fd, ffd);
                        found = true;
                        break;
                    }
                }
            } else {
                horizon_add(I, td, fd, W);
                for (int add = 1; add <= ffd; add++) {
                    rest += static_cast<float>(p.dt_rot);
                    if (T[td * ffd + (add % ffd)] >= p.freeze_T) {
                        const double rot_fi = static_cast<double>(add - fd) / ffd * 2.0 * kPi;
                        const double cs = cos(rot_fi), sn = sin(rot_fi);
                        double s[3];
                        get_pos(h, s);
                        const double n0 = s[0] * cs - s[1] * sn, n1 = s[0] * sn + s[1] * cs;
                        s[0] = n0;
                        s[1] = n1;
                        set_pos(h, s);
                        fd = add % ffd;
                        fi = column_centre<R>(fd, ffd);
                        found = true;
                        break;
                    }
                }
            }
            a.s.rest[i] = rest;
            if (!found) {
                horizon_add(I, td, fd, W);
                return DSMC_FATE_FROZEN;
            }
            local_T = static_cast<R>(T[td * ffd + fd]);
        }
    }
    if (!launch<kCfg, kRoll>(a, i, I, h, st, local_T, thi, fi)) return DSMC_FATE_ESCAPED;
    // the running weight restarts from its exact value at every launch (and at every cell
    // change): points of the particle's own trajectory, so results do not depend on where
    // kernel launches begin or end (the launch changes neither w0 nor the day count)
    h.W = W;
    if (first)
        enter_cell(I, h, b, cell_from_scratch<R>(I, pos(h, 0), pos(h, 1), pos(h, 2)));
    else
        enter_cell_near(I, h, b);
    return 0;
}

// Latitude and longitude of the current position in FP32 (the reference model's relaunch
// angles, ballistic.c:245-247).
__device__ __forceinline__ void angles_of_f(const Hot &h, float &thi, float &fi) {
    const float x = h.sh[0] + h.sl[0], y = h.sh[1] + h.sl[1], z = h.sh[2] + h.sl[2];
    thi = asinf(fminf(1.0f, fmaxf(-1.0f, z * rsqrtf(fmaf(x, x, fmaf(y, y, z * z))))));
    fi = atan2f(x, y);
    if (fi < 0.0f) fi += 2.0f * kPiF;
}

// Face of the icosphere containing unit direction n, from the FP32 tables: the nearest of the 20
// base-face centroids, then one corner-cut test triple per subdivision level (the FP64 descent of
// locate_face on FP32 copies).
__device__ __forceinline__ int locate_face_f(const float4 *tab, int nlevel, const float n[3]) {
    int node = 0;
    float best = -2.0f;
#pragma unroll 4
    for (int f = 0; f < 20; f++) {
        const float4 c = __ldg(tab + f);
        const float d = c.x * n[0] + c.y * n[1] + c.z * n[2];
        if (d > best) { best = d; node = f; }
    }
    int offset = 0, width = 20;
    for (int level = 0; level < nlevel; level++) {
        const float4 *pl = tab + 20 + 3 * (offset + node);
        const float4 a = __ldg(pl), b = __ldg(pl + 1), c = __ldg(pl + 2);
        const int child = (a.x * n[0] + a.y * n[1] + a.z * n[2] > 0.0f) ? 0
                        : (b.x * n[0] + b.y * n[1] + b.z * n[2] > 0.0f) ? 1
                        : (c.x * n[0] + c.y * n[1] + c.z * n[2] > 0.0f) ? 2 : 3;
        node = node * 4 + child;
        offset += width;
        width *= 4;
    }
    return node;
}

// Landing (ballistic.c:239-264): polar deposit (reference) or night freeze-out / day-side
// re-emission point (config). Returns 0 to start a new hop, else the fate.
template <bool kCfg, typename R>
__device__ int land(const FastArgsT<R> &a, long long i, const FastInst &I, HotT<R> &h, R &thi,
                    R &fi, R &local_T) {
    const dsmc_params &p = I.p;
    int td, fd;
    if (!kCfg && p.model == DSMC_MODEL_REFERENCE) {
        if constexpr (is_f64<R>()) angles_of(h, thi, fi);
        else angles_of_f(h, thi, fi);
        ref_index(thi, fi, p.ftd, p.ffd, td, fd);
        if (td <= 1 || td >= p.ftd - 2) {
            horizon_add(I, td, fd, static_cast<R>(0.05) * weight(I, h));
            h.w0 *= static_cast<R>(0.95);
        }
        return 0;
    }
    if constexpr (is_f64<R>()) {
        // FP64 normal and face descent (the plain kernel's landing arithmetic)
        double s[3];
        get_pos(h, s);
        const double r2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
        const double Ri = sqrt(r2);
        const double nd[3] = {s[0] / Ri, s[1] / Ri, s[2] / Ri};
        if (nd[0] * p.sun[0] + nd[1] * p.sun[1] + nd[2] * p.sun[2] <= 0.0) {
            td = (h.cell >> 8) & 0xff;
            fd = h.cell & 0xff;
            track_angles<double>(I, s[0], s[1], s[2], r2, td, fd);
            horizon_add(I, td, fd, weight(I, h));
            return DSMC_FATE_FROZEN;
        }
        const double sn[3] = {nd[0] * p.Radii, nd[1] * p.Radii, nd[2] * p.Radii};
        set_pos(h, sn);
        const int face = locate_face(I.t, nd);
        a.s.face[i] = face;
        local_T = I.t.face_T[face];
        return 0;
    } else {
        // FP32 normal; the landing cell of a night-side freeze-out by comparison walks from the
        // last cell (the upper-inclusive cells of grid_spherical_to_index without asin or atan2)
        const float x = h.sh[0] + h.sl[0], y = h.sh[1] + h.sl[1], z = h.sh[2] + h.sl[2];
        const float r2 = fmaf(x, x, fmaf(y, y, z * z));
        const float ir = rsqrtf(r2);
        const float n[3] = {x * ir, y * ir, z * ir};
        if (fmaf(n[0], static_cast<float>(p.sun[0]), fmaf(n[1], static_cast<float>(p.sun[1]),
                                                          n[2] * static_cast<float>(p.sun[2]))) <= 0.0f) {
            td = (h.cell >> 8) & 0xff;
            fd = h.cell & 0xff;
            track_angles<float>(I, x, y, z, r2, td, fd);
            horizon_add(I, td, fd, weight(I, h));
            return DSMC_FATE_FROZEN;
        }
        // day side: re-emission from the surface point below the landing point
        const double nd[3] = {n[0], n[1], n[2]};
        const double s[3] = {nd[0] * p.Radii, nd[1] * p.Radii, nd[2] * p.Radii};
        set_pos(h, s);
        int face;
        if (I.face_f) {
            // hops are short next to the face size on high-gravity bodies: try the face of the
            // last launch point first (three sign tests), descend the tree only when the point
            // left it
            const int last = a.s.face[i];
            const int nnode = 20 * ((1 << (2 * I.t.nlevel)) - 1) / 3;
            const float4 *ed = I.face_f + 20 + 3 * nnode + 3 * last;
            bool inside = last >= 0;
            if (inside) {
                const float4 e0 = __ldg(ed), e1 = __ldg(ed + 1), e2 = __ldg(ed + 2);
                inside = (e0.x * n[0] + e0.y * n[1] + e0.z * n[2] >= 0.0f) &
                         (e1.x * n[0] + e1.y * n[1] + e1.z * n[2] >= 0.0f) &
                         (e2.x * n[0] + e2.y * n[1] + e2.z * n[2] >= 0.0f);
            }
            face = inside ? last : locate_face_f(I.face_f, I.t.nlevel, n);
            a.s.face[i] = face;
        } else {
            face = locate_face(I.t, nd);
        }
        local_T = static_cast<float>(I.t.face_T[face]);
        return 0;
    }
}

// End of a particle's life: per-particle rows (layout of ballistic.c:120,273-276 and
// advanced.c:262-267,439-444), counters, deposits flushed.
template <typename R>
__device__ void finish(const FastArgsT<R> &a, long long i, const FastInst &I, HotT<R> &h,
                       StatAcc &st, int fate) {
    const dsmc_params &p = I.p;
    const DevTables &t = I.t;
    const bool ref = p.model == DSMC_MODEL_REFERENCE, adv = p.runner == DSMC_RUNNER_ADVANCED;
    const unsigned pid = a.s.pid[i];
    const int ncol = a.s.ncol[i];
    const long long slot = static_cast<long long>(pid) - t.out_base;
    if (slot >= 0 && slot < t.out_cap) {
        if (t.ttime && (fate != DSMC_FATE_ESCAPED || !ref)) {
            R thi, fi;
            angles_of(h, thi, fi);
            const float rest = a.s.rest[i];
            const double flight = static_cast<double>(h.steps) * p.dt_step;
            t.ttime[1 * t.out_cap + slot] = thi;
            t.ttime[2 * t.out_cap + slot] = flight + rest;
            t.ttime[3 * t.out_cap + slot] = weight(I, h);
            t.ttime[4 * t.out_cap + slot] = flight;
            if (adv || !ref) {
                t.ttime[7 * t.out_cap + slot] = rest;
                t.ttime[8 * t.out_cap + slot] = ncol;
            }
        }
        if (t.fate) t.fate[slot] = fate;
        if (t.steps) t.steps[slot] = h.steps;
    }
    st.finished++;
    st.collisions += ncol;
    if (fate == DSMC_FATE_ESCAPED) st.escaped++;
    flush_cell(I, h);
    flush_hist(I, h);
    h.ci = -1;
    h.inst = -1;
}

// A collision against a partner drawn from the cell's fitted speed CDF (advanced.c:374-396).
template <bool kRoll, typename R>
__device__ void collide(const FastArgsT<R> &a, long long i, const FastInst &I, HotT<R> &h,
                        long long pidx) {
    const dsmc_params &p = I.p;
    const DevTables &t = I.t;
    Philox rng;
    rng.init(p.seed, p.instance, a.s.pid[i]);
    rng.event = a.s.evt[i];
    philox_next<kRoll>(rng);
    const double *coef = t.cdf_coef + DSMC_CDF_STRIDE * pidx;
    const double *box = t.cdf_box + 4 * pidx;
    double v[3];
    get_vel(h, v);
    const double vv2 = cdf_sample(coef, box, t.cdf_total[pidx], t.cdf_degree, rng.raw(0) / kTwo32);
    double col_p = -1.0;
    if (p.scatter == DSMC_SCATTER_REFERENCE) {
        const double thi2 = kPi * rng.raw(1) / kTwo32 - kPi / 2.0;
        const double fi2 = 2.0 * kPi * rng.raw(2) / kTwo32;
        const double v2[3] = {vv2 * cos(thi2) * cos(fi2), vv2 * cos(thi2) * sin(fi2), vv2 * sin(thi2)};
        for (int k = 0; k < 3; k++) v[k] = (v[k] + v2[k]) + 0.5 * (v[k] - v2[k]);
        if (p.redraw_col_threshold) col_p = rng.raw(3) / kTwo32;
    } else {
        double d2[3], om[3];
        if constexpr (is_f64<R>()) {
            // the plain FP64 kernel's maps of the random words
            unit_sphere_d(rng.raw(1) / kTwo32, rng.raw(2) / kTwo32, d2);
            if (p.redraw_col_threshold) col_p = rng.raw(3) / kTwo32;
            philox_next<kRoll>(rng);
            unit_sphere_d(rng.raw(0) / kTwo32, rng.raw(1) / kTwo32, om);
        } else {
            float d2f[3], omf[3];
            unit_sphere_f(unit_open(rng.w[1]), unit_open(rng.w[2]), d2f);
            if (p.redraw_col_threshold) col_p = rng.raw(3) / kTwo32;
            philox_next<kRoll>(rng);
            unit_sphere_f(unit_open(rng.w[0]), unit_open(rng.w[1]), omf);
            for (int k = 0; k < 3; k++) { d2[k] = d2f[k]; om[k] = omf[k]; }
        }
        double g2 = 0.0, vcm[3];
        for (int k = 0; k < 3; k++) {
            const double v2k = vv2 * d2[k];
            g2 += (v[k] - v2k) * (v[k] - v2k);
            vcm[k] = 0.5 * (v[k] + v2k);
        }
        const double hg = 0.5 * sqrt(g2);
        for (int k = 0; k < 3; k++) v[k] = vcm[k] + hg * om[k];
    }
    a.s.evt[i] = rng.event;
    a.s.ncol[i] += 1;
    if (col_p >= 0.0) {
        if constexpr (is_f64<R>()) h.pthr = -log1p(-col_p);
        else h.pthr = -log1pf(-static_cast<float>(col_p));
    }
    set_vel(h, v);
    h.pcol = R(0);
    drift_start(a, i, I, h);
}

// Next work index of the device queue: one atomic per group of lanes asking together.
__device__ __forceinline__ unsigned long long grab_work(FastCounters *ctr) {
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    const unsigned rank = __popc(m & ((1u << lane) - 1u));
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(&ctr->next, static_cast<unsigned long long>(__popc(m)));
    base = __shfl_sync(m, base, leader);
    return base + rank;
}

template <typename A>
__device__ __forceinline__ int find_inst(const A &a, unsigned long long w) {
    int lo = 0, hi = static_cast<int>(a.ctr->ninst) - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (static_cast<unsigned long long>(a.inst[mid].work_base) <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Fill an empty slot with the next particle from the queue and launch it; particles that end
// at their first launch are finished here and the next one is taken. Returns false when the
// queue is empty.
template <bool kCfg, bool kRoll, typename R>
__device__ bool start_next(const FastArgsT<R> &a, long long i, HotT<R> &h, BoundsT<R> &b,
                           StatAcc &st) {
    for (;;) {
        const unsigned long long w = grab_work(a.ctr);
        if (w >= a.ctr->total) return false;
        const int ii = find_inst(a, w);
        const FastInst &I = a.inst[ii];
        const dsmc_params &p = I.p;
        if (ii != st.inst) {
            flush_stats_lane(a, st);
            st.inst = ii;
        }
        const unsigned pid = static_cast<unsigned>(I.pid_begin + static_cast<long long>(w - I.work_base));
        h.inst = ii;
        Philox rng;
        rng.init(p.seed, p.instance, pid);
        philox_next<kRoll>(rng);
        h.w0 = R(1);
        h.nday = 0;
        h.steps = 0;
        h.hop = 0;
        h.pcol = R(0);
        h.ci = -1;
        h.run_w = R(0);
        h.hist_key = -1;
        h.hist_cnt = 0;
        const double zero[3] = {0.0, 0.0, 0.0};
        set_vel(h, zero);
        R thi, fi, local_T = R(0);
        double col_p = 0.0;
        double s[3];
        if (!kCfg && p.model == DSMC_MODEL_REFERENCE) {
            const bool adv = p.runner == DSMC_RUNNER_ADVANCED;
            if (adv) col_p = rng.raw(0) / kTwo32;
            const int o = adv ? 1 : 0;
            const double th = rng.raw(o) / kTwo32 * kPi - kPi / 2.0;
            const double ph = rng.raw(o + 1) / kTwo32 * 2.0 * kPi;
            s[0] = p.Radii * cos(th) * sin(ph);
            s[1] = p.Radii * cos(th) * cos(ph);
            s[2] = p.Radii * sin(th);
            thi = static_cast<R>(th);
            fi = static_cast<R>(ph);
            int td, fd;
            ref_index(thi, fi, p.ftd, p.ffd, td, fd);
            local_T = static_cast<R>(I.t.T_map[td * p.ffd + fd]);
        } else {
            const int f = pick_face(I.t, rng.raw(0) / kTwo32);
            a.s.face[i] = f;
            double u1 = rng.raw(1) / kTwo32, u2 = rng.raw(2) / kTwo32;
            col_p = rng.raw(3) / kTwo32;
            if (u1 + u2 > 1.0) { u1 = 1.0 - u1; u2 = 1.0 - u2; }
            const double *fv = I.t.face_verts + 9 * f;
            double q[3];
            for (int k = 0; k < 3; k++) q[k] = fv[k] + u1 * (fv[3 + k] - fv[k]) + u2 * (fv[6 + k] - fv[k]);
            // |q|^-1 from the FP32 estimate and one Newton step in FP64 (relative error ~1e-14)
            const double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
            double iq = rsqrtf(static_cast<float>(q2));
            iq = iq * (1.5 - 0.5 * q2 * iq * iq);
            for (int k = 0; k < 3; k++) s[k] = q[k] * (p.Radii * iq);
            local_T = static_cast<R>(I.t.face_T[f]);
            thi = fi = R(0);   // the config model's launch does not use the angles
        }
        a.s.pid[i] = pid;
        a.s.evt[i] = rng.event;
        a.s.ncol[i] = 0;
        a.s.rest[i] = 0.0f;
        if (p.runner != DSMC_RUNNER_ADVANCED) {
            h.pthr = R(0);
        } else {
            if constexpr (is_f64<R>()) h.pthr = -log1p(-col_p);
            else h.pthr = -log1pf(-static_cast<float>(col_p));
        }
        set_pos(h, s);
        const long long slot = static_cast<long long>(pid) - I.t.out_base;
        if (I.t.ttime && slot >= 0 && slot < I.t.out_cap) {
            if (p.model != DSMC_MODEL_REFERENCE) angles_of(h, thi, fi);
            I.t.ttime[slot] = thi;
            if (p.runner == DSMC_RUNNER_ADVANCED || p.model != DSMC_MODEL_REFERENCE) {
                I.t.ttime[5 * I.t.out_cap + slot] = fi;
                I.t.ttime[6 * I.t.out_cap + slot] = local_T;
            }
        }
        const int fate = hop_top<kCfg, kRoll>(a, i, I, h, b, st, thi, fi, local_T, true);
        if (fate == 0) return true;
        finish(a, i, I, h, st, fate);
    }
}

// One Verlet step of the reference's variant. FP32: (hi, lo) position and velocity sums, and the
// acceleration carried as the velocity change a * dt (GM passed as GM dt, c1 = 1.5 dt,
// c2 = dt / 6; three multiplies fewer per step, and at a power-of-two dt the same roundings as
// a and dt kept apart); FP64: plain doubles with c1 = 1.5 dt^2, c2 = dt^2 / 6. (x, y, z, r2)
// hold the current position on entry and the new one on exit; d the displacement.
__device__ __forceinline__ void verlet_step(Hot &h, float &x, float &y, float &z, float &r2,
                                            float GM, float dt, float c1, float c2, float d[3]) {
    const float ir = rsqrtf(r2);
    const float g = GM * (ir * ir * ir);
    const float acc[3] = {g * x, g * y, g * z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        d[k] = fmaf(h.vh[k], dt, fmaf(h.vl[k], dt, -fmaf(acc[k], c1, h.oa[k] * c2)));
        accumulate(h.sh[k], h.sl[k], d[k]);
        accumulate(h.vh[k], h.vl[k], -acc[k]);
        h.oa[k] = acc[k];
    }
    x = h.sh[0] + h.sl[0];
    y = h.sh[1] + h.sl[1];
    z = h.sh[2] + h.sl[2];
    r2 = fmaf(x, x, fmaf(y, y, z * z));
}

__device__ __forceinline__ void verlet_step(HotT<double> &h, double &x, double &y, double &z,
                                            double &r2, double GM, double dt, double c1, double c2,
                                            double d[3]) {
    const double ir = rsqrt(r2);
    const double g = GM * (ir * ir * ir);
    const double acc[3] = {g * x, g * y, g * z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        d[k] = fma(h.vh[k], dt, -fma(acc[k], c1, h.oa[k] * c2));
        h.sh[k] += d[k];
        h.vh[k] -= acc[k] * dt;
        h.oa[k] = acc[k];
    }
    x = h.sh[0];
    y = h.sh[1];
    z = h.sh[2];
    r2 = fma(x, x, fma(y, y, z * z));
}

enum Flag { kRef = 1, kSkipFirst = 2, kCollide = 4, kHist = 8 };

// Event gathering (see fast_kernel): Verlet steps per chunk between the warp's votes.
constexpr int kChunk = 32;

// kMaxThreads x kMinBlocks: the register budget the allocation must respect (65536 registers
// per SM shared by kMinBlocks blocks of kMaxThreads). The launch shape picks the variant.
// kMode 0: the general loop. kMode 1 (lean): every instance of the launch is a config-model
// problem without speed histograms whose hop cap is not below its life cap and that has no
// collisions, so the reference-model, collision and histogram branches and the per-hop step
// counter drop out of the loop. kMode 2: the same, with the collision branch kept (config-model
// collisional instances). R: float (FAST_FP32) or double (FAST_FP64).
// The step loop runs in segments: an inner loop pushes the particle until an event (landing,
// escape, cap) or the end of the launch's step budget, so the per-step path carries no instance
// or restart checks, and the lean loops settle their step counters once per segment. This
// structure measured 21 % faster than one flat loop over steps with the same arithmetic (and
// bit-identical results).
template <int kMaxThreads, int kMinBlocks, int kMode, typename R>
__global__ void __launch_bounds__(kMaxThreads, kMinBlocks) fast_kernel(const FastArgsT<R> a) {
    constexpr bool kLean = kMode != 0;
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    HotT<R> h;
    load_hot(a.s, i, a.nslots, h);
    StatAcc st;
    st.inst = h.inst;
    BoundsT<R> b;
    bool alive = h.inst >= 0;
    if (alive) {
        // reload the cached bounds of the saved cell without flushing its pending deposits
        const int ci = h.ci;
        const R run_w = h.run_w;
        h.ci = -1;
        enter_cell(a.inst[h.inst], h, b, h.cell);
        h.ci = ci;
        h.run_w = run_w;
    } else {
        alive = start_next<kLean, kMode == 2>(a, i, h, b, st);
    }
    int cur = -1, flags = 0, half_ffd = 0, life_cap = 0, hop_cap = 0, col_ht = 0, nbins = 0;
    R GM = R(0), dt = R(0), c1 = R(0), c2 = R(0), rl2 = R(0), re2 = R(0), sx = R(0), sy = R(0),
      sz = R(0), fday = R(0);
    float inv_bw = 0.f;
    const FastInst *I = nullptr;
    int budget = a.K;

    while (alive && budget > 0) {
        if (h.inst != cur) {
            cur = h.inst;
            I = &a.inst[cur];
            const dsmc_params &p = I->p;
            dt = static_cast<R>(p.dt_step);
            if constexpr (is_f64<R>()) {
                GM = p.GM;
                c1 = 1.5 * p.dt_step * p.dt_step;
                c2 = p.dt_step * p.dt_step / 6.0;
                rl2 = p.Radii * p.Radii;
                re2 = p.max_height * p.max_height;
            } else {
                GM = static_cast<R>(p.GM * p.dt_step);
                c1 = static_cast<R>(1.5 * p.dt_step);
                c2 = static_cast<R>(p.dt_step / 6.0);
                rl2 = I->r_land2;
                re2 = I->r_esc2;
            }
            fday = static_cast<R>(p.wdecay);
            sx = static_cast<R>(p.sun[0]);
            sy = static_cast<R>(p.sun[1]);
            sz = static_cast<R>(p.sun[2]);
            half_ffd = p.ffd / 2;
            flags = (p.model == DSMC_MODEL_REFERENCE ? kRef : 0) |
                    (p.skip_first_deposit ? kSkipFirst : 0) |
                    (p.runner == DSMC_RUNNER_ADVANCED && I->t.n_bg ? kCollide : 0) |
                    (I->t.speed_hist && p.n_speed_bins > 0 ? kHist : 0);
            life_cap = p.life_step_cap > 0
                           ? static_cast<int>(min(static_cast<long long>(p.life_step_cap), 0x7fffffffLL))
                           : 0x7fffffff;
            hop_cap = static_cast<int>(min(static_cast<long long>(p.hop_step_cap), 0x7fffffffLL));
            col_ht = p.collide_ht_max;
            nbins = p.n_speed_bins;
            inv_bw = nbins > 0 ? static_cast<float>(1.0 / p.speed_bin_width) : 0.f;
        }
        // One segment: steps until an event or the end of the launch's budget. The lean loop
        // also stops at the life cap, so its step counters are settled once per segment.
        R x = pos(h, 0), y = pos(h, 1), z = pos(h, 2);
        R r2 = fma_r(x, x, fma_r(y, y, z * z));
        const int n = kLean ? min(budget, life_cap - h.steps) : budget;
        int taken = 0;
        int event = 0;   // 1 landed (or hop cap), 2 escaped, 3 life cap
        // Lanes whose particle lands leave the step loop and run their event code while the warp
        // serialises it against the lanes still stepping. Where hops are short (high-gravity
        // bodies, a landing every ~200 steps) that leaves most lanes idle, so there the warp
        // steps in chunks of kChunk and, between chunks, lets the stopped lanes wait until they
        // have idled `limit` lane-chunks in all: then every waiting lane takes its event
        // together. Long hops (Ceres-like) keep the free-running loop. The limit is the largest
        // of the instances of the lanes that enter the segment together, so it is uniform.
        const unsigned peers = __activemask();
        const int limit = static_cast<int>(__reduce_max_sync(peers, static_cast<unsigned>(I->gather)));
        const bool gather = limit > 0;
        const int npeer = __popc(peers);
        int idle = 0;
        for (;;) {
        const int lim = gather ? min(n, taken + kChunk) : n;
        while (!event && taken < lim) {
            R d[3];
            verlet_step(h, x, y, z, r2, GM, dt, c1, c2, d);
            taken++;
            const int ii = kLean ? 1 : h.hop;
            if (!kLean) {
                h.steps++;
                h.hop++;
            }
            const R zz = z * fabs(z);
            const bool in_r = (r2 > b.r2lo) & (r2 <= b.r2hi);
            const bool in_t = (zz > r2 * b.zlo) & (zz <= r2 * b.zhi);
            const bool in_f = (x * b.c0 - y * b.s0 > R(0)) & (x * b.c1 - y * b.s1 <= R(0));
            if (!(in_r & in_t & in_f)) {
                if (r2 <= rl2) {
                    event = 1;
                    break;
                }
                if (r2 >= re2) {
                    event = 2;
                    break;
                }
                move_cell<kMode == 1>(*I, h, b, x, y, r2, zz, in_r, in_t, in_f);
            }
            const bool day = (!kLean && (flags & kRef)) ? ((h.cell & 0xff) < half_ffd)
                                                        : (fma_r(x, sx, fma_r(y, sy, z * sz)) > R(0));
            if (day) {
                h.nday++;
                h.W *= fday;
            }
            if (kLean || !((flags & kSkipFirst) && ii == 0)) {
                bool collided = false;
                if ((kMode == 0 ? (flags & kCollide) != 0 : kMode == 2) && h.nsig > R(0)) {
                    h.pcol = fma_r(sqrt(fma_r(d[0], d[0], fma_r(d[1], d[1], d[2] * d[2]))), h.nsig, h.pcol);
                    if (h.pcol > h.pthr) {
                        const int ht = h.cell >> 16, td = (h.cell >> 8) & 0xff, fd = h.cell & 0xff;
                        const long long pidx = (static_cast<long long>(td) * I->p.ffd + fd) * I->p.hd + ht;
                        if (ht < col_ht && __ldg(I->t.cdf_valid + pidx)) {
                            collide<kMode == 2>(a, i, *I, h, pidx);
                            collided = true;
                        }
                    }
                }
                if (!collided) {
                    h.run_w += h.W;
                    if (!kLean && (flags & kHist)) {
                        const R sp = sqrt(fma_r(h.vh[0], h.vh[0], fma_r(h.vh[1], h.vh[1], h.vh[2] * h.vh[2])));
                        const int key = h.ci * nbins + min(static_cast<int>(static_cast<float>(sp) * inv_bw), nbins - 1);
                        if (key == h.hist_key) {
                            h.hist_cnt++;
                        } else {
                            flush_hist(*I, h);
                            h.hist_key = key;
                            h.hist_cnt = 1;
                        }
                    }
                }
            }
            if (!kLean) {
                if (h.steps >= life_cap) event = 3;
                else if (h.hop >= hop_cap) event = 1;
            }
        }
        if (!gather) break;
        const int k = __popc(__ballot_sync(peers, event != 0 || taken >= n));
        idle += k;
        if (k == npeer || idle >= limit) break;
        }
        budget -= taken;
        st.steps += taken;
        if (kLean) {
            h.steps += taken;
            if (!event && h.steps >= life_cap) event = 3;
        }
        if (event) {
            drift_check(a, i, *I, h, st);
            int fate = 0;
            if (event == 2) {
                fate = DSMC_FATE_ESCAPED;
            } else if (event == 3) {
                fate = DSMC_FATE_STEP_CAP;
            } else {
                R thi, fi, local_T = R(0);
                fate = land<kLean>(a, i, *I, h, thi, fi, local_T);
                if (fate == 0) fate = hop_top<kLean, kMode == 2>(a, i, *I, h, b, st, thi, fi, local_T, false);
            }
            if (fate) {
                finish(a, i, *I, h, st, fate);
                alive = start_next<kLean, kMode == 2>(a, i, h, b, st);
            }
        }
    }
    store_hot(a.s, i, a.nslots, h);
    // statistics of this launch, per instance; the finished count also drives the host loop
    const unsigned fin = st.finished;
    flush_stats(a, st);
    const unsigned wfin = __reduce_add_sync(0xffffffffu, fin);
    if ((threadIdx.x & 31) == 0 && wfin) atomicAdd(&a.ctr->finished, static_cast<unsigned long long>(wfin));
}

// Fed-state FP32 push (dsmc_push_host with FAST_FP32).
__global__ void push_fp32_kernel(const dsmc_params p, long long n, int nsteps, double *pos,
                                 double *vel, int *status, int *taken) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Hot h;
    const double s[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    const double v[3] = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    set_pos(h, s);
    set_vel(h, v);
    const double R0 = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    const double g0 = p.GM / (R0 * R0 * R0);
    for (int k = 0; k < 3; k++) h.oa[k] = static_cast<float>(g0 * s[k] * p.dt_step);
    const float GM = static_cast<float>(p.GM * p.dt_step), dt = static_cast<float>(p.dt_step);
    const float c1 = static_cast<float>(1.5 * p.dt_step);
    const float c2 = static_cast<float>(p.dt_step / 6.0);
    const float rl2 = static_cast<float>(p.Radii * p.Radii);
    const float re2 = static_cast<float>(p.max_height * p.max_height);
    float x = h.sh[0] + h.sl[0], y = h.sh[1] + h.sl[1], z = h.sh[2] + h.sl[2];
    float r2 = fmaf(x, x, fmaf(y, y, z * z));
    int st = 0, k = 0;
    for (; k < nsteps && st == 0; k++) {
        float d[3];
        verlet_step(h, x, y, z, r2, GM, dt, c1, c2, d);
        st = r2 <= rl2 ? 1 : (r2 >= re2 ? 2 : 0);
    }
    double so[3], vo[3];
    get_pos(h, so);
    get_vel(h, vo);
    for (int j = 0; j < 3; j++) { pos[3 * i + j] = so[j]; vel[3 * i + j] = vo[j]; }
    status[i] = st;
    taken[i] = k;
}

}  // namespace

cudaError_t launch_push_fp32(const dsmc_params &p, long long n, int nsteps, double *pos,
                             double *vel, int *status, int *taken, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    push_fp32_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, stream>>>(p, n, nsteps, pos, vel,
                                                                                status, taken);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// Host side.

FastEngine::~FastEngine() { free_all(); }

void FastEngine::free_all() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    for (cudaGraphExec_t &g : graph_mode_) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    if (slot_mem_) cudaFree(slot_mem_);
    slot_mem_ = nullptr;
    if (d_inst_) cudaFree(d_inst_);
    d_inst_ = nullptr;
    if (d_tab_) cudaFree(d_tab_);
    d_tab_ = nullptr;
    if (d_ctr_) cudaFree(d_ctr_);
    d_ctr_ = nullptr;
    if (h_ctr_) cudaFreeHost(h_ctr_);
    h_ctr_ = nullptr;
    if (d_stats_) cudaFree(d_stats_);
    d_stats_ = nullptr;
    stats_cap_ = 0;
    ninst_cap_ = 0;
    for (void *p : inst_tabs_)
        if (p) cudaFree(p);
    inst_tabs_.clear();
    nslots_ = 0;
}

namespace {

// Register budgets of fast_kernel: 0: 256 x 2 (128 registers a thread), 1: 256 x 3 (80),
// 2: 128 x 3 (168), 3: 128 x 2 (255), 4: 128 x 4 (128), 5: 128 x 5 (96).
// The lean loops (modes 1 and 2) exist for budgets 0, 2, 4 and 5; elsewhere the general loop
// runs. The FP64 engine exists for budgets 2 and 4 (its double state needs the larger budgets).
template <int kT, int kB, typename R>
void (*by_mode(int mode))(FastArgsT<R>) {
    return mode == 2 ? fast_kernel<kT, kB, 2, R> : mode == 1 ? fast_kernel<kT, kB, 1, R>
                                                             : fast_kernel<kT, kB, 0, R>;
}

void (*kernel_variant(int variant, int mode))(FastArgs) {
    switch (variant) {
        case 1: return fast_kernel<256, 3, 0, float>;
        case 2: return by_mode<128, 3, float>(mode);
        case 3: return fast_kernel<128, 2, 0, float>;
        case 4: return by_mode<128, 4, float>(mode);
        case 5: return by_mode<128, 5, float>(mode);
        default: return by_mode<256, 2, float>(mode);
    }
}

void (*kernel_variant64(int variant, int mode))(FastArgsT<double>) {
    return variant == 2 ? by_mode<128, 3, double>(mode) : by_mode<128, 4, double>(mode);
}

// FP64 variant for a launch shape: 128 x 4 (128 registers) unless 3 blocks per SM are asked.
// On the 1e7-particle Ceres-like workload 128 x 4 runs 1.59e11 particle-steps/s against 1.37e11
// at 128 x 3 (168 registers, no spills): more resident warps beat spill-free code, as in FP32.
int pick_variant64(int blocks_per_sm) { return blocks_per_sm == 3 ? 2 : 4; }

// Variant for a launch shape: blocks_per_sm names the register budget. The default (0) is the
// fastest measured on B200 for each loop, although ptxas reports spills for all three: the lean
// loop at 96 registers (20 warps per SM) beats 128 registers (16 warps) by 6 % and 80 (24 warps)
// by 3 %; the collision loop at 96 beats 128 by 1.5 % and 168 (no spills, 12 warps) by 15 %;
// the general loop at 128 beats 168 by 19 % and 96 by 18 %.
int pick_variant(int block, int blocks_per_sm, int mode) {
    if (block > 128) return blocks_per_sm >= 3 ? 1 : 0;
    if (blocks_per_sm == 2) return 3;
    if (blocks_per_sm == 3) return 2;
    if (blocks_per_sm == 4) return 4;
    if (blocks_per_sm == 5) return 5;
    return mode == 0 ? 4 : 5;
}

// Loop mode of one instance (see fast_kernel): 1 lean, 2 lean with collisions, 0 general.
int instance_mode(const dsmc_params &p, const DevTables &t) {
    if (p.model != DSMC_MODEL_CONFIG || p.skip_first_deposit || (t.speed_hist && p.n_speed_bins > 0) ||
        p.life_step_cap <= 0 || p.hop_step_cap < p.life_step_cap)
        return 0;
    return p.runner == DSMC_RUNNER_ADVANCED && t.n_bg ? 2 : 1;
}

// The loop that can run every instance of a launch: general if any needs it, else lean with
// collisions if any collides, else lean.
int launch_mode(const std::vector<dsmc_params> &ps, const std::vector<DevTables> &ts) {
    int m = 1;
    for (size_t k = 0; k < ps.size(); k++) {
        const int mk = instance_mode(ps[k], ts[k]);
        if (mk == 0) return 0;
        m = std::max(m, mk);
    }
    return m;
}

}  // namespace

namespace {

// FP32 copies of the icosphere's base-face centroids and corner-cut planes, as float4 (xyz, 0):
// [0, 20) centroids, then 3 planes per subdivision node, then per leaf face the normals of the 3
// planes through the origin and its edges, turned so that the face's cone is on their positive
// side (a point lies in face f iff its direction is on the positive side of all three). Built on
// the device from the problem's FP64 tables.
__global__ void face_tables_kernel(const double *cent, const double *planes, const double *verts,
                                   int nnode, int nface, float4 *out) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long np = 20 + 3ll * nnode;
    if (i < 20) {
        out[i] = make_float4(static_cast<float>(cent[3 * i]), static_cast<float>(cent[3 * i + 1]),
                             static_cast<float>(cent[3 * i + 2]), 0.0f);
    } else if (i < np) {
        const double *q = planes + 3 * (i - 20);   // node (i-20)/3, plane (i-20)%3
        out[i] = make_float4(static_cast<float>(q[0]), static_cast<float>(q[1]), static_cast<float>(q[2]), 0.0f);
    } else if (i < np + 3ll * nface) {
        const long long f = (i - np) / 3;
        const int e = static_cast<int>((i - np) % 3);
        const double *v = verts + 9 * f;
        const double *p = v + 3 * e, *q = v + 3 * ((e + 1) % 3);
        double c[3] = {p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]};
        const double m[3] = {v[0] + v[3] + v[6], v[1] + v[4] + v[7], v[2] + v[5] + v[8]};
        if (c[0] * m[0] + c[1] * m[1] + c[2] * m[2] < 0.0)
            for (int k = 0; k < 3; k++) c[k] = -c[k];
        out[i] = make_float4(static_cast<float>(c[0]), static_cast<float>(c[1]), static_cast<float>(c[2]), 0.0f);
    }
}

}  // namespace

size_t face_floats_for(int nlevel) {
    const size_t nnode = static_cast<size_t>(20 * ((1 << (2 * nlevel)) - 1) / 3);
    const size_t nface = static_cast<size_t>(20) << (2 * nlevel);
    return 4 * (20 + 3 * nnode + 3 * nface);
}

size_t face_table_floats(const dsmc_params &p, const DevTables &t) {
    if (p.model != DSMC_MODEL_CONFIG || !t.base_centroid || !t.split_planes || !t.face_verts ||
        t.nlevel < 0)
        return 0;
    return face_floats_for(t.nlevel);
}

cudaError_t build_face_tables(const DevTables &t, float4 *out, cudaStream_t stream) {
    const int nnode = 20 * ((1 << (2 * t.nlevel)) - 1) / 3;
    const int nface = 20 << (2 * t.nlevel);
    const int n = 20 + 3 * nnode + 3 * nface;
    face_tables_kernel<<<(n + 127) / 128, 128, 0, stream>>>(t.base_centroid, t.split_planes,
                                                            t.face_verts, nnode, nface, out);
    return cudaGetLastError();
}

cudaError_t FastEngine::ensure_slots(int num_sms) {
    // one wave: as many blocks per SM as can be resident together
    int resident = 0;
    cudaError_t e0;
    if (fp64_) {
        if (block != 128) return cudaErrorInvalidValue;   // the FP64 engine runs 128-thread blocks
        variant_ = pick_variant64(blocks_per_sm);
        e0 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel_variant64(variant_, mode_), block, 0);
    } else {
        variant_ = pick_variant(block, blocks_per_sm, mode_);
        e0 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel_variant(variant_, mode_), block, 0);
    }
    if (e0 != cudaSuccess) return e0;
    if (resident < 1) return cudaErrorInvalidConfiguration;
    const int per_sm = (blocks_per_sm > resident || blocks_per_sm < 1) ? resident : blocks_per_sm;
    nslots_want_changed_ = false;
    const long long want = static_cast<long long>(num_sms) * per_sm * block;
    if (slot_mem_ && nslots_ == want && slot_fp64_ == fp64_) return cudaSuccess;
    if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    for (cudaGraphExec_t &g : graph_mode_)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    if (slot_mem_) { cudaFree(slot_mem_); slot_mem_ = nullptr; }
    const long long S = want;
    cudaError_t e = cudaMalloc(&slot_mem_, fast_slot_bytes(S, fp64_));
    if (e != cudaSuccess) return e;
    slots_ = Slots{};
    slots64_ = SlotsT<double>{};
    if (fp64_) slots64_ = carve_slots<double>(slot_mem_, S);
    else slots_ = carve_slots<float>(slot_mem_, S);
    slot_fp64_ = fp64_;
    nslots_ = S;
    if (!d_ctr_) {
        if ((e = cudaMalloc(&d_ctr_, sizeof(FastCounters))) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&h_ctr_, sizeof(FastCounters))) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t FastEngine::upload_instances(const std::vector<dsmc_params> &ps,
                                         const std::vector<DevTables> &ts,
                                         const std::vector<long long> &counts,
                                         const std::vector<long long> &pid_begins,
                                         cudaStream_t stream) {
    const int n = static_cast<int>(ps.size());
    // boundary tables, one block per instance: rb2 [hd+1], sbs [ftd+1], lonb [2*(ffd+1)]
    // and, for config-model instances, the FP32 icosphere tables (face_table_floats)
    // and, for FP64 solves, the same boundary tables in double (rb2, sbs, lonb as double2)
    std::vector<size_t> off(n), foff(n, 0), doff(n, 0);
    size_t total = 0;
    for (int k = 0; k < n; k++) {
        off[k] = total;
        total += (ps[k].hd + 1) + (ps[k].ftd + 1);
        total = (total + 1) & ~static_cast<size_t>(1);  // float2 alignment
        total += 2 * (ps[k].ffd + 1);
        const size_t ff = face_table_floats(ps[k], ts[k]);
        if (ff) {
            total = (total + 3) & ~static_cast<size_t>(3);   // float4 alignment
            foff[k] = total;
            total += ff;
        }
        if (fp64_) {
            total = (total + 3) & ~static_cast<size_t>(3);   // double2 alignment (16 bytes)
            doff[k] = total;
            // (hd+1) + (ftd+1) doubles, rounded up to even for the double2 table, + 2 (ffd+1)
            const size_t nd = ((static_cast<size_t>(ps[k].hd + 1) + (ps[k].ftd + 1) + 1) & ~static_cast<size_t>(1)) +
                              2 * static_cast<size_t>(ps[k].ffd + 1);
            total += 2 * nd;
        }
    }
    std::vector<float> tab(total, 0.0f);
    std::vector<FastInst> inst(n);
    long long base = 0;
    for (int k = 0; k < n; k++) {
        const dsmc_params &p = ps[k];
        float *rb2 = tab.data() + off[k];
        float *sbs = rb2 + (p.hd + 1);
        size_t lo = off[k] + (p.hd + 1) + (p.ftd + 1);
        lo = (lo + 1) & ~static_cast<size_t>(1);
        float *lon = tab.data() + lo;
        for (int j = 0; j <= p.hd; j++) {
            const double rj = p.use_exp_grid
                                  ? p.Radii + p.unih * (std::pow(1.0 + p.alpha2, j) - 1.0) / p.alpha2
                                  : p.Radii + j * p.unih;
            rb2[j] = static_cast<float>(rj * rj);
        }
        for (int j = 0; j <= p.ftd; j++) {
            const double b = static_cast<double>(j) / p.ftd * kPi - kPi / 2.0;
            const double sb = std::sin(b);
            sbs[j] = static_cast<float>(sb * std::fabs(sb));
        }
        sbs[0] = -1.0f;
        sbs[p.ftd] = 1.0f;
        for (int j = 0; j <= p.ffd; j++) {
            const double ph = 2.0 * kPi * j / p.ffd;
            lon[2 * j] = static_cast<float>(std::sin(ph));
            lon[2 * j + 1] = static_cast<float>(std::cos(ph));
        }
        lon[0] = 0.0f; lon[1] = 1.0f;
        lon[2 * p.ffd] = 0.0f; lon[2 * p.ffd + 1] = 1.0f;
        size_t d_lo = 0;
        if (fp64_) {
            double *db = reinterpret_cast<double *>(tab.data() + doff[k]);
            double *drb2 = db, *dsbs = db + (p.hd + 1);
            d_lo = ((static_cast<size_t>(p.hd + 1) + (p.ftd + 1) + 1) & ~static_cast<size_t>(1));
            double *dlon = db + d_lo;
            for (int j = 0; j <= p.hd; j++) {
                const double rj = p.use_exp_grid
                                      ? p.Radii + p.unih * (std::pow(1.0 + p.alpha2, j) - 1.0) / p.alpha2
                                      : p.Radii + j * p.unih;
                drb2[j] = rj * rj;
            }
            for (int j = 0; j <= p.ftd; j++) {
                const double sb = std::sin(static_cast<double>(j) / p.ftd * kPi - kPi / 2.0);
                dsbs[j] = sb * std::fabs(sb);
            }
            dsbs[0] = -1.0;
            dsbs[p.ftd] = 1.0;
            for (int j = 0; j <= p.ffd; j++) {
                const double ph = 2.0 * kPi * j / p.ffd;
                dlon[2 * j] = std::sin(ph);
                dlon[2 * j + 1] = std::cos(ph);
            }
            dlon[0] = 0.0; dlon[1] = 1.0;
            dlon[2 * p.ffd] = 0.0; dlon[2 * p.ffd + 1] = 1.0;
        }
        FastInst &I = inst[k];
        std::memset(&I, 0, sizeof I);
        I.p = p;
        I.t = ts[k];
        I.work_base = base;
        I.n = counts[k];
        I.pid_begin = pid_begins[k];
        I.c_day = static_cast<float>(p.dt_step / p.lifetime / std::log(2.0));
        I.c_day_d = p.dt_step / p.lifetime / std::log(2.0);
        I.gather = gather_chunks(p);
        I.drift_abs = p.drift_tol > 0.0 ? p.drift_tol * p.GM / p.Radii : 0.0;
        I.r_land2 = static_cast<float>(p.Radii * p.Radii);
        I.r_esc2 = static_cast<float>(p.max_height * p.max_height);
        // device addresses filled below
        I.rb2 = reinterpret_cast<const float *>(off[k]);
        I.sbs = reinterpret_cast<const float *>(off[k] + (p.hd + 1));
        I.lonb = reinterpret_cast<const float2 *>(lo);
        I.face_f = foff[k] ? reinterpret_cast<const float4 *>(foff[k]) : nullptr;
        if (fp64_) {
            I.rb2d = reinterpret_cast<const double *>(doff[k]);
            I.sbsd = reinterpret_cast<const double *>(doff[k] + 2 * static_cast<size_t>(p.hd + 1));
            I.lonbd = reinterpret_cast<const double2 *>(doff[k] + 2 * d_lo);
        }
        base += counts[k];
    }
    cudaError_t e;
    if (total > tab_cap_) {
        if (d_tab_) cudaFree(d_tab_);
        d_tab_ = nullptr;
        if ((e = cudaMalloc(&d_tab_, total * sizeof(float))) != cudaSuccess) return e;
        tab_cap_ = total;
        if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    }
    if (n > ninst_cap_) {
        if (d_inst_) cudaFree(d_inst_);
        d_inst_ = nullptr;
        if ((e = cudaMalloc(&d_inst_, n * sizeof(FastInst))) != cudaSuccess) return e;
        ninst_cap_ = n;
        if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    }
    for (auto &I : inst) {
        I.rb2 = d_tab_ + reinterpret_cast<size_t>(I.rb2);
        I.sbs = d_tab_ + reinterpret_cast<size_t>(I.sbs);
        I.lonb = reinterpret_cast<const float2 *>(d_tab_ + reinterpret_cast<size_t>(I.lonb));
        if (I.face_f) I.face_f = reinterpret_cast<const float4 *>(d_tab_ + reinterpret_cast<size_t>(I.face_f));
        if (fp64_) {
            I.rb2d = reinterpret_cast<const double *>(d_tab_ + reinterpret_cast<size_t>(I.rb2d));
            I.sbsd = reinterpret_cast<const double *>(d_tab_ + reinterpret_cast<size_t>(I.sbsd));
            I.lonbd = reinterpret_cast<const double2 *>(d_tab_ + reinterpret_cast<size_t>(I.lonbd));
        }
    }
    if ((e = cudaMemcpyAsync(d_tab_, tab.data(), total * sizeof(float), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(d_inst_, inst.data(), n * sizeof(FastInst), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    for (int k = 0; k < n; k++)
        if (inst[k].face_f && (e = build_face_tables(ts[k], const_cast<float4 *>(inst[k].face_f), stream)) != cudaSuccess)
            return e;
    ninst_ = n;
    // the host staging vectors die here: wait for the copies
    return cudaStreamSynchronize(stream);
}

// Captures G launches of the current kernel variant into graph_ unless an identical graph exists.
cudaError_t FastEngine::prepare_graph(cudaStream_t stream) {
    const int key[4] = {static_cast<int>(nslots_), (variant_ * 4 + mode_) * 2 + (fp64_ ? 1 : 0),
                        static_cast<int>(reinterpret_cast<uintptr_t>(d_inst_) >> 8),
                        steps_per_launch * 64 + launches_per_graph};
    if (graph_ && graph_stream_ == stream && std::memcmp(key, graph_key_, sizeof key) == 0)
        return cudaSuccess;
    if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    const cudaError_t e = capture(stream, mode_, &graph_);
    if (e != cudaSuccess) return e;
    graph_stream_ = stream;
    std::memcpy(graph_key_, key, sizeof key);
    return cudaSuccess;
}

// G launches of the current variant (lean or general loop) captured as one graph.
// One launch of the current variant over every slot, in the precision the slots are carved for.
void FastEngine::launch_kernel(cudaStream_t stream, int mode, unsigned grid) {
    if (slot_fp64_) {
        FastArgsT<double> a{};
        a.inst = d_inst_;
        a.s = slots64_;
        a.nslots = nslots_;
        a.ctr = d_ctr_;
        a.K = steps_per_launch;
        kernel_variant64(variant_, mode)<<<grid, block, 0, stream>>>(a);
    } else {
        FastArgs a{};
        a.inst = d_inst_;
        a.s = slots_;
        a.nslots = nslots_;
        a.ctr = d_ctr_;
        a.K = steps_per_launch;
        kernel_variant(variant_, mode)<<<grid, block, 0, stream>>>(a);
    }
}

cudaError_t FastEngine::capture(cudaStream_t stream, int mode, cudaGraphExec_t *out) {
    const unsigned grid = static_cast<unsigned>(nslots_ / block);
    cudaError_t e;
    cudaGraph_t g;
    *out = nullptr;
    if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
    for (int k = 0; k < launches_per_graph; k++) launch_kernel(stream, mode, grid);
    if ((e = cudaStreamEndCapture(stream, &g)) != cudaSuccess) return e;
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) *out = nullptr;
    return e;
}

// One round: the captured graph (or one plain launch), then the counters copied back.
cudaError_t FastEngine::round(cudaStream_t stream) {
    cudaError_t e;
    if (launches_per_graph > 1) {
        if ((e = cudaGraphLaunch(graph_, stream)) != cudaSuccess) return e;
        launches += launches_per_graph;
    } else {
        launch_kernel(stream, mode_, static_cast<unsigned>(nslots_ / block));
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        launches += 1;
    }
    if ((e = cudaMemcpyAsync(h_ctr_, d_ctr_, sizeof(FastCounters), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(stream);
}

cudaError_t FastEngine::drain(long long total, cudaStream_t stream) {
    cudaError_t e;
    launches = 0;
    if (total <= 0) return cudaSuccess;
    h_ctr_->next = 0;
    h_ctr_->finished = 0;
    h_ctr_->total = static_cast<unsigned long long>(total);
    h_ctr_->ninst = ninst_;
    if ((e = cudaMemcpyAsync(d_ctr_, h_ctr_, sizeof(FastCounters), cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return e;
    int *inst = slot_fp64_ ? slots64_.inst : slots_.inst;
    if ((e = cudaMemsetAsync(inst, 0xff, nslots_ * sizeof(int), stream)) != cudaSuccess) return e;
    if (launches_per_graph > 1 && (e = prepare_graph(stream)) != cudaSuccess) return e;
    // Every launch advances each live particle by K steps or ends it, and every life is bounded
    // by its step caps, so the queue drains. The loop still gives up (launch-timeout status) if
    // no particle finishes for 4096 rounds, which would mean a logic error, not a long solve.
    unsigned long long last = 0;
    long long stalled = 0;
    for (;;) {
        if (stalled > 4096) return cudaErrorLaunchTimeout;
        if ((e = round(stream)) != cudaSuccess) return e;
        if (h_ctr_->finished >= static_cast<unsigned long long>(total)) return cudaSuccess;
        stalled = h_ctr_->finished == last ? stalled + 1 : 0;
        last = h_ctr_->finished;
    }
}

cudaError_t FastEngine::run(const dsmc_params &p, const DevTables &t, bool fp64, long long pid_begin,
                            long long n, int num_sms, cudaStream_t stream) {
    if (p.ftd > 255 || p.ffd > 255 || p.hd > 32767) return cudaErrorInvalidValue;
    fp64_ = fp64;
    mode_ = launch_mode({p}, {t});
    cudaError_t e = ensure_slots(num_sms);
    if (e != cudaSuccess) return e;
    e = upload_instances({p}, {t}, {n}, {pid_begin}, stream);
    if (e != cudaSuccess) return e;
    return drain(n, stream);
}

cudaError_t FastEngine::serve_open(int num_sms, int max_instances, cudaStream_t stream) {
    if (max_instances < 1) return cudaErrorInvalidValue;
    fp64_ = false;   // serving runs the FP32 engine
    mode_ = 0;   // the slots are sized for the general loop; every round picks its own loop
    cudaError_t e = ensure_slots(num_sms);
    if (e != cudaSuccess) return e;
    for (void *p : inst_tabs_)
        if (p) cudaFreeAsync(p, stream);
    inst_tabs_.assign(static_cast<size_t>(max_instances), nullptr);
    if (max_instances > ninst_cap_) {
        if (d_inst_) cudaFree(d_inst_);
        d_inst_ = nullptr;
        if ((e = cudaMalloc(&d_inst_, static_cast<size_t>(max_instances) * sizeof(FastInst))) != cudaSuccess) return e;
        ninst_cap_ = max_instances;
        if (graph_) { cudaGraphExecDestroy(graph_); graph_ = nullptr; }
    }
    if (!d_stats_ || stats_cap_ < max_instances) {
        if (d_stats_) cudaFree(d_stats_);
        d_stats_ = nullptr;
        if ((e = cudaMalloc(&d_stats_, static_cast<size_t>(max_instances) * kStatCount * sizeof(unsigned long long))) != cudaSuccess)
            return e;
        stats_cap_ = max_instances;
    }
    if ((e = cudaMemsetAsync(d_stats_, 0, static_cast<size_t>(max_instances) * kStatCount * sizeof(unsigned long long), stream)) != cudaSuccess)
        return e;
    ninst_ = 0;
    serve_total_ = 0;
    launches = 0;
    if ((e = cudaMemsetAsync(d_ctr_, 0, sizeof(FastCounters), stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(slots_.inst, 0xff, nslots_ * sizeof(int), stream)) != cudaSuccess) return e;
    if (launches_per_graph > 1 && (e = prepare_graph(stream)) != cudaSuccess) return e;
    // the lean loops over the same slots, for rounds in which every queued instance qualifies
    for (int m = 1; m <= 2; m++) {
        if (graph_mode_[m]) { cudaGraphExecDestroy(graph_mode_[m]); graph_mode_[m] = nullptr; }
        if (launches_per_graph > 1 && (e = capture(stream, m, &graph_mode_[m])) != cudaSuccess) return e;
    }
    return cudaStreamSynchronize(stream);
}

int FastEngine::loop_mode(const dsmc_params &p, const DevTables &t) { return instance_mode(p, t); }

namespace {

// Grows the served queue to `total` work items over `ninst` instances. Grabs made while the
// queue was empty pushed `next` past the old end without taking work (start_next returns on
// w >= total), so those indices are handed back first.
__global__ void publish_queue_kernel(FastCounters *c, unsigned long long old_total,
                                     unsigned long long total, long long ninst) {
    if (c->next > old_total) c->next = old_total;
    c->total = total;
    c->ninst = ninst;
}

}  // namespace

cudaError_t FastEngine::serve_append(const dsmc_params &p, const DevTables &t, long long n,
                                     int *index, cudaStream_t upload, cudaStream_t compute) {
    if (ninst_ >= ninst_cap_ || !d_stats_) return cudaErrorMemoryAllocation;
    if (p.ftd > 255 || p.ffd > 255 || p.hd > 32767 || n < 0 || n > (1ll << 32)) return cudaErrorInvalidValue;
    const size_t need = serve_table_floats(p, face_table_floats(p, t) ? t.nlevel : -1);
    const size_t base_need = static_cast<size_t>(p.hd + 1) + (p.ftd + 1) + 1 + 2 * static_cast<size_t>(p.ffd + 1);
    void *d_tab = nullptr;
    cudaError_t e = pool_ ? cudaMallocFromPoolAsync(&d_tab, need * sizeof(float), pool_, upload)
                          : cudaMallocAsync(&d_tab, need * sizeof(float), upload);
    if (e != cudaSuccess) return e;
    std::vector<float> tab(need, 0.0f);
    FastInst host;
    DevTables tt = t;
    tt.stats = d_stats_ + static_cast<size_t>(ninst_) * kStatCount;
    if ((e = fast_fill_instance(p, tt, 0, n, static_cast<float *>(d_tab), need, &host, tab.data())) != cudaSuccess) {
        cudaFreeAsync(d_tab, upload);
        return e;
    }
    host.work_base = static_cast<long long>(serve_total_);
    float4 *face = nullptr;
    if (face_table_floats(p, t)) {
        face = reinterpret_cast<float4 *>(static_cast<float *>(d_tab) + ((base_need + 3) & ~static_cast<size_t>(3)));
        host.face_f = face;
    }
    // The new descriptor lies beyond the instances the kernels in flight can see; it is written
    // on the upload stream while they run, and published on the compute stream after them.
    if ((e = cudaMemcpyAsync(d_tab, tab.data(), need * sizeof(float), cudaMemcpyHostToDevice, upload)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_inst_ + ninst_, &host, sizeof host, cudaMemcpyHostToDevice, upload)) != cudaSuccess ||
        (face && (e = build_face_tables(t, face, upload)) != cudaSuccess) ||
        (e = cudaStreamSynchronize(upload)) != cudaSuccess) {
        cudaFreeAsync(d_tab, upload);
        return e;
    }
    inst_tabs_[static_cast<size_t>(ninst_)] = d_tab;
    const unsigned long long old_total = serve_total_;
    serve_total_ += static_cast<unsigned long long>(n);
    publish_queue_kernel<<<1, 1, 0, compute>>>(d_ctr_, old_total, serve_total_, ninst_ + 1);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        serve_total_ = old_total;
        return e;
    }
    *index = ninst_++;
    return cudaSuccess;
}

cudaError_t FastEngine::serve_launch(cudaStream_t stream, int mode) {
    if (launches_per_graph > 1) {
        const cudaError_t e = cudaGraphLaunch(mode ? graph_mode_[mode] : graph_, stream);
        if (e == cudaSuccess) launches += launches_per_graph;
        return e;
    }
    launch_kernel(stream, mode, static_cast<unsigned>(nslots_ / block));
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) launches += 1;
    return e;
}

void FastEngine::serve_release(int index, cudaStream_t stream) {
    if (index < 0 || index >= static_cast<int>(inst_tabs_.size())) return;
    if (inst_tabs_[static_cast<size_t>(index)]) cudaFreeAsync(inst_tabs_[static_cast<size_t>(index)], stream);
    inst_tabs_[static_cast<size_t>(index)] = nullptr;
}

void FastEngine::serve_close(cudaStream_t stream) {
    for (void *p : inst_tabs_)
        if (p) cudaFreeAsync(p, stream);
    inst_tabs_.clear();
}

size_t FastEngine::serve_table_floats(const dsmc_params &p, int nlevel) {
    // boundary tables, then (config model, icosphere of nlevel levels) the FP32 face tables
    const size_t base = static_cast<size_t>(p.hd + 1) + (p.ftd + 1) + 1 + 2 * static_cast<size_t>(p.ffd + 1);
    if (p.model != DSMC_MODEL_CONFIG || nlevel < 0) return base;
    return ((base + 3) & ~static_cast<size_t>(3)) + face_floats_for(nlevel);
}

size_t FastEngine::serve_fixed_bytes(int max_instances) const {
    return fast_slot_bytes(nslots_) + static_cast<size_t>(max_instances) * (sizeof(FastInst) + kStatCount * 8) +
           sizeof(FastCounters);
}

size_t fast_slot_bytes(long long nslots, bool fp64) {
    return static_cast<size_t>(nslots) * (fp64 ? slot_bytes_per_slot<double>() : slot_bytes_per_slot<float>()) + 256;
}

template <typename R>
SlotsT<R> carve_slots(void *mem, long long S) {
    char *b = static_cast<char *>(mem);
    auto take = [&](size_t each) { char *q = b; b += static_cast<size_t>(S) * each; return q; };
    constexpr size_t r = sizeof(R);
    SlotsT<R> s{};
    s.run_w = reinterpret_cast<R *>(take(8));
    s.inst = reinterpret_cast<int *>(take(4));
    s.pid = reinterpret_cast<unsigned *>(take(4));
    s.evt = reinterpret_cast<unsigned *>(take(4));
    s.sh = reinterpret_cast<R *>(take(3 * r));
    s.sl = reinterpret_cast<R *>(take(3 * r));
    s.vh = reinterpret_cast<R *>(take(3 * r));
    s.vl = reinterpret_cast<R *>(take(3 * r));
    s.oa = reinterpret_cast<R *>(take(3 * r));
    s.w0 = reinterpret_cast<R *>(take(r));
    s.nday = reinterpret_cast<int *>(take(4));
    s.steps = reinterpret_cast<int *>(take(4));
    s.hop = reinterpret_cast<int *>(take(4));
    s.cell = reinterpret_cast<int *>(take(4));
    s.run_cell = reinterpret_cast<int *>(take(4));
    s.hist_key = reinterpret_cast<int *>(take(4));
    s.hist_cnt = reinterpret_cast<int *>(take(4));
    s.pcol = reinterpret_cast<R *>(take(r));
    s.pthr = reinterpret_cast<R *>(take(r));
    s.ncol = reinterpret_cast<int *>(take(4));
    s.rest = reinterpret_cast<float *>(take(4));
    s.wcur = reinterpret_cast<R *>(take(r));
    s.face = reinterpret_cast<int *>(take(4));
    s.e0 = reinterpret_cast<float *>(take(4));
    return s;
}

template SlotsT<float> carve_slots<float>(void *, long long);
template SlotsT<double> carve_slots<double>(void *, long long);

size_t fast_inst_bytes() { return sizeof(FastInst); }

double fast_hop_steps(const dsmc_params &p) {
    const double g = p.GM / (p.Radii * p.Radii);
    const double v = std::sqrt(p.kB_over_m * 235.0);
    return g > 0.0 && p.dt_step > 0.0 ? 2.0 * v / (g * p.dt_step) : 1e30;
}

// Measured on B200 (particle-steps/s, gathering against the free-running loop): Moon-like
// (~200 steps per hop) 1.24e11 vs 8.2e10 at 16 lane-chunks, 1.17e11 at 4; Europa-like (~250)
// 1.31e11 vs 9.3e10; the reference model (dt 5 s, ~480) 6.8e10 at 4 vs 6.2e10 at 16; Ceres-like
// (~1160) and its collisional phase 2 are fastest free-running (gathering at 16 cost 5 %).
int gather_chunks(const dsmc_params &p) {
    const double hop = fast_hop_steps(p);
    return hop < 300.0 ? 16 : (hop < 600.0 ? 4 : 0);
}

size_t fast_counter_bytes() { return sizeof(FastCounters); }

cudaError_t fast_fill_instance(const dsmc_params &p, const DevTables &t, long long pid_begin,
                               long long n, float *d_tab, size_t tab_floats, void *inst_host,
                               float *tab_host) {
    const size_t need = static_cast<size_t>(p.hd + 1) + (p.ftd + 1) + 1 + 2 * (p.ffd + 1);
    if (need > tab_floats) return cudaErrorInvalidValue;
    float *rb2 = tab_host, *sbs = rb2 + (p.hd + 1);
    size_t lo = static_cast<size_t>(p.hd + 1) + (p.ftd + 1);
    lo = (lo + 1) & ~static_cast<size_t>(1);
    float *lon = tab_host + lo;
    for (int j = 0; j <= p.hd; j++) {
        const double rj = p.use_exp_grid ? p.Radii + p.unih * (std::pow(1.0 + p.alpha2, j) - 1.0) / p.alpha2
                                         : p.Radii + j * p.unih;
        rb2[j] = static_cast<float>(rj * rj);
    }
    for (int j = 0; j <= p.ftd; j++) {
        const double sb = std::sin(static_cast<double>(j) / p.ftd * kPi - kPi / 2.0);
        sbs[j] = static_cast<float>(sb * std::fabs(sb));
    }
    sbs[0] = -1.0f;
    sbs[p.ftd] = 1.0f;
    for (int j = 0; j <= p.ffd; j++) {
        const double ph = 2.0 * kPi * j / p.ffd;
        lon[2 * j] = static_cast<float>(std::sin(ph));
        lon[2 * j + 1] = static_cast<float>(std::cos(ph));
    }
    lon[0] = 0.0f; lon[1] = 1.0f;
    lon[2 * p.ffd] = 0.0f; lon[2 * p.ffd + 1] = 1.0f;
    FastInst &I = *static_cast<FastInst *>(inst_host);
    std::memset(&I, 0, sizeof I);
    I.p = p;
    I.t = t;
    I.rb2 = d_tab;
    I.sbs = d_tab + (p.hd + 1);
    I.lonb = reinterpret_cast<const float2 *>(d_tab + lo);
    I.work_base = 0;
    I.n = n;
    I.pid_begin = pid_begin;
    I.c_day = static_cast<float>(p.dt_step / p.lifetime / std::log(2.0));
    I.c_day_d = p.dt_step / p.lifetime / std::log(2.0);
    I.gather = gather_chunks(p);
    I.drift_abs = p.drift_tol > 0.0 ? p.drift_tol * p.GM / p.Radii : 0.0;
    I.r_land2 = static_cast<float>(p.Radii * p.Radii);
    I.r_esc2 = static_cast<float>(p.max_height * p.max_height);
    return cudaSuccess;
}

cudaError_t fast_drain_external(const void *d_inst, void *slot_mem, long long nslots, void *d_ctr,
                                long long total, int steps_per_launch, int block,
                                long long stall_launches, cudaStream_t stream,
                                long long *launches) {
    *launches = 0;
    if (total <= 0) return cudaSuccess;
    if (nslots % block) return cudaErrorInvalidValue;
    const long long S = nslots;
    const Slots s = carve_slots<float>(slot_mem, S);
    cudaError_t e;
    FastCounters host{};
    host.total = static_cast<unsigned long long>(total);
    host.ninst = 1;
    if ((e = cudaMemcpyAsync(d_ctr, &host, sizeof host, cudaMemcpyHostToDevice, stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(s.inst, 0xff, S * sizeof(int), stream)) != cudaSuccess) return e;
    // the pageable source must stay valid until the copy has been made
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    FastArgs a{};
    a.inst = static_cast<const FastInst *>(d_inst);
    a.s = s;
    a.nslots = S;
    a.ctr = static_cast<FastCounters *>(d_ctr);
    a.K = steps_per_launch;
    const unsigned grid = static_cast<unsigned>(S / block);
    unsigned long long last = 0;
    long long stalled = 0;
    for (;;) {
        if (stalled > stall_launches) return cudaErrorLaunchTimeout;
        fast_kernel<256, 2, 0, float><<<grid, block, 0, stream>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        *launches += 1;
        if ((e = cudaMemcpyAsync(&host, d_ctr, sizeof host, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
        if (host.finished >= static_cast<unsigned long long>(total)) return cudaSuccess;
        stalled = host.finished == last ? stalled + 1 : 0;
        last = host.finished;
    }
}

}  // namespace dsmc
