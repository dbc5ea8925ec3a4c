// kernel_plain.cu - the plain FP64 path: one thread per test particle for its whole life.
//
// This translation unit is compiled with -fmad=false so that every double operation rounds on
// its own, as the reference's x86-64 build does (SSE2, no FMA contraction). With fed initial
// states the push is then bit-identical to the reference's verlet_step
// (src/common/integrator.c:4-55). Transcendentals (sin, cos, asin, atan2, log, exp) come from
// CUDA's libm and may differ from glibc in the last place; everything else follows the reference
// runners' operation order (src/dsmc/ballistic.c:97-281, src/dsmc/advanced.c:236-451).
//
// Deposits are unsigned 64-bit fixed point (W * 2^24, rounded to nearest), one atomicAdd per
// deposited step, so the grids are independent of thread order and bit-reproducible.
#include "dsmc_device.cuh"
#include "dsmc_kernels.h"

namespace dsmc {
namespace {

__device__ __forceinline__ double len3(const double a[3]) {
    return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}

__device__ __forceinline__ void to_angles(const double s[3], double Ri, double &thi, double &fi) {
    thi = asin(s[2] / Ri);
    fi = atan2(s[0], s[1]);
    if (fi < 0) fi += 2.0 * kPi;
}

__device__ __forceinline__ void to_index(double thi, double fi, int ftd, int ffd, int &td,
                                         int &fd) {
    td = static_cast<int>(ceil((thi + kPi / 2.0) / kPi * ftd)) - 1;
    fd = static_cast<int>(ceil(fi / (2.0 * kPi) * ffd)) - 1;
    td = td < 0 ? 0 : (td >= ftd ? ftd - 1 : td);
    fd = fd < 0 ? 0 : (fd >= ffd ? ffd - 1 : fd);
}

__device__ __forceinline__ double cdf_eval(const double *coef, const double *box, int degree,
                                           double x) {
    double t = (x - box[2]) / box[3];
    double r = 0.0;
    for (int i = 0; i <= degree; i++) r = r * t + coef[i];
    return r;
}

// collision_sample_speed, src/common/collision.c:43-101: bisection of the fitted
// reverse-cumulative speed distribution.
__device__ double cdf_sample(const double *coef, const double *box, double total, int degree,
                             double u) {
    double vmax = box[1];
    double at_max = cdf_eval(coef, box, degree, vmax);
    double ranking = u * (total - at_max) + at_max;
    double v0 = box[0], v1 = vmax;
    for (int iter = 0; iter < 100; iter++) {
        double vm = (v0 + v1) * 0.5;
        double fm = cdf_eval(coef, box, degree, vm) - ranking;
        double f1 = cdf_eval(coef, box, degree, v1) - ranking;
        if (fm * f1 < 0) v0 = vm;
        else v1 = vm;
        if (fabs(v1 - v0) < 0.01) break;
    }
    return (v0 + v1) * 0.5;
}

__device__ __forceinline__ void unit_sphere(double zu, double pu, double o[3]) {
    double z = 2.0 * zu - 1.0;
    double r = sqrt(fmax(0.0, 1.0 - z * z));
    double ph = 2.0 * kPi * pu;
    o[0] = r * cos(ph);
    o[1] = r * sin(ph);
    o[2] = z;
}

struct Acc {
    unsigned long long steps = 0, escaped = 0, collisions = 0, bound = 0, finished = 0, drift = 0;
};

// Orbital energy per unit mass |v|^2 / 2 - GM / |s| of the per-hop energy-drift guard.
__device__ __forceinline__ double orbital_energy(const dsmc_params &p, const double s[3],
                                                 const double v[3]) {
    return 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - p.GM / len3(s);
}

// Velocity-record replay modes (see launch_plain_record): kCount counts the deposited visits of
// each particle per (td, ht) bucket into the particle's own row; kRecord turns those rows into
// write cursors and stores the visits that fall below the per-bucket cap. Both modes leave the
// density and horizon grids untouched.
enum Mode { kSolve = 0, kCount = 1, kRecord = 2 };

template <int kMode>
__device__ void particle_life(const dsmc_params &p, const DevTables &t, long long pid,
                              Acc &acc, const RecordArgs &ra) {
    const int ftd = p.ftd, ffd = p.ffd, hd = p.hd;
    const bool ref = p.model == DSMC_MODEL_REFERENCE;
    const bool adv = p.runner == DSMC_RUNNER_ADVANCED;
    const double h = p.dt_step;

    Philox rng;
    rng.init(p.seed, p.instance, static_cast<uint32_t>(pid));

    int fate = DSMC_FATE_ALIVE, num_col = 0, td, fd;
    long long steps = 0;
    double real_col_p = 0.0, col_p = 0.0, time = 0.0, W = 1.0, flight_time = 0.0,
           rest_time = 0.0, thi, fi, local_T, s[3], v[3] = {0.0, 0.0, 0.0};
    // energy-drift guard: E at the hop's launch (or last collision) against E where it ends
    const double drift_abs = p.drift_tol * p.GM / p.Radii;
    double E_start = 0.0;

    rng.next();
    if (ref) {
        if (adv) col_p = rng.raw(0) / kTwo32;
        const int o = adv ? 1 : 0;
        thi = rng.raw(o) / kTwo32 * kPi - kPi / 2.0;
        fi = rng.raw(o + 1) / kTwo32 * 2.0 * kPi;
        s[0] = p.Radii * cos(thi) * sin(fi);
        s[1] = p.Radii * cos(thi) * cos(fi);
        s[2] = p.Radii * sin(thi);
        to_index(thi, fi, ftd, ffd, td, fd);
        local_T = t.T_map[td * ffd + fd];
    } else {
        const int f = pick_face(t, rng.raw(0) / kTwo32);
        double u1 = rng.raw(1) / kTwo32, u2 = rng.raw(2) / kTwo32;
        col_p = rng.raw(3) / kTwo32;
        if (u1 + u2 > 1.0) { u1 = 1.0 - u1; u2 = 1.0 - u2; }
        const double *a = t.face_verts + 9 * f;
        double q[3];
        for (int k = 0; k < 3; k++)
            q[k] = a[k] + u1 * (a[3 + k] - a[k]) + u2 * (a[6 + k] - a[k]);
        const double lq = len3(q);
        for (int k = 0; k < 3; k++) s[k] = q[k] * (p.Radii / lq);
        to_angles(s, len3(s), thi, fi);
        to_index(thi, fi, ftd, ffd, td, fd);
        local_T = t.face_T[f];
    }
    const long long slot = pid - t.out_base;
    const bool record = kMode == kSolve && t.ttime && slot >= 0 && slot < t.out_cap;
    if (record) {
        t.ttime[0 * t.out_cap + slot] = thi;
        if (adv || !ref) {
            t.ttime[5 * t.out_cap + slot] = fi;
            t.ttime[6 * t.out_cap + slot] = local_T;
        }
    }

    for (;;) {
        if (W < p.w_min) { fate = DSMC_FATE_PHOTOLYSED; break; }
        if (p.life_step_cap > 0 && steps >= p.life_step_cap) { fate = DSMC_FATE_STEP_CAP; break; }

        if (ref) {
            // Launch, ballistic.c:125-173 and advanced.c:272-326.
            const double KF = 2.0 * kPi * p.Radii * fabs(cos(thi)) / p.P;
            to_index(thi, fi, ftd, ffd, td, fd);
            local_T = t.T_map[td * ffd + fd];
            if (local_T < p.freeze_T) {
                bool found = false;
                if (!adv) {
                    for (int add = 0; add < ffd; add++) {
                        time += p.dt_rot;
                        const int check = (fd + add + 1) % ffd;
                        if (t.T_map[td * ffd + check] >= p.freeze_T) {
                            fd = check;
                            fi = (fd + 0.5) / ffd * 2.0 * kPi;
                            found = true;
                            break;
                        }
                    }
                } else {
                    if (kMode == kSolve) atomicAdd(&t.horizon[td * ffd + fd], to_fixed(W));
                    for (int add = 1; add <= ffd; add++) {
                        time += p.dt_rot;
                        rest_time += p.dt_rot;
                        if (t.T_map[td * ffd + (add % ffd)] >= p.freeze_T) {
                            const double rot_fi = static_cast<double>(add - fd) / ffd * 2.0 * kPi;
                            const double cs = cos(rot_fi), sn = sin(rot_fi);
                            const double n0 = s[0] * cs - s[1] * sn, n1 = s[0] * sn + s[1] * cs;
                            s[0] = n0;
                            s[1] = n1;
                            fd = add % ffd;
                            fi = (fd + 0.5) / ffd * 2.0 * kPi;
                            found = true;
                            break;
                        }
                    }
                }
                if (!found) {
                    if (kMode == kSolve) atomicAdd(&t.horizon[td * ffd + fd], to_fixed(W));
                    fate = DSMC_FATE_FROZEN;
                    break;
                }
                local_T = t.T_map[td * ffd + fd];
            }
            rng.next();
            // velocity_sample (velocity.c:49-68) and velocity_sticking (velocity.c:70-73)
            int idx = local_T >= 220.0 ? 20 : static_cast<int>(ceil(local_T / 10.0)) - 2;
            idx = idx < 0 ? 0 : (idx >= 23 ? 22 : idx);
            const double vr = t.vt_speeds[idx * 1000 + rng.w[0] % static_cast<uint32_t>(t.vt_count[idx])];
            const double v_old_sq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            const double vout = sqrt(p.alpha * vr * vr + (1.0 - p.alpha) * v_old_sq);
            const double flyd = rng.raw(1) / kTwo32 * kPi + thi - kPi / 2.0;
            const double xi = rng.raw(2) / kTwo32 * kPi + fi - kPi / 2.0;
            v[0] = cos(flyd) * sin(xi) * vout;
            v[1] = cos(flyd) * cos(xi) * vout;
            v[2] = sin(flyd) * vout;
            v[0] += KF * sin(fi + kPi / 2.0);
            v[1] += KF * cos(fi + kPi / 2.0);
            if (len3(v) >= p.ve) { fate = DSMC_FATE_ESCAPED; break; }
        } else {
            // Flux-weighted Maxwell-Boltzmann: Rayleigh normal, Gaussian tangential components.
            rng.next();
            const double sigma = sqrt(p.kB_over_m * local_T);
            const double vn = sigma * sqrt(-2.0 * log(1.0 - rng.raw(0) / kTwo32));
            const double rho = sqrt(-2.0 * log(1.0 - rng.raw(1) / kTwo32));
            const double ang = 2.0 * kPi * (rng.raw(2) / kTwo32);
            const double t1 = rho * cos(ang), t2 = rho * sin(ang);
            const double R = len3(s);
            const double n[3] = {s[0] / R, s[1] / R, s[2] / R};
            double e[3] = {-n[1], n[0], 0.0};
            const double le = sqrt(e[0] * e[0] + e[1] * e[1]);
            if (le < 1e-12) { e[0] = 1.0; e[1] = 0.0; }
            else { e[0] /= le; e[1] /= le; }
            const double nt[3] = {n[1] * e[2] - n[2] * e[1], n[2] * e[0] - n[0] * e[2],
                                  n[0] * e[1] - n[1] * e[0]};
            const double omega = p.P > 0.0 ? 2.0 * kPi / p.P : 0.0;
            const double rot[3] = {omega * s[1], -omega * s[0], 0.0};
            for (int k = 0; k < 3; k++)
                v[k] = vn * n[k] + (sigma * t1) * e[k] + (sigma * t2) * nt[k] + rot[k];
            const double E = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - p.GM / len3(s);
            if (E < 0.0) acc.bound++;
        }

        double Ri = len3(s);
        double oa[3];
        for (int k = 0; k < 3; k++) oa[k] = p.GM * s[k] / (Ri * Ri * Ri);
        E_start = orbital_energy(p, s, v);

        for (long long ii = 0; ii < p.hop_step_cap; ii++) {
            flight_time += h;
            time += h;
            steps++;
            // verlet_step, integrator.c:12-54
            const double R0 = len3(s);
            const double R03 = R0 * R0 * R0;
            const double h2 = h * h;
            const double g = p.GM / R03;
            double ns[3];
            for (int k = 0; k < 3; k++)
                ns[k] = s[k] + v[k] * h - g * s[k] * (1.5 * h2) - oa[k] * (h2 / 6.0);
            const double dx = ns[0] - s[0], dy = ns[1] - s[1], dz = ns[2] - s[2];
            const double ds = sqrt(dx * dx + dy * dy + dz * dz);
            for (int k = 0; k < 3; k++) v[k] -= g * s[k] * h;
            for (int k = 0; k < 3; k++) oa[k] = g * s[k];
            s[0] = ns[0]; s[1] = ns[1]; s[2] = ns[2];
            Ri = len3(s);
            if (Ri <= p.Radii) break;
            if (Ri >= p.max_height) { fate = DSMC_FATE_ESCAPED; break; }

            to_angles(s, Ri, thi, fi);
            to_index(thi, fi, ftd, ffd, td, fd);
            const bool day = ref ? (fd < ffd / 2)
                                 : (s[0] * p.sun[0] + s[1] * p.sun[1] + s[2] * p.sun[2] > 0.0);
            if (day) W *= p.wdecay;

            bool deposit = !(p.skip_first_deposit && ii == 0);
            int ht = 0;
            if (deposit) {
                if (p.use_exp_grid) {
                    const double arg = p.alpha2 * (Ri - p.Radii) / p.unih + 1.0;
                    ht = arg <= 1.0 ? 0 : static_cast<int>(ceil(log(arg) / p.log1p_alpha2)) - 1;
                } else {
                    ht = static_cast<int>(ceil((Ri - p.Radii) / p.unih)) - 1;
                }
                if (ht < 0) ht = 0;
                if (ht >= hd) deposit = false;
            }
            if (deposit) {
                bool collided = false;
                if (adv && t.n_bg && ht < p.collide_ht_max) {
                    const long long atm = static_cast<long long>(ht) * ftd * ffd + td * ffd + fd;
                    const double nloc = atm < t.n_bg_len ? t.n_bg[atm] : 0.0;
                    real_col_p += ds * nloc * p.cross_section;
                    const long long pc = static_cast<long long>(td) * ffd * hd +
                                         static_cast<long long>(fd) * hd + ht;
                    if (col_p < 1.0 - exp(-real_col_p) && t.cdf_valid[pc]) {
                        real_col_p = 0.0;
                        num_col++;
                        const double *coef = t.cdf_coef + DSMC_CDF_STRIDE * pc;
                        const double *box = t.cdf_box + 4 * pc;
                        rng.next();
                        if (p.scatter == DSMC_SCATTER_REFERENCE) {
                            // advanced.c:381-395 and collision.c:35-40
                            const double vv2 = cdf_sample(coef, box, t.cdf_total[pc],
                                                          t.cdf_degree, rng.raw(0) / kTwo32);
                            const double thi2 = kPi * rng.raw(1) / kTwo32 - kPi / 2.0;
                            const double fi2 = 2.0 * kPi * rng.raw(2) / kTwo32;
                            const double v2[3] = {vv2 * cos(thi2) * cos(fi2),
                                                  vv2 * cos(thi2) * sin(fi2), vv2 * sin(thi2)};
                            for (int k = 0; k < 3; k++) {
                                const double del = v[k] - v2[k], vcm = v[k] + v2[k];
                                v[k] = vcm + 0.5 * del;
                            }
                            if (p.redraw_col_threshold) col_p = rng.raw(3) / kTwo32;
                        } else {
                            // isotropic elastic hard sphere, equal masses
                            const double vv2 = cdf_sample(coef, box, t.cdf_total[pc],
                                                          t.cdf_degree, rng.raw(0) / kTwo32);
                            double d2[3], om[3];
                            unit_sphere(rng.raw(1) / kTwo32, rng.raw(2) / kTwo32, d2);
                            if (p.redraw_col_threshold) col_p = rng.raw(3) / kTwo32;
                            rng.next();
                            unit_sphere(rng.raw(0) / kTwo32, rng.raw(1) / kTwo32, om);
                            double gv[3], vcm[3];
                            for (int k = 0; k < 3; k++) {
                                const double v2k = vv2 * d2[k];
                                gv[k] = v[k] - v2k;
                                vcm[k] = 0.5 * (v[k] + v2k);
                            }
                            const double gl = len3(gv);
                            for (int k = 0; k < 3; k++) v[k] = vcm[k] + 0.5 * gl * om[k];
                        }
                        collided = true;
                        E_start = orbital_energy(p, s, v);
                    }
                }
                if (kMode != kSolve) {
                    // count_nn is keyed by (td, ht) without fd, ballistic.c:216-229
                    int *row = ra.rows + (pid - ra.row_base) * static_cast<long long>(ftd * hd);
                    const int b = td * hd + ht;
                    const int cur = row[b];
                    row[b] = cur + 1;
                    if (kMode == kRecord && cur < ra.cap) {
                        const long long slot = static_cast<long long>(b) * ra.cap + cur;
                        ra.rec_v[3 * slot] = v[0];
                        ra.rec_v[3 * slot + 1] = v[1];
                        ra.rec_v[3 * slot + 2] = v[2];
                        ra.rec_fd[slot] = fd;
                        ra.rec_key[slot] = (static_cast<unsigned long long>(pid) << 32) |
                                           static_cast<unsigned long long>(steps);
                    }
                } else if (!collided) {
                    const long long cell = static_cast<long long>(ht) * ftd * ffd + td * ffd + fd;
                    atomicAdd(&t.density[cell], to_fixed(W));
                    if (t.speed_hist && p.n_speed_bins > 0) {
                        int b = static_cast<int>(len3(v) / p.speed_bin_width);
                        if (b >= p.n_speed_bins) b = p.n_speed_bins - 1;
                        atomicAdd(&t.speed_hist[cell * p.n_speed_bins + b], 1ull);
                    }
                }
            }
            if (p.life_step_cap > 0 && steps >= p.life_step_cap) {
                fate = DSMC_FATE_STEP_CAP;
                break;
            }
        }
        // the hop ended (landing, escape radius, hop or life cap)
        if (p.drift_tol > 0.0 && fabs(orbital_energy(p, s, v) - E_start) > drift_abs) acc.drift++;
        if (fate != DSMC_FATE_ALIVE) break;

        // Landing, ballistic.c:239-264.
        Ri = len3(s);
        to_angles(s, Ri, thi, fi);
        to_index(thi, fi, ftd, ffd, td, fd);
        if (ref) {
            if (td <= 1 || td >= ftd - 2) {
                if (kMode == kSolve) atomicAdd(&t.horizon[td * ffd + fd], to_fixed(0.05 * W));
                W *= 0.95;
            }
        } else {
            const double nrm[3] = {s[0] / Ri, s[1] / Ri, s[2] / Ri};
            if (nrm[0] * p.sun[0] + nrm[1] * p.sun[1] + nrm[2] * p.sun[2] <= 0.0) {
                if (kMode == kSolve) atomicAdd(&t.horizon[td * ffd + fd], to_fixed(W));
                fate = DSMC_FATE_FROZEN;
                break;
            }
            for (int k = 0; k < 3; k++) s[k] = nrm[k] * p.Radii;
            local_T = t.face_T[locate_face(t, nrm)];
        }
    }

    acc.steps += steps;
    acc.collisions += num_col;
    acc.finished++;
    if (fate == DSMC_FATE_ESCAPED) acc.escaped++;
    if (kMode == kSolve && t.fate && slot >= 0 && slot < t.out_cap) t.fate[slot] = fate;
    if (kMode == kSolve && t.steps && slot >= 0 && slot < t.out_cap) t.steps[slot] = steps;
    if (record && (fate != DSMC_FATE_ESCAPED || !ref)) {
        t.ttime[1 * t.out_cap + slot] = thi;
        t.ttime[2 * t.out_cap + slot] = time;
        t.ttime[3 * t.out_cap + slot] = W;
        t.ttime[4 * t.out_cap + slot] = flight_time;
        if (adv || !ref) {
            t.ttime[7 * t.out_cap + slot] = rest_time;
            t.ttime[8 * t.out_cap + slot] = static_cast<double>(num_col);
        }
    }
}

template <int kMode>
__global__ void __launch_bounds__(128) plain_fp64_kernel(const dsmc_params p, const DevTables t,
                                                          long long pid_begin, long long n,
                                                          const RecordArgs ra) {
    Acc acc;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += stride)
        particle_life<kMode>(p, t, pid_begin + i, acc, ra);
    if (kMode == kSolve) {
        warp_add_stat(&t.stats[kStatSteps], acc.steps);
        warp_add_stat(&t.stats[kStatEscaped], acc.escaped);
        warp_add_stat(&t.stats[kStatCollisions], acc.collisions);
        warp_add_stat(&t.stats[kStatBound], acc.bound);
        warp_add_stat(&t.stats[kStatFinished], acc.finished);
        warp_add_stat(&t.stats[kStatDrift], acc.drift);
    }
}

// Turns per-particle visit counts into write cursors: for each bucket, an exclusive scan over
// the chunk's particles in pid order, starting from the records the bucket already holds.
__global__ void record_scan_kernel(int *rows, int nrows, int nb, int *filled) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int run = filled[b];
    for (int q = 0; q < nrows; q++) {
        const long long i = static_cast<long long>(q) * nb + b;
        const int c = rows[i];
        rows[i] = run;
        run += c;
    }
    filled[b] = run;
}

long long plain_blocks(long long n, int num_sms) {
    const int block = 128;
    long long blocks = (n + block - 1) / block;
    // Enough blocks for every particle its own thread, capped at a few waves of resident blocks
    // (the grid-stride loop covers the rest).
    const long long cap = static_cast<long long>(num_sms) * 16 * 64;
    return blocks > cap ? cap : blocks;
}

// Fed-state push: integrate each (s, v) with the reference's Verlet variant for up to nsteps
// steps, starting from oa = GM s / r^3 (ballistic.c:176-181), stopping at landing or escape.
__global__ void push_fp64_kernel(const dsmc_params p, long long n, int nsteps, double *pos,
                                 double *vel, int *status, int *taken) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    double v[3] = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    const double h = p.dt_step;
    double Ri = len3(s);
    double oa[3];
    for (int k = 0; k < 3; k++) oa[k] = p.GM * s[k] / (Ri * Ri * Ri);
    int st = 0, k = 0;
    for (; k < nsteps && st == 0; k++) {
        const double R0 = len3(s);
        const double g = p.GM / (R0 * R0 * R0);
        const double h2 = h * h;
        double ns[3];
        for (int j = 0; j < 3; j++)
            ns[j] = s[j] + v[j] * h - g * s[j] * (1.5 * h2) - oa[j] * (h2 / 6.0);
        for (int j = 0; j < 3; j++) v[j] -= g * s[j] * h;
        for (int j = 0; j < 3; j++) oa[j] = g * s[j];
        s[0] = ns[0]; s[1] = ns[1]; s[2] = ns[2];
        Ri = len3(s);
        st = Ri <= p.Radii ? 1 : (Ri >= p.max_height ? 2 : 0);
    }
    for (int j = 0; j < 3; j++) { pos[3 * i + j] = s[j]; vel[3 * i + j] = v[j]; }
    status[i] = st;
    taken[i] = k;
}

}  // namespace

cudaError_t launch_push_fp64(const dsmc_params &p, long long n, int nsteps, double *pos,
                             double *vel, int *status, int *taken, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    push_fp64_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, stream>>>(p, n, nsteps, pos, vel,
                                                                                status, taken);
    return cudaGetLastError();
}

cudaError_t launch_plain_fp64(const dsmc_params &p, const DevTables &t, long long pid_begin,
                              long long n, int num_sms, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const RecordArgs ra{};
    plain_fp64_kernel<kSolve><<<static_cast<unsigned>(plain_blocks(n, num_sms)), 128, 0, stream>>>(
        p, t, pid_begin, n, ra);
    return cudaGetLastError();
}

cudaError_t launch_plain_record(const dsmc_params &p, const DevTables &t, long long pid_begin,
                                long long n, const RecordArgs &ra, int *filled, int num_sms,
                                cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>(plain_blocks(n, num_sms));
    plain_fp64_kernel<kCount><<<blocks, 128, 0, stream>>>(p, t, pid_begin, n, ra);
    const int nb = p.ftd * p.hd;
    record_scan_kernel<<<(nb + 127) / 128, 128, 0, stream>>>(ra.rows, static_cast<int>(n), nb, filled);
    plain_fp64_kernel<kRecord><<<blocks, 128, 0, stream>>>(p, t, pid_begin, n, ra);
    return cudaGetLastError();
}

}  // namespace dsmc
