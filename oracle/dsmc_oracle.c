/* dsmc_oracle.c - CPU oracle of the DSMC test-particle hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this file, as the
 * checker; the product never links it. It restates the reference (rubby0605/dsmc_suite) in plain
 * C, keeping the reference's floating-point operation order so that, compiled without FMA
 * contraction, it reproduces the reference binary bit for bit (tests pin it against the reference
 * compiled from its own sources, and against the reference's known answers in
 * tests/test_verlet.c).
 */
#include "dsmc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define OR_RAND_MAX 2147483647.0   /* glibc RAND_MAX */
#define OR_TWO32 4294967296.0

/* ------------------------------------------------------------------------------------------ */
/* Philox4x32-10, as published by Salmon et al. (SC'11): 10 rounds of two 32x32->64 multiplies
 * with Weyl-sequence key bumps between rounds. */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Random stream of one particle. In rand_r mode every draw calls rand_r on the shared seed in
 * the reference's order; in Philox mode each event takes one 4-word block with counter
 * (pid, event, instance, 0) under key (seed_lo, seed_hi). */
typedef struct {
    int kind;
    unsigned *rr;
    uint32_t key[2];
    uint32_t pid, inst, event;
    uint32_t w[4];
    double div;
} or_rng;

static void rng_event(or_rng *r)
{
    if (r->kind != OR_RNG_PHILOX) return;
    uint32_t ctr[4] = {r->pid, r->event, r->inst, 0u};
    or_philox4x32(ctr, r->key, r->w);
    r->event++;
}

/* Raw draw as a double in [0, div]: rand_r() with div = RAND_MAX, or a Philox word with
 * div = 2^32. */
static double rng_raw(or_rng *r, int slot)
{
    if (r->kind == OR_RNG_PHILOX) return (double)r->w[slot];
    return (double)rand_r(r->rr);
}

static uint32_t rng_word(or_rng *r, int slot)
{
    if (r->kind == OR_RNG_PHILOX) return r->w[slot];
    return (uint32_t)rand_r(r->rr);
}

/* ------------------------------------------------------------------------------------------ */
/* Scalar functions. */

static double len3(const double a[3])
{
    /* vec3_len, include/types.h:23-25 */
    return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}

/* verlet_step, src/common/integrator.c:4-55. Returns 0 ok, 1 landed, 2 escaped. */
int or_verlet_step(double s[3], double v[3], double oa[3], double GM, double h, double Radii,
                   double max_height, double *ds_out)
{
    double Ri = len3(s);
    double Ri3 = Ri * Ri * Ri;
    double h2 = h * h;
    double g = GM / Ri3;
    double ns[3];
    for (int k = 0; k < 3; k++)
        ns[k] = s[k] + v[k] * h - g * s[k] * (1.5 * h2) - oa[k] * (h2 / 6.0);
    if (ds_out) {
        double d[3] = {ns[0] - s[0], ns[1] - s[1], ns[2] - s[2]};
        *ds_out = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    for (int k = 0; k < 3; k++) v[k] -= g * s[k] * h;
    for (int k = 0; k < 3; k++) oa[k] = g * s[k];
    s[0] = ns[0]; s[1] = ns[1]; s[2] = ns[2];
    double Rn = len3(s);
    if (Rn <= Radii) return 1;
    if (Rn >= max_height) return 2;
    return 0;
}

/* grid_spherical_to_index, src/common/grid.c:28-39. */
void or_spherical_to_index(double thi, double fi, int ftd, int ffd, int *td, int *fd)
{
    *td = (int)ceil((thi + M_PI / 2.0) / M_PI * ftd) - 1;
    *fd = (int)ceil(fi / (2.0 * M_PI) * ffd) - 1;
    if (*td < 0) *td = 0;
    if (*td >= ftd) *td = ftd - 1;
    if (*fd < 0) *fd = 0;
    if (*fd >= ffd) *fd = ffd - 1;
}

/* grid_exp_ht_index, src/common/grid.c:91-99; log(1 + alpha2) is passed in, formed by the
 * caller as log(1.0 + alpha2). */
int or_exp_ht_index(double Ri, double Radii, double unih, double alpha2, double log1p_alpha2)
{
    double arg = alpha2 * (Ri - Radii) / unih + 1.0;
    if (arg <= 1.0) return 0;
    int ht = (int)ceil(log(arg) / log1p_alpha2) - 1;
    if (ht < 0) ht = 0;
    return ht;
}

/* pos_to_angles, src/dsmc/ballistic.c:29-33. */
static void pos_to_angles(const double s[3], double Ri, double *thi, double *fi)
{
    *thi = asin(s[2] / Ri);
    *fi = atan2(s[0], s[1]);
    if (*fi < 0) *fi += 2.0 * M_PI;
}

/* velocity_table_init, src/common/velocity.c:6-47. */
void or_velocity_table_init(or_vtable *vt, double mmass, double mole, double k_B)
{
    double dT = (240.0 - 20.0) / (23 - 1);
    double m = mmass / mole;
    for (int i = 0; i < 23; i++) {
        double T = 20.0 + i * dT;
        vt->temps[i] = T;
        int n_v = 0;
        for (int j = 0; j <= 100; j++) {
            double vv = j * 10.0;
            double factor = 1.0 / (2.0 * M_PI) * m / (k_B * T);
            double aa = 4.0 * M_PI * vv * vv * pow(factor, 1.5)
                        * exp(-m * 3.0 * vv * vv / (2.0 * k_B * T));
            aa *= 5e5;
            int count = (int)floor(aa);
            for (int k = 0; k < count && n_v < 1000; k++) vt->speeds[i][n_v++] = vv;
        }
        if (n_v == 0) n_v = 1;
        vt->count[i] = n_v;
    }
}

/* velocity_sample, src/common/velocity.c:49-68, with the random word passed in. */
double or_velocity_sample_word(const or_vtable *vt, double T_local, uint32_t word)
{
    int idx;
    if (T_local >= 220.0) idx = 20;
    else idx = (int)ceil(T_local / 10.0) - 2;
    if (idx < 0) idx = 0;
    if (idx >= 23) idx = 22;
    return vt->speeds[idx][word % (uint32_t)vt->count[idx]];
}

/* Horner evaluation of one CDF row at speed x, in t = (x - xc) / xs (polyval,
 * src/common/polyfit.c:103-110, started from 0 as collision.c:57-60 does). */
static double cdf_eval(const double *coef, const double *box, int degree, double x)
{
    double t = (x - box[2]) / box[3];
    double r = 0.0;
    for (int i = 0; i <= degree; i++) r = r * t + coef[i];
    return r;
}

/* collision_sample_speed, src/common/collision.c:43-101. */
double or_cdf_sample(const double *coef, const double *box, double total, int degree, double u)
{
    double min_v = box[0], max_v = box[1];
    double val_at_max = cdf_eval(coef, box, degree, max_v);
    double ranking = u * (total - val_at_max) + val_at_max;
    double v0 = min_v, v1 = max_v;
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

/* polyfit, src/common/polyfit.c:10-101: normal equations, Gaussian elimination with partial
 * pivoting, coefficients returned highest power first. */
int or_polyfit(const double *x, const double *y, int n, int degree, double *coeffs)
{
    int m = degree + 1;
    if (n < m || degree > 6) return -1;
    double S[14] = {0};
    for (int i = 0; i < n; i++) {
        double xp = 1.0;
        for (int k = 0; k <= 2 * degree; k++) { S[k] += xp; xp *= x[i]; }
    }
    double a[7] = {0}, rhs[7] = {0};
    for (int i = 0; i < n; i++) {
        double xp = 1.0;
        for (int j = 0; j < m; j++) { rhs[j] += xp * y[i]; xp *= x[i]; }
    }
    double mat[7][8];
    memset(mat, 0, sizeof(mat));
    for (int r = 0; r < m; r++) {
        for (int c = 0; c < m; c++) mat[r][c] = S[r + c];
        mat[r][m] = rhs[r];
    }
    for (int col = 0; col < m; col++) {
        int max_row = col;
        double max_val = fabs(mat[col][col]);
        for (int row = col + 1; row < m; row++)
            if (fabs(mat[row][col]) > max_val) { max_val = fabs(mat[row][col]); max_row = row; }
        if (max_val < 1e-30) return -1;
        if (max_row != col)
            for (int k = 0; k <= m; k++) {
                double tmp = mat[col][k]; mat[col][k] = mat[max_row][k]; mat[max_row][k] = tmp;
            }
        for (int row = col + 1; row < m; row++) {
            double factor = mat[row][col] / mat[col][col];
            for (int k = col; k <= m; k++) mat[row][k] -= factor * mat[col][k];
        }
    }
    for (int row = m - 1; row >= 0; row--) {
        a[row] = mat[row][m];
        for (int col = row + 1; col < m; col++) a[row] -= mat[row][col] * a[col];
        a[row] /= mat[row][row];
    }
    for (int i = 0; i < m; i++) coeffs[i] = a[degree - i];
    return 0;
}

/* One cell of build_poly_fits, src/dsmc/advanced.c:44-108: sort the speeds, histogram them into
 * max(4, (nn+1)/2) bins between min and max, fit the reverse-cumulative counts. Writes the
 * coefficient row (xc = 0, xs = 1, so t = v) and returns 1 when the fit is valid. */
int or_fit_cell_from_samples(const double *speeds, int nn, int degree, double *coef,
                             double *box, double *total)
{
    if (nn <= 8) return 0;
    double v[64];
    if (nn > 64) return 0;
    for (int i = 0; i < nn; i++) v[i] = speeds[i];
    for (int i = 0; i < nn; i++)
        for (int j = i + 1; j < nn; j++)
            if (v[j] < v[i]) { double t = v[j]; v[j] = v[i]; v[i] = t; }
    double min_v = v[0], max_v = v[nn - 1];
    int nbins = (nn + 1) / 2;
    if (nbins < 4) nbins = 4;
    double xx[64], yy[64], yy2[64];
    double dv = (max_v - min_v) / nbins;
    for (int i = 0; i < nbins; i++) { xx[i] = min_v + (i + 0.5) * dv; yy[i] = 0; }
    for (int i = 0; i < nn; i++) {
        int bin = (int)((v[i] - min_v) / dv);
        if (bin >= nbins) bin = nbins - 1;
        if (bin < 0) bin = 0;
        yy[bin]++;
    }
    for (int i = 0; i < nbins; i++) {
        yy2[i] = 0;
        for (int j = i; j < nbins; j++) yy2[i] += yy[j];
    }
    double c[7];
    if (or_polyfit(xx, yy2, nbins, degree, c) != 0) return 0;
    for (int i = 0; i < DSMC_CDF_STRIDE; i++) coef[i] = i <= degree ? c[i] : 0.0;
    box[0] = min_v; box[1] = max_v; box[2] = 0.0; box[3] = 1.0;
    *total = (double)nn;
    return 1;
}

/* Config-model fit of one cell from its speed histogram: the same reverse-cumulative form over
 * the occupied bin range, with speeds mapped to t in [-1, 1] and counts normalised by the total,
 * which keeps the degree-6 normal equations well conditioned in FP64. */
int or_fit_cell_from_hist(const uint64_t *hist, int nbins, double bin_width, int degree,
                          double *coef, double *box, double *total)
{
    int lo = -1, hi = -1;
    uint64_t nn = 0;
    for (int i = 0; i < nbins; i++)
        if (hist[i]) { if (lo < 0) lo = i; hi = i; nn += hist[i]; }
    if (lo < 0) return 0;
    int m = hi - lo + 1;
    if (m < degree + 2 || nn <= 8) return 0;
    double min_v = lo * bin_width, max_v = (hi + 1) * bin_width;
    double xc = 0.5 * (min_v + max_v), xs = 0.5 * (max_v - min_v);
    double t[64], y[64];
    double acc = 0.0, inv = 1.0 / (double)nn;
    for (int i = hi; i >= lo; i--) {
        acc += (double)hist[i];
        t[i - lo] = ((lo + (i - lo) + 0.5) * bin_width - xc) / xs;
        y[i - lo] = acc * inv;
    }
    double c[7];
    if (or_polyfit(t, y, m, degree, c) != 0) return 0;
    for (int i = 0; i < DSMC_CDF_STRIDE; i++) coef[i] = i <= degree ? c[i] : 0.0;
    box[0] = min_v; box[1] = max_v; box[2] = xc; box[3] = xs;
    *total = 1.0;
    return 1;
}

/* Face of the icosphere whose cone contains direction p, by testing every face's three edge
 * planes (brute force; the product descends the subdivision tree instead). */
int or_locate_face(const dsmc_surface *surf, const double p[3])
{
    int best = 0;
    double best_dot = -2.0;
    for (int f = 0; f < surf->nface; f++) {
        const double *a = surf->face_verts + 9 * f, *b = a + 3, *c = a + 6;
        const double *e[3][2] = {{a, b}, {b, c}, {c, a}};
        int in = 1;
        for (int k = 0; k < 3 && in; k++) {
            const double *u = e[k][0], *w = e[k][1];
            double n0 = u[1] * w[2] - u[2] * w[1];
            double n1 = u[2] * w[0] - u[0] * w[2];
            double n2 = u[0] * w[1] - u[1] * w[0];
            if (n0 * p[0] + n1 * p[1] + n2 * p[2] < 0.0) in = 0;
        }
        if (in) return f;
        double cx = a[0] + b[0] + c[0], cy = a[1] + b[1] + c[1], cz = a[2] + b[2] + c[2];
        double d = (cx * p[0] + cy * p[1] + cz * p[2]) / sqrt(cx * cx + cy * cy + cz * cz);
        if (d > best_dot) { best_dot = d; best = f; }
    }
    return best;
}

/* ------------------------------------------------------------------------------------------ */
/* Particle life. */

typedef struct {
    const dsmc_params *p;
    const dsmc_surface *surf;
    const dsmc_collision *col;
    const or_vtable *vt;
    or_outputs *out;
    int64_t pid_begin, n;
    int serial;          /* 1: plain adds (one thread, double sums in deposit order) */
} or_ctx;

static void add_f64(double *a, double x, int serial)
{
    if (serial) { *a += x; return; }
#pragma omp atomic
    *a += x;
}

static void add_u64(uint64_t *a, uint64_t x, int serial)
{
    if (serial) { *a += x; return; }
#pragma omp atomic
    *a += x;
}

static void add_i64(int64_t *a, int64_t x, int serial)
{
    if (serial) { *a += x; return; }
#pragma omp atomic
    *a += x;
}

static uint64_t to_fixed(double W)
{
    return (uint64_t)llrint(W * DSMC_FIXED_SCALE);
}

static void deposit_grid(or_ctx *c, int64_t idx, double W)
{
    if (c->out->density_f64) add_f64(&c->out->density_f64[idx], W, c->serial);
    if (c->out->density_fx) add_u64(&c->out->density_fx[idx], to_fixed(W), c->serial);
}

static void deposit_horizon(or_ctx *c, int64_t idx, double W)
{
    if (c->out->horizon_f64) add_f64(&c->out->horizon_f64[idx], W, c->serial);
    if (c->out->horizon_fx) add_u64(&c->out->horizon_fx[idx], to_fixed(W), c->serial);
}

static void sample_unit_sphere(double z_u, double phi_u, double o[3])
{
    double z = 2.0 * z_u - 1.0;
    double r = sqrt(fmax(0.0, 1.0 - z * z));
    double ph = 2.0 * M_PI * phi_u;
    o[0] = r * cos(ph); o[1] = r * sin(ph); o[2] = z;
}

/* Config-model launch velocity: flux-weighted Maxwell-Boltzmann at temperature T, i.e. a Rayleigh
 * normal component and Gaussian tangential components, plus the rotation of the surface. */
static void config_launch(const dsmc_params *p, const double s[3], double T, or_rng *r,
                          double v[3])
{
    rng_event(r);
    double u0 = rng_raw(r, 0) / OR_TWO32, u1 = rng_raw(r, 1) / OR_TWO32,
           u2 = rng_raw(r, 2) / OR_TWO32;
    double sigma = sqrt(p->kB_over_m * T);
    double vn = sigma * sqrt(-2.0 * log(1.0 - u0));
    double rho = sqrt(-2.0 * log(1.0 - u1));
    double ang = 2.0 * M_PI * u2;
    double t1 = rho * cos(ang), t2 = rho * sin(ang);
    double R = len3(s);
    double n[3] = {s[0] / R, s[1] / R, s[2] / R};
    double e[3] = {-n[1], n[0], 0.0};
    double le = sqrt(e[0] * e[0] + e[1] * e[1]);
    if (le < 1e-12) { e[0] = 1.0; e[1] = 0.0; }
    else { e[0] /= le; e[1] /= le; }
    double nt[3] = {n[1] * e[2] - n[2] * e[1], n[2] * e[0] - n[0] * e[2],
                    n[0] * e[1] - n[1] * e[0]};
    double omega = p->P > 0.0 ? 2.0 * M_PI / p->P : 0.0;
    double rot[3] = {omega * s[1], -omega * s[0], 0.0};
    for (int k = 0; k < 3; k++)
        v[k] = vn * n[k] + (sigma * t1) * e[k] + (sigma * t2) * nt[k] + rot[k];
}

static int pick_face(const dsmc_surface *surf, double u)
{
    if (!surf->face_cdf) {
        int f = (int)(u * surf->nface);
        return f < surf->nface ? f : surf->nface - 1;
    }
    int lo = 0, hi = surf->nface - 1;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (surf->face_cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

/* Orbital energy per unit mass |v|^2 / 2 - GM / |s| of the drift guard. */
static double orbital_energy(const dsmc_params *p, const double s[3], const double v[3])
{
    return 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - p->GM / len3(s);
}

static void run_particle(or_ctx *c, int64_t pid, or_rng *r)
{
    const dsmc_params *p = c->p;
    or_outputs *out = c->out;
    const int ftd = p->ftd, ffd = p->ffd, hd = p->hd;
    const int64_t nslot = c->n;
    const int64_t n = pid - c->pid_begin;
    const int ref = p->model == DSMC_MODEL_REFERENCE;
    const int adv = p->runner == DSMC_RUNNER_ADVANCED;
    const double h = p->dt_step;
    const double *T = c->surf->T_map;
    double *tt = out->ttime;

    int fate = DSMC_FATE_ALIVE;
    int num_col = 0;
    int64_t steps = 0;
    double real_col_p = 0.0, col_p = 0.0;
    double time = 0.0, W = 1.0, flight_time = 0.0, rest_time = 0.0;
    double thi, fi, s[3], v[3] = {0.0, 0.0, 0.0};
    double local_T = 0.0;
    int td, fd;
    /* energy-drift guard: E at the hop's launch (or last collision) against E where it ends */
    const double drift_abs = p->drift_tol * p->GM / p->Radii;
    double E_start = 0.0;

    r->pid = (uint32_t)pid;
    r->event = 0;
    rng_event(r);
    if (ref) {
        /* ballistic.c:112-118; advanced.c:246,254-260 (col_p is drawn first there). */
        if (adv) col_p = rng_raw(r, 0) / r->div;
        int o = adv ? 1 : 0;
        thi = rng_raw(r, o) / r->div * M_PI - M_PI / 2.0;
        fi = rng_raw(r, o + 1) / r->div * 2.0 * M_PI;
        s[0] = p->Radii * cos(thi) * sin(fi);
        s[1] = p->Radii * cos(thi) * cos(fi);
        s[2] = p->Radii * sin(thi);
        or_spherical_to_index(thi, fi, ftd, ffd, &td, &fd);
        local_T = T[td * ffd + fd];
    } else {
        int f = pick_face(c->surf, rng_raw(r, 0) / OR_TWO32);
        double u1 = rng_raw(r, 1) / OR_TWO32, u2 = rng_raw(r, 2) / OR_TWO32;
        col_p = rng_raw(r, 3) / OR_TWO32;
        if (u1 + u2 > 1.0) { u1 = 1.0 - u1; u2 = 1.0 - u2; }
        const double *a = c->surf->face_verts + 9 * f, *b = a + 3, *cc = a + 6;
        double q[3];
        for (int k = 0; k < 3; k++) q[k] = a[k] + u1 * (b[k] - a[k]) + u2 * (cc[k] - a[k]);
        double lq = len3(q);
        for (int k = 0; k < 3; k++) s[k] = q[k] * (p->Radii / lq);
        pos_to_angles(s, len3(s), &thi, &fi);
        or_spherical_to_index(thi, fi, ftd, ffd, &td, &fd);
        local_T = c->surf->face_T[f];
    }
    if (tt) {
        tt[0 * nslot + n] = thi;
        if (adv || !ref) { tt[5 * nslot + n] = fi; tt[6 * nslot + n] = local_T; }
    }

    for (;;) {
        if (W < p->w_min) { fate = DSMC_FATE_PHOTOLYSED; break; }
        if (p->life_step_cap > 0 && steps >= p->life_step_cap) { fate = DSMC_FATE_STEP_CAP; break; }

        if (ref) {
            double KF = 2.0 * M_PI * p->Radii * fabs(cos(thi)) / p->P;
            or_spherical_to_index(thi, fi, ftd, ffd, &td, &fd);
            local_T = T[td * ffd + fd];
            if (local_T < p->freeze_T) {
                int found = 0;
                if (!adv) {
                    /* ballistic.c:132-153: scan columns relative to fd; s is not moved. */
                    for (int add = 0; add < ffd; add++) {
                        time += p->dt_rot;
                        int check_fd = (fd + add + 1) % ffd;
                        if (T[td * ffd + check_fd] >= p->freeze_T) {
                            fd = check_fd;
                            fi = (fd + 0.5) / ffd * 2.0 * M_PI;
                            found = 1;
                            break;
                        }
                    }
                    if (!found) { deposit_horizon(c, td * ffd + fd, W); fate = DSMC_FATE_FROZEN; break; }
                } else {
                    /* advanced.c:278-309: horizon at entry, absolute column scan, s rotated. */
                    deposit_horizon(c, td * ffd + fd, W);
                    for (int add = 1; add <= ffd; add++) {
                        time += p->dt_rot;
                        rest_time += p->dt_rot;
                        if (T[td * ffd + (add % ffd)] >= p->freeze_T) {
                            double rot_fi = (double)(add - fd) / ffd * 2.0 * M_PI;
                            double cs = cos(rot_fi), sn = sin(rot_fi);
                            double ns0 = s[0] * cs - s[1] * sn, ns1 = s[0] * sn + s[1] * cs;
                            s[0] = ns0; s[1] = ns1;
                            fd = add % ffd;
                            fi = (fd + 0.5) / ffd * 2.0 * M_PI;
                            found = 1;
                            break;
                        }
                    }
                    if (!found) { deposit_horizon(c, td * ffd + fd, W); fate = DSMC_FATE_FROZEN; break; }
                }
                local_T = T[td * ffd + fd];
            }
            /* ballistic.c:156-173 */
            rng_event(r);
            double vr = or_velocity_sample_word(c->vt, local_T, rng_word(r, 0));
            double v_old_sq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            double vout = sqrt(p->alpha * vr * vr + (1.0 - p->alpha) * v_old_sq);
            double flyd = rng_raw(r, 1) / r->div * M_PI + thi - M_PI / 2.0;
            double xi = rng_raw(r, 2) / r->div * M_PI + fi - M_PI / 2.0;
            v[0] = cos(flyd) * sin(xi) * vout;
            v[1] = cos(flyd) * cos(xi) * vout;
            v[2] = sin(flyd) * vout;
            v[0] += KF * sin(fi + M_PI / 2.0);
            v[1] += KF * cos(fi + M_PI / 2.0);
            if (len3(v) >= p->ve) { fate = DSMC_FATE_ESCAPED; break; }
        } else {
            config_launch(p, s, local_T, r, v);
            double E = 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - p->GM / len3(s);
            if (E < 0.0) add_i64(&out->n_bound_launch, 1, c->serial);
        }

        double Ri = len3(s);
        double oa[3];
        for (int k = 0; k < 3; k++) oa[k] = p->GM * s[k] / (Ri * Ri * Ri);
        E_start = orbital_energy(p, s, v);

        for (int64_t ii = 0; ii < p->hop_step_cap; ii++) {
            flight_time += h;
            time += h;
            steps++;
            double ds;
            int st = or_verlet_step(s, v, oa, p->GM, h, p->Radii, p->max_height, &ds);
            if (st == 1) break;
            if (st == 2) { fate = DSMC_FATE_ESCAPED; break; }

            Ri = len3(s);
            pos_to_angles(s, Ri, &thi, &fi);
            or_spherical_to_index(thi, fi, ftd, ffd, &td, &fd);

            int day = ref ? (fd < ffd / 2)
                          : (s[0] * p->sun[0] + s[1] * p->sun[1] + s[2] * p->sun[2] > 0.0);
            if (day) W *= p->wdecay;

            int deposit = !(p->skip_first_deposit && ii == 0);
            int ht = -1;
            if (deposit) {
                if (p->use_exp_grid)
                    ht = or_exp_ht_index(Ri, p->Radii, p->unih, p->alpha2, p->log1p_alpha2);
                else
                    ht = (int)ceil((Ri - p->Radii) / p->unih) - 1;
                if (ht < 0) ht = 0;
                if (ht >= hd) deposit = 0;
            }
            if (deposit) {
                /* velocity record, ballistic.c:216-232 (serial pinning mode only) */
                if (ref && !adv && c->serial && out->v_record &&
                    out->v_count_nn[td * hd + ht] < 200 && out->n_records < out->v_cap) {
                    int64_t ridx = out->n_records++;
                    out->v_record[3 * ridx] = v[0];
                    out->v_record[3 * ridx + 1] = v[1];
                    out->v_record[3 * ridx + 2] = v[2];
                    out->v_td[ridx] = td; out->v_fd[ridx] = fd; out->v_ht[ridx] = ht;
                    out->v_count_nn[td * hd + ht]++;
                }
                int collided = 0;
                if (adv && c->col && c->col->n_bg && ht < p->collide_ht_max) {
                    int64_t atm_idx = (int64_t)ht * ftd * ffd + td * ffd + fd;
                    double nloc = atm_idx < c->col->n_bg_len ? c->col->n_bg[atm_idx] : 0.0;
                    real_col_p += ds * nloc * p->cross_section;
                    int64_t pidx = (int64_t)td * ffd * hd + (int64_t)fd * hd + ht;
                    if (col_p < 1.0 - exp(-real_col_p) && c->col->cdf_valid[pidx]) {
                        real_col_p = 0.0;
                        num_col++;
                        const double *coef = c->col->cdf_coef + DSMC_CDF_STRIDE * pidx;
                        const double *box = c->col->cdf_box + 4 * pidx;
                        double total = c->col->cdf_total[pidx];
                        rng_event(r);
                        if (p->scatter == DSMC_SCATTER_REFERENCE) {
                            /* advanced.c:381-395, collision.c:15-41 */
                            double rand_val = rng_raw(r, 0) / r->div;
                            double vv2 = or_cdf_sample(coef, box, total, c->col->cdf_degree,
                                                       rand_val);
                            double thi2 = M_PI * rng_raw(r, 1) / r->div - M_PI / 2.0;
                            double fi2 = 2.0 * M_PI * rng_raw(r, 2) / r->div;
                            double v2[3] = {vv2 * cos(thi2) * cos(fi2),
                                            vv2 * cos(thi2) * sin(fi2), vv2 * sin(thi2)};
                            for (int k = 0; k < 3; k++) {
                                double del = v[k] - v2[k], vcm = v[k] + v2[k];
                                v[k] = vcm + 0.5 * del;
                            }
                            if (p->redraw_col_threshold) col_p = rng_raw(r, 3) / r->div;
                        } else {
                            double vv2 = or_cdf_sample(coef, box, total, c->col->cdf_degree,
                                                       rng_raw(r, 0) / OR_TWO32);
                            double d2[3], om[3];
                            sample_unit_sphere(rng_raw(r, 1) / OR_TWO32,
                                               rng_raw(r, 2) / OR_TWO32, d2);
                            if (p->redraw_col_threshold) col_p = rng_raw(r, 3) / OR_TWO32;
                            rng_event(r);
                            sample_unit_sphere(rng_raw(r, 0) / OR_TWO32,
                                               rng_raw(r, 1) / OR_TWO32, om);
                            double g[3], vcm[3];
                            for (int k = 0; k < 3; k++) {
                                double v2k = vv2 * d2[k];
                                g[k] = v[k] - v2k;
                                vcm[k] = 0.5 * (v[k] + v2k);
                            }
                            double gl = len3(g);
                            for (int k = 0; k < 3; k++) v[k] = vcm[k] + 0.5 * gl * om[k];
                        }
                        collided = 1;
                        E_start = orbital_energy(p, s, v);
                    }
                }
                if (!collided) {
                    int64_t cell = (int64_t)ht * ftd * ffd + td * ffd + fd;
                    deposit_grid(c, cell, W);
                    if (out->speed_hist && p->n_speed_bins > 0) {
                        double sp = len3(v);
                        int b = (int)(sp / p->speed_bin_width);
                        if (b >= p->n_speed_bins) b = p->n_speed_bins - 1;
                        add_u64(&out->speed_hist[cell * p->n_speed_bins + b], 1, c->serial);
                    }
                }
            }
            if (p->life_step_cap > 0 && steps >= p->life_step_cap) {
                fate = DSMC_FATE_STEP_CAP;
                break;
            }
        }
        /* the hop ended (landing, escape radius, hop or life cap) */
        if (p->drift_tol > 0.0 && fabs(orbital_energy(p, s, v) - E_start) > drift_abs)
            add_i64(&out->n_drift_flagged, 1, c->serial);
        if (fate != DSMC_FATE_ALIVE) break;

        /* landing (or a hop that ran out of steps): ballistic.c:239-264 */
        Ri = len3(s);
        pos_to_angles(s, Ri, &thi, &fi);
        or_spherical_to_index(thi, fi, ftd, ffd, &td, &fd);
        if (ref) {
            if (td <= 1 || td >= ftd - 2) {
                deposit_horizon(c, td * ffd + fd, 0.05 * W);
                W *= 0.95;
            }
        } else {
            double nrm[3] = {s[0] / Ri, s[1] / Ri, s[2] / Ri};
            if (nrm[0] * p->sun[0] + nrm[1] * p->sun[1] + nrm[2] * p->sun[2] <= 0.0) {
                deposit_horizon(c, td * ffd + fd, W);
                fate = DSMC_FATE_FROZEN;
                break;
            }
            for (int k = 0; k < 3; k++) s[k] = nrm[k] * p->Radii;
            local_T = c->surf->face_T[or_locate_face(c->surf, nrm)];
        }
    }

    if (out->fate) out->fate[n] = fate;
    if (out->steps) out->steps[n] = steps;
    if (fate == DSMC_FATE_ESCAPED) add_i64(&out->n_escaped, 1, c->serial);
    add_i64(&out->total_steps, steps, c->serial);
    add_i64(&out->n_collisions, num_col, c->serial);
    if (tt && (fate != DSMC_FATE_ESCAPED || !ref)) {
        tt[1 * nslot + n] = thi;
        tt[2 * nslot + n] = time;
        tt[3 * nslot + n] = W;
        tt[4 * nslot + n] = flight_time;
        if (adv || !ref) {
            tt[7 * nslot + n] = rest_time;
            tt[8 * nslot + n] = (double)num_col;
        }
    }
}

int or_run(const dsmc_params *p, const dsmc_surface *surf, const dsmc_collision *col,
           const or_vtable *vt, int rng_kind, unsigned rr_seed, int64_t pid_begin, int64_t n,
           int nthreads, or_outputs *out)
{
    if (!p || !surf || !out || n < 0) return -1;
    if (p->model == DSMC_MODEL_REFERENCE && (!surf->T_map || !vt)) return -2;
    if (p->model == DSMC_MODEL_CONFIG && (!surf->face_verts || !surf->face_T)) return -3;
    if (rng_kind == OR_RNG_RAND_R && nthreads != 1) return -4;
    or_ctx c = {p, surf, col, vt, out, pid_begin, n, nthreads == 1};
    if (rng_kind == OR_RNG_RAND_R) {
        unsigned seed = rr_seed;
        or_rng r = {OR_RNG_RAND_R, &seed, {0, 0}, 0, 0, 0, {0, 0, 0, 0}, OR_RAND_MAX};
        for (int64_t i = 0; i < n; i++) run_particle(&c, pid_begin + i, &r);
        return 0;
    }
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
    {
        or_rng r = {OR_RNG_PHILOX, NULL, {(uint32_t)p->seed, (uint32_t)(p->seed >> 32)},
                    0, p->instance, 0, {0, 0, 0, 0}, OR_TWO32};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 100)
#endif
        for (int64_t i = 0; i < n; i++) run_particle(&c, pid_begin + i, &r);
    }
    return 0;
}
