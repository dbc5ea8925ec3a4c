/* dsmc_oracle.h - CPU oracle of the DSMC test-particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (dsmc_suite_b200/, include/) links or calls
 * this code; only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py do, as the
 * checker. The oracle restates the reference's algorithm (rubby0605/dsmc_suite,
 * src/dsmc/ballistic.c, src/dsmc/advanced.c and the files of src/common/) in plain C with the reference's
 * operation order, and adds the config-model physics of include/dsmc_params.h.
 *
 * Two random streams:
 *   OR_RNG_RAND_R - glibc rand_r on one seed, drawn in the reference's order; with one thread this
 *                   reproduces the reference binary's `-t 1` run draw for draw (pinning mode).
 *   OR_RNG_PHILOX - Philox4x32-10 keyed (seed, instance, particle id), the stream the CUDA kernels
 *                   use, so oracle and GPU see identical draws (comparison mode).
 */
#ifndef DSMC_ORACLE_H
#define DSMC_ORACLE_H

#include <stdint.h>
#include "../include/dsmc_params.h"
#include "../include/thermal.h"

enum { OR_RNG_RAND_R = 0, OR_RNG_PHILOX = 1 };

/* Same layout as the reference's VelocityTable (include/types.h:80-86). */
typedef struct or_vtable {
    double temps[23];
    double speeds[23][1000];
    int count[23];
} or_vtable;

typedef struct or_outputs {
    double   *density_f64;   /* [hd*ftd*ffd] double sums in deposit order, or NULL */
    uint64_t *density_fx;    /* [hd*ftd*ffd] fixed-point sums, or NULL */
    double   *horizon_f64;   /* [ftd*ffd], or NULL */
    uint64_t *horizon_fx;    /* [ftd*ffd], or NULL */
    double   *ttime;         /* [9][n] per-particle rows (ballistic.c:120,273-276;
                                advanced.c:262-267,439-444), or NULL */
    int32_t  *fate;          /* [n], or NULL */
    int64_t  *steps;         /* [n] Verlet steps per particle, or NULL */
    uint64_t *speed_hist;    /* [hd*ftd*ffd][n_speed_bins], or NULL */
    /* velocity record of the reference ballistic runner (ballistic.c:216-232) */
    double   *v_record;      /* [v_cap][3], or NULL */
    int32_t  *v_td, *v_fd, *v_ht;
    int32_t  *v_count_nn;    /* [ftd*hd] records per (td, ht), zeroed by the caller */
    int64_t   v_cap;         /* 100*ftd*hd in the reference */
    int64_t   n_records;
    /* totals */
    int64_t total_steps, n_escaped, n_collisions, n_bound_launch;
    int64_t n_drift_flagged;   /* hops that failed the energy-drift guard (dsmc_params.drift_tol) */
} or_outputs;

/* Philox4x32-10 block function (Salmon, Moraes, Dror, Shaw, SC'11). */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Scalar restatements. */
int or_verlet_step(double s[3], double v[3], double oa[3], double GM, double h, double Radii,
                   double max_height, double *ds_out);
void or_spherical_to_index(double thi, double fi, int ftd, int ffd, int *td, int *fd);
int or_exp_ht_index(double Ri, double Radii, double unih, double alpha2, double log1p_alpha2);
void or_velocity_table_init(or_vtable *vt, double mmass, double mole, double k_B);
double or_velocity_sample_word(const or_vtable *vt, double T_local, uint32_t word);
double or_cdf_sample(const double *coef, const double *box, double total, int degree,
                     double u);
int or_polyfit(const double *x, const double *y, int n, int degree, double *coeffs);
int or_fit_cell_from_samples(const double *speeds, int nn, int degree, double *coef,
                             double *box, double *total);
int or_fit_cell_from_hist(const uint64_t *hist, int nbins, double bin_width, int degree,
                          double *coef, double *box, double *total);
int or_locate_face(const dsmc_surface *surf, const double p[3]);

/* One solve over particles [pid_begin, pid_begin + n). Deposits are added into the output
 * arrays, which the caller zeroes. rr_seed is the rand_r seed (OR_RNG_RAND_R only; the reference
 * uses 67890 for ballistic and 98765 for advanced at thread 0). nthreads > 1 is allowed only
 * with OR_RNG_PHILOX and fixed-point outputs. Returns 0, or a negative value on bad input. */
int or_run(const dsmc_params *p, const dsmc_surface *surf, const dsmc_collision *col,
           const or_vtable *vt, int rng_kind, unsigned rr_seed, int64_t pid_begin, int64_t n,
           int nthreads, or_outputs *out);

/* Thermal column model (thermal_oracle.c): surface temperature [ftd][ffd]; flux NULL = the
 * reference's analytic flux. Returns 0, or < 0 on bad input / no memory. */
int or_thermal_solve(int ftd, int ffd, const ThermalParams *tp, const double *flux,
                     double *T_out, int *h_depth);

/* Monte Carlo shadow flux (raytrace_oracle.c): F [nface][tt]; facet 0-based. */
int or_shadow_flux(int npoint, const double *spot, int nface, const int32_t *facet,
                   const double *normal, double za, int tt, int nmonte, double *F, int nthreads);

#endif
