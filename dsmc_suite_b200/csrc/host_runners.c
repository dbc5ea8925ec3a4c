/* host_runners.c - drop-in run_ballistic / run_advanced (signatures of the reference's
 * src/dsmc/ballistic.c:35-36 and src/dsmc/advanced.c:119-121) on top of the C ABI.
 *
 * The runners keep the reference's file contract and console summary lines; the particle loops
 * themselves run on the GPU. Reference-model physics comes from dsmc_params_reference. */
#include "dsmc_cuda.h"
#include "dsmc_runners.h"
#include "fileio.h"
#include "types.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int env_int(const char *name, int dflt)
{
    const char *v = getenv(name);
    return v && *v ? atoi(v) : dflt;
}

static int env_path(void)
{
    const char *v = getenv("DSMC_PATH");
    if (!v || !*v || !strcmp(v, "plain")) return DSMC_PATH_PLAIN_FP64;
    if (!strcmp(v, "fast32") || !strcmp(v, "fast")) return DSMC_PATH_FAST_FP32;
    if (!strcmp(v, "fast64")) return DSMC_PATH_FAST_FP64;
    return DSMC_PATH_PLAIN_FP64;
}

static void apply_seed(dsmc_params *p)
{
    const char *v = getenv("DSMC_SEED");
    if (v && *v) p->seed = strtoull(v, NULL, 10);
}

static int report(dsmc_ctx *ctx, int rc, const char *what)
{
    if (rc != DSMC_OK)
        fprintf(stderr, "%s failed: %s (%s)\n", what, dsmc_status_string(rc), dsmc_last_error(ctx));
    return rc;
}

static double *fixed_to_double(const uint64_t *fx, long n)
{
    double *d = malloc((size_t)n * sizeof(double));
    if (!d) return NULL;
    for (long i = 0; i < n; i++) d[i] = (double)fx[i] / DSMC_FIXED_SCALE;
    return d;
}

/* Solve, then copy grids and per-particle rows back. Returns DSMC_OK or a status. */
static int solve(dsmc_ctx *ctx, const dsmc_params *p, const dsmc_surface *s,
                 const dsmc_collision *col, int totaln, uint64_t *den, uint64_t *hor,
                 double *ttime, dsmc_stats *st)
{
    int rc;
    if ((rc = report(ctx, dsmc_setup(ctx, p, s, col), "dsmc_setup"))) return rc;
    if ((rc = report(ctx, dsmc_enable_particle_outputs(ctx, totaln), "particle outputs"))) return rc;
    if ((rc = report(ctx, dsmc_zero(ctx), "dsmc_zero"))) return rc;
    if ((rc = report(ctx, dsmc_run(ctx, env_path(), 0, totaln), "dsmc_run"))) return rc;
    if ((rc = report(ctx, dsmc_sync(ctx), "dsmc_sync"))) return rc;
    if ((rc = report(ctx, dsmc_get_density(ctx, den), "density"))) return rc;
    if ((rc = report(ctx, dsmc_get_horizon(ctx, hor), "horizon"))) return rc;
    if ((rc = report(ctx, dsmc_get_particle_outputs(ctx, totaln, ttime, NULL, NULL), "ttime")))
        return rc;
    return report(ctx, dsmc_get_stats(ctx, st), "stats");
}

static void write_grids(const char *prefix, const uint64_t *den, const uint64_t *hor,
                        const double *ttime, int nrows, int totaln, const dsmc_params *p)
{
    char fname[1024];
    const long ncell = (long)p->hd * p->ftd * p->ffd, nh = (long)p->ftd * p->ffd;
    double *dd = fixed_to_double(den, ncell), *hh = fixed_to_double(hor, nh);
    if (dd && hh) {
        snprintf(fname, sizeof fname, "%s_den.dat", prefix);
        write_density_dat(fname, dd, p->ftd, p->ffd, p->hd);
        snprintf(fname, sizeof fname, "%s_horizon.dat", prefix);
        write_horizon_dat(fname, hh, p->ftd, p->ffd);
        snprintf(fname, sizeof fname, "%s_ttime.dat", prefix);
        write_ttime_dat(fname, ttime, nrows, totaln);
        const char *rate = getenv("DSMC_NDENSITY_RATE");
        if (rate && *rate && totaln > 0) {
            /* FP64 number density [m^-3] per cell, physical cell volumes */
            double *nd = malloc((size_t)ncell * sizeof(double));
            snprintf(fname, sizeof fname, "%s_ndensity.dat", prefix);
            if (!nd || dsmc_number_density_host(p, den, totaln, strtod(rate, NULL),
                                                DSMC_VOLUME_PHYSICAL, nd) != DSMC_OK ||
                write_ndensity_dat(fname, nd, p->ftd, p->ffd, p->hd))
                fprintf(stderr, "cannot write %s\n", fname);
            free(nd);
        }
        if (env_int("DSMC_SIDECAR", 0)) {
            snprintf(fname, sizeof fname, "%s_grids.bin", prefix);
            if (write_grids_bin(fname, den, hor, ttime, p->ftd, p->ffd, p->hd, nrows, totaln,
                                DSMC_FIXED_SCALE))
                fprintf(stderr, "cannot write %s\n", fname);
        }
    } else {
        fprintf(stderr, "out of host memory writing results\n");
    }
    free(dd);
    free(hh);
}

void run_ballistic(int totaln, const char *temp_file, const char *output_prefix, int nthreads)
{
    (void)nthreads;
    int ftd, ffd;
    double *T = read_temperature_dat(temp_file, &ftd, &ffd);
    if (!T) { fprintf(stderr, "Failed to read temperature file\n"); return; }
    if (totaln < 0) totaln = 0;
    dsmc_params p;
    dsmc_params_reference(&p, DSMC_RUNNER_BALLISTIC, ftd, ffd);
    apply_seed(&p);
    printf("Starting ballistic simulation: %d particles\n", totaln);
    printf("  ftd=%d, ffd=%d, hd=%d\n", ftd, ffd, p.hd);
    printf("  Escape velocity = %.2f m/s\n", p.ve);
    printf("  Lifetime = %.1f s\n", p.lifetime);

    dsmc_ctx *ctx = NULL;
    if (report(NULL, dsmc_ctx_create(env_int("DSMC_DEVICE", 0), &ctx), "dsmc_ctx_create")) {
        free(T);
        return;
    }
    const long ncell = (long)p.hd * ftd * ffd;
    uint64_t *den = calloc((size_t)ncell, sizeof(uint64_t));
    uint64_t *hor = calloc((size_t)ftd * ffd, sizeof(uint64_t));
    double *ttime = calloc((size_t)9 * (totaln > 0 ? totaln : 1), sizeof(double));
    dsmc_surface s;
    memset(&s, 0, sizeof s);
    s.T_map = T;
    dsmc_stats st;
    if (den && hor && ttime && solve(ctx, &p, &s, NULL, totaln, den, hor, ttime, &st) == DSMC_OK) {
        printf("Simulation complete. Escaped: %lld/%d\n", (long long)st.n_escaped, totaln);
        write_grids(output_prefix, den, hor, ttime, 5, totaln, &p);
        /* Velocity record of the phase-1 run (ballistic.c:216-232). */
        const long cap = 100L * ftd * p.hd;
        double *vr = calloc((size_t)cap * 3 + 3, sizeof(double));
        int32_t *rtd = calloc((size_t)cap + 1, sizeof(int32_t)), *rfd = calloc((size_t)cap + 1, sizeof(int32_t)),
                *rht = calloc((size_t)cap + 1, sizeof(int32_t));
        int64_t nrec = 0;
        if (vr && rtd && rfd && rht &&
            report(ctx, dsmc_velocity_record(ctx, totaln, 200, cap, vr, rtd, rfd, rht, &nrec),
                   "velocity record") == DSMC_OK) {
            char fname[1024];
            snprintf(fname, sizeof fname, "%s_v_record.dat", output_prefix);
            write_v_record_dat(fname, vr, rtd, rfd, rht, (int)nrec);
        }
        free(vr); free(rtd); free(rfd); free(rht);
    }
    dsmc_ctx_destroy(ctx);
    free(den);
    free(hor);
    free(ttime);
    free(T);
}

void run_advanced(int totaln, const char *temp_file, const char *prev_den_file,
                  const char *prev_v_record_file, const char *output_prefix, int nthreads)
{
    (void)nthreads;
    int ftd, ffd;
    double *T = read_temperature_dat(temp_file, &ftd, &ffd);
    if (!T) { fprintf(stderr, "Failed to read temperature file\n"); return; }
    if (totaln < 0) totaln = 0;
    dsmc_params p;
    dsmc_params_reference(&p, DSMC_RUNNER_ADVANCED, ftd, ffd);
    apply_seed(&p);
    const int hd = p.hd, max_per_cell = 50;
    const long ncell = (long)hd * ftd * ffd;

    /* Phase-1 background (advanced.c:160-166). */
    int pftd = 0, pffd = 0, phd = 0;
    double *copy_atm = prev_den_file ? read_density_dat(prev_den_file, &pftd, &pffd, &phd, 1) : NULL;

    /* Phase-1 speeds per cell, at most 50, in [td][fd][ht] order (advanced.c:168-209). */
    int32_t *count_num = calloc((size_t)ncell, sizeof(int32_t));
    double *speeds = calloc((size_t)ncell * max_per_cell, sizeof(double));
    if (!count_num || !speeds) { fprintf(stderr, "out of host memory\n"); goto out_early; }
    if (prev_v_record_file) {
        double *vrec;
        int *tdl, *fdl, *htl, nrec;
        if (read_v_record_dat(prev_v_record_file, &vrec, &tdl, &fdl, &htl, &nrec) == 0) {
            printf("Read %d velocity records\n", nrec);
            for (int i = 0; i < nrec; i++) {
                const int td = tdl[i], fd = fdl[i], ht = htl[i];
                if (td < 0 || td >= ftd || fd < 0 || fd >= ffd || ht < 0 || ht >= hd) continue;
                const long idx3 = (long)td * ffd * hd + (long)fd * hd + ht;
                if (count_num[idx3] < max_per_cell) {
                    const double *v = vrec + 3 * i;
                    speeds[idx3 * max_per_cell + count_num[idx3]] =
                        sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    count_num[idx3]++;
                }
            }
            free(vrec); free(tdl); free(fdl); free(htl);
        }
    }

    dsmc_ctx *ctx = NULL;
    if (report(NULL, dsmc_ctx_create(env_int("DSMC_DEVICE", 0), &ctx), "dsmc_ctx_create"))
        goto out_early;
    {
        printf("Building polynomial velocity fits...\n");
        double *coef = calloc((size_t)ncell * DSMC_CDF_STRIDE, sizeof(double));
        double *box = calloc((size_t)ncell * 4, sizeof(double));
        double *total = calloc((size_t)ncell, sizeof(double));
        int32_t *valid = calloc((size_t)ncell, sizeof(int32_t));
        uint64_t *den = calloc((size_t)ncell, sizeof(uint64_t));
        uint64_t *hor = calloc((size_t)ftd * ffd, sizeof(uint64_t));
        double *ttime = calloc((size_t)9 * (totaln > 0 ? totaln : 1), sizeof(double));
        if (coef && box && total && valid && den && hor && ttime &&
            report(ctx, dsmc_fit_cdf_samples_host(ctx, ncell, max_per_cell, speeds, count_num,
                                                  POLY_DEGREE, coef, box, total, valid),
                   "CDF fit") == DSMC_OK) {
            long nvalid = 0;
            for (long i = 0; i < ncell; i++) nvalid += valid[i] != 0;
            printf("Valid polynomial fits: %ld / %ld\n", nvalid, ncell);
            printf("Starting advanced DSMC: %d particles with collisions\n", totaln);
            dsmc_collision col;
            memset(&col, 0, sizeof col);
            col.n_bg = copy_atm;
            col.n_bg_len = copy_atm ? (int64_t)phd * pftd * pffd : 0;
            col.cdf_coef = coef;
            col.cdf_box = box;
            col.cdf_total = total;
            col.cdf_valid = valid;
            col.cdf_degree = POLY_DEGREE;
            dsmc_surface s;
            memset(&s, 0, sizeof s);
            s.T_map = T;
            dsmc_stats st;
            if (solve(ctx, &p, &s, &col, totaln, den, hor, ttime, &st) == DSMC_OK) {
                printf("Advanced DSMC complete. Escaped: %lld/%d, Total collisions: %lld\n",
                       (long long)st.n_escaped, totaln, (long long)st.n_collisions);
                write_grids(output_prefix, den, hor, ttime, 9, totaln, &p);
            }
        } else {
            fprintf(stderr, "out of host memory or fit failure\n");
        }
        free(coef); free(box); free(total); free(valid); free(den); free(hor); free(ttime);
    }
    dsmc_ctx_destroy(ctx);
out_early:
    free(count_num);
    free(speeds);
    free(copy_atm);
    free(T);
}
