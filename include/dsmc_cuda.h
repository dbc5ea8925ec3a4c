/* dsmc_cuda.h - the C ABI between the DSMC host code and the sm_100a kernels.
 *
 * The reference runs its particle loops inside run_ballistic (src/dsmc/ballistic.c:35-36) and
 * run_advanced (src/dsmc/advanced.c:119-121), declared only as `extern` in src/main.c:18-23, with
 * OpenMP threads over particles. This header is the seam that replaces those loops: the drop-in
 * runners (same signatures, include/dsmc_runners.h) and the CLI call these functions, and every
 * one is plain C: pointers, sizes and status codes, no exceptions and no C++ or torch types.
 *
 * Conventions
 *   - Every function returns int status: DSMC_OK (0) or a negative dsmc_status.
 *   - A context owns one device, one stream and the device buffers of one problem. A context is
 *     not thread-safe; use one per host thread. Several contexts may share a device.
 *   - Functions named *_host take host pointers and copy inside the call. Functions without that
 *     suffix work on device-resident state and are asynchronous on the context stream.
 *   - There is no CPU fallback: without a usable CUDA device, dsmc_ctx_create fails with
 *     DSMC_ERR_NO_DEVICE.
 */
#ifndef DSMC_CUDA_H
#define DSMC_CUDA_H

#include <stddef.h>
#include <stdint.h>
#include "dsmc_params.h"
#include "thermal.h"

#ifdef __cplusplus
extern "C" {
#endif

enum dsmc_status {
    DSMC_OK = 0,
    DSMC_ERR_INVALID = -1,      /* bad argument or inconsistent sizes */
    DSMC_ERR_CUDA = -2,         /* a CUDA runtime call failed (see dsmc_last_error) */
    DSMC_ERR_NO_DEVICE = -3,    /* no CUDA device, or the device index is out of range */
    DSMC_ERR_NO_MEMORY = -4,    /* device or pinned host allocation failed */
    DSMC_ERR_STATE = -5,        /* call out of order (e.g. run before setup) */
    DSMC_ERR_BUDGET = -6,       /* admission refused: the request exceeds the memory budget */
    DSMC_ERR_IO = -7            /* file could not be read or written */
};

/* ---------------------------------------------------------------------------------------- */
/* Host-side set-up helpers (no device needed).                                              */

/* Reference-model parameters exactly as the reference runners fill them:
 * runner DSMC_RUNNER_BALLISTIC -> src/dsmc/ballistic.c:49-67 (100 uniform shells, dt 5 s);
 * runner DSMC_RUNNER_ADVANCED  -> src/dsmc/advanced.c:131-152 (50 exponential shells, dt 0.5 s).
 * ftd/ffd come from the temperature file. */
int dsmc_params_reference(dsmc_params *p, int runner, int ftd, int ffd);

/* Config-model parameters: body radius [m], GM [m^3/s^2], shells hd (exponential, to 10 R),
 * 36 x 72 angular grid, dt 2 s, 20,000-step life cap, photolysis lifetime 2.6e5 s, H2O
 * m = 2.99e-26 kg, sun on +x (sub-solar longitude pi/2). */
int dsmc_params_config(dsmc_params *p, int runner, double Radii, double GM, int hd,
                       uint64_t seed);

/* Icosphere of 20 * 4^nlevel faces (1280 at nlevel 3, 642 vertices), built by midpoint
 * subdivision of the icosahedron with faces kept in subdivision order (face index =
 * base * 4^nlevel + child path). Fills face_verts [nface][3][3], base_centroid [20][3] and
 * split_planes [20 * (4^nlevel - 1) / 3][3][3] (corner-cut planes used to locate a point). */
int dsmc_icosphere_nface(int nlevel);
int dsmc_icosphere_nnode(int nlevel);
int dsmc_icosphere_build(int nlevel, double *face_verts, double *base_centroid,
                         double *split_planes);
/* Face containing unit direction p, by descending the subdivision tree. */
int dsmc_icosphere_locate(int nlevel, const double *base_centroid, const double *split_planes,
                          const double p[3]);

/* Synthetic temperature field T = max(T_floor, T_ss * cos(z)^(1/4)), z the solar zenith:
 * per face at the face centroid, or per latitude-longitude cell centre. */
int dsmc_face_temperature(int nface, const double *face_verts, const double sun[3],
                          double T_ss, double T_floor, double *face_T);
int dsmc_latlon_temperature(int ftd, int ffd, const double sun[3], double T_ss,
                            double T_floor, double *T_map);

/* Antoine sublimation flux of H2O [molecules m^-2 s^-1] at T (vapour pressure of
 * src/thermal/thermal_model.c:50-55 with the constants of :33-38, divided by sqrt(2 pi m k T)). */
double dsmc_sublimation_flux(double T, double mmass_kg);

/* Launch-face CDF weighted by face area x sublimation flux. Returns the total production rate
 * for a unit-radius body [molecules/s per m^2 of R^2] in *rate_per_R2. */
int dsmc_source_cdf(int nface, const double *face_verts, const double *face_T, double mmass_kg,
                    double *face_cdf, double *rate_per_R2);

/* ---------------------------------------------------------------------------------------- */
/* Device contexts.                                                                          */

typedef struct dsmc_ctx dsmc_ctx;

/* Solve paths. PLAIN_FP64 is the straight port: one thread per particle for its whole life,
 * the reference's FP64 arithmetic without FMA contraction, one atomic per deposited step.
 * FAST_FP32 keeps resident particle slots that refill from a work queue, pushes in FP32 with
 * two-sum compensated positions and velocities, tracks cells by comparisons, and aggregates
 * deposits in registers. FAST_FP64 is the same resident-slot engine on FP64 state and FP64
 * boundary tables (no compensation needed), with the plain path's FP64 maps of the random words
 * at launches and collisions: it follows the same Philox streams as PLAIN_FP64 and differs from
 * it only by rounding, so it serves as the full-size FP64 reference of FAST_FP32. FAST_FP64
 * runs 128-thread blocks, 4 (default) or 3 resident per SM. */
enum dsmc_path { DSMC_PATH_PLAIN_FP64 = 0, DSMC_PATH_FAST_FP32 = 1, DSMC_PATH_FAST_FP64 = 2 };

typedef struct dsmc_stats {
    int64_t total_steps;      /* Verlet steps executed */
    int64_t n_escaped;
    int64_t n_collisions;
    int64_t n_bound_launch;   /* config model: launches with negative energy */
    int64_t n_finished;       /* particles whose life ended */
    int64_t n_drift_flagged;  /* trajectories whose energy drift exceeded the guard */
} dsmc_stats;

const char *dsmc_status_string(int status);
/* Text of the last error on this context (or of the last failed dsmc_ctx_create). */
const char *dsmc_last_error(const dsmc_ctx *ctx);

int dsmc_ctx_create(int device, dsmc_ctx **out);
int dsmc_ctx_destroy(dsmc_ctx *ctx);
/* Run on the caller's stream (a cudaStream_t passed as void*), or NULL for the context's own. */
int dsmc_ctx_set_stream(dsmc_ctx *ctx, void *stream);

/* Upload one problem: parameters, surface and (advanced runner) collision tables. Allocates the
 * density [hd][ftd][ffd] and horizon [ftd][ffd] fixed-point grids and zeroes them. */
int dsmc_setup(dsmc_ctx *ctx, const dsmc_params *p, const dsmc_surface *surf,
               const dsmc_collision *col);
/* Allocate per-particle outputs for up to n particles (ttime rows, fate, steps); 0 frees them. */
int dsmc_enable_particle_outputs(dsmc_ctx *ctx, int64_t n);
/* Zero grids, per-particle outputs and statistics. */
int dsmc_zero(dsmc_ctx *ctx);
/* Solve particles [pid_begin, pid_begin + n) on the device, adding into the grids. Async. */
int dsmc_run(dsmc_ctx *ctx, int path, int64_t pid_begin, int64_t n);
int dsmc_sync(dsmc_ctx *ctx);

/* Launch shape of the FAST paths: threads per block, resident blocks per SM (0 = as many as
 * fit), Verlet steps per slot per launch, and launches per captured CUDA graph (1 = no graph).
 * Results do not depend on the shape: every particle's trajectory is a function of its id and
 * the deposits are integer sums. */
int dsmc_set_launch_shape(dsmc_ctx *ctx, int block, int blocks_per_sm, int steps_per_launch,
                          int launches_per_graph);
/* Kernel launches issued by the last dsmc_run and the resident slot count of the FAST paths. */
int dsmc_get_launch_info(dsmc_ctx *ctx, int64_t *launches, int64_t *nslots);

/* Measured FMA throughput of this device [TFLOP/s] for FP32 (fp64 = 0) or FP64 (fp64 = 1):
 * 8 independent FMA chains per thread over a few full waves, timed with CUDA events. The
 * denominator of the push kernels' roofline fraction. */
int dsmc_measure_fma_peak(dsmc_ctx *ctx, int fp64, double *tflops);

/* Results (synchronous copies to host memory). */
int dsmc_get_density(dsmc_ctx *ctx, uint64_t *density_fx);
int dsmc_get_horizon(dsmc_ctx *ctx, uint64_t *horizon_fx);
int dsmc_get_stats(dsmc_ctx *ctx, dsmc_stats *out);
/* Per-cell speed histogram [hd*ftd*ffd][n_speed_bins] (when params.n_speed_bins > 0). */
int dsmc_get_speed_hist(dsmc_ctx *ctx, uint64_t *hist);
/* ttime [9][n], fate [n], steps [n] for the particles of the last runs, indexed pid - pid_begin
 * of the run that produced them. Any pointer may be NULL. */
int dsmc_get_particle_outputs(dsmc_ctx *ctx, int64_t n, double *ttime, int32_t *fate,
                              int64_t *steps);
/* Device-to-device copy of the fixed-point grids into caller buffers on the same device
 * (asynchronous on the context stream), e.g. into communication buffers for a reduction across
 * GPUs. Either destination may be NULL. */
int dsmc_copy_grids_device(dsmc_ctx *ctx, uint64_t *density_dst, uint64_t *horizon_dst);
/* Device address of the fixed-point density grid and its length in cells, for collectives. */
int dsmc_density_device(dsmc_ctx *ctx, uint64_t **dev_ptr, int64_t *ncell);
int dsmc_horizon_device(dsmc_ctx *ctx, uint64_t **dev_ptr, int64_t *ncell);

/* FP64 fits of per-cell collision-partner speed CDFs, computed on the device; host buffers in
 * and out. From speed samples (the reference's build_poly_fits, src/dsmc/advanced.c:32-117):
 * speeds [ncell][max_per_cell] with counts [ncell] (max_per_cell <= 64). From speed histograms
 * (config model): hist [ncell][nbins] of width bin_width. Outputs coef [ncell][DSMC_CDF_STRIDE],
 * box [ncell][4], total [ncell] and valid [ncell], ready for a dsmc_collision. */
int dsmc_fit_cdf_samples_host(dsmc_ctx *ctx, int64_t ncell, int max_per_cell,
                              const double *speeds, const int32_t *counts, int degree,
                              double *coef, double *box, double *total, int32_t *valid);
int dsmc_fit_cdf_hist_host(dsmc_ctx *ctx, int64_t ncell, int nbins, double bin_width,
                           const uint64_t *hist, int degree, double *coef, double *box,
                           double *total, int32_t *valid);

/* Fed-state push: integrate n particles from the given positions and velocities (host arrays
 * [n][3], updated in place) with the reference's Verlet variant (verlet_step,
 * src/common/integrator.c:4-55) and the context's GM, dt, Radii and max_height, for up to nsteps
 * steps each, starting from oa = GM s / r^3 (src/dsmc/ballistic.c:176-181). A particle stops at
 * landing (status 1) or escape (status 2); status 0 means it ran all nsteps. steps_taken may be
 * NULL. PLAIN_FP64 (and FAST_FP64) use the FP64 arithmetic of the plain kernel; FAST_FP32 uses
 * the compensated FP32 push of the fast path. */
int dsmc_push_host(dsmc_ctx *ctx, int path, int64_t n, int nsteps, double *pos, double *vel,
                   int32_t *status, int32_t *steps_taken);

/* Velocity record of the ballistic runner (src/dsmc/ballistic.c:216-232): for each
 * (latitude row, shell) bucket, the first per_bucket visits in (particle id, step) order, i.e.
 * the records the reference keeps in a one-thread run, at most total_cap records in that order.
 * Replays particles [0, n) of the problem set up on ctx in chunks (count pass, per-bucket scan,
 * record pass) and stops once every bucket or the total is full. The grids are not touched.
 * v_out [total_cap][3], td/fd/ht [total_cap]; *n_out receives the count. */
int dsmc_velocity_record(dsmc_ctx *ctx, int64_t n, int per_bucket, int64_t total_cap,
                         double *v_out, int32_t *td, int32_t *fd, int32_t *ht, int64_t *n_out);

/* Host-buffer solve: set-up, n particles from pid 0, results copied back into host buffers.
 * This is the one call a plugin makes; density_fx [hd*ftd*ffd] and horizon_fx [ftd*ffd] may be
 * NULL. */
int dsmc_solve_host(dsmc_ctx *ctx, int path, const dsmc_params *p, const dsmc_surface *surf,
                    const dsmc_collision *col, int64_t n, uint64_t *density_fx,
                    uint64_t *horizon_fx, dsmc_stats *stats);

/* ---------------------------------------------------------------------------------------- */
/* FP64 number density (host, no device needed).                                             */
/* The reference writes raw weight sums (src/dsmc/ballistic.c:235-236) and never divides by the */
/* volumes that src/common/grid.c:41-84 computes. These turn the fixed-point grid of a solve    */
/* into molecules per m^3: n test particles stand for production_rate molecules/s, one         */
/* deposited weight-step is dt_step seconds of residence, so                                  */
/*     nden[c] = density_fx[c] / 2^24 * production_rate / n * dt_step / volume[c]             */
/* in FP64. DSMC_VOLUME_PHYSICAL: spherical-shell cells (r_o^3 - r^3) / 3 * dphi *            */
/* |sin b_o - sin b|; DSMC_VOLUME_REFERENCE: the reference's grid_compute_volume_uniform /     */
/* _exp (grid.c:41-84, which adds the two cubes). Arrays [hd][ftd][ffd].                      */
enum dsmc_volume { DSMC_VOLUME_PHYSICAL = 0, DSMC_VOLUME_REFERENCE = 1 };
int dsmc_cell_volumes(const dsmc_params *p, int volume_mode, double *volume);
int dsmc_number_density_host(const dsmc_params *p, const uint64_t *density_fx, int64_t n,
                             double production_rate, int volume_mode, double *nden);

/* ---------------------------------------------------------------------------------------- */
/* FAST_FP32 solve without any device allocation.                                            */
/* (This entry point has no counterpart in the reference.)                                   */
/*                                                                                           */
/* For callers that cannot call cudaMalloc - code whose host framework owns all device       */
/* memory through its own pool, or a plugin whose process intercepts or budgets allocation   */
/* calls - but can pass device buffers they already hold. Solves the ballistic runner for    */
/* particles [pid_begin, pid_begin + n) on the current device, like dsmc_run with            */
/* DSMC_PATH_FAST_FP32, and returns when the solve is done.                                  */
/*   surf     the surface with DEVICE pointers (T_map for the reference model; face_verts,   */
/*            face_T, face_cdf (may be NULL), base_centroid, split_planes for the config     */
/*            model), in the layouts of dsmc_surface.                                        */
/*   density  device [hd*ftd*ffd] and horizon device [ftd*ffd] fixed-point grids: the solve  */
/*            ADDS into them, so zero them first for a fresh result.                         */
/*   stats    device [6] unsigned 64-bit counters in dsmc_stats order; zeroed by the call.   */
/*   stream   a cudaStream_t, or NULL for the legacy default stream.                         */
/* Scratch: one fixed device array of about 10.0 MB inside the library (at most 32,768      */
/* resident particle slots and (hd+1) + (ftd+1) + 2 (ffd+1) + 1 <= 4096 table floats, ftd  */
/* and ffd <= 255). Every GPU that loads the library holds that array until the process     */
/* exits. Larger grids are rejected with DSMC_ERR_INVALID. The first call on a device looks  */
/* up the array's device address (cudaGetSymbolAddress); make that first call before any     */
/* stream capture. Every call shares the array and it keeps the last call's contents (the   */
/* call resets what must start at zero). Calls whose GPU work overlapped would race on the  */
/* array; the library prevents that within a process: calls are serialised by a lock and    */
/* each returns only after its GPU work has finished (the host reads the work-queue counters */
/* after every launch). dsmc_noalloc_last_error() describes the last failure. */
int dsmc_solve_fast_noalloc(const dsmc_params *p, const dsmc_surface *surf, int64_t pid_begin,
                            int64_t n, uint64_t *density, uint64_t *horizon, uint64_t *stats,
                            void *stream);
const char *dsmc_noalloc_last_error(void);

/* ---- Thermal model -------------------------------------------------------------------------- */
/* Replaces the column loop of thermal_solve (src/thermal/thermal_model.c:105-283): the 1-D heat  */
/* equation of every surface cell, n_substep implicit steps of one rotation step each, with the  */
/* surface temperature from the energy balance (solar flux, conduction, thermal emission, H2O    */
/* sublimation) by bisection and a zero-flux bottom. One GPU thread per (td, fd) column, FP64.   */
/* flux [ftd][ffd] absorbed flux [W/m^2], or NULL for the reference's analytic flux; writes the  */
/* surface temperature T_surface [ftd][ffd] and, when h_depth is not NULL, the depth points.     */
int dsmc_thermal_solve_host(dsmc_ctx *ctx, int ftd, int ffd, const ThermalParams *tp,
                            const double *flux, double *T_surface, int *h_depth);

/* Device time [ms] of the kernel of the last dsmc_thermal_solve_host / dsmc_shadow_flux_host
 * call on this context (CUDA events around the launch; host set-up and copies excluded). */
int dsmc_last_kernel_ms(const dsmc_ctx *ctx, double *ms);

/* ---- Shadow flux ------------------------------------------------------------------------------ */
/* Replaces the Embree loop of the reference's ray tracer (src/raytracer/shadow_maker.c:198-238):  */
/* for rotation phase t in [0, tt) and face f, F[f][t] = (1 - shadowed / nmonte) (s . n_f), 0 when  */
/* s . n_f < 0, with s the sun direction at declination -za [rad] and the shadow rays from nmonte  */
/* rand_r points of the face (seed t * nface + f + 42) lifted 1e-3 along n_f. spot [npoint][3]     */
/* vertices, facet [nface][3] 0-based vertex indices, face_normal [nface][3] outward unit normals   */
/* (mesh_compute_normals). The mesh's BVH is built on the host; the rays are traced on the GPU.   */
int dsmc_shadow_flux_host(dsmc_ctx *ctx, int npoint, const double *spot, int nface,
                          const int32_t *facet, const double *face_normal, double za, int tt,
                          int nmonte, double *F);

/* ---- Batched and served solves ------------------------------------------------------------- */
/* No counterpart in the reference, whose runners solve one problem per call                   */
/* (src/dsmc/ballistic.c:38, src/dsmc/advanced.c:132). A server owns one GPU: a fixed set of     */
/* resident particle slots (FAST_FP32 engine), one device work queue and a memory budget.       */
/* Each request is a whole problem (params, surface, optional collision tables, n particles     */
/* with ids [0, n)); at the next poll its particles join the queue behind the ones already      */
/* queued, and slots freed by ended particles take them while earlier requests are still        */
/* running. The requests admitted between two polls join grouped by estimated hop length,       */
/* longest first (ties in admission order), which keeps warps on one kind of trajectory. A      */
/* batch is a set of requests submitted before the first poll. Results of a request are         */
/* bit-identical whatever else shares the queue, in whatever order, and whatever the launch     */
/* shape. Not thread-safe: one host thread drives a server; several servers may coexist.        */
typedef struct dsmc_server dsmc_server;

typedef struct dsmc_server_info {
    int64_t submitted, completed, fetched, rejected;  /* requests */
    int64_t active;             /* submitted and not yet complete */
    int64_t bytes_in_use;       /* device bytes held: engine + unfetched requests */
    int64_t bytes_budget;
    int64_t slots;              /* resident particle slots */
    int64_t rounds, launches;   /* rounds (graph replays) and kernel launches issued */
    int64_t total_steps;        /* particle steps of completed requests */
    double busy_ms;             /* device time of the rounds (CUDA events) */
} dsmc_server_info;

typedef struct dsmc_request_info {
    int64_t n;                  /* particles */
    int64_t ncell, nhcell;      /* density and horizon grid sizes */
    double t_submit, t_done;    /* server clock [s] (dsmc_server_now) at admission and at the */
                                /* poll that saw the last particle end */
} dsmc_request_info;

/* hbm_budget: device bytes the server may hold (engine slots and tables plus every admitted,  */
/* unfetched request); max_requests: requests the queue can hold before it must drain (it     */
/* restarts from empty whenever no request is active). */
int dsmc_server_create(int device, int64_t hbm_budget, int max_requests, dsmc_server **out);
int dsmc_server_destroy(dsmc_server *srv);
const char *dsmc_server_last_error(const dsmc_server *srv);
/* Launch shape of the engine (see dsmc_set_launch_shape); only while no request is active. */
int dsmc_server_set_shape(dsmc_server *srv, int block, int blocks_per_sm, int steps_per_launch,
                          int launches_per_graph);
/* Admit one request: its tables are uploaded now, its particles queued by the next poll.      */
/* DSMC_ERR_BUDGET (nothing allocated) when it does not fit the budget or the queue is full;    */
/* retry after fetching results. On success *ticket names the request.                          */
int dsmc_server_submit(dsmc_server *srv, const dsmc_params *p, const dsmc_surface *surf,
                       const dsmc_collision *col, int64_t n, int64_t *ticket);
/* Advance the queue: queues the requests admitted since the last call, keeps up to two rounds */
/* in flight and waits for the oldest. Writes the tickets that completed in this call to       */
/* done[0..*ndone) (at most cap; the rest are reported by later calls). Returns at once with   */
/* *ndone = 0 when nothing is active or pending. */
int dsmc_server_poll(dsmc_server *srv, int64_t *done, int cap, int *ndone);
/* Copy a completed request's results to host memory (any pointer may be NULL) and free its   */
/* device memory. DSMC_ERR_STATE while the request is still running. */
int dsmc_server_fetch(dsmc_server *srv, int64_t ticket, uint64_t *density, uint64_t *horizon,
                      dsmc_stats *stats, dsmc_request_info *info);
int dsmc_server_info_get(const dsmc_server *srv, dsmc_server_info *info);
/* Seconds since the server was created, on the clock of dsmc_request_info. */
double dsmc_server_now(const dsmc_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* DSMC_CUDA_H */
