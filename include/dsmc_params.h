/* dsmc_params.h - plain-C parameter block shared by every DSMC solve entry point.
 *
 * One struct carries everything a solve needs besides its arrays. It replaces the hard-coded
 * parameter fills of the reference runners (src/dsmc/ballistic.c:49-67,
 * src/dsmc/advanced.c:131-152) and the compile-time constants of include/constants.h:5-41, so
 * that the same kernels serve two physics models:
 *
 *   DSMC_MODEL_REFERENCE - the reference's own physics, quirks included: table-based launch
 *       speeds (src/common/velocity.c:6-68), launch angles uniform over a half-space
 *       (ballistic.c:161-170), escape by launch speed (ballistic.c:173), the T<100 K freeze scan
 *       (ballistic.c:132-153, advanced.c:278-309), polar deposit on landing (ballistic.c:252-256),
 *       first step of each hop not deposited (ballistic.c:208), 1e7-step cap per hop.
 *   DSMC_MODEL_CONFIG - flux-weighted Maxwell-Boltzmann launch with a cosine (Lambert)
 *       direction from an icosphere surface, night-side freeze-out and day-side re-emission,
 *       a life-time step cap, and isotropic elastic hard-sphere scattering.
 *
 * All fields are plain C types so the struct crosses the C ABI (ctypes, cgo, JNI) unchanged.
 */
#ifndef DSMC_PARAMS_H
#define DSMC_PARAMS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum dsmc_model  { DSMC_MODEL_REFERENCE = 0, DSMC_MODEL_CONFIG = 1 };
enum dsmc_runner { DSMC_RUNNER_BALLISTIC = 0, DSMC_RUNNER_ADVANCED = 1 };
enum dsmc_scatter { DSMC_SCATTER_REFERENCE = 0, DSMC_SCATTER_ISOTROPIC = 1 };

/* Fixed-point scale of every deposit: one unit of test-particle weight for one time step is
 * 2^24 counts in an unsigned 64-bit cell, so a cell holds 1.1e12 unit deposits before wrap. */
#define DSMC_FIXED_SHIFT 24
#define DSMC_FIXED_SCALE 16777216.0

/* Per-particle end states (the "fate" output). */
enum dsmc_fate {
    DSMC_FATE_ALIVE = 0,
    DSMC_FATE_PHOTOLYSED = 1,   /* weight fell below 0.01 at a hop boundary (ballistic.c:124) */
    DSMC_FATE_ESCAPED = 2,      /* launch speed >= ve (reference) or r >= max_height */
    DSMC_FATE_FROZEN = 3,       /* no warm column (reference) / night-side landing (config) */
    DSMC_FATE_STEP_CAP = 4      /* life-time step cap reached (config) */
};

typedef struct dsmc_params {
    int32_t model;          /* enum dsmc_model */
    int32_t runner;         /* enum dsmc_runner: selects the ballistic or the advanced variant */
    int32_t ftd, ffd, hd;   /* latitude rows, longitude columns, radial shells */
    int32_t use_exp_grid;   /* 0: uniform shells of unih; 1: exponential (grid.c:91-99) */

    double GM;              /* G*M, formed as the reference forms it (integrator.c:12) */
    double Radii;           /* body radius [m] */
    double ve;              /* escape speed used by the reference launch test [m/s] */
    double lifetime;        /* photodissociation lifetime [s] */
    double P;               /* rotation period [s] */
    double dt_step;         /* Verlet step h [s] */
    double dt_rot;          /* P / ffd [s] */
    double max_height;      /* escape radius [m] */
    double unih;            /* base shell thickness [m] */
    double alpha2;          /* exponential shell growth */
    double log1p_alpha2;    /* log(1 + alpha2), formed on the host */
    double wdecay;          /* exp(-h / lifetime), formed on the host */
    double alpha;           /* sticking mix of the reference launch (velocity.c:70-73) */
    double cross_section;   /* hard-sphere cross-section [m^2] */
    double kB_over_m;       /* k_B / m [J/K/kg]: config launch scale sigma = sqrt(kB_over_m * T) */
    double freeze_T;        /* reference freeze threshold, 100 K */
    double w_min;           /* weight at which a particle is dropped, 0.01 */
    double sun[3];          /* config model: unit vector to the sub-solar point */

    int64_t hop_step_cap;   /* steps per hop before the loop gives up (reference 1e7) */
    int64_t life_step_cap;  /* steps per particle life (config 20,000; 0 = none) */
    int32_t skip_first_deposit;  /* 1: the first step of each hop is not deposited */
    int32_t scatter;        /* enum dsmc_scatter */
    int32_t collide_ht_max; /* collisions only in shells ht < collide_ht_max (reference hd/3) */
    int32_t redraw_col_threshold; /* 1: draw a new collision threshold after each collision */

    uint64_t seed;          /* Philox key */
    uint32_t instance;      /* Philox counter word, distinguishes instances of one batch */
    int32_t n_speed_bins;   /* config phase-1 speed histogram bins per cell (0 = off) */
    double speed_bin_width; /* [m/s] */
    /* Per-hop energy-drift guard (FP64). E = |v|^2 / 2 - GM / |s| is taken at every launch and
     * after every collision, and again where the hop ends (landing, escape radius, hop or life
     * cap); a hop whose |E_end - E_start| exceeds drift_tol * GM / Radii is counted in
     * dsmc_stats.n_drift_flagged. The trajectory itself is not changed. 0 turns the guard off.
     * The reference's integrator (src/common/integrator.c:4-55: first-order velocity update)
     * drifts by about 1e-3 GM / R over a typical hop at its time steps; the presets use 1e-2. */
    double drift_tol;
} dsmc_params;

/* Surface description. The reference model reads a latitude-longitude temperature map
 * (fileio.c:47-62, indexed T[td*ffd+fd] at ballistic.c:129); the config model uses an icosphere
 * with one temperature per face. */
typedef struct dsmc_surface {
    const double *T_map;         /* reference model: [ftd][ffd] surface temperature [K] */
    int32_t nface;               /* config model: icosphere faces (1280 at 3 subdivisions) */
    int32_t nlevel;              /* subdivision levels of the icosphere (3) */
    const double *face_verts;    /* [nface][3][3] unit-sphere vertices, faces in subdivision order */
    const double *face_T;        /* [nface] face temperature [K] */
    const double *face_cdf;      /* [nface] cumulative launch weight ending at 1, or NULL: uniform */
    const double *base_centroid; /* [20][3] unit centroids of the 20 icosahedron faces */
    const double *split_planes;  /* [nnode][3][3] corner-cut plane normals of every parent face */
} dsmc_surface;

/* Largest polynomial degree of a collision-partner speed CDF, and the stride of one cell's
 * coefficient row. The reference fits degree 3 (include/types.h:89); its polyfit supports up to
 * degree 6 (src/common/polyfit.c:17-45). */
#define DSMC_CDF_MAX_DEGREE 6
#define DSMC_CDF_STRIDE 8

/* Collision inputs of the advanced runner: the phase-1 background and the per-cell partner
 * speed CDFs. CDF rows are in the reference's [td][fd][ht] order (advanced.c:41), which differs
 * from the [ht][td][fd] order of the density grid. */
typedef struct dsmc_collision {
    const double *n_bg;          /* background per cell, indexed ht*ftd*ffd + td*ffd + fd */
    int64_t n_bg_len;            /* entries of n_bg (the phase-1 grid may have more shells) */
    const double *cdf_coef;      /* [ncell][DSMC_CDF_STRIDE], highest power first, in t */
    const double *cdf_box;       /* [ncell][4]: min_v, max_v, xc, xs with t = (v - xc) / xs */
    const double *cdf_total;     /* [ncell]: sample count nn (reference) or 1 (normalised fits) */
    const int32_t *cdf_valid;    /* [ncell] */
    int32_t cdf_degree;
} dsmc_collision;

#ifdef __cplusplus
}
#endif
#endif /* DSMC_PARAMS_H */
