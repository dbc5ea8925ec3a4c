/* host_setup.c - parameter presets and surface construction (host only, no device needed). */
#include "dsmc_cuda.h"

#include <math.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Reference constants, include/constants.h:5-35 of the reference. */
#define REF_G        6.67e-11
#define REF_M_CERES  9.39e20
#define REF_R_CERES  476.2e3
#define REF_K_B      1.38e-23
#define REF_MOLE     6.02e23
#define REF_MMASS    18e-3
#define REF_P_CERES  (9.07417 * 3600.0)
#define REF_LIFETIME (1.0 / 1.02e-5 * (2.8 * 2.8))
#define REF_SIGMA_X  1e-19

static void common_reference(dsmc_params *p, int ftd, int ffd)
{
    memset(p, 0, sizeof(*p));
    p->model = DSMC_MODEL_REFERENCE;
    p->ftd = ftd;
    p->ffd = ffd;
    p->GM = REF_G * REF_M_CERES;
    p->Radii = REF_R_CERES;
    p->ve = sqrt(2.0 * REF_G * REF_M_CERES / REF_R_CERES);
    p->lifetime = REF_LIFETIME;
    p->P = REF_P_CERES;
    p->alpha = 0.5;
    p->dt_rot = p->P / ffd;
    p->kB_over_m = REF_K_B / (REF_MMASS / REF_MOLE);
    p->freeze_T = 100.0;
    p->w_min = 0.01;
    p->hop_step_cap = 10000000;
    p->life_step_cap = 0;
    p->drift_tol = 1e-2;
    p->scatter = DSMC_SCATTER_REFERENCE;
    p->seed = 20261203u;
}

int dsmc_params_reference(dsmc_params *p, int runner, int ftd, int ffd)
{
    if (!p || ftd < 4 || ffd < 2) return DSMC_ERR_INVALID;
    common_reference(p, ftd, ffd);
    p->runner = runner;
    if (runner == DSMC_RUNNER_BALLISTIC) {
        /* ballistic.c:60-67 */
        p->dt_step = 5.0;
        p->use_exp_grid = 0;
        p->unih = p->Radii * 0.1;
        p->alpha2 = 0.0;
        p->hd = 100;
        p->max_height = p->unih * p->hd + p->Radii;
        p->skip_first_deposit = 1;
        p->collide_ht_max = 0;
    } else if (runner == DSMC_RUNNER_ADVANCED) {
        /* advanced.c:142-152 */
        p->dt_step = 0.5;
        p->cross_section = REF_SIGMA_X;
        p->use_exp_grid = 1;
        p->hd = 50;
        p->max_height = 3e6 * sqrt(2.0);
        p->alpha2 = 0.04;
        p->unih = (p->max_height - p->Radii) / (pow(1.0 + p->alpha2, p->hd) - 1.0) * p->alpha2;
        p->skip_first_deposit = 1;
        p->collide_ht_max = p->hd / 3;   /* advanced.c:369 */
    } else {
        return DSMC_ERR_INVALID;
    }
    p->log1p_alpha2 = log(1.0 + p->alpha2);
    p->wdecay = exp(-p->dt_step / p->lifetime);   /* ballistic.c:204 */
    return DSMC_OK;
}

int dsmc_params_config(dsmc_params *p, int runner, double Radii, double GM, int hd,
                       uint64_t seed)
{
    if (!p || Radii <= 0.0 || GM <= 0.0 || hd < 1) return DSMC_ERR_INVALID;
    if (runner != DSMC_RUNNER_BALLISTIC && runner != DSMC_RUNNER_ADVANCED)
        return DSMC_ERR_INVALID;
    memset(p, 0, sizeof(*p));
    const double k_B = 1.380649e-23, m = 2.99e-26, d = 4.6e-10;
    p->model = DSMC_MODEL_CONFIG;
    p->runner = runner;
    p->ftd = 36;
    p->ffd = 72;
    p->hd = hd;
    p->use_exp_grid = 1;
    p->GM = GM;
    p->Radii = Radii;
    p->ve = sqrt(2.0 * GM / Radii);
    p->lifetime = 2.6e5;
    p->P = REF_P_CERES;
    p->dt_step = 2.0;
    p->dt_rot = p->P / p->ffd;
    p->max_height = 10.0 * Radii;
    p->alpha2 = 0.04;
    p->unih = (p->max_height - Radii) / (pow(1.0 + p->alpha2, hd) - 1.0) * p->alpha2;
    p->log1p_alpha2 = log(1.0 + p->alpha2);
    p->wdecay = exp(-p->dt_step / p->lifetime);
    p->alpha = 1.0;
    p->cross_section = M_PI * d * d;
    p->kB_over_m = k_B / m;
    p->freeze_T = 0.0;
    p->w_min = 0.01;
    p->sun[0] = 1.0;
    p->hop_step_cap = 20000;
    p->life_step_cap = 20000;
    p->skip_first_deposit = 0;
    p->scatter = DSMC_SCATTER_ISOTROPIC;
    p->collide_ht_max = hd;
    p->redraw_col_threshold = 1;
    p->seed = seed;
    p->n_speed_bins = 0;
    p->speed_bin_width = 25.0;
    p->drift_tol = 1e-2;
    return DSMC_OK;
}

/* ---------------------------------------------------------------------------------------- */
/* Icosphere. */

static void v_norm(double v[3])
{
    double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= l; v[1] /= l; v[2] /= l;
}

static void v_cross(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

static double v_dot(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

int dsmc_icosphere_nface(int nlevel)
{
    if (nlevel < 0 || nlevel > 6) return DSMC_ERR_INVALID;
    return 20 << (2 * nlevel);
}

int dsmc_icosphere_nnode(int nlevel)
{
    if (nlevel < 0 || nlevel > 6) return DSMC_ERR_INVALID;
    return 20 * ((1 << (2 * nlevel)) - 1) / 3;
}

static int node_offset(int level)
{
    return 20 * ((1 << (2 * level)) - 1) / 3;
}

/* Recursive subdivision of one triangle. Children are numbered 0: corner a, 1: corner b,
 * 2: corner c, 3: centre, and their vertices are the unit midpoints of the parent's edges. */
static void subdivide(const double a[3], const double b[3], const double c[3], int level,
                      int nlevel, int node, double *face_verts, double *split_planes)
{
    if (level == nlevel) {
        double *f = face_verts + 9 * node;
        memcpy(f, a, 3 * sizeof(double));
        memcpy(f + 3, b, 3 * sizeof(double));
        memcpy(f + 6, c, 3 * sizeof(double));
        return;
    }
    double ab[3], bc[3], ca[3];
    for (int k = 0; k < 3; k++) {
        ab[k] = 0.5 * (a[k] + b[k]);
        bc[k] = 0.5 * (b[k] + c[k]);
        ca[k] = 0.5 * (c[k] + a[k]);
    }
    v_norm(ab); v_norm(bc); v_norm(ca);
    if (split_planes) {
        double *pl = split_planes + 9 * (node_offset(level) + node);
        const double *corner[3] = {a, b, c};
        const double *e0[3] = {ab, bc, ca}, *e1[3] = {ca, ab, bc};
        for (int k = 0; k < 3; k++) {
            double n[3];
            v_cross(e0[k], e1[k], n);
            if (v_dot(n, corner[k]) < 0.0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
            memcpy(pl + 3 * k, n, 3 * sizeof(double));
        }
    }
    subdivide(a, ab, ca, level + 1, nlevel, node * 4 + 0, face_verts, split_planes);
    subdivide(b, bc, ab, level + 1, nlevel, node * 4 + 1, face_verts, split_planes);
    subdivide(c, ca, bc, level + 1, nlevel, node * 4 + 2, face_verts, split_planes);
    subdivide(ab, bc, ca, level + 1, nlevel, node * 4 + 3, face_verts, split_planes);
}

int dsmc_icosphere_build(int nlevel, double *face_verts, double *base_centroid,
                         double *split_planes)
{
    if (nlevel < 0 || nlevel > 6 || !face_verts) return DSMC_ERR_INVALID;
    /* The 12 icosahedron vertices are the cyclic permutations of (0, +-1, +-t), t the golden
     * ratio; its 20 faces are the vertex triples that are pairwise at the edge length 2. */
    const double t = (1.0 + sqrt(5.0)) / 2.0;
    double V[12][3];
    int nv = 0;
    for (int perm = 0; perm < 3; perm++)
        for (int s1 = -1; s1 <= 1; s1 += 2)
            for (int s2 = -1; s2 <= 1; s2 += 2) {
                double q[3] = {0.0, s1 * 1.0, s2 * t};
                V[nv][0] = q[(3 - perm) % 3];
                V[nv][1] = q[(4 - perm) % 3];
                V[nv][2] = q[(5 - perm) % 3];
                nv++;
            }
    int nf = 0;
    for (int i = 0; i < 12; i++)
        for (int j = i + 1; j < 12; j++)
            for (int k = j + 1; k < 12; k++) {
                double dij = 0, djk = 0, dki = 0;
                for (int x = 0; x < 3; x++) {
                    dij += (V[i][x] - V[j][x]) * (V[i][x] - V[j][x]);
                    djk += (V[j][x] - V[k][x]) * (V[j][x] - V[k][x]);
                    dki += (V[k][x] - V[i][x]) * (V[k][x] - V[i][x]);
                }
                if (fabs(dij - 4.0) > 1e-9 || fabs(djk - 4.0) > 1e-9 || fabs(dki - 4.0) > 1e-9)
                    continue;
                double a[3], b[3], c[3], e1[3], e2[3], n[3], s[3];
                memcpy(a, V[i], sizeof a); memcpy(b, V[j], sizeof b); memcpy(c, V[k], sizeof c);
                for (int x = 0; x < 3; x++) {
                    e1[x] = b[x] - a[x]; e2[x] = c[x] - a[x]; s[x] = a[x] + b[x] + c[x];
                }
                v_cross(e1, e2, n);
                if (v_dot(n, s) < 0.0) { double tmp[3]; memcpy(tmp, b, sizeof tmp);
                                         memcpy(b, c, sizeof tmp); memcpy(c, tmp, sizeof tmp); }
                v_norm(a); v_norm(b); v_norm(c);
                if (base_centroid) {
                    double *bc = base_centroid + 3 * nf;
                    for (int x = 0; x < 3; x++) bc[x] = a[x] + b[x] + c[x];
                    v_norm(bc);
                }
                subdivide(a, b, c, 0, nlevel, nf, face_verts, split_planes);
                nf++;
            }
    return nf == 20 ? DSMC_OK : DSMC_ERR_INVALID;
}

int dsmc_icosphere_locate(int nlevel, const double *base_centroid, const double *split_planes,
                          const double p[3])
{
    int node = 0;
    double best = -2.0;
    for (int f = 0; f < 20; f++) {
        double d = v_dot(base_centroid + 3 * f, p);
        if (d > best) { best = d; node = f; }
    }
    for (int level = 0; level < nlevel; level++) {
        const double *pl = split_planes + 9 * (node_offset(level) + node);
        int child = v_dot(pl, p) > 0.0 ? 0 : v_dot(pl + 3, p) > 0.0 ? 1
                  : v_dot(pl + 6, p) > 0.0 ? 2 : 3;
        node = node * 4 + child;
    }
    return node;
}

int dsmc_face_temperature(int nface, const double *face_verts, const double sun[3],
                          double T_ss, double T_floor, double *face_T)
{
    if (nface <= 0 || !face_verts || !sun || !face_T) return DSMC_ERR_INVALID;
    for (int f = 0; f < nface; f++) {
        const double *a = face_verts + 9 * f;
        double c[3] = {a[0] + a[3] + a[6], a[1] + a[4] + a[7], a[2] + a[5] + a[8]};
        v_norm(c);
        double cz = v_dot(c, sun);
        double T = cz > 0.0 ? T_ss * pow(cz, 0.25) : 0.0;
        face_T[f] = T > T_floor ? T : T_floor;
    }
    return DSMC_OK;
}

int dsmc_latlon_temperature(int ftd, int ffd, const double sun[3], double T_ss,
                            double T_floor, double *T_map)
{
    if (ftd <= 0 || ffd <= 0 || !sun || !T_map) return DSMC_ERR_INVALID;
    for (int td = 0; td < ftd; td++) {
        double th = (td + 0.5) / ftd * M_PI - M_PI / 2.0;
        for (int fd = 0; fd < ffd; fd++) {
            double fi = (fd + 0.5) / ffd * 2.0 * M_PI;
            /* position direction in the reference's convention: (cos th sin fi, cos th cos fi,
             * sin th), ballistic.c:114-118 */
            double n[3] = {cos(th) * sin(fi), cos(th) * cos(fi), sin(th)};
            double cz = v_dot(n, sun);
            double T = cz > 0.0 ? T_ss * pow(cz, 0.25) : 0.0;
            T_map[td * ffd + fd] = T > T_floor ? T : T_floor;
        }
    }
    return DSMC_OK;
}

double dsmc_sublimation_flux(double T, double mmass_kg)
{
    /* H2O vapour pressure (Torr) log10 form and the Torr->Pa factor as in
     * src/thermal/thermal_model.c:33-38 and :50-55 of the reference. */
    const double c0 = -2445.5646, c1 = -6.757169, c2 = -0.01677006, c3 = 1.20514e-5,
                 c4 = 8.2312, torr = 133.32237, k_B = 1.380649e-23;
    double log10_p = c0 / T + c1 + c2 * T + c3 * T * T + c4 * log10(T);
    double p = torr * pow(10.0, log10_p);
    return p / sqrt(2.0 * M_PI * mmass_kg * k_B * T);
}

int dsmc_source_cdf(int nface, const double *face_verts, const double *face_T, double mmass_kg,
                    double *face_cdf, double *rate_per_R2)
{
    if (nface <= 0 || !face_verts || !face_T || !face_cdf) return DSMC_ERR_INVALID;
    double acc = 0.0;
    for (int f = 0; f < nface; f++) {
        const double *a = face_verts + 9 * f, *b = a + 3, *c = a + 6;
        double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        double n[3];
        v_cross(e1, e2, n);
        double area = 0.5 * sqrt(v_dot(n, n));
        acc += area * dsmc_sublimation_flux(face_T[f], mmass_kg);
        face_cdf[f] = acc;
    }
    if (!(acc > 0.0)) return DSMC_ERR_INVALID;
    for (int f = 0; f < nface; f++) face_cdf[f] /= acc;
    face_cdf[nface - 1] = 1.0;
    if (rate_per_R2) *rate_per_R2 = acc;
    return DSMC_OK;
}
