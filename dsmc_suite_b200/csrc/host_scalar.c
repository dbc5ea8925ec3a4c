/* host_scalar.c - the reference's scalar C entry points, kept with their signatures.
 *
 * integrator.h, velocity.h, collision.h, grid.h and polyfit.h of the reference declare
 * per-particle C functions that the runners call. They stay available here for code linked
 * against the reference: single-particle host arithmetic, written with the reference's operation
 * order so results are bit-identical to the reference's src/common/ files when compiled without FMA
 * contraction (the library builds with -ffp-contract=off). The GPU kernels do not call these; they run the
 * same arithmetic on the device.
 */
#include "types.h"
#include "integrator.h"
#include "velocity.h"
#include "collision.h"
#include "grid.h"
#include "polyfit.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Reference: src/common/integrator.c:4-55. */
VerletStatus verlet_step(Particle *p, const PhysicsParams *params, double h, Vec3 *oa,
                         double *ds_out)
{
    const double GM = params->G * params->M;
    const double r = vec3_len(p->pos);
    const double g = GM / (r * r * r);
    const double h2 = h * h;
    const double c1 = 1.5 * h2, c2 = h2 / 6.0;
    Vec3 s = p->pos;
    Vec3 n;
    n.x = s.x + p->vel.x * h - g * s.x * c1 - oa->x * c2;
    n.y = s.y + p->vel.y * h - g * s.y * c1 - oa->y * c2;
    n.z = s.z + p->vel.z * h - g * s.z * c1 - oa->z * c2;
    if (ds_out) {
        Vec3 d = vec3_sub(n, s);
        *ds_out = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    }
    p->vel.x -= g * s.x * h;
    p->vel.y -= g * s.y * h;
    p->vel.z -= g * s.z * h;
    oa->x = g * s.x;
    oa->y = g * s.y;
    oa->z = g * s.z;
    p->pos = n;
    const double rn = vec3_len(n);
    if (rn <= params->Radii) return VERLET_LANDED;
    if (rn >= params->max_height) return VERLET_ESCAPED;
    return VERLET_OK;
}

/* Reference: src/common/velocity.c:6-47. Speeds 0..1000 m/s in steps of 10 are repeated
 * floor(5e5 * 4 pi v^2 (m / 2 pi k T)^1.5 exp(-3 m v^2 / 2 k T)) times, at most 1000 entries. */
void velocity_table_init(VelocityTable *vt, double mmass, double mole, double k_B)
{
    const double dT = (240.0 - 20.0) / (VEL_TABLE_NTEMP - 1);
    const double m = mmass / mole;
    for (int i = 0; i < VEL_TABLE_NTEMP; i++) {
        const double T = 20.0 + i * dT;
        vt->temps[i] = T;
        int fill = 0;
        for (int j = 0; j <= 100 && fill < VEL_TABLE_NVEL; j++) {
            const double vv = j * 10.0;
            const double factor = 1.0 / (2.0 * M_PI) * m / (k_B * T);
            double aa = 4.0 * M_PI * vv * vv * pow(factor, 1.5) *
                        exp(-m * 3.0 * vv * vv / (2.0 * k_B * T));
            aa *= 5e5;
            const int reps = (int)floor(aa);
            for (int k = 0; k < reps && fill < VEL_TABLE_NVEL; k++) vt->speeds[i][fill++] = vv;
        }
        vt->count[i] = fill > 0 ? fill : 1;
    }
}

/* Reference: src/common/velocity.c:49-68. */
double velocity_sample(const VelocityTable *vt, double T_local, unsigned int *seed)
{
    int row = T_local >= 220.0 ? 20 : (int)ceil(T_local / 10.0) - 2;
    if (row < 0) row = 0;
    if (row >= VEL_TABLE_NTEMP) row = VEL_TABLE_NTEMP - 1;
    return vt->speeds[row][rand_r(seed) % vt->count[row]];
}

/* Reference: src/common/velocity.c:70-73. */
double velocity_sticking(double vr, double v_old_sq, double alpha)
{
    return sqrt(alpha * vr * vr + (1.0 - alpha) * v_old_sq);
}

/* Reference: src/common/collision.c:4-13. */
int collision_check(double *real_col_p, double col_threshold, double ds, double local_density,
                    double cross_section)
{
    *real_col_p += ds * local_density * cross_section;
    return col_threshold < 1.0 - exp(-(*real_col_p));
}

/* Reference: src/common/collision.c:15-41 (its documented v <- (v + v2) + 0.5 (v - v2)). */
void collision_execute(Vec3 *v, Vec3 v2)
{
    const Vec3 d = vec3_sub(*v, v2), c = vec3_add(*v, v2);
    v->x = c.x + 0.5 * d.x;
    v->y = c.y + 0.5 * d.y;
    v->z = c.z + 0.5 * d.z;
}

static double horner0(const double *c, int degree, double x)
{
    double r = 0.0;
    for (int i = 0; i <= degree; i++) r = r * x + c[i];
    return r;
}

/* Reference: src/common/collision.c:43-101. */
double collision_sample_speed(const PolyFit *pf, double rand_val, int nn)
{
    if (!pf->valid) return 0.0;
    const double top = horner0(pf->coeffs, POLY_DEGREE, pf->max_v);
    const double target = rand_val * ((double)nn - top) + top;
    double lo = pf->min_v, hi = pf->max_v;
    for (int it = 0; it < 100; it++) {
        const double mid = (lo + hi) * 0.5;
        const double fm = horner0(pf->coeffs, POLY_DEGREE, mid) - target;
        const double fh = horner0(pf->coeffs, POLY_DEGREE, hi) - target;
        if (fm * fh < 0) lo = mid;
        else hi = mid;
        if (fabs(hi - lo) < 0.01) break;
    }
    return (lo + hi) * 0.5;
}

/* Reference: src/common/grid.c:7-26 (callee allocates, grid_free releases). */
SphericalGrid *grid_create(int ftd, int ffd, int hd)
{
    SphericalGrid *g = calloc(1, sizeof(*g));
    if (!g) return NULL;
    g->ftd = ftd;
    g->ffd = ffd;
    g->hd = hd;
    const size_t n3 = (size_t)hd * ftd * ffd, n2 = (size_t)ftd * ffd;
    g->density = calloc(n3, sizeof(double));
    g->temperature = calloc(n2, sizeof(double));
    g->volume = calloc(n3, sizeof(double));
    g->horizon = calloc(n2, sizeof(double));
    if (!g->density || !g->temperature || !g->volume || !g->horizon) {
        grid_free(g);
        return NULL;
    }
    return g;
}

void grid_free(SphericalGrid *g)
{
    if (!g) return;
    free(g->density);
    free(g->temperature);
    free(g->volume);
    free(g->horizon);
    free(g);
}

/* Reference: src/common/grid.c:28-39; cell k covers (k, k+1] in units of the cell width. */
void grid_spherical_to_index(double thi, double fi, int ftd, int ffd, int *td, int *fd)
{
    int a = (int)ceil((thi + M_PI / 2.0) / M_PI * ftd) - 1;
    int b = (int)ceil(fi / (2.0 * M_PI) * ffd) - 1;
    *td = a < 0 ? 0 : (a >= ftd ? ftd - 1 : a);
    *fd = b < 0 ? 0 : (b >= ffd ? ffd - 1 : b);
}

/* Reference: src/common/grid.c:41-63. */
void grid_compute_volume_uniform(SphericalGrid *g, double Radii, double unih)
{
    const double dfi = 2.0 * M_PI / g->ffd;
    double r_in = Radii;
    for (int ht = 0; ht < g->hd; ht++) {
        const double r_out = r_in + unih;
        double lat_lo = -M_PI / 2.0;
        for (int td = 0; td < g->ftd; td++) {
            const double lat_hi = (td + 1.0) / g->ftd * M_PI - M_PI / 2.0;
            const double vol = fabs(r_in * r_in * r_in + r_out * r_out * r_out) / 6.0 * dfi *
                               fabs(sin(lat_lo) - sin(lat_hi));
            for (int fd = 0; fd < g->ffd; fd++) g->volume[grid_index(ht, td, fd, g->ftd, g->ffd)] = vol;
            lat_lo = lat_hi;
        }
        r_in = r_out;
    }
}

/* Reference: src/common/grid.c:65-84. */
void grid_compute_volume_exp(SphericalGrid *g, double Radii, double unih, double alpha2)
{
    const double dfi = 2.0 * M_PI / g->ffd;
    double r_in = Radii;
    for (int ht = 0; ht < g->hd; ht++) {
        const double r_out = r_in + unih * pow(1.0 + alpha2, ht);
        for (int td = 0; td < g->ftd; td++) {
            const double lat_lo = td > 0 ? (double)td / g->ftd * M_PI - M_PI / 2.0 : -M_PI / 2.0;
            const double lat_hi = (td + 1.0) / g->ftd * M_PI - M_PI / 2.0;
            const double vol = fabs(r_in * r_in * r_in + r_out * r_out * r_out) / 6.0 * dfi *
                               fabs(sin(lat_lo) - sin(lat_hi));
            for (int fd = 0; fd < g->ffd; fd++) g->volume[grid_index(ht, td, fd, g->ftd, g->ffd)] = vol;
        }
        r_in = r_out;
    }
}

/* Reference: src/common/grid.c:86-89. */
double grid_exp_height(int ht, double alpha2, double unih, double Radii)
{
    return (pow(1.0 + alpha2, ht + 1) - 1.0) / alpha2 * unih + Radii;
}

/* Reference: src/common/grid.c:91-99. */
int grid_exp_ht_index(double Ri, double Radii, double unih, double alpha2)
{
    const double arg = alpha2 * (Ri - Radii) / unih + 1.0;
    if (arg <= 1.0) return 0;
    const int ht = (int)ceil(log(arg) / log(1.0 + alpha2)) - 1;
    return ht < 0 ? 0 : ht;
}

/* Reference: src/common/polyfit.c:10-101. Power sums S_k and moments b_j feed the normal
 * equations, solved by Gaussian elimination with partial pivoting; degree <= 6. */
int polyfit(const double *x, const double *y, int n, int degree, double *coeffs)
{
    const int m = degree + 1;
    if (n < m || degree < 0 || degree > 6) return -1;
    double S[13] = {0}, b[7] = {0}, a[7] = {0};
    for (int i = 0; i < n; i++) {
        double xp = 1.0;
        for (int k = 0; k <= 2 * degree; k++) { S[k] += xp; xp *= x[i]; }
    }
    for (int i = 0; i < n; i++) {
        double xp = 1.0;
        for (int j = 0; j < m; j++) { b[j] += xp * y[i]; xp *= x[i]; }
    }
    double A[7][8];
    for (int r = 0; r < m; r++) {
        for (int c = 0; c < m; c++) A[r][c] = S[r + c];
        A[r][m] = b[r];
    }
    for (int col = 0; col < m; col++) {
        int piv = col;
        double best = fabs(A[col][col]);
        for (int r = col + 1; r < m; r++)
            if (fabs(A[r][col]) > best) { best = fabs(A[r][col]); piv = r; }
        if (best < 1e-30) return -1;
        if (piv != col)
            for (int k = 0; k <= m; k++) { double t = A[col][k]; A[col][k] = A[piv][k]; A[piv][k] = t; }
        for (int r = col + 1; r < m; r++) {
            const double f = A[r][col] / A[col][col];
            for (int k = col; k <= m; k++) A[r][k] -= f * A[col][k];
        }
    }
    for (int r = m - 1; r >= 0; r--) {
        a[r] = A[r][m];
        for (int c = r + 1; c < m; c++) a[r] -= A[r][c] * a[c];
        a[r] /= A[r][r];
    }
    for (int i = 0; i < m; i++) coeffs[i] = a[degree - i];
    return 0;
}

/* Reference: src/common/polyfit.c:103-110. */
double polyval(const double *coeffs, int degree, double x)
{
    double r = coeffs[0];
    for (int i = 1; i <= degree; i++) r = r * x + coeffs[i];
    return r;
}
