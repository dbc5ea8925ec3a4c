/* types.h - data types of the DSMC C interface.
 *
 * Layout-compatible with the reference's include/types.h:7-106 (same members, same order), so
 * code written against the reference's structs links against this library unchanged. The small
 * vector helpers are static inline as in the reference. */
#ifndef TYPES_H
#define TYPES_H

#include <math.h>

typedef struct {
    double x, y, z;
} Vec3;

static inline double vec3_dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static inline Vec3 vec3_cross(Vec3 a, Vec3 b)
{
    Vec3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}

static inline double vec3_len(Vec3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

static inline Vec3 vec3_scale(Vec3 v, double s)
{
    Vec3 r = {v.x * s, v.y * s, v.z * s};
    return r;
}

static inline Vec3 vec3_add(Vec3 a, Vec3 b)
{
    Vec3 r = {a.x + b.x, a.y + b.y, a.z + b.z};
    return r;
}

static inline Vec3 vec3_sub(Vec3 a, Vec3 b)
{
    Vec3 r = {a.x - b.x, a.y - b.y, a.z - b.z};
    return r;
}

static inline Vec3 vec3_normalize(Vec3 v)
{
    double l = vec3_len(v);
    if (l < 1e-30) { Vec3 z = {0, 0, 0}; return z; }
    return vec3_scale(v, 1.0 / l);
}

/* One test particle (array-of-structs form used by the scalar entry points). */
typedef struct {
    Vec3 pos;
    Vec3 vel;
    double weight;
    int td, fd, ht;
    double flight_time;
    int collision_count;
} Particle;

/* Latitude x longitude x shell grid; arrays are [hd][ftd][ffd] or [ftd][ffd]. */
typedef struct {
    int ftd;
    int ffd;
    int hd;
    double *density;
    double *temperature;
    double *volume;
    double *horizon;
} SphericalGrid;

typedef struct {
    double G, M, k_B, mmass, mole;
    double Radii, ve, lifetime, P;
    double cross_section, alpha;
    double dt_step;
    double dt_rot;
    double max_height;
    double unih;
    double alpha2;
    int use_exp_grid;
} PhysicsParams;

#define VEL_TABLE_NTEMP 23
#define VEL_TABLE_NVEL  1000
typedef struct {
    double temps[VEL_TABLE_NTEMP];
    double speeds[VEL_TABLE_NTEMP][VEL_TABLE_NVEL];
    int count[VEL_TABLE_NTEMP];
} VelocityTable;

#define POLY_DEGREE 3
typedef struct {
    double coeffs[POLY_DEGREE + 1];
    double min_v, max_v;
    int valid;
} PolyFit;

typedef struct {
    int npoint;
    int nface;
    double (*spot)[3];
    int (*facet)[3];
    double (*face_normal)[3];
    double *face_area;
    double (*loc_xyz)[3];
    double (*dir)[2];
} Mesh;

#endif /* TYPES_H */
