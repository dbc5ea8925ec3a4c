/* collision.h - test-particle collision helpers (replaces the reference's
 * include/collision.h:7-16, same signatures). */
#ifndef COLLISION_H
#define COLLISION_H

#include "types.h"

/* *real_col_p += ds * local_density * cross_section; returns 1 when
 * col_threshold < 1 - exp(-*real_col_p). */
int collision_check(double *real_col_p, double col_threshold, double ds, double local_density,
                    double cross_section);

/* The reference's velocity update v <- (v + v2) + 0.5 (v - v2). */
void collision_execute(Vec3 *v, Vec3 v2);

/* Partner speed from the fitted reverse-cumulative distribution, by bisection. */
double collision_sample_speed(const PolyFit *pf, double rand_val, int nn);

#endif /* COLLISION_H */
