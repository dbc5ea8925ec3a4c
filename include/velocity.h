/* velocity.h - launch-speed sampling (replaces the reference's include/velocity.h:7-15, same
 * signatures). */
#ifndef VELOCITY_H
#define VELOCITY_H

#include "types.h"

/* Speed table for 23 temperatures from 20 K to 240 K (reference velocity.c:6-47 semantics). */
void velocity_table_init(VelocityTable *vt, double mmass, double mole, double k_B);

/* Draw a speed for local temperature T_local with glibc rand_r on *seed. */
double velocity_sample(const VelocityTable *vt, double T_local, unsigned int *seed);

/* sqrt(alpha * vr^2 + (1 - alpha) * v_old_sq). */
double velocity_sticking(double vr, double v_old_sq, double alpha);

#endif /* VELOCITY_H */
