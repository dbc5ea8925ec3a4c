/* integrator.h - orbit push of one particle (replaces the reference's include/integrator.h:7-20,
 * same enum and signature). */
#ifndef INTEGRATOR_H
#define INTEGRATOR_H

#include "types.h"

typedef enum {
    VERLET_OK = 0,
    VERLET_LANDED,
    VERLET_ESCAPED
} VerletStatus;

/* One step of the reference's Stormer-Verlet variant:
 *   s' = s + v h - (GM/r^3) s (1.5 h^2) - oa h^2 / 6,   v' = v - (GM/r^3) s h,   oa' = (GM/r^3) s
 * Updates p->pos, p->vel and *oa; *ds_out (may be NULL) receives |s' - s|. Returns
 * VERLET_LANDED when |s'| <= Radii and VERLET_ESCAPED when |s'| >= max_height. */
VerletStatus verlet_step(Particle *p, const PhysicsParams *params, double h, Vec3 *oa,
                         double *ds_out);

#endif /* INTEGRATOR_H */
