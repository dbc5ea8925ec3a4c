/* grid.h - spherical grid helpers (replaces the reference's include/grid.h:7-30, same
 * signatures). */
#ifndef GRID_H
#define GRID_H

#include "types.h"

SphericalGrid *grid_create(int ftd, int ffd, int hd);
void grid_free(SphericalGrid *g);

/* Flat index of [ht][td][fd], all 0-based. */
static inline int grid_index(int ht, int td, int fd, int ftd, int ffd)
{
    return ht * ftd * ffd + td * ffd + fd;
}

/* Latitude thi in [-pi/2, pi/2] and longitude fi in [0, 2 pi) to 0-based cell indices. */
void grid_spherical_to_index(double thi, double fi, int ftd, int ffd, int *td, int *fd);

/* Cell volumes as the reference computes them (|r_o^3 + r^3| / 6 * dphi * |dsin|). */
void grid_compute_volume_uniform(SphericalGrid *g, double Radii, double unih);
void grid_compute_volume_exp(SphericalGrid *g, double Radii, double unih, double alpha2);

/* Outer radius of exponential shell ht. */
double grid_exp_height(int ht, double alpha2, double unih, double Radii);

/* Exponential shell index (0-based) of radius Ri. */
int grid_exp_ht_index(double Ri, double Radii, double unih, double alpha2);

#endif /* GRID_H */
