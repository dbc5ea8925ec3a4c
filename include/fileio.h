/* fileio.h - ASCII .dat readers and writers (replaces the reference's include/fileio.h:6-43,
 * same signatures and byte-compatible formats). Readers return malloc'd buffers the caller
 * frees, or NULL / -1 on failure. */
#ifndef FILEIO_H
#define FILEIO_H

#include <stdint.h>

#include "types.h"

double *read_density_dat(const char *filename, int *ftd, int *ffd, int *hd, int has_hd);
int write_density_dat(const char *filename, const double *den, int ftd, int ffd, int hd);
double *read_temperature_dat(const char *filename, int *ftd, int *ffd);
double *read_temperature_time_dat(const char *filename, int *ftd, int *ffd);
int write_ttime_dat(const char *filename, const double *ttime, int nrows, int totaln);
int write_v_record_dat(const char *filename, const double *v_record, const int *td_list,
                       const int *fd_list, const int *ht_list, int nrecords);
int read_v_record_dat(const char *filename, double **v_record, int **td_list, int **fd_list,
                      int **ht_list, int *nrecords);
double *read_flux_dat(const char *filename, int *nface, int *tt);
int write_flux_dat(const char *filename, const double *F, int nface, int tt);
int write_horizon_dat(const char *filename, const double *horizon, int ftd, int ffd);

/* Addition (no reference counterpart): the run's exact fixed-point grids and FP64 per-particle
 * rows as one binary side-car, <prefix>_grids.bin, for comparisons the printed precision of the
 * .dat files cannot settle. Layout in host_fileio.c; 0 on success, -1 on an I/O failure. */
int write_grids_bin(const char *filename, const uint64_t *den, const uint64_t *hor,
                    const double *ttime, int ftd, int ffd, int hd, int nrows, int totaln,
                    double fixed_scale);

/* Addition (no reference counterpart): <prefix>_ndensity.dat, the FP64 number density [m^-3]
 * of dsmc_number_density_host: header ftd, ffd, hd, then [hd][ftd][ffd] values in %.9e. */
int write_ndensity_dat(const char *filename, const double *nden, int ftd, int ffd, int hd);

#endif /* FILEIO_H */
