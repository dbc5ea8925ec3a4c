/* dsmc_runners.h - the reference's module runners, kept with their signatures.
 *
 * The reference declares these only as `extern` in src/main.c:18-23 (defined in
 * src/dsmc/ballistic.c:35-36 and src/dsmc/advanced.c:119-121). Here they read the same input
 * files, solve on the GPU through include/dsmc_cuda.h and write the same output files:
 *   <prefix>_den.dat, <prefix>_horizon.dat, <prefix>_v_record.dat (ballistic), <prefix>_ttime.dat
 * nthreads is accepted for compatibility; the solve runs on one CUDA device (DSMC_DEVICE,
 * default 0). DSMC_PATH selects the kernel path (plain, fast32 or fast64; default plain) and
 * DSMC_SEED the Philox seed. DSMC_SIDECAR=1 (the CLI's --bin) also writes <prefix>_grids.bin, the exact
 * fixed-point grids and FP64 per-particle rows (layout in fileio.h / host_fileio.c). On failure
 * a message goes to stderr and no file is written. DSMC_NDENSITY_RATE=Q (the CLI's --ndensity Q)
 * also writes <prefix>_ndensity.dat, the FP64 number density [m^-3] for a production rate of
 * Q molecules/s (dsmc_number_density_host, physical cell volumes). */
#ifndef DSMC_RUNNERS_H
#define DSMC_RUNNERS_H

#ifdef __cplusplus
extern "C" {
#endif

void run_ballistic(int totaln, const char *temp_file, const char *output_prefix, int nthreads);
void run_advanced(int totaln, const char *temp_file, const char *prev_den_file,
                  const char *prev_v_record_file, const char *output_prefix, int nthreads);

#ifdef __cplusplus
}
#endif
#endif /* DSMC_RUNNERS_H */
