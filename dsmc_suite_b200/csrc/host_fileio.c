/* host_fileio.c - the reference's ASCII .dat formats (include/fileio.h of the reference,
 * src/common/fileio.c:6-219), byte-compatible on output. Readers check every conversion and
 * return NULL / -1 on a missing or short file instead of returning partly filled buffers. */
#include "fileio.h"

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static FILE *open_or_report(const char *filename, const char *mode)
{
    FILE *fp = fopen(filename, mode);
    if (!fp && mode[0] == 'r') fprintf(stderr, "Cannot open %s\n", filename);
    return fp;
}

static double *read_values(FILE *fp, long count)
{
    if (count <= 0 || count > (1L << 31)) return NULL;
    double *data = calloc((size_t)count, sizeof(double));
    if (!data) return NULL;
    for (long i = 0; i < count; i++) {
        if (fscanf(fp, "%lf", &data[i]) != 1) { free(data); return NULL; }
    }
    return data;
}

/* Reference: fileio.c:6-25. Header ftd, ffd (and hd when has_hd), then [hd][ftd][ffd]. */
double *read_density_dat(const char *filename, int *ftd, int *ffd, int *hd, int has_hd)
{
    FILE *fp = open_or_report(filename, "r");
    if (!fp) return NULL;
    double *data = NULL;
    if (fscanf(fp, "%d", ftd) == 1 && fscanf(fp, "%d", ffd) == 1 &&
        (!has_hd || fscanf(fp, "%d", hd) == 1))
        data = read_values(fp, (long)(*hd) * (*ftd) * (*ffd));
    fclose(fp);
    if (!data) fprintf(stderr, "Malformed density file %s\n", filename);
    return data;
}

/* Reference: fileio.c:27-45. */
int write_density_dat(const char *filename, const double *den, int ftd, int ffd, int hd)
{
    FILE *fp = open_or_report(filename, "w");
    if (!fp) return -1;
    fprintf(fp, "%d\n%d\n%d\n", ftd, ffd, hd);
    const long n = (long)hd * ftd * ffd;
    for (long i = 0; i < n; i++) fprintf(fp, "%9.6f\n", den[i]);
    return fclose(fp) == 0 ? 0 : -1;
}

/* Addition (no reference counterpart): number density [m^-3], header ftd, ffd, hd as the
 * density file, then [hd][ftd][ffd] values in %.9e (the density file's %9.6f is fixed point). */
int write_ndensity_dat(const char *filename, const double *nden, int ftd, int ffd, int hd)
{
    FILE *fp = open_or_report(filename, "w");
    if (!fp) return -1;
    fprintf(fp, "%d\n%d\n%d\n", ftd, ffd, hd);
    const long n = (long)hd * ftd * ffd;
    for (long i = 0; i < n; i++) fprintf(fp, "%.9e\n", nden[i]);
    return fclose(fp) == 0 ? 0 : -1;
}

/* Reference: fileio.c:47-62. Header ftd, ffd, then [ftd][ffd]. */
double *read_temperature_dat(const char *filename, int *ftd, int *ffd)
{
    FILE *fp = open_or_report(filename, "r");
    if (!fp) return NULL;
    double *data = NULL;
    if (fscanf(fp, "%d", ftd) == 1 && fscanf(fp, "%d", ffd) == 1)
        data = read_values(fp, (long)(*ftd) * (*ffd));
    fclose(fp);
    if (!data) fprintf(stderr, "Malformed temperature file %s\n", filename);
    return data;
}

/* Reference: fileio.c:64-109. ffd copies of the map, copy t shifted left by t columns. */
double *read_temperature_time_dat(const char *filename, int *ftd, int *ffd)
{
    double *T = read_temperature_dat(filename, ftd, ffd);
    if (!T) return NULL;
    const int nt = *ftd, nf = *ffd;
    double *out = calloc((size_t)nf * nt * nf, sizeof(double));
    if (!out) { free(T); return NULL; }
    for (int t = 0; t < nf; t++)
        for (int td = 0; td < nt; td++)
            for (int fd = 0; fd < nf; fd++)
                out[((size_t)t * nt + td) * nf + fd] = T[td * nf + (fd + t) % nf];
    free(T);
    return out;
}

/* Reference: fileio.c:111-123. Row-major [nrows][totaln], one value per line. */
int write_ttime_dat(const char *filename, const double *ttime, int nrows, int totaln)
{
    FILE *fp = open_or_report(filename, "w");
    if (!fp) return -1;
    const long n = (long)nrows * totaln;
    for (long i = 0; i < n; i++) fprintf(fp, "%9.5f\n", ttime[i]);
    return fclose(fp) == 0 ? 0 : -1;
}

/* Reference: fileio.c:125-141. */
int write_v_record_dat(const char *filename, const double *v_record, const int *td_list,
                       const int *fd_list, const int *ht_list, int nrecords)
{
    FILE *fp = open_or_report(filename, "w");
    if (!fp) return -1;
    fprintf(fp, "%d\n", nrecords);
    for (int i = 0; i < nrecords; i++)
        fprintf(fp, "%f %f %f\n%d\n%d\n%d\n", v_record[3 * i], v_record[3 * i + 1],
                v_record[3 * i + 2], td_list[i], fd_list[i], ht_list[i]);
    return fclose(fp) == 0 ? 0 : -1;
}

/* Reference: fileio.c:143-167. */
int read_v_record_dat(const char *filename, double **v_record, int **td_list, int **fd_list,
                      int **ht_list, int *nrecords)
{
    FILE *fp = fopen(filename, "r");
    if (!fp) return -1;
    int n = 0;
    if (fscanf(fp, "%d", &n) != 1 || n < 0) { fclose(fp); return -1; }
    double *v = calloc((size_t)n * 3 + 1, sizeof(double));
    int *a = calloc((size_t)n + 1, sizeof(int)), *b = calloc((size_t)n + 1, sizeof(int)),
        *c = calloc((size_t)n + 1, sizeof(int));
    int ok = v && a && b && c;
    for (int i = 0; ok && i < n; i++)
        ok = fscanf(fp, "%lf %lf %lf", &v[3 * i], &v[3 * i + 1], &v[3 * i + 2]) == 3 &&
             fscanf(fp, "%d", &a[i]) == 1 && fscanf(fp, "%d", &b[i]) == 1 &&
             fscanf(fp, "%d", &c[i]) == 1;
    fclose(fp);
    if (!ok) { free(v); free(a); free(b); free(c); return -1; }
    *v_record = v; *td_list = a; *fd_list = b; *ht_list = c; *nrecords = n;
    return 0;
}

/* Reference: fileio.c:169-186. */
double *read_flux_dat(const char *filename, int *nface, int *tt)
{
    FILE *fp = fopen(filename, "r");
    if (!fp) return NULL;
    double *F = NULL;
    if (fscanf(fp, "%d", nface) == 1 && fscanf(fp, "%d", tt) == 1)
        F = read_values(fp, (long)(*nface) * (*tt));
    fclose(fp);
    return F;
}

/* Reference: fileio.c:188-203. */
int write_flux_dat(const char *filename, const double *F, int nface, int tt)
{
    FILE *fp = open_or_report(filename, "w");
    if (!fp) return -1;
    fprintf(fp, "%d\n%d\n", nface, tt);
    const long n = (long)nface * tt;
    for (long i = 0; i < n; i++) fprintf(fp, "%9.7f\n", F[i]);
    return fclose(fp) == 0 ? 0 : -1;
}

/* Reference: fileio.c:205-219. */
int write_horizon_dat(const char *filename, const double *horizon, int ftd, int ffd)
{
    FILE *fp = open_or_report(filename, "w");
    if (!fp) return -1;
    fprintf(fp, "%d\n%d\n", ftd, ffd);
    const long n = (long)ftd * ffd;
    for (long i = 0; i < n; i++) fprintf(fp, "%9.6f\n", horizon[i]);
    return fclose(fp) == 0 ? 0 : -1;
}

/* Binary side-car of one run (not in the reference): the exact fixed-point density and horizon
 * grids and the FP64 per-particle rows that _den.dat, _horizon.dat and _ttime.dat print rounded
 * to 6 and 5 decimals. Little-endian, naturally aligned:
 *   char magic[8] = "DSMCBIN1"; int32 ftd, ffd, hd, nrows; int64 totaln; double fixed_scale;
 *   uint64 den[hd * ftd * ffd]   (the order of _den.dat)
 *   uint64 horizon[ftd * ffd]    (the order of _horizon.dat)
 *   double ttime[nrows * totaln] (the order of _ttime.dat)
 * A grid value is count / fixed_scale, which is what the .dat files print. */
int write_grids_bin(const char *filename, const uint64_t *den, const uint64_t *hor,
                    const double *ttime, int ftd, int ffd, int hd, int nrows, int totaln,
                    double fixed_scale)
{
    FILE *fp = open_or_report(filename, "wb");
    if (!fp) return -1;
    const int32_t dims[4] = {ftd, ffd, hd, nrows};
    const int64_t n = totaln;
    const size_t ncell = (size_t)hd * ftd * ffd, nh = (size_t)ftd * ffd,
                 nt = (size_t)nrows * (totaln > 0 ? totaln : 0);
    int ok = fwrite("DSMCBIN1", 1, 8, fp) == 8 && fwrite(dims, sizeof dims, 1, fp) == 1 &&
             fwrite(&n, sizeof n, 1, fp) == 1 && fwrite(&fixed_scale, sizeof fixed_scale, 1, fp) == 1 &&
             fwrite(den, sizeof *den, ncell, fp) == ncell &&
             fwrite(hor, sizeof *hor, nh, fp) == nh &&
             (nt == 0 || fwrite(ttime, sizeof *ttime, nt, fp) == nt);
    return fclose(fp) == 0 && ok ? 0 : -1;
}
