/* polyfit.h - least-squares polynomial fit (replaces the reference's include/polyfit.h:4-15,
 * same signatures). Coefficients are highest power first. */
#ifndef POLYFIT_H
#define POLYFIT_H

int polyfit(const double *x, const double *y, int n, int degree, double *coeffs);
double polyval(const double *coeffs, int degree, double x);

#endif /* POLYFIT_H */
