/* constants.h - physical constants of the reference model (Ceres, H2O), with the values of the
 * reference's include/constants.h:5-41. */
#ifndef CONSTANTS_H
#define CONSTANTS_H

#define CONST_G             6.67e-11                 /* m^3 kg^-1 s^-2 */
#define CONST_M_CERES       9.39e20                  /* kg */
#define CONST_R_CERES       476.2e3                  /* m */
#define CONST_K_B           1.38e-23                 /* J/K */
#define CONST_MOLE          6.02e23                  /* 1/mol */
#define CONST_MMASS_H2O     18e-3                    /* kg/mol */
#define CONST_MMOL_H2O      (CONST_MMASS_H2O / CONST_MOLE)
#define CONST_VE_CERES      (sqrt(2.0 * CONST_G * CONST_M_CERES / CONST_R_CERES))
#define CONST_P_CERES       (9.07417 * 3600.0)       /* s */
#define CONST_LIFETIME      (1.0 / 1.02e-5 * (2.8 * 2.8))  /* s, at 2.8 AU */
#define CONST_CROSS_SECTION 1e-19                    /* m^2 */
#define CONST_SIGMA         5.6704e-8                /* W m^-2 K^-4 */
#define CONST_SOLAR_1AU     1368.0                   /* W/m^2 */

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#endif /* CONSTANTS_H */
