#ifndef ORACLE_STUB_GSL_SPLINE_H
#define ORACLE_STUB_GSL_SPLINE_H
typedef struct gsl_spline_s gsl_spline;
typedef struct gsl_interp_accel_s gsl_interp_accel;
#endif
