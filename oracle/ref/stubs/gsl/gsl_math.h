#ifndef ORACLE_STUB_GSL_MATH_H
#define ORACLE_STUB_GSL_MATH_H
#include <math.h>
typedef struct
{
  double (*function)(double x, void *params);
  void *params;
} gsl_function;
#define GSL_MAX(a, b) ((a) > (b) ? (a) : (b))
#define GSL_MIN(a, b) ((a) < (b) ? (a) : (b))
#endif
