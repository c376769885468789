#ifndef ORACLE_STUB_GSL_RNG_H
#define ORACLE_STUB_GSL_RNG_H
typedef struct gsl_rng_type_s gsl_rng_type;
typedef struct gsl_rng_s gsl_rng;
extern const gsl_rng_type *gsl_rng_ranlxd1;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_set(const gsl_rng *r, unsigned long seed);
double gsl_rng_uniform(const gsl_rng *r);
void gsl_rng_free(gsl_rng *r);
#endif
