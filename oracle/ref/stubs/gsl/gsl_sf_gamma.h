#ifndef ORACLE_STUB_gsl_sf_gamma_H
#define ORACLE_STUB_gsl_sf_gamma_H
#endif
