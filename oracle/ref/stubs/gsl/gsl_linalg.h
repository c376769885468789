#ifndef ORACLE_STUB_gsl_linalg_H
#define ORACLE_STUB_gsl_linalg_H
#endif
