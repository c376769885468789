#ifndef ORACLE_STUB_gsl_heapsort_H
#define ORACLE_STUB_gsl_heapsort_H
#endif
