#ifndef ORACLE_STUB_GSL_ERRNO_H
#define ORACLE_STUB_GSL_ERRNO_H
typedef void gsl_error_handler_t(const char *reason, const char *file, int line, int gsl_errno);
gsl_error_handler_t *gsl_set_error_handler(gsl_error_handler_t *h);
#define GSL_SUCCESS 0
#endif
