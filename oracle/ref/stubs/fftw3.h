#ifndef ORACLE_STUB_FFTW3_H
#define ORACLE_STUB_FFTW3_H
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct fftw_plan_s *fftw_plan;
typedef struct fftwf_plan_s *fftwf_plan;
#define FFTW_ESTIMATE 0
#define FFTW_UNALIGNED 0
#define FFTW_IN_PLACE 0
#define FFTW_FORWARD -1
#define FFTW_BACKWARD 1
#define FFTW_DESTROY_INPUT 0
/* the double-precision entry points the periodic PM uses (implemented by oracle/ref/fftw_shim.c) */
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride, int odist, int sign, unsigned flags);
void fftw_destroy_plan(fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
#endif
