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
#endif
