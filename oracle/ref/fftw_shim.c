/*
 * fftw_shim.c -- TEST INFRASTRUCTURE ONLY (oracle).  The few FFTW-3 entry points that the
 * reference's periodic PM (gravity/pm/pm_periodic.c:193-237, gravity/pm/pm_mpi_fft.c) calls, in
 * double precision (DOUBLEPRECISION_FFTW), so that pmforce_periodic can run in the harness without
 * the FFTW library:
 *
 *   fftw_plan_many_dft_r2c / _c2r / fftw_plan_many_dft with rank 1 and howmany 1 (a strided 1-D
 *   transform of length n), and fftw_execute_dft_r2c / _c2r / fftw_execute_dft on new arrays with the
 *   plan's strides.
 *
 * Transforms are unnormalised, with FFTW's sign convention (FFTW_FORWARD = -1: X_k = sum_j x_j
 * exp(-2 pi i j k / n)).  Algorithm: iterative radix-2 Cooley-Tukey (decimation in time, bit-reversed
 * input order) for power-of-two lengths, the plain O(n^2) DFT otherwise; twiddle factors from
 * cos/sin of the exact angle in long double.  Real-to-complex transforms run the complex transform on
 * the real data and keep the n/2+1 independent coefficients; complex-to-real transforms rebuild the
 * Hermitian-symmetric spectrum and keep the real part of the backward transform.  The rounding
 * differs from FFTW's, so results agree with FFTW to a few units of the last place, not bit for bit.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

struct fftw_plan_s
{
  int kind; /* 0 r2c, 1 c2c, 2 c2r */
  int n, sign, istride, ostride;
};

static fftw_plan new_plan(int kind, const int *n, int sign, int istride, int ostride)
{
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  p->kind     = kind;
  p->n        = n[0];
  p->sign     = sign;
  p->istride  = istride;
  p->ostride  = ostride;
  return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist, unsigned flags)
{
  return new_plan(0, n, FFTW_FORWARD, istride, ostride);
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist, unsigned flags)
{
  return new_plan(2, n, FFTW_BACKWARD, istride, ostride);
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride, int odist, int sign, unsigned flags)
{
  return new_plan(1, n, sign, istride, ostride);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }

/* in-place complex transform of length n (contiguous re, im pairs) */
static void dft(double *a, int n, int sign)
{
  if(n <= 1)
    return;
  if((n & (n - 1)) == 0)
    {
      for(int i = 1, j = 0; i < n; i++)
        {
          int bit = n >> 1;
          for(; j & bit; bit >>= 1)
            j ^= bit;
          j ^= bit;
          if(i < j)
            {
              double tr = a[2 * i], ti = a[2 * i + 1];
              a[2 * i]     = a[2 * j];
              a[2 * i + 1] = a[2 * j + 1];
              a[2 * j]     = tr;
              a[2 * j + 1] = ti;
            }
        }
      for(int len = 2; len <= n; len <<= 1)
        for(int k = 0; k < len / 2; k++)
          {
            const long double ang = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L * k / len;
            const double wr = (double)cosl(ang), wi = (double)sinl(ang);
            for(int s = 0; s < n; s += len)
              {
                double *u = a + 2 * (s + k), *v = a + 2 * (s + k + len / 2);
                const double tr = v[0] * wr - v[1] * wi, ti = v[0] * wi + v[1] * wr;
                v[0] = u[0] - tr;
                v[1] = u[1] - ti;
                u[0] += tr;
                u[1] += ti;
              }
          }
      return;
    }
  double *b = (double *)malloc(sizeof(double) * 2 * n);
  for(int k = 0; k < n; k++)
    {
      double sr = 0, si = 0;
      for(int j = 0; j < n; j++)
        {
          const long double ang = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L * (((long)j * k) % n) / n;
          const double wr = (double)cosl(ang), wi = (double)sinl(ang);
          sr += a[2 * j] * wr - a[2 * j + 1] * wi;
          si += a[2 * j] * wi + a[2 * j + 1] * wr;
        }
      b[2 * k]     = sr;
      b[2 * k + 1] = si;
    }
  memcpy(a, b, sizeof(double) * 2 * n);
  free(b);
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out)
{
  const int n = p->n;
  double *a   = (double *)malloc(sizeof(double) * 2 * n);
  for(int j = 0; j < n; j++)
    {
      a[2 * j]     = in[(long)j * p->istride][0];
      a[2 * j + 1] = in[(long)j * p->istride][1];
    }
  dft(a, n, p->sign);
  for(int k = 0; k < n; k++)
    {
      out[(long)k * p->ostride][0] = a[2 * k];
      out[(long)k * p->ostride][1] = a[2 * k + 1];
    }
  free(a);
}

void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out)
{
  const int n = p->n;
  double *a   = (double *)malloc(sizeof(double) * 2 * n);
  for(int j = 0; j < n; j++)
    {
      a[2 * j]     = in[(long)j * p->istride];
      a[2 * j + 1] = 0;
    }
  dft(a, n, FFTW_FORWARD);
  for(int k = 0; k <= n / 2; k++)
    {
      out[(long)k * p->ostride][0] = a[2 * k];
      out[(long)k * p->ostride][1] = a[2 * k + 1];
    }
  free(a);
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out)
{
  const int n = p->n;
  double *a   = (double *)malloc(sizeof(double) * 2 * n);
  for(int k = 0; k <= n / 2; k++)
    {
      a[2 * k]     = in[(long)k * p->istride][0];
      a[2 * k + 1] = in[(long)k * p->istride][1];
    }
  for(int k = n / 2 + 1; k < n; k++) /* Hermitian symmetry */
    {
      a[2 * k]     = a[2 * (n - k)];
      a[2 * k + 1] = -a[2 * (n - k) + 1];
    }
  dft(a, n, FFTW_BACKWARD);
  for(int j = 0; j < n; j++)
    out[(long)j * p->ostride] = a[2 * j];
  free(a);
}
