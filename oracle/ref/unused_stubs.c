/*
 * unused_stubs.c -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Link-time stand-ins for library entry points (FFTW, GMP, a few GSL helpers)
 * and generated build files that the reference's translation units reference
 * on paths the oracle never executes (PM long-range force, Voronoi mesh,
 * snapshot I/O).  Each aborts loudly if it is ever reached.
 */
#include <stdio.h>
#include <stdlib.h>

static void unused(const char *name)
{
  fprintf(stderr, "oracle build: %s is outside the short-range gravity path and is not available\n", name);
  abort();
}

#define UNUSED_FN(name) \
  void name(void) { unused(#name); }

UNUSED_FN(fftwf_execute_dft)
UNUSED_FN(fftwf_execute_dft_c2r)
UNUSED_FN(fftwf_execute_dft_r2c)
UNUSED_FN(gsl_finite)
UNUSED_FN(gsl_rng_size)
UNUSED_FN(gsl_rng_state)
UNUSED_FN(mpz_add)
UNUSED_FN(mpz_add_ui)
UNUSED_FN(mpz_cdiv_q)
UNUSED_FN(mpz_clear)
UNUSED_FN(mpz_get_d)
UNUSED_FN(mpz_init)
UNUSED_FN(mpz_mul)
UNUSED_FN(mpz_mul_2exp)
UNUSED_FN(mpz_set)
UNUSED_FN(mpz_set_si)
UNUSED_FN(mpz_sgn)
UNUSED_FN(mpz_sub)
UNUSED_FN(mpz_tdiv_q_2exp)
UNUSED_FN(output_compile_time_options)
#ifndef HAVE_PM_PERIODIC /* the pmfft harness build links the reference's own periodic PM */
UNUSED_FN(pm_init_periodic)
UNUSED_FN(pmforce_periodic)
#endif
UNUSED_FN(write_only_delaunay_triangulation)

/* endrun() is defined next to main() in the reference; the harness has its own main */
void endrun(void)
{
  fflush(stdout);
  exit(0);
}
