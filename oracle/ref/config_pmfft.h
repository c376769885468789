/* Compile-time options of the periodic TreePM build with the reference's own PM long-range force
 * (gravity/pm/pm_periodic.c, double-precision mesh, FFT calls served by fftw_shim.c). */
#define SELFGRAVITY
#define PMGRID 64
#define DOUBLEPRECISION 1
#define DOUBLEPRECISION_FFTW
#define EVALPOTENTIAL
#define DO_NOT_RANDOMIZE_DOMAINCENTER
#define NSOFTTYPES 2
#define ALLOW_DIRECT_SUMMATION
