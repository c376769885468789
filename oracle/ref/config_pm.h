/* Compile-time options of the periodic TreePM oracle build of the reference. */
#define SELFGRAVITY
#define PMGRID 64
#define DOUBLEPRECISION 1
#define EVALPOTENTIAL
#define DO_NOT_RANDOMIZE_DOMAINCENTER
#define NSOFTTYPES 2
#define ALLOW_DIRECT_SUMMATION
