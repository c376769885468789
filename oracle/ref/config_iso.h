/* Compile-time options of the isolated (non-periodic, no PM) oracle build of the reference. */
#define SELFGRAVITY
#define GRAVITY_NOT_PERIODIC
#define DOUBLEPRECISION 1
#define EVALPOTENTIAL
#define DO_NOT_RANDOMIZE_DOMAINCENTER
#define NSOFTTYPES 2
#define ALLOW_DIRECT_SUMMATION
