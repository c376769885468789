/* Compile-time options of the periodic pure-tree (no PM, Ewald-corrected) oracle build of the reference. */
#define SELFGRAVITY
#define DOUBLEPRECISION 1
#define EVALPOTENTIAL
#define DO_NOT_RANDOMIZE_DOMAINCENTER
#define NSOFTTYPES 2
#define ALLOW_DIRECT_SUMMATION
