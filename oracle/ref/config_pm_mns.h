/* Compile-time options of the periodic TreePM oracle build with MULTIPLE_NODE_SOFTENING. */
#define SELFGRAVITY
#define PMGRID 64
#define DOUBLEPRECISION 1
#define EVALPOTENTIAL
#define DO_NOT_RANDOMIZE_DOMAINCENTER
#define NSOFTTYPES 2
#define MULTIPLE_NODE_SOFTENING
