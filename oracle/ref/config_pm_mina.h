/* Compile-time options of the periodic TreePM oracle build with ACTIVATE_MINIMUM_OPENING_ANGLE
 * (the relative criterion's mass test also needs a minimum opening angle, forcetree_walk.c:266-271). */
#define SELFGRAVITY
#define PMGRID 64
#define DOUBLEPRECISION 1
#define EVALPOTENTIAL
#define DO_NOT_RANDOMIZE_DOMAINCENTER
#define NSOFTTYPES 2
#define ACTIVATE_MINIMUM_OPENING_ANGLE
