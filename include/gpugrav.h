/*
 * gpugrav.h -- C ABI of libarepo_gpugrav, a B200 (sm_100a) engine for AREPO's
 * short-range TreePM tree gravity.
 *
 * The library replaces the pair
 *     construct_forcetree(0, ...);   src/gravity/forcetree.c:110-149
 *     gravity_tree(timebin);         src/gravity/gravtree.c:357-707
 * inside gravity() (src/gravity/accel.c:127-134), including the Peano-Hilbert
 * key generation and key sort that precede it (src/domain/domain_toplevel.c:120-135,
 * src/domain/peano.c:74-133).  gravity_force_finalize(), the PM long-range
 * force, the rest of the domain decomposition and the hydro stay in the caller.
 *
 * Conventions (all as in the reference):
 *   - accelerations are returned WITHOUT the factor G (gravity_force_finalize
 *     multiplies by G, src/gravity/accel.c:258-265);
 *   - OldAcc is a float per particle (src/main/allvars.h:1266);
 *   - particles are addressed in the caller's order; the library sorts them
 *     internally (stable, by 126-bit Peano-Hilbert key) and scatters results back;
 *   - negative status codes mirror force_treebuild_construct's -1/-2/-3
 *     (src/gravity/forcetree.c:313-318); the library never exits or aborts.
 *
 * Plain pointers and sizes only.  `mem` arguments say whether an array lives
 * in host memory (GPUGRAV_MEM_HOST, copied through pinned staging buffers) or
 * in device memory of the context's GPU (GPUGRAV_MEM_DEVICE).
 */
#ifndef GPUGRAV_H
#define GPUGRAV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GPUGRAV_ABI_VERSION 1
#define GPUGRAV_MAX_SOFTTYPES 16 /* NSOFTTYPES + NSOFTTYPES_HYDRO supported by this build */
#define GPUGRAV_NTAB 127         /* NTAB, src/gravity/forcetree.h:86 */

typedef enum gpugrav_status
{
  GPUGRAV_OK              = 0,
  GPUGRAV_ERR_TREE_FULL   = -1,  /* force_treebuild_construct: -1, node storage too small */
  GPUGRAV_ERR_TOPNODES    = -2,  /* force_treebuild_construct: -2, top-level nodes invalid / do not fit */
  GPUGRAV_ERR_OUT_OF_BOX  = -3,  /* force_treebuild_construct: -3, particle outside the domain box:
                                    the caller must redo the domain decomposition (src/gravity/forcetree.c:197-208) */
  GPUGRAV_ERR_INVALID     = -10, /* bad argument */
  GPUGRAV_ERR_OOM         = -11, /* device or pinned host allocation failed */
  GPUGRAV_ERR_CUDA        = -12, /* CUDA runtime error; gpugrav_last_error() has the text */
  GPUGRAV_ERR_TIMEOUT     = -13, /* reserved for a bounded device-side wait that gives up; no entry point of this
                                    build waits on the device (every wait is a stream synchronisation) */
  GPUGRAV_ERR_STATE       = -14, /* call order violated (e.g. walk before build) */
  GPUGRAV_ERR_DEEP_TREE   = -15, /* tree deeper than the walk's fixed limits (pathological input) */
  GPUGRAV_ERR_UNSUPPORTED = -16, /* option not available in this build */
  GPUGRAV_ERR_TOO_LARGE   = -17  /* request exceeds a fixed capacity (gpugrav_direct_noalloc: 4096 targets) */
} gpugrav_status;

enum
{
  GPUGRAV_MEM_HOST   = 0,
  GPUGRAV_MEM_DEVICE = 1
};

enum
{
  GPUGRAV_PREC_FP64       = 0, /* parity walk: reference arithmetic, per-target opening decisions */
  GPUGRAV_PREC_FP32       = 1, /* fast walk: FP32 arithmetic, FP64 separations, compensated sums */
  GPUGRAV_PREC_FP64_GROUP = 2  /* the fast walk's algorithm (groups, interaction lists) in FP64 arithmetic:
                                  the precision ablation of GPUGRAV_PREC_FP32 (no Ewald-corrected mode) */
};

/* Run parameters: the All.* fields the path reads. */
typedef struct gpugrav_params
{
  int32_t abi_version;                 /* GPUGRAV_ABI_VERSION */
  int32_t periodic;                    /* 1: periodic box: TreePM short-range force (PMGRID builds) if asmth > 0,
                                          Ewald-corrected tree (periodic builds without PMGRID) if asmth == 0;
                                          0: isolated, plain Newtonian tree (GRAVITY_NOT_PERIODIC, no PMGRID) */
  double box_size;                     /* All.BoxSize */
  double asmth;                        /* All.Asmth[0] (periodic only) */
  double rcut;                         /* All.Rcut[0] = RCUT * Asmth[0] (periodic only) */
  double rcut_cells;                   /* RCUT: extent of the tabulated short-range factor (default 4.5) */
  int32_t nsofttypes;                  /* number of softening types (NSOFTTYPES + NSOFTTYPES_HYDRO) */
  int32_t type_of_opening_criterion;   /* All.TypeOfOpeningCriterion (0: Barnes-Hut, 1: relative) */
  double force_softening[GPUGRAV_MAX_SOFTTYPES + 1]; /* All.ForceSoftening[0..nsofttypes], last entry 0
                                                        (set_softenings, src/gravity/grav_softening.c:92-95) */
  double err_tol_theta;                /* All.ErrTolTheta; > 0 selects the Barnes-Hut criterion in gpugrav_walk */
  double err_tol_force_acc;            /* All.ErrTolForceAcc */
  double top_node_factor;              /* All.TopNodeFactor (library-built top tree only) */
  int32_t multiple_domains;            /* All.MultipleDomains (library-built top tree only) */
  int32_t precision;                   /* GPUGRAV_PREC_* */
  int32_t flags;                       /* GPUGRAV_FLAG_* */
  int32_t reserved;                    /* 0 */
} gpugrav_params;

/* gpugrav_params.flags */
enum
{
  /* MULTIPLE_NODE_SOFTENING: a node whose largest softening exceeds the target's is used once per
   * softening type with that type's mass (ExtNodes[].mass_per_type) instead of being opened
   * (src/gravity/forcetree_walk.c:296-308, 382-401; src/gravity/forcetree.c:1222-1308) */
  GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING = 1,
  /* ACTIVATE_MINIMUM_OPENING_ANGLE: the relative criterion's mass test opens a node only if it also
   * spans more than 0.4 (len > 0.4 r) (src/gravity/forcetree_walk.c:266-271) */
  GPUGRAV_FLAG_MINIMUM_OPENING_ANGLE = 2,
  /* ALLOW_DIRECT_SUMMATION: gpugrav_compute of fewer than GPUGRAV_DIRECT_SUMMATION_THRESHOLD particles runs
   * gpugrav_gravity_direct instead of the tree, as gravity() does (src/gravity/accel.c:103-110) */
  GPUGRAV_FLAG_ALLOW_DIRECT_SUMMATION = 4
};
#define GPUGRAV_DIRECT_SUMMATION_THRESHOLD 3000 /* DIRECT_SUMMATION_THRESHOLD, src/main/allvars.h:245-247 */

/* Domain geometry: the globals set by domain_findExtent (src/domain/domain_box.c:169-196). */
typedef struct gpugrav_domain
{
  double corner[3];   /* DomainCorner */
  double center[3];   /* DomainCenter */
  double len;         /* DomainLen */
  double inverse_len; /* DomainInverseLen */
  double big_fac;     /* DomainBigFac = DomainLen / 2^52 */
} gpugrav_domain;

/* One top-level node: struct topnode_data (src/main/allvars.h:769-782), keys split in two 64-bit halves. */
typedef struct gpugrav_topnode
{
  uint64_t start_key_hi, start_key_lo; /* StartKey (126-bit Peano-Hilbert key) */
  uint64_t size_hi, size_lo;           /* Size */
  int32_t daughter;                    /* Daughter: index of the first of 8 daughters, -1 for a leaf */
  int32_t leaf;                        /* Leaf: top-leaf number (leaves only) */
  uint8_t morton_to_peano[8];          /* MortonToPeanoSubnode */
} gpugrav_topnode;

/* Summary of the last build (gpugrav_build). Node indices follow the reference:
 * particles are [0, max_part), the root node is max_part (Tree_MaxPart), top-level
 * nodes follow it, first_non_top is Tree_FirstNonTopLevelNode. */
typedef struct gpugrav_tree_info
{
  int64_t num_particles;
  int64_t max_part;      /* = num_particles */
  int64_t num_nodes;     /* Tree_NumNodes */
  int64_t first_non_top; /* Tree_FirstNonTopLevelNode */
  int32_t num_topnodes;  /* NTopnodes */
  int32_t num_topleaves; /* NTopleaves */
  int32_t max_depth;     /* deepest node level (root = 0) */
  int32_t coincident_cells; /* cells at MAX_TREE_LEVEL holding >= 2 particles */
} gpugrav_tree_info;

/* Device-time breakdown of the last calls, milliseconds (CUDA events on the library stream). */
typedef struct gpugrav_timings
{
  double upload_ms, domain_ms, sort_ms, toptree_ms, build_ms, moments_ms, walk_ms, download_ms;
  int64_t interactions; /* sum of per-target interaction counts of the last walk */
  int32_t walk_kernel_launches;
  int32_t build_kernel_launches;
  double pm_ms; /* last gpugrav_pm_periodic: deposit, FFTs, Green's function, readout */
} gpugrav_timings;

typedef struct gpugrav_ctx gpugrav_ctx;

/* ---- lifetime ---- */
const char *gpugrav_status_string(int32_t status);
const char *gpugrav_last_error(gpugrav_ctx *ctx);
int32_t gpugrav_abi_version(void);
/* Create a context on CUDA device `device`; replaces force_treeallocate (src/gravity/forcetree.c:1677-1696):
 * the context owns all device memory and grows it as needed. */
int32_t gpugrav_create(gpugrav_ctx **ctx, int32_t device, const gpugrav_params *params);
int32_t gpugrav_destroy(gpugrav_ctx *ctx);
int32_t gpugrav_set_params(gpugrav_ctx *ctx, const gpugrav_params *params);
/* Run all library work on a caller-owned cudaStream_t (NULL: the context's own non-blocking stream,
 * which does not order against the caller's work; the legacy default stream is cudaStreamLegacy). */
int32_t gpugrav_set_stream(gpugrav_ctx *ctx, void *cuda_stream);
int32_t gpugrav_synchronize(gpugrav_ctx *ctx);

/* ---- domain stage ----
 * Replaces do_box_wrapping (periodic wrap, src/domain/domain_box.c:259-275), domain_findExtent
 * (src/domain/domain_box.c:107-197, with DO_NOT_RANDOMIZE_DOMAINCENTER), the key computation of
 * domain_determineTopTree (src/domain/domain_toplevel.c:120-126) and peano_hilbert_order
 * (src/domain/peano.c:74-133, a stable sort by key).
 * pos: n*3 doubles (x,y,z per particle), mass: n doubles, softtype: n bytes (P[].SofteningType).
 * dom: NULL -> the library computes the extent; otherwise the caller's DomainCorner/Len are used and
 * a particle outside them yields GPUGRAV_ERR_OUT_OF_BOX (isolated runs, src/gravity/forcetree.c:411-430). */
int32_t gpugrav_load(gpugrav_ctx *ctx, int64_t n, const double *pos, const double *mass, const uint8_t *softtype,
                     int32_t mem, const gpugrav_domain *dom);

/* ---- build ----
 * Replaces force_treebuild (src/gravity/forcetree.c:162-288): top-level skeleton
 * (force_create_empty_nodes :1131-1180), octree over the 52-bit integer coordinates
 * (force_treebuild_insert_single_point :835-938, including the MAX_TREE_LEVEL rule for
 * coincident points), multipole moments and the nextnode/sibling threading
 * (force_update_node_recursive :1217-1429).
 * top: the caller's TopNodes (domain_determineTopTree output) or NULL, in which case the library
 * derives the top tree from the sorted keys with the same refinement rule (one rank, work load =
 * particle count). */
int32_t gpugrav_build(gpugrav_ctx *ctx, const gpugrav_topnode *top, int32_t ntop);

/* ---- walk ----
 * Replaces gravity_tree (src/gravity/gravtree.c:357-707) / force_treeevaluate
 * (src/gravity/forcetree_walk.c:115-514) for every loaded particle as a target.
 * The opening criterion follows err_tol_theta: > 0 Barnes-Hut, == 0 relative (uses oldacc).
 * oldacc: n floats in caller order or NULL (zeros); acc: n*3 doubles; pot, ninter: n each or NULL.
 * All arrays in caller order, in memory of kind `mem`. */
int32_t gpugrav_walk(gpugrav_ctx *ctx, const float *oldacc, double *acc, double *pot, int32_t *ninter, int32_t mem);
/* The walk of an active subset: gravity_tree(timebin) builds TargetList from
 * TimeBinsGravity.ActiveParticleList (src/gravity/gravtree.c:494-520) and walks only those particles
 * while the tree holds all of them (the production caller under HIERARCHICAL_GRAVITY,
 * src/time_integration/do_gravity_hydro.c:126-270).  targets: ntargets caller indices in [0, n), any
 * order, each at most once (GPUGRAV_ERR_INVALID otherwise); the library walks them in Peano-Hilbert
 * order.  oldacc: n floats in caller order (every particle's OldAcc, as for gpugrav_walk) or NULL;
 * acc: ntargets*3, pot, ninter: ntargets each or NULL, in the order of `targets`.  FP64: per-target
 * results bit-identical to gpugrav_walk's for the same particles; FP32: walk groups are formed from
 * consecutive active targets.  Arrays (targets included) in memory of kind `mem`. */
int32_t gpugrav_walk_targets(gpugrav_ctx *ctx, int64_t ntargets, const int32_t *targets, const float *oldacc, double *acc,
                             double *pot, int32_t *ninter, int32_t mem);
/* Restrict the following walks (gpugrav_walk, gpugrav_walk_targets, gpugrav_compute) to slice `slice` of `nslices`
 * contiguous slices of the targets in Peano-Hilbert order -- the reference's domain
 * decomposition into key segments (src/domain/domain_toplevel.c), applied to targets only: the
 * tree still holds every particle. FP32: slices are whole walk groups; FP64: target ranges.
 * Outputs of targets outside the slice are written as zero, so the slices' outputs of G callers
 * sum exactly to the unsliced result. Default 0 of 1 (all targets). */
int32_t gpugrav_set_target_slice(gpugrav_ctx *ctx, int32_t slice, int32_t nslices);

/* Read-back of ExtNodes[].mass_per_type under MULTIPLE_NODE_SOFTENING: num_nodes x nsofttypes
 * doubles in the reference's node order (parity checks). */
int32_t gpugrav_export_mass_per_type(gpugrav_ctx *ctx, double *out);

/* The same with slices of equal COST instead of equal target counts: cost (n floats in caller order,
 * e.g. the interaction counts of the previous step, the load measure force_assign_cost_values gives the
 * reference's domain decomposition, src/gravity/forcetree.c:945-1010) is summed per FP32 walk group or
 * FP64 target in key order, and slice s gets the units from the first whose cost prefix reaches s/nslices
 * of the total to the first that reaches (s+1)/nslices.  Every rank must pass the same costs.  NULL cost:
 * equal counts (gpugrav_set_target_slice).  n must be the particle count of the following walks; the
 * costs are copied (active-target walks ignore them). */
int32_t gpugrav_set_target_slice_cost(gpugrav_ctx *ctx, int32_t slice, int32_t nslices, int64_t n, const float *cost,
                                      int32_t mem);

/* Periodic box without PM (params: periodic = 1, asmth = 0): the walks use the nearest image of
 * every node and particle plus the reference's Ewald correction per interaction
 * (src/gravity/forcetree_walk.c:469-477, forcetree_ewald.c:268-391). The correction tables are those
 * of ewald_init (forcetree_ewald.c:89-254): by default the library computes them on the host on
 * first use (the reference's sums, bit-identical; a few seconds, once per process) and scales them
 * to box_size; a caller that already holds AREPO's tables (Ewd_fcorrx/y/z, Ewd_potcorr after
 * ewald_init, i.e. scaled to its box) passes them here: en = EN = 64, (en+1)^3 doubles each,
 * last index fastest. They are copied; they stay in use until the next call. */
int32_t gpugrav_set_ewald_table(gpugrav_ctx *ctx, int32_t en, const double *fcorrx, const double *fcorry,
                                const double *fcorrz, const double *potcorr);

/* Long-range periodic PM accelerations (without G) and potentials of n particles; replaces
 * pmforce_periodic(0, NULL) (src/gravity/pm/pm_periodic.c:1572-1936): CIC assignment on a
 * pmgrid^3 mesh, FFT, Green's function -exp(-k^2 Asmth^2)/k^2 with the CIC deconvolution, inverse
 * FFT, 4-point finite differences, CIC readout (FP64 mesh). Uses the context's box_size and asmth
 * (Asmth = ASMTH * BoxSize / PMGRID); positions in [0, box_size); independent of the tree state.
 * pos n*3, mass n, acc n*3 (required), pot n (may be NULL); host or device arrays per `mem`.
 * 8 <= pmgrid <= 2048. */
int32_t gpugrav_pm_periodic(gpugrav_ctx *ctx, int32_t pmgrid, int64_t n, const double *pos, const double *mass, double *acc,
                            double *pot, int32_t mem);

/* ---- one call: load + build + walk (the drop-in for construct_forcetree + gravity_tree) ----
 * With GPUGRAV_FLAG_ALLOW_DIRECT_SUMMATION and n < GPUGRAV_DIRECT_SUMMATION_THRESHOLD: gpugrav_gravity_direct
 * (ninter, if given, is n for every particle); dom, top and oldacc are then unused. */
int32_t gpugrav_compute(gpugrav_ctx *ctx, int64_t n, const double *pos, const double *mass, const uint8_t *softtype,
                        const float *oldacc, const gpugrav_domain *dom, const gpugrav_topnode *top, int32_t ntop,
                        double *acc, double *pot, int32_t *ninter, int32_t mem);

/* ---- introspection (parity checks; host buffers) ---- */
int32_t gpugrav_get_domain(gpugrav_ctx *ctx, gpugrav_domain *dom);
/* order[i] = caller index of the particle at sorted position i (P[i].ID-1 after peano_hilbert_order) */
int32_t gpugrav_get_order(gpugrav_ctx *ctx, int64_t *order);
/* 126-bit keys in sorted order */
int32_t gpugrav_get_keys(gpugrav_ctx *ctx, uint64_t *key_hi, uint64_t *key_lo);
int32_t gpugrav_get_topnodes(gpugrav_ctx *ctx, gpugrav_topnode *top, int32_t capacity, int32_t *ntop);
int32_t gpugrav_get_tree_info(gpugrav_ctx *ctx, gpugrav_tree_info *info);
/* Nodes in the reference's numbering: entry k describes node max_part + k, k < num_nodes.
 * center, s: 3 doubles per node; p_next, p_father: per particle (sorted order). Any pointer may be NULL. */
int32_t gpugrav_export_tree(gpugrav_ctx *ctx, double *center, double *len, double *s, double *mass, int32_t *sibling,
                            int32_t *nextnode, int32_t *father, uint8_t *maxsofttype, int32_t *p_next, int32_t *p_father);
int32_t gpugrav_get_timings(gpugrav_ctx *ctx, gpugrav_timings *t);

/* ---- direct summation (accuracy instrument; gravity_forcetest_evaluate,
 *      src/gravity/gravtree_forcetest.c:421-648, without Ewald images) ----
 * FP64 direct sum over all loaded particles for the given targets (caller indices):
 * the TreePM short-range force with the exact erfc factor (periodic) or Newtonian (isolated).
 * mode GPUGRAV_DIRECT_FULL sums every pair (gravtree_forcetest.c:583-601); GPUGRAV_DIRECT_CUT keeps
 * only pairs closer than Rcut, the range the tree walk evaluates (forcetree_walk.c:369-372), so that
 * the difference to the walk is the tree approximation error alone. */
enum
{
  GPUGRAV_DIRECT_FULL = 0,
  GPUGRAV_DIRECT_CUT  = 1
};
int32_t gpugrav_direct(gpugrav_ctx *ctx, int64_t ntargets, const int64_t *targets, int32_t mode, double *acc, double *pot);
/* FORCETEST's split (gravity_forcetest_evaluate, src/gravity/gravtree_forcetest.c:537-620) for the given
 * targets: acc_total/pot_total the correct direct-summation force and potential (spline-softened
 * Newtonian pairs plus, in a periodic box, the Ewald correction of every pair -- ftrue), and for a
 * TreePM context acc_short/pot_short the short-range part with the exact erfc factor (fsr, the best the
 * tree can deliver; the potential with the reference's constant M_total pi / (Asmth^2 V)), so that
 * ftrue - fsr is the long-range force the PM should deliver.  Any output may be NULL; the short-range
 * outputs need periodic with asmth > 0. */
int32_t gpugrav_direct_split(gpugrav_ctx *ctx, int64_t ntargets, const int64_t *targets, double *acc_total, double *pot_total,
                             double *acc_short, double *pot_short);

/* ---- small-N direct summation (gravity_direct, src/gravity/gravdirect.c:61-257) ----
 * What gravity() runs instead of the tree when fewer than DIRECT_SUMMATION_THRESHOLD particles are
 * active (src/gravity/accel.c:103-110): the n given particles (the active ones) attract each other,
 * every pair with force_evaluate_direct's arithmetic (src/gravity/forcetree_walk.c:557-708: tabulated
 * short-range factor for TreePM, Ewald correction for a periodic box without PM, spline softening),
 * summed in the given order -- FP64 results bit-identical to the reference's.  Accelerations without G
 * and potentials (pot may be NULL) in the given order; one particle gets zero force.  Uses the
 * context's parameters and replaces its loaded particles (load and build again before a walk). */
int32_t gpugrav_gravity_direct(gpugrav_ctx *ctx, int64_t n, const double *pos, const double *mass, const uint8_t *softtype,
                               double *acc, double *pot, int32_t mem);

/* ---- gravity time steps and time bins (src/time_integration/timestep.c) ----
 * get_timestep_gravity (timestep.c:284-353) for every particle, then the bin of
 * timebins_get_bin_and_do_validity_checks (timestep.c:725-770): the step rounded down to a power of two
 * of the integer timeline, raised only into synchronized bins, 0 at the end of the timeline.  Then the
 * list of active particles of a time bin (TimeBinsGravity.ActiveParticleList for the bins that are
 * synchronized now), ready for gpugrav_walk_targets.  Parameters are AREPO's All.* fields; the
 * softening lengths come from the context (ForceSoftening). */
typedef struct gpugrav_timestep_params
{
  double err_tol_int_accuracy;       /* All.ErrTolIntAccuracy */
  double cf_atime, cf_a2inv, cf_hubble_a; /* All.cf_* (1 without comoving integration) */
  double max_size_timestep;          /* All.MaxSizeTimestep */
  double min_size_timestep;          /* All.MinSizeTimestep */
  double dt_displacement;            /* All.DtDisplacement (PMGRID builds); 0: no such limit */
  double timebase_interval;          /* All.Timebase_interval */
  int64_t timebase;                  /* TIMEBASE of the build (1 << TIMEBINS) */
  int64_t ti_current;                /* All.Ti_Current */
  int32_t nostop_below_min;          /* NOSTOP_WHEN_BELOW_MINTIMESTEP: clamp instead of failing */
  int32_t pad;
  uint8_t synchronized[64];          /* TimeBinSynchronized[bin] */
} gpugrav_timestep_params;

/* grav_accel: n*3 accelerations as gravity_force_finalize leaves them (with G); grav_pm: n*3 (PMGRID) or
 * NULL; ids: P[].ID or NULL (a particle with mass 0 and ID 0 takes the maximum step); bin_old: the
 * current TimeBinGrav of each particle.  Outputs ti_step (integer steps before the power-of-two
 * rounding, as get_timestep_gravity returns them) and bin (the new TimeBinGrav).  Errors the reference
 * stops on: GPUGRAV_ERR_INVALID (a step below MinSizeTimestep without nostop_below_min, an integer step
 * outside (0, TIMEBASE), a step of integer size 1, a step beyond the end of the timeline); `failed`
 * (may be NULL) receives the first failing particle. */
int32_t gpugrav_timestep_gravity(gpugrav_ctx *ctx, const gpugrav_timestep_params *tp, int64_t n, const double *grav_accel,
                                 const double *grav_pm, const double *mass, const uint64_t *ids, const uint8_t *softtype,
                                 const int8_t *bin_old, int64_t *ti_step, int8_t *bin, int64_t *failed, int32_t mem);
/* Particles whose bin is synchronized (synchronized[bin] != 0), in index order: list (capacity n) and
 * their count. */
int32_t gpugrav_active_particles(gpugrav_ctx *ctx, int64_t n, const int8_t *bin, const uint8_t *synchronized, int32_t *list,
                                 int64_t *count, int32_t mem);

/* ---- serving loop: many independent isolated systems, continuously batched ----
 * Each submitted request is one isolated N-body system (G = 1 units of the params' softening table)
 * that runs what the reference runs on its first step and afterwards: a Barnes-Hut force pass
 * (err_tol_theta), a relative-criterion pass (err_tol_force_acc), then nsteps kick-drift-kick
 * leapfrog steps of size dt (kick_particle, src/time_integration/do_gravity_hydro.c:63-83;
 * drift_particle, src/time_integration/predict.c:357-425), with the FP32 walk.
 * Requests are admitted at tick boundaries in arrival order while system slots, the particle pool
 * and the device-memory budget allow; gpugrav_serve_tick advances every admitted system by one
 * force evaluation in one batched build and one persistent walk. Results stay in device memory
 * until polled. A serving handle has no internal lock: call it from one host thread at a time.
 * No counterpart in the reference (it integrates one system per run). */
typedef struct gpugrav_serve gpugrav_serve;

typedef struct gpugrav_serve_config
{
  int32_t abi_version;          /* GPUGRAV_ABI_VERSION */
  int32_t max_systems;          /* systems in flight at once (1 = one request at a time) */
  int64_t max_particles;        /* particle pool: particles in flight at once */
  int64_t memory_budget_bytes;  /* admission budget for the device footprint of the particles in flight (0: pool only) */
} gpugrav_serve_config;

typedef struct gpugrav_serve_stats
{
  int64_t submitted, admitted, completed, cancelled;
  int64_t waiting, running, in_flight_particles;
  int64_t ticks, particle_steps;  /* force evaluations x particles, summed over ticks */
  double last_tick_s;
  int64_t last_tick_particles;
  int32_t last_tick_systems;
  int32_t pad;
  int64_t graph_captures;  /* walk + store/kick captured as a CUDA graph (again after a buffer moved) */
  int64_t graph_replays;   /* ticks that launched the captured graph */
  /* cumulative seconds: admission (host packing + uploads), keys/sort/build/layout (device),
   * walk + store/kick (device), completion (downloads + unpacking) */
  double admit_s, build_s, walk_s, finish_s;
  int64_t interactions;  /* particle-node and particle-particle interactions of all walks */
  double keys_s, tree_s; /* parts of build_s: kick/drift + keys + sort + gather; octree build */
} gpugrav_serve_stats;

int32_t gpugrav_serve_create(gpugrav_serve **srv, int32_t device, const gpugrav_params *params,
                             const gpugrav_serve_config *cfg);
int32_t gpugrav_serve_destroy(gpugrav_serve *srv);
const char *gpugrav_serve_last_error(gpugrav_serve *srv);
/* host arrays, copied: pos, vel n*3; mass n; softtype n. id >= 0 (poll returns -1 for "none"). */
int32_t gpugrav_serve_submit(gpugrav_serve *srv, int64_t id, int64_t n, const double *pos, const double *vel,
                             const double *mass, const uint8_t *softtype, int32_t nsteps, double dt);
int32_t gpugrav_serve_cancel(gpugrav_serve *srv, int64_t id);
/* one force evaluation for every admitted system (admission first); n_active may be NULL */
int32_t gpugrav_serve_tick(gpugrav_serve *srv, int32_t *n_active);
/* oldest finished request: *id = -1 when none. With capacity < *n only id and n are returned and the
 * result stays queued. times (may be NULL): submit, admit, done (seconds, steady clock).
 * A finished request keeps its particles on the device (counted against the memory budget) until
 * it is polled; pos, vel, acc (host, n*3 each, any may be NULL) are then copied from the device. */
int32_t gpugrav_serve_poll(gpugrav_serve *srv, int64_t *id, int64_t *n, double *pos, double *vel, double *acc,
                           int64_t capacity, double *times);
int32_t gpugrav_serve_get_stats(gpugrav_serve *srv, gpugrav_serve_stats *stats);

/* ---- direct summation without allocation (no counterpart in the reference) ----
 * The same FP64 sum as gpugrav_direct, for callers that cannot allocate device memory at the point
 * of the call (their device memory belongs to their own pool allocator, or they cannot accept the
 * device-wide synchronisation of cudaMalloc/cudaFree mid-step). Needs no context: every array is the
 * caller's, in device memory of `device` -- pos (n*3), mass (n), softtype (n) of the sources, inside
 * the periodic box for periodic runs; target_pos (ntargets*3), target_softtype (ntargets); outputs
 * acc (ntargets*3) and pot (ntargets or NULL). Launches on `stream` (a cudaStream_t, NULL = default)
 * and returns without synchronising. At most 4096 targets per call (GPUGRAV_ERR_TOO_LARGE beyond);
 * its scratch is a fixed 4 MiB device array per GPU, held until exit and shared by all calls: calls
 * that overlap on the GPU race. The first call in a CUDA context (the device's primary context, or a
 * caller's own context made current on `device`) resolves the array's address in that context; make it
 * before any stream capture. Softening types must lie in [0, nsofttypes): a target of another type gets
 * NaN outputs, and a source of another type makes every pair it enters NaN. The parameters are checked
 * as gpugrav_create checks them; a periodic box needs asmth > 0 (the Ewald mode needs its tables, an
 * allocation). Allocates nothing (no cudaMalloc/cudaFree). */
int32_t gpugrav_direct_noalloc(int32_t device, const gpugrav_params *params, int64_t n, const double *pos,
                               const double *mass, const uint8_t *softtype, int64_t ntargets, const double *target_pos,
                               const uint8_t *target_softtype, int32_t mode, double *acc, double *pot, void *stream);

/* ---- diagnostics (no counterpart in the reference) ----
 * CUDA-core fused multiply-add throughput of `device` in TFLOP/s for GPUGRAV_PREC_FP32 or
 * GPUGRAV_PREC_FP64 (2 flops per FMA): the denominator of the tree walk's roofline. */
int32_t gpugrav_measure_fma_peak(int32_t device, int32_t precision, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* GPUGRAV_H */
