// internal.h -- shared definitions of libarepo_gpugrav (not part of the C ABI).
//
// Floating point on the parity path (keys, build, moments, FP64 walk) must
// round exactly like the reference's plain C doubles: the translation units
// that implement it are compiled with -fmad=false, and the helpers below spell
// out the IEEE operations where a contraction would otherwise be tempting.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/gpugrav.h"

// return a failing CUDA status from a cudaError_t function
#define GG_TRY(x)             \
  do                          \
    {                         \
      cudaError_t _e = (x);   \
      if(_e != cudaSuccess)   \
        return _e;            \
    }                         \
  while(0)

namespace gg
{
typedef unsigned __int128 u128;

constexpr int kBits         = 42;  // BITS_PER_DIMENSION (src/main/allvars.h:370-372)
constexpr int kMaxTreeLevel = 30;  // MAX_TREE_LEVEL (src/gravity/forcetree.h:106)
constexpr int kNtab         = GPUGRAV_NTAB;
constexpr int kMaxTop       = 4096;  // top-level nodes held in shared memory by the build kernels
constexpr int32_t kNodeFlag = 1 << 8;

// Per-build constants (small, read by every kernel): lives in device memory, copied to
// registers/shared memory by the kernels.
struct BuildConst
{
  gpugrav_domain dom;
  int64_t n;         // particles
  int32_t ntop;      // skeleton nodes (NTopnodes, root included)
  int32_t nleaves;   // NTopleaves
  int32_t periodic;
  int32_t nsoft;
  int32_t mns;       // MULTIPLE_NODE_SOFTENING: per-type node masses
  int32_t pad;
  double box;
  double soft[GPUGRAV_MAX_SOFTTYPES + 1];
};

// Walk constants
constexpr int kEwaldN = 64;  // EN of the Ewald correction tables (src/gravity/forcetree.h:90)

struct WalkConst
{
  int32_t periodic;  // nearest-image separations
  int32_t pm;        // TreePM split: Rcut prune and erfc table (periodic with Asmth > 0)
  int32_t ewald;     // pure periodic tree: Ewald correction per interaction (periodic without PM)
  int32_t mns;       // MULTIPLE_NODE_SOFTENING: nodes used per softening type
  int32_t nsoft;
  int32_t minangle;  // ACTIVATE_MINIMUM_OPENING_ANGLE: minimum opening angle in the relative criterion
  const double *w_mpt;  // FP64 walk: per-type masses of each walk entry (nodes), nsoft each
  double ewd_fac_intp;       // 2 EN / L
  const double *ewd;         // device tables fx | fy | fz | pot, (EN+1)^3 each
  int32_t bh;        // 1: Barnes-Hut criterion (ErrTolTheta > 0), 0: relative criterion
  double box, half_box;
  double theta;      // ErrTolTheta
  double erracc;     // ErrTolForceAcc
  double rcut, rcut2, asmthinv2, asmthfac;
  double soft[GPUGRAV_MAX_SOFTTYPES + 1];
  float tab_force[kNtab + 1];
  float tab_pot[kNtab + 1];
};

#ifdef __CUDACC__
// Ewald correction force and potential for the separation (dx, dy, dz) = source - target: trilinear
// interpolation of the octant tables with the sign flips of ewald_corr / ewald_pot_corr
// (src/gravity/forcetree_ewald.c:268-391), same operations in the same order (FP64).
__device__ __forceinline__ void ewald_corr(double dx, double dy, double dz, const WalkConst &w, double *fper, double &pcorr)
{
  constexpr int m = kEwaldN + 1;
  const size_t total = (size_t)m * m * m;
  int signx, signy, signz;
  if(dx < 0)
    {
      dx    = -dx;
      signx = +1;
    }
  else
    signx = -1;
  if(dy < 0)
    {
      dy    = -dy;
      signy = +1;
    }
  else
    signy = -1;
  if(dz < 0)
    {
      dz    = -dz;
      signz = +1;
    }
  else
    signz = -1;
  double u = dx * w.ewd_fac_intp;
  int i    = (int)u;
  if(i >= kEwaldN)
    i = kEwaldN - 1;
  u -= i;
  double v = dy * w.ewd_fac_intp;
  int j    = (int)v;
  if(j >= kEwaldN)
    j = kEwaldN - 1;
  v -= j;
  double ww = dz * w.ewd_fac_intp;
  int k     = (int)ww;
  if(k >= kEwaldN)
    k = kEwaldN - 1;
  ww -= k;
  const double f1 = (1 - u) * (1 - v) * (1 - ww), f2 = (1 - u) * (1 - v) * (ww), f3 = (1 - u) * (v) * (1 - ww),
               f4 = (1 - u) * (v) * (ww), f5 = (u) * (1 - v) * (1 - ww), f6 = (u) * (1 - v) * (ww), f7 = (u) * (v) * (1 - ww),
               f8 = (u) * (v) * (ww);
  const size_t b = ((size_t)i * m + j) * m + k;
  double r[4];
#pragma unroll
  for(int c = 0; c < 4; c++)
    {
      const double *t = w.ewd + c * total;
      r[c] = t[b] * f1 + t[b + 1] * f2 + t[b + m] * f3 + t[b + m + 1] * f4 + t[b + m * m] * f5 + t[b + m * m + 1] * f6 +
             t[b + m * m + m] * f7 + t[b + m * m + m + 1] * f8;
    }
  fper[0] = signx * r[0];
  fper[1] = signy * r[1];
  fper[2] = signz * r[2];
  pcorr   = r[3];
}
#endif

// Device buffer that only grows.
struct DevBuf
{
  void *p    = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes);
  void release();
  template <class T>
  T *as() const
  {
    return (T *)p;
  }
};

struct PinnedBuf
{
  void *p    = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes);
  void release();
};

}  // namespace gg

struct gpugrav_ctx
{
  int device            = 0;
  cudaStream_t stream   = nullptr;
  bool own_stream       = false;
  gpugrav_params prm{};
  std::string err;
  // GPUGRAV_PROFILE=1: host wall time per build step (the stream is synchronised after each step),
  // printed to stderr when the context is destroyed
  bool profile = false;
  std::map<std::string, double> prof;
  double prof_t = 0;
  void mark(const char *what);

  // ---- state ----
  int64_t n          = 0;
  bool loaded        = false;
  bool built         = false;
  int32_t ntop       = 0;  // skeleton nodes
  int32_t nleaves    = 0;
  int64_t num_nodes  = 0;  // total nodes (skeleton + dynamic)
  int64_t n_entries  = 0;  // walk entries = n + num_nodes
  int32_t max_depth  = 0;
  int32_t hack_cells = 0;
  gpugrav_domain dom{};
  std::vector<gpugrav_topnode> top_host;

  // ---- device buffers ----
  gg::DevBuf bconst, wconst;
  gg::DevBuf pos_in, mass_in, st_in;          // caller order
  gg::DevBuf key, key_alt, idx, perm;         // keys / sort
  gg::DevBuf sort_tmp;
  gg::DevBuf s_pm, s_ix, s_iy, s_iz, s_st;    // sorted SoA: (x,y,z,m) double4, 52-bit coordinates, softening type
  gg::DevBuf s_cd, s_tl, s_tlnode;            // pair depth, top-leaf depth / node
  gg::DevBuf cnt, base, hcnt, hack_list, hack_scratch, counters;
  gg::DevBuf top, skel;                       // top nodes, skeleton description
  gg::DevBuf n_suns, n_depth, n_cl, n_sm, n_maxsoft, n_size, n_father, n_sibling, n_next, n_dfs, n_first;
  gg::DevBuf n_mpt, w_mpt, g_mpt;             // MULTIPLE_NODE_SOFTENING: per-type node masses (node, walk, FP32 layouts)
  gg::DevBuf p_next, p_father, p_dfs;
  gg::DevBuf depth_hist, depth_order;
  gg::DevBuf w_sm, w_cl, w_link;              // walk layout (DFS order)
  // FP32 group walk: nodes in breadth-first order (children contiguous), particles grouped by parent
  gg::DevBuf g_key, g_key_alt, g_val, g_val_alt, g_bfs;   // (depth, dfs) sort -> breadth-first rank
  gg::DevBuf g_np, g_poff;                    // particle children per node (bfs order), their offsets
  gg::DevBuf g_sm, g_rel, g_kids;             // node: (CoM, mass) double4; (centre - CoM, len) float4; int4 links
  gg::DevBuf g_pm, g_pst;                     // particles in parent order: (x, y, z, m) double4; softening type
  gg::DevBuf g_stack;                         // per-warp traversal stacks
  gg::DevBuf g_groups, g_ngroups;             // walk groups (first, count, root, criterion), their count
  gg::DevBuf g_gpd, g_gseg, g_gflag, g_gid;   // group construction scratch
  gg::DevBuf t_cd, t_pd;                      // active list: pair depths of consecutive targets, their cell depths
  int32_t slice = 0, nslices = 1;             // target slice of the walks (gpugrav_set_target_slice)
  // active targets of the current walk (gpugrav_walk_targets): sorted particle positions in key order
  // (t_pos_alt) and their places in the caller's list (t_idx_alt); w_tlist is null for a walk of every particle
  gg::DevBuf iperm, t_in, t_pos, t_pos_alt, t_idx, t_idx_alt;
  const int32_t *w_tlist = nullptr;
  // cost-balanced slices (gpugrav_set_target_slice_cost): per-particle cost in caller order, per-unit
  // costs and their prefix sums, the slice range computed on the device
  gg::DevBuf cost_in, cost_u, cost_p, slice_rng;
  bool cost_set     = false;
  int64_t cost_n    = 0;
  bool slice_rng_on = false;
  int64_t w_ntargets     = 0;
  bool groups_active     = false;  // the FP32 group table describes an active list, not every particle
  // Ewald correction tables (ewald.cu): FP64 and float4 copies, scaled to ewd_box (or the caller's)
  gg::DevBuf ewd, ewd32;
  double ewd_box = 0;
  bool ewd_user  = false;
  // periodic PM long-range force (pm.cu): mesh size of the cuFFT plans, plans, meshes, particles
  int32_t pm_grid = 0, pm_plan_f = 0, pm_plan_b = 0;
  gg::DevBuf pm_rho, pm_rhok, pm_pos, pm_mass, pm_acc, pm_pot, pm_tab;
  int group_slack = 99;                       // group cuts between cells (< 64) or key order only (GPUGRAV_GROUP_SLACK)
  int active_slack = 2;                       // the same for groups of an active list (GPUGRAV_ACTIVE_GROUP_SLACK)
  bool layout32_valid = false;
  // several independent systems in one build (serving): system of each sorted particle, domain of
  // each system (walk groups never span two systems)
  bool multi = false;
  gg::DevBuf m_sys, m_doms;
  // FP32 walk launch plan (walk32_prepare)
  void *w32_kernel   = nullptr;
  int32_t w32_blocks = 0;
  bool want_pot       = true;  // potential requested by the current walk call
  int walk32_tpl      = 0;     // targets per lane of the group walk: 0 auto, 1 or 2 (GPUGRAV_WALK32_TPL)
  gg::DevBuf acc_s, pot_s, nint_s, oldacc_s, oldacc_in;  // per target (sorted), inputs
  gg::DevBuf out_acc, out_pot, out_nint;      // caller order staging for host copies
  gg::DevBuf scratch;                         // reductions
  gg::PinnedBuf pinned;

  cudaEvent_t ev[20] = {};
  gpugrav_timings timings{};
};

// depth of the deepest tree cell holding two particles, from their integer positions (52 bits per
// axis below the domain cube; 52 when they coincide)
__device__ __forceinline__ int common_depth(uint64_t ax, uint64_t ay, uint64_t az, uint64_t bx, uint64_t by, uint64_t bz)
{
  uint64_t d = (ax ^ bx) | (ay ^ by) | (az ^ bz);
  return d == 0 ? 52 : (__clzll((long long)d) - 12);
}

namespace gg
{
// launchers implemented in the .cu files; each returns cudaGetLastError() of its launches
cudaError_t domain_stage(gpugrav_ctx *c, bool compute_extent, int *out_of_box);
cudaError_t sort_stage(gpugrav_ctx *c);
cudaError_t gather_stage(gpugrav_ctx *c);
cudaError_t toptree_stage(gpugrav_ctx *c, int *status);
cudaError_t skeleton_stage(gpugrav_ctx *c, int *status);
cudaError_t build_stage(gpugrav_ctx *c, int *status);
cudaError_t walk64_stage(gpugrav_ctx *c, const WalkConst &wc);
cudaError_t walk32_stage(gpugrav_ctx *c, const WalkConst &wc);
cudaError_t walk32_prepare(gpugrav_ctx *c, const WalkConst &wc);
cudaError_t walk32_launch(gpugrav_ctx *c);
cudaError_t groups_stage(gpugrav_ctx *c);
cudaError_t timestep_stage(gpugrav_ctx *c, const gpugrav_timestep_params *tp, int64_t n, const double *acc, const double *pm,
                           const double *mass, const uint64_t *ids, const uint8_t *st, const int8_t *bin_old, int64_t *ti,
                           int8_t *bin, int *fail_code, int64_t *first);
cudaError_t active_stage(gpugrav_ctx *c, int64_t n, const int8_t *bin, const uint8_t *d_sync, int32_t *list, int64_t *d_count);
cudaError_t targets_stage(gpugrav_ctx *c, int64_t nt, const int32_t *d_targets, int *flags);
cudaError_t groups_active_stage(gpugrav_ctx *c, int64_t nt, int cap);
cudaError_t targets_scatter(gpugrav_ctx *c, int64_t nt, int64_t a, int64_t b, double *acc, double *pot, int32_t *nint);
cudaError_t slice_mask_stage(gpugrav_ctx *c, bool fp32);
cudaError_t slice_cost_stage(gpugrav_ctx *c, bool fp32);
const std::vector<double> &ewald_unit_table();
cudaError_t ewald_upload(gpugrav_ctx *c, const double *user);
cudaError_t ewald_ensure(gpugrav_ctx *c);
cudaError_t pm_stage(gpugrav_ctx *c, int pmgrid, int64_t np, const double *pos, const double *mass, double *acc, double *pot,
                     int *cufft_status);
void pm_release(gpugrav_ctx *c);
cudaError_t layout32_buffers(gpugrav_ctx *c, int64_t n, int64_t nn);
cudaError_t layout32_reserve(gpugrav_ctx *c, int64_t n, int64_t nn);
cudaError_t build_reserve(gpugrav_ctx *c, int64_t n, int64_t nn, int32_t ntop);
cudaError_t node_arrays(gpugrav_ctx *c, int64_t nn);
cudaError_t layout32_stage(gpugrav_ctx *c);
cudaError_t direct_stage(gpugrav_ctx *c, const WalkConst &wc, int64_t nt, const int64_t *d_targets, int cut, double *d_acc,
                         double *d_pot);
cudaError_t gravity_direct_stage(gpugrav_ctx *c, int64_t n, const double *d_pos, const double *d_mass, const uint8_t *d_st,
                                 double *d_acc, double *d_pot, int32_t *d_nint, int *d_flag);
void make_walk_const(const gpugrav_params &p, WalkConst *wc);
// targets per lane of the group walk (FP32, or its FP64 form; TreePM or isolated): by default 2 (groups
// of 64 targets) for one system and 1 for the serving loop's batched systems; GPUGRAV_WALK32_TPL=1 or 2
// forces either.  The Ewald walk and the per-target walk: 1.
inline int walk32_tpl(const gpugrav_ctx *c)
{
  const bool ewald = c->prm.periodic && !(c->prm.asmth > 0);
  const bool group = c->prm.precision == GPUGRAV_PREC_FP32 || c->prm.precision == GPUGRAV_PREC_FP64_GROUP;
  if(ewald || !group || c->walk32_tpl == 1)
    return 1;
  return (c->walk32_tpl == 2 || !c->multi) ? 2 : 1;
}
// GPUGRAV_OK or GPUGRAV_ERR_INVALID: ABI version, softening table (finite, >= 0, zero end entry),
// box size, TreePM split (asmth, rcut, rcut_cells > 0 unless asmth == 0), tolerances, flags
int validate_params(const gpugrav_params *p);
}  // namespace gg
