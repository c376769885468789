// walk32.cu -- FP32 group walk (the fast path).
//
// Physics as in force_treeevaluate (src/gravity/forcetree_walk.c:115-514): the
// tabulated erfc short-range factor cut at Rcut, the cubic-spline softening, the
// periodic nearest image, the relative criterion (ErrTolForceAcc x OldAcc) after
// a Barnes-Hut pass.  Different arithmetic organisation:
//
//  * a warp walks the tree for a group of 32 targets that are consecutive in key
//    order (compact in space); nodes are tested 32 at a time, one per lane,
//    against the group's bounding box with the reference's tests made
//    conservative for the whole group (a node is accepted only if every target of
//    the group would accept it), so each target's error is at most that of its
//    own reference walk;
//  * accepted nodes and the particles of opened nodes go to an interaction list
//    in shared memory; the list is evaluated densely -- every lane computes its
//    own target against every entry -- in FP32;
//  * separations: the group centre g is subtracted in FP64 from every list
//    entry and from every target before rounding to FP32, so an FP32 difference
//    never carries the absolute position (error ~ eps32 x |x - g|, not eps32 x |x|);
//  * sums: FP32 within a list batch, batch partials accumulated in FP64.
//
// Layout: nodes in breadth-first order with contiguous children (ranked by
// (depth, depth-first position)), particles grouped by parent node.
#include <cub/cub.cuh>

#include "internal.h"

namespace gg
{
namespace
{
#ifndef GG_W32_WARPS
#define GG_W32_WARPS 4
#endif
#ifndef GG_W32_EVAL_AT
#define GG_W32_EVAL_AT 192
#endif
#ifndef GG_W32_UNROLL
#define GG_W32_UNROLL 8
#endif
constexpr int kWarps   = GG_W32_WARPS;    // warps per block
constexpr int kEvalAt  = GG_W32_EVAL_AT;  // evaluate once this many entries are queued
#ifndef GG_W32_MINBLOCKS
#define GG_W32_MINBLOCKS 7  // blocks per SM the register budget is sized for (72 registers a thread, 31 KB of shared memory a block)
#endif
// two targets per lane: fewer entries in flight, 80 registers (6 blocks per SM, 35 KB of shared memory a block)
#ifndef GG_W32_UNROLL2
#define GG_W32_UNROLL2 4
#endif
#ifndef GG_W32_MINBLOCKS2
#define GG_W32_MINBLOCKS2 6
#endif
// list entries in flight per lane in the evaluation loop
template <int TPL>
constexpr int kUnroll = TPL == 2 ? GG_W32_UNROLL2 : GG_W32_UNROLL;
// capacity (Cap below): accepted nodes (<= 32) join a list holding fewer than kEvalAt entries;
// particles are added at most 32 per round and the list is evaluated first whenever a round could
// overflow it.  Entries inside some target's softening length go to a separate, smaller near list,
// evaluated as soon as it holds kNearAt entries.
constexpr int kNearAt = 64;
constexpr int kStackCap = 16384;  // traversal stack entries per warp (global memory)
// A node that the group-box test opens although it is smaller than 1/kVote of the box's largest side
// and nearer to the box than that is tested against every target of the group instead (opened
// only if some target's own criterion opens it).  For a compact group this never happens; for a
// group whose targets are far apart (outskirts of an isolated system, where consecutive targets
// in key order can lie on both sides of a dense core) the box test alone would open the whole
// core down to single particles.
constexpr float kVote = 16.0f;

// cubic-spline softening coefficients (src/main/allvars.h:557-573), rounded to the walk's type
#define SF1 10.666666666667
#define SF2 32.0
#define SF3 (-38.4)
#define SF4 (-2.8)
#define SF5 5.333333333333
#define SF6 6.4
#define SF7 (-9.6)
#define SF8 21.333333333333
#define SF9 (-48.0)
#define SF10 38.4
#define SF11 (-10.666666666667)
#define SF12 (-0.066666666667)
#define SF13 (-3.2)
#define SF14 0.066666666667
#define SF15 (-16.0)
#define SF16 9.6
#define SF17 (-2.133333333333)

// The arithmetic type R of the evaluation: float (the fast form) or double (the same group walk in
// FP64, the precision ablation of the fast form).  List capacities per type: double entries take
// twice the shared memory.
template <typename R>
struct Cap
{
  static constexpr int eval     = sizeof(R) == 4 ? kEvalAt : 96;
  static constexpr int list     = eval + 64;
  static constexpr int near_at  = sizeof(R) == 4 ? kNearAt : 32;
  static constexpr int near_cap = near_at + 32;
};
template <typename R>
struct V4T;
template <>
struct V4T<float>
{
  typedef float4 type;
};
template <>
struct V4T<double>
{
  typedef double4 type;
};
template <typename R>
using V4 = typename V4T<R>::type;
template <typename R>
__device__ __forceinline__ V4<R> mk4(double x, double y, double z, double m)
{
  V4<R> v;
  v.x = (R)x;
  v.y = (R)y;
  v.z = (R)z;
  v.w = (R)m;
  return v;
}
__device__ __forceinline__ float fmaR(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmaR(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float maxR(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double maxR(double a, double b) { return fmax(a, b); }

struct W32Const
{
  double box, half_box;
  float rcut, rcut2, asmthfac;
  float rcut2_all;  // an entry whose farthest distance from the group box is below this is inside Rcut of every target
  float theta2, erracc;
  int periodic, bh;
  float soft[GPUGRAV_MAX_SOFTTYPES + 1];
  float4 tab[kNtab + 1];  // (f[i], f[i+1] - f[i], p[i], p[i+1] - p[i]): force table times 1/Asmth^2, potential table
  const float4 *ewd;       // Ewald correction (fx, fy, fz, pot) per table entry (pure periodic tree)
  float ewd_fac;           // 2 EN / L
  int mns;                 // MULTIPLE_NODE_SOFTENING: nodes used per softening type
  const float *mpt;        // per-type node masses, breadth-first order, nsoft each
  int nsoft;
  int minangle;            // ACTIVATE_MINIMUM_OPENING_ANGLE
  // FP64 form only (the FP32 kernels do not copy these into shared memory)
  double rcut2_d, asmthfac_d;  // Rcut^2 and the table index factor in double
  double4 tab64[kNtab + 1];    // the table above in double
};
// bytes of the constants a kernel of arithmetic type R keeps in shared memory
template <typename R>
constexpr int kW32Bytes = sizeof(R) == 4 ? (int)offsetof(W32Const, rcut2_d) : (int)sizeof(W32Const);

// ------------------------------------------------------------------------------
// layout
// ------------------------------------------------------------------------------
__global__ void k_g_keys(int64_t nn, const uint8_t *__restrict__ depth, const int32_t *__restrict__ ndfs,
                         uint64_t *__restrict__ key, int32_t *__restrict__ val)
{
  for(int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nn; k += (int64_t)gridDim.x * blockDim.x)
    {
      key[k] = ((uint64_t)depth[k] << 32) | (uint32_t)ndfs[k];
      val[k] = (int32_t)k;
    }
}

__global__ void k_g_rank(int64_t nn, int64_t n, const int32_t *__restrict__ sorted, const int32_t *__restrict__ suns,
                         int32_t *__restrict__ bfs, int32_t *__restrict__ np)
{
  for(int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nn; b += (int64_t)gridDim.x * blockDim.x)
    {
      int32_t k = sorted[b];
      bfs[k]    = (int32_t)b;
      int c     = 0;
      for(int q = 0; q < 8; q++)
        {
          int32_t v = suns[8 * (int64_t)k + q];
          c += (v >= 0 && v < n) ? 1 : 0;
        }
      np[b] = c;
    }
}

__global__ void k_g_fill(int64_t nn, int64_t n, const int32_t *__restrict__ sorted, const int32_t *__restrict__ suns,
                         const int32_t *__restrict__ bfs, const int32_t *__restrict__ poff, const double4 *__restrict__ sm,
                         const double4 *__restrict__ cl, const uint8_t *__restrict__ maxsoft, const double4 *__restrict__ pm,
                         const uint8_t *__restrict__ st, double4 *__restrict__ g_sm, float4 *__restrict__ g_rel,
                         int4 *__restrict__ g_kids, double4 *__restrict__ g_pm, uint8_t *__restrict__ g_pst, int *err,
                         const double *__restrict__ mpt, int nsoft, float *__restrict__ g_mpt)
{
  for(int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nn; b += (int64_t)gridDim.x * blockDim.x)
    {
      int32_t k = sorted[b];
      double4 s = sm[k], c = cl[k];
      g_sm[b]   = s;
      g_rel[b]  = make_float4((float)(c.x - s.x), (float)(c.y - s.y), (float)(c.z - s.z), (float)c.w);
      int32_t fc = -1, nc = 0, npc = 0;
      int32_t fp = poff[b];
      for(int q = 0; q < 8; q++)
        {
          int32_t v = suns[8 * (int64_t)k + q];
          if(v < 0)
            continue;
          if(v < n)
            {
              g_pm[fp + npc]  = pm[v];
              g_pst[fp + npc] = st[v];
              npc++;
            }
          else
            {
              int32_t cb = bfs[v - n];
              if(fc < 0)
                fc = cb;
              else if(cb != fc + nc)
                atomicOr(err, 8);  // children must be contiguous in breadth-first order
              nc++;
            }
        }
      g_kids[b] = make_int4(fc, fp, nc | (npc << 4), (int)maxsoft[k]);
      if(g_mpt)
        for(int q = 0; q < nsoft; q++)
          g_mpt[b * nsoft + q] = (float)mpt[(int64_t)k * nsoft + q];
    }
}

// ------------------------------------------------------------------------------
// walk
// ------------------------------------------------------------------------------
__device__ __forceinline__ double wrapd(double d, const W32Const &w)
{
  if(!w.periodic)
    return d;
  return (d > w.half_box) ? d - w.box : ((d < -w.half_box) ? d + w.box : d);
}

__device__ __forceinline__ double wmin(double v)
{
  for(int o = 16; o > 0; o >>= 1)
    v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double wmax(double v)
{
  for(int o = 16; o > 0; o >>= 1)
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float wminf(float v)
{
  for(int o = 16; o > 0; o >>= 1)
    v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float wmaxf(float v)
{
  for(int o = 16; o > 0; o >>= 1)
    v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int wscan_incl(int v, int lane)
{
  for(int o = 1; o < 32; o <<= 1)
    {
      int u = __shfl_up_sync(0xffffffffu, v, o);
      if(lane >= o)
        v += u;
    }
  return v;
}

// Reciprocal square root of a normal (never subnormal) argument: the hardware approximation
// without the subnormal handling that a general rsqrtf needs (the walk clamps r^2 >= 1e-30).
__device__ __forceinline__ float rsqrt_normal(float x)
{
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float rsqrtR(float x) { return rsqrt_normal(x); }
__device__ __forceinline__ double rsqrtR(double x) { return rsqrt(x); }
__device__ __forceinline__ float rcut2_of(const W32Const &w, float) { return w.rcut2; }
__device__ __forceinline__ double rcut2_of(const W32Const &w, double) { return w.rcut2_d; }

// Short-range factors of the TreePM split at separation r: linear interpolation of the force
// (scaled by 1/Asmth^2) and potential tables between nodes floor(te) and floor(te) + 1,
// te = r * asmthfac, as the reference does (src/gravity/forcetree_walk.c:366-379).  Adding 1.5 * 2^23 with rounding toward minus
// infinity leaves floor(te) in the low mantissa bits (no conversion instruction).  CLAMP: the index
// is clamped to the last interval, which only entries beyond Rcut reach (they are masked); without
// CLAMP the entry is inside Rcut, so floor(te) <= NTAB (the table has NTAB + 1 rows).
template <bool CLAMP = true>
__device__ __forceinline__ void short_range(float r, const W32Const &w, float &ff, float &fpt)
{
  const float tr  = __fmaf_rd(r, w.asmthfac, 12582912.0f);
  const float tb0 = CLAMP ? fminf(tr, 12582912.0f + (float)(kNtab - 1)) : tr;
  const float tw  = fmaf(r, w.asmthfac, 12582912.0f - tb0);
  const float4 t  = w.tab[__float_as_int(tb0) - 0x4B400000];
  ff              = fmaf(tw, t.y, t.x);
  fpt             = fmaf(tw, t.w, t.z);
}
// the same in double: floor(te) by conversion
template <bool CLAMP = true>
__device__ __forceinline__ void short_range(double r, const W32Const &w, double &ff, double &fpt)
{
  const double te = r * w.asmthfac_d;
  int i           = (int)te;
  if(CLAMP)
    i = min(i, kNtab - 1);
  const double tw = te - i;
  const double4 t = w.tab64[i];
  ff              = fma(tw, t.y, t.x);
  fpt             = fma(tw, t.w, t.z);
}

// Per-target state of a lane (targets per lane: TPL).
template <typename R>
struct Tgt
{
  R x, y, z, h;             // position relative to the group centre, softening
  R ax, ay, az, pot;        // partial sums of the current list batch (folded into FP64 sums in shared memory)
  int ni;
};

// Ewald correction (force, potential) for the separation (dx, dy, dz) = source - target:
// the trilinear interpolation and sign flips of ewald_corr (src/gravity/forcetree_ewald.c:268-342)
// in FP32 on the float4 table.
__device__ __forceinline__ float4 ewald_corr32(float dx, float dy, float dz, const W32Const &w)
{
  constexpr int m = kEwaldN + 1;
  const float sx = dx < 0.0f ? 1.0f : -1.0f, sy = dy < 0.0f ? 1.0f : -1.0f, sz = dz < 0.0f ? 1.0f : -1.0f;
  float u = fabsf(dx) * w.ewd_fac, v = fabsf(dy) * w.ewd_fac, s = fabsf(dz) * w.ewd_fac;
  const int i = min((int)u, kEwaldN - 1), j = min((int)v, kEwaldN - 1), k = min((int)s, kEwaldN - 1);
  u -= i;
  v -= j;
  s -= k;
  const float4 *t = w.ewd + ((i * m + j) * m + k);
  const float4 a0 = __ldg(t), a1 = __ldg(t + 1), a2 = __ldg(t + m), a3 = __ldg(t + m + 1);
  const float4 b0 = __ldg(t + m * m), b1 = __ldg(t + m * m + 1), b2 = __ldg(t + m * m + m), b3 = __ldg(t + m * m + m + 1);
  const float f1 = (1 - u) * (1 - v) * (1 - s), f2 = (1 - u) * (1 - v) * s, f3 = (1 - u) * v * (1 - s), f4 = (1 - u) * v * s;
  const float f5 = u * (1 - v) * (1 - s), f6 = u * (1 - v) * s, f7 = u * v * (1 - s), f8 = u * v * s;
  float4 r;
  r.x = a0.x * f1 + a1.x * f2 + a2.x * f3 + a3.x * f4 + b0.x * f5 + b1.x * f6 + b2.x * f7 + b3.x * f8;
  r.y = a0.y * f1 + a1.y * f2 + a2.y * f3 + a3.y * f4 + b0.y * f5 + b1.y * f6 + b2.y * f7 + b3.y * f8;
  r.z = a0.z * f1 + a1.z * f2 + a2.z * f3 + a3.z * f4 + b0.z * f5 + b1.z * f6 + b2.z * f7 + b3.z * f8;
  r.w = a0.w * f1 + a1.w * f2 + a2.w * f3 + a3.w * f4 + b0.w * f5 + b1.w * f6 + b2.w * f7 + b3.w * f8;
  return make_float4(sx * r.x, sy * r.y, sz * r.z, r.w);
}

// Separation of a list entry from a target: (dx, dy, dz) = entry - target, r^2, 1/r and r.  A zero
// separation (the target itself) gives a huge 1/r but r = 0 (CLAMP); it lies inside the softening
// length unless that is zero, where the reference's kernel has no finite value either.  far() and
// near() both call this, so they agree on which side of the softening length every pair lies.
template <typename R>
struct Sep
{
  R dx, dy, dz, r2, rinv, r;
};
template <typename R, bool CLAMP = true>
__device__ __forceinline__ Sep<R> separation(const V4<R> e, const Tgt<R> &T)
{
  Sep<R> s;
  s.dx   = e.x - T.x;
  s.dy   = e.y - T.y;
  s.dz   = e.z - T.z;
  s.r2   = fmaR(s.dx, s.dx, fmaR(s.dy, s.dy, s.dz * s.dz));
  s.rinv = rsqrtR(CLAMP ? maxR(s.r2, (R)(sizeof(R) == 4 ? 1.0e-30 : 1.0e-60)) : s.r2);
  s.r    = s.r2 * s.rinv;
  return s;
}

// One target against one list entry, outside the softening length (r >= max(h_i, h_j)): the
// Newtonian kernel, times the TreePM short-range factor when PERIODIC.  MASK: an entry beyond Rcut
// of this target (periodic) is masked, not branched around, so that the interactions of an unrolled
// block schedule together, and the pair is counted only inside Rcut; without MASK the entry is known
// to lie inside Rcut of every target of the group and its interactions are counted per list region.
// CHECK: the entry may lie inside the softening length of this target; such a pair is masked as well
// and reported by the return value, and near() adds the spline kernel for it.  Without CHECK the list
// entry is known to lie outside the softening length of every target of the group.  The Ewald
// correction (EWALD: pure periodic tree, nearest image) is taken here for every pair.
template <typename R, bool PERIODIC, bool POT, bool EWALD = false, bool CHECK = true, bool MASK = true>
__device__ __forceinline__ bool far(const V4<R> e, const R hj, Tgt<R> &T, const W32Const &w)
{
  constexpr bool PAIRWISE = MASK || CHECK;  // Rcut mask and count per pair
  // outside every target's softening length (no CHECK) r > 0 unless the softening is zero
  const Sep<R> s = separation<R, CHECK>(e, T);
  bool in        = true;
  R ff = 0, fpt = 0;
  if(PERIODIC)
    {
      if(PAIRWISE)
        in = s.r2 < rcut2_of(w, R(0));
      short_range<PAIRWISE>(s.r, w, ff, fpt);
    }
  // force m (1/r^3 + f_s / (r Asmth^2)) = (m/r) (1/r^2 + f_s'), potential (m/r) p_s (Newtonian: -m/r);
  // 1/r^2 stays finite at the clamped r = 0, so masking m/r masks both
  const bool soft = CHECK && s.r < maxR(T.h, hj);
  const R m       = in ? e.w : R(0);
  const R mr      = soft ? R(0) : m * s.rinv;
  const R fm      = mr * (PERIODIC ? fmaR(s.rinv, s.rinv, ff) : s.rinv * s.rinv);
  T.ax            = fmaR(s.dx, fm, T.ax);
  T.ay            = fmaR(s.dy, fm, T.ay);
  T.az            = fmaR(s.dz, fm, T.az);
  if(POT)
    T.pot = PERIODIC ? fmaR(mr, fpt, T.pot) : T.pot - mr;
  if(EWALD)
    {
      const float4 c = ewald_corr32((float)s.dx, (float)s.dy, (float)s.dz, w);
      T.ax           = fmaR(m, (R)c.x, T.ax);
      T.ay           = fmaR(m, (R)c.y, T.ay);
      T.az           = fmaR(m, (R)c.z, T.az);
      if(POT)
        T.pot = fmaR(m, (R)c.w, T.pot);
    }
  if(PAIRWISE)
    T.ni += in ? 1 : 0;  // list entries all have mass != 0
  return soft;
}

// The softened kernel of one target against one list entry, for a pair inside the softening length
// (nothing otherwise): the reference's spline (src/gravity/forcetree_walk.c:421-455), plus the
// TreePM short-range correction of the Newtonian part away from r = 0.
template <typename R, bool PERIODIC, bool POT>
__device__ __forceinline__ void near(const V4<R> e, const R hj, Tgt<R> &T, const W32Const &w)
{
  const Sep<R> s = separation<R>(e, T);
  const R hmax   = maxR(T.h, hj);
  if(!(s.r < hmax))
    return;
  const R h_inv  = R(1) / hmax;
  const R h3_inv = h_inv * h_inv * h_inv;
  const R u      = s.r * h_inv;
  const R u2     = u * u;
  R fac, wp = 0;
  if(u < R(0.5))
    {
      fac = h3_inv * fmaR(u2, fmaR((R)SF2, u, (R)SF3), (R)SF1);
      if(POT)
        wp = h_inv * fmaR(u2, fmaR(u2, fmaR((R)SF6, u, (R)SF7), (R)SF5), (R)SF4);
    }
  else
    {
      const R u3 = u2 * u;
      fac = h3_inv * ((R)SF8 + (R)SF9 * u + (R)SF10 * u2 + (R)SF11 * u3 + (R)SF12 / u3);
      if(POT)
        wp = h_inv * ((R)SF13 + (R)SF14 / u + u2 * ((R)SF1 + u * ((R)SF15 + u * ((R)SF16 + (R)SF17 * u))));
    }
  bool in = true;
  if(PERIODIC)
    {
      in = s.r2 < rcut2_of(w, R(0));
      if(s.r > R(0))
        {
          R ff, fpt;
          short_range(s.r, w, ff, fpt);
          fac = fmaR(s.rinv, ff, fac);
          if(POT)
            wp = fmaR(s.rinv, fpt + R(1), wp);
        }
    }
  const R m  = in ? e.w : R(0);
  const R fm = fac * m;
  T.ax       = fmaR(s.dx, fm, T.ax);
  T.ay       = fmaR(s.dy, fm, T.ay);
  T.az       = fmaR(s.dz, fm, T.az);
  if(POT)
    T.pot = fmaR(m, wp, T.pot);
}

#ifdef GG_WALK32_STATS
}  // namespace
// measurement build only: [0] list entries evaluated per lane, [1] node tests, [2] particle candidates,
// [3] groups, [4] entries inside Rcut of every target, [5] border entries, [6] warp steps, [7] steps
// with a per-target vote, [8] voting nodes, [9] particle rounds, [10] list evaluations
constexpr int kWalkStats = 12;
__device__ unsigned long long g_walk_stats[kWalkStats];
namespace
{
#define WALK_STAT(i, v)                       \
  do                                          \
    {                                         \
      if((threadIdx.x & 31) == 0)             \
        atomicAdd(&g_walk_stats[i], (unsigned long long)(v)); \
    }                                         \
  while(0)
#else
#define WALK_STAT(i, v) \
  do                    \
    {                   \
    }                   \
  while(0)
#endif

// The lane's TPL targets against one region of the warp's list (each entry read once for all of
// them), in blocks of kUnroll entries evaluated without branches.  CHECK (near list): a block in
// which some pair lies inside the softening length (the targets' own particles, close neighbours)
// is revisited for those pairs.  MASK: per-pair Rcut mask and count (see far()).
template <typename R, bool PERIODIC, bool POT, int TPL, bool EWALD, bool CHECK, bool MASK>
__device__ __forceinline__ void evaluate_region(const V4<R> *__restrict__ LP, const R *__restrict__ LH, int nl, Tgt<R> (&T)[TPL],
                                                const W32Const &w)
{
  int j = 0;
  constexpr int U = kUnroll<TPL>;
  for(; j + U <= nl; j += U)
    {
      V4<R> e[U];
      R hj[U];
#pragma unroll
      for(int u = 0; u < U; u++)
        {
          e[u]  = LP[j + u];
          hj[u] = CHECK ? LH[j + u] : R(0);
        }
      bool soft = false;
#pragma unroll
      for(int u = 0; u < U; u++)
#pragma unroll
        for(int k = 0; k < TPL; k++)
          soft |= far<R, PERIODIC, POT, EWALD, CHECK, MASK>(e[u], hj[u], T[k], w);
      if(CHECK && soft)
        {
#pragma unroll 1
          for(int u = 0; u < U; u++)
            {
              const V4<R> eu = LP[j + u];
              const R hu     = LH[j + u];
#pragma unroll
              for(int k = 0; k < TPL; k++)
                near<R, PERIODIC, POT>(eu, hu, T[k], w);
            }
        }
    }
  for(; j < nl; j++)
    {
      const V4<R> e = LP[j];
      const R hj    = CHECK ? LH[j] : R(0);
#pragma unroll
      for(int k = 0; k < TPL; k++)
        if(far<R, PERIODIC, POT, EWALD, CHECK, MASK>(e, hj, T[k], w) && CHECK)
          near<R, PERIODIC, POT>(e, hj, T[k], w);
    }
}

// The warp's interaction list in shared memory.  Main buffer: entries outside the softening length of
// every target of the group, those inside Rcut of every target at the bottom (growing up, `na`),
// the others at the top (growing down, `nb`).  Near buffer (`nn`): entries inside some target's
// softening length, with their softening lengths.
template <typename R>
struct List
{
  V4<R> *P;
  V4<R> *NP;
  R *NH;
  int na, nb, nn;
};

// Evaluates and empties the list, then folds the batch partials into the lane's FP64 sums (shared
// memory, dsum[(4k + c) * 32] for target k and component c = x, y, z, potential).
template <typename R, bool PERIODIC, bool POT, int TPL, bool EWALD = false>
__device__ __forceinline__ void evaluate(List<R> &L, Tgt<R> (&T)[TPL], double *dsum, const W32Const &w)
{
  WALK_STAT(4, L.na);
  WALK_STAT(5, L.nb);
  evaluate_region<R, PERIODIC, POT, TPL, EWALD, false, false>(L.P, nullptr, L.na, T, w);
  evaluate_region<R, PERIODIC, POT, TPL, EWALD, false, true>(L.P + Cap<R>::list - L.nb, nullptr, L.nb, T, w);
  evaluate_region<R, PERIODIC, POT, TPL, EWALD, true, true>(L.NP, L.NH, L.nn, T, w);
#pragma unroll
  for(int k = 0; k < TPL; k++)
    {
      T[k].ni += L.na;
      dsum[(4 * k + 0) * 32] += T[k].ax;
      dsum[(4 * k + 1) * 32] += T[k].ay;
      dsum[(4 * k + 2) * 32] += T[k].az;
      if(POT)
        dsum[(4 * k + 3) * 32] += T[k].pot;
      T[k].ax = T[k].ay = T[k].az = T[k].pot = R(0);
    }
  L.na = L.nb = L.nn = 0;
}

// true when a push round of up to 32 entries could overflow a buffer
template <typename R>
__device__ __forceinline__ bool list_full(const List<R> &L)
{
  return L.na + L.nb + 32 > Cap<R>::list || L.nn + 32 > Cap<R>::near_cap;
}

// Appends one entry per lane that keeps one to the warp's list.  The entry (x, y, z relative to the
// group centre, mass) lies at squared distance d2 from the nearest point of the group box (half
// extents bx, by, bz); hn is the larger of the group's largest softening (with margin) and the
// entry's own.  Closer than hn: near list.  Otherwise, when its farthest distance from the box is
// below Rcut (with margin) or there is no Rcut: inside Rcut of every target; else the border region.
template <typename R, bool PERIODIC>
__device__ __forceinline__ void push(List<R> &L, bool keep, const V4<R> e, R h, float d2, float hn, float bx, float by, float bz,
                                     const W32Const &w, unsigned lt_mask)
{
  int cls = 2;
  if(!(d2 < hn * hn))
    {
      cls = 0;
      if(PERIODIC)
        {
          const float fx = fabsf((float)e.x) + bx, fy = fabsf((float)e.y) + by, fz = fabsf((float)e.z) + bz;
          cls = (fmaf(fx, fx, fmaf(fy, fy, fz * fz)) < w.rcut2_all) ? 0 : 1;
        }
    }
  const unsigned ka = __ballot_sync(0xffffffffu, keep && cls == 0), kb = __ballot_sync(0xffffffffu, keep && cls == 1),
                 kn = __ballot_sync(0xffffffffu, keep && cls == 2);
  if(keep)
    {
      if(cls == 0)
        L.P[L.na + __popc(ka & lt_mask)] = e;
      else if(cls == 1)
        L.P[Cap<R>::list - 1 - (L.nb + __popc(kb & lt_mask))] = e;
      else
        {
          const int q = L.nn + __popc(kn & lt_mask);
          L.NP[q]     = e;
          L.NH[q]     = h;
        }
    }
  L.na += __popc(ka);
  L.nb += __popc(kb);
  L.nn += __popc(kn);
}

// A warp's group: centre (FP64), half extents, smallest and (with margin) largest target softening,
// smallest ErrTolForceAcc x |OldAcc|, and the per-target vote's squared size bound.
struct GroupSh
{
  double gx, gy, gz;
  float ex, ey, ez, h_min, h_grp, aold_min, vote_r2;
};

template <bool PERIODIC, bool POT, int TPL, bool EWALD = false, typename R = float>
__global__ void __launch_bounds__(32 * kWarps, sizeof(R) == 4 ? (TPL == 2 ? GG_W32_MINBLOCKS2 : GG_W32_MINBLOCKS) : 3) k_walk32(const double4 *__restrict__ g_sm, const float4 *__restrict__ g_rel,
                                                        const int4 *__restrict__ g_kids, const double4 *__restrict__ g_pm,
                                                        const uint8_t *__restrict__ g_pst, const double4 *__restrict__ tpm,
                                                        const uint8_t *__restrict__ tst, const float *__restrict__ oldacc,
                                                        const int *__restrict__ ngroups_dev, const int4 *__restrict__ groups,
                                                        const int32_t *__restrict__ tlist, int slice, int nslices,
                                                        const int64_t *__restrict__ slice_rng,
                                                        const W32Const *__restrict__ wcp,
                                                        int *__restrict__ stack_base, int *__restrict__ work,
                                                        double *__restrict__ acc_out, double *__restrict__ pot_out,
                                                        int32_t *__restrict__ nint_out, unsigned long long *__restrict__ total,
                                                        int *__restrict__ err)
{
  __shared__ __align__(16) unsigned char w_raw[kW32Bytes<R>];
  const W32Const &w = *reinterpret_cast<const W32Const *>(w_raw);
  __shared__ V4<R> il_p[kWarps][Cap<R>::list];
  __shared__ V4<R> il_np[kWarps][Cap<R>::near_cap];
  __shared__ R il_nh[kWarps][Cap<R>::near_cap];
  // cold per-lane and per-warp state kept out of registers: the FP64 sums of the lanes' targets,
  // ErrTolForceAcc x |OldAcc| of the targets (read by the per-target vote), the warp's interaction total
  __shared__ double dsum_sh[kWarps][4 * TPL][32];
  __shared__ float aold_sh[kWarps][32 * TPL];
  __shared__ unsigned long long total_sh[kWarps];
  __shared__ GroupSh group_sh[kWarps];
  static_assert(kW32Bytes<R> % 4 == 0, "constants copied in 4-byte words");
  for(int t = threadIdx.x; t < kW32Bytes<R> / 4; t += blockDim.x)
    ((int *)w_raw)[t] = ((const int *)wcp)[t];
  __syncthreads();

  const int warp         = threadIdx.x >> 5;
  const int lane         = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  int *stack             = stack_base + ((int64_t)blockIdx.x * kWarps + warp) * kStackCap;
  List<R> L;
  L.P  = il_p[warp];
  L.NP = il_np[warp];
  L.NH = il_nh[warp];
  double *dsum = &dsum_sh[warp][0][lane];
  if(lane == 0)
    total_sh[warp] = 0;
  // groups of this target slice; the count lives on the device (no host round trip, graph replays)
  const int64_t ng       = *ngroups_dev;
  // (or the cost-balanced range computed on the device, slice_rng[0..1])
  const int g_begin = slice_rng ? (int)slice_rng[0] : (int)(ng * slice / nslices);
  const int g_end   = slice_rng ? (int)slice_rng[1] : (int)(ng * (slice + 1) / nslices);

  while(true)
    {
      int grp = 0;
      if(lane == 0)
        grp = atomicAdd(work, 1);
      grp = g_begin + __shfl_sync(0xffffffffu, grp, 0);
      if(grp >= g_end)
        break;
      // group of up to 32*TPL consecutive targets; lane holds targets t0 + lane + 32k.  A group lies
      // inside one system and walks that system's tree (root).
      const int4 G       = groups[grp];
      const int64_t t0   = G.x;
      const int cnt      = G.y;
      const int root     = G.z;
      const int bh       = G.w >= 0 ? G.w : w.bh;
      WALK_STAT(3, 1);
      double4 p[TPL];
      double mnx = 1e300, mxx = -1e300, mny = 1e300, mxy = -1e300, mnz = 1e300, mxz = -1e300;
      float hmin_l = 3.0e38f, hmax_l = 0.0f, amin_l = 3.0e38f;
#pragma unroll
      for(int k = 0; k < TPL; k++)
        {
          const int s      = lane + 32 * k;
          // idle slots repeat the group's first target; a group of active targets (tlist) holds
          // consecutive entries of the active list
          const int64_t tt = tlist ? (int64_t)tlist[t0 + (s < cnt ? s : 0)] : t0 + (s < cnt ? s : 0);
          p[k]             = tpm[tt];
          const float a_l  = w.erracc * oldacc[tt];
          aold_sh[warp][s] = a_l;
          mnx = fmin(mnx, p[k].x), mxx = fmax(mxx, p[k].x);
          mny = fmin(mny, p[k].y), mxy = fmax(mxy, p[k].y);
          mnz = fmin(mnz, p[k].z), mxz = fmax(mxz, p[k].z);
          hmin_l = fminf(hmin_l, w.soft[tst[tt]]);
          hmax_l = fmaxf(hmax_l, w.soft[tst[tt]]);
          amin_l = fminf(amin_l, a_l);
        }
      // group box (FP64), centre g, half extent (rounded up)
      mnx = wmin(mnx), mxx = wmax(mxx), mny = wmin(mny), mxy = wmax(mxy), mnz = wmin(mnz), mxz = wmax(mxz);
      {
        GroupSh g;
        g.gx = 0.5 * (mnx + mxx), g.gy = 0.5 * (mny + mxy), g.gz = 0.5 * (mnz + mxz);
        g.ex = (float)(0.5 * (mxx - mnx)) * 1.000001f, g.ey = (float)(0.5 * (mxy - mny)) * 1.000001f,
        g.ez = (float)(0.5 * (mxz - mnz)) * 1.000001f;
        g.h_min = wminf(hmin_l);
        // an entry farther than max(h_grp, h_j) from the group box is outside the softening length of
        // every target (the margin covers the rounding of the FP32 separations)
        g.h_grp    = wmaxf(hmax_l) * 1.001f;
        g.aold_min = wminf(amin_l);
        // box side squared over kVote^2: a node smaller than this and closer than it gets the per-target vote
        const float side = 2.0f * fmaxf(g.ex, fmaxf(g.ey, g.ez));
        g.vote_r2        = side * side * (1.0f / (kVote * kVote));
        if(lane == 0)
          group_sh[warp] = g;
      }
      __syncwarp();
      // the group's constants are read from shared memory where they are used (out of registers)
      const GroupSh &gs = group_sh[warp];
      const double &gx = gs.gx, &gy = gs.gy, &gz = gs.gz;
      const float &ex = gs.ex, &ey = gs.ey, &ez = gs.ez, &h_min = gs.h_min, &h_grp = gs.h_grp, &aold_min = gs.aold_min,
                  &vote_r2 = gs.vote_r2;
      Tgt<R> T[TPL];
#pragma unroll
      for(int k = 0; k < TPL; k++)
        {
          T[k].x = (R)(p[k].x - gx), T[k].y = (R)(p[k].y - gy), T[k].z = (R)(p[k].z - gz);
          const int sk = lane + 32 * k < cnt ? lane + 32 * k : 0;
          T[k].h       = (R)w.soft[tst[tlist ? (int64_t)tlist[t0 + sk] : t0 + sk]];
          T[k].ax = T[k].ay = T[k].az = T[k].pot = R(0);
#pragma unroll
          for(int c = 0; c < 4; c++)
            dsum[(4 * k + c) * 32] = 0.0;
          T[k].ni = 0;
        }

      int sp = 1;
      L.na = L.nb = L.nn = 0;
      if(lane == 0)
        stack[0] = root;
      __syncwarp();

      // The walk is a loop over warp-uniform work items, so that the list evaluation has a single
      // (inlined) site: a pending softening-type entry of MULTIPLE_NODE_SOFTENING nodes (t_next <
      // t_end), a pending round of up to 32 particles of opened nodes (q0 < ptot), or a step over
      // up to 32 stack nodes.  The list is evaluated first when the next item could overflow it,
      // when it is full enough at a node step, and at the end.
      int t_next = 0, t_end = 0;  // MULTIPLE_NODE_SOFTENING entries of the last node step
      int q0 = 0, ptot = 0;       // particle rounds of the last node step
      // per-lane state of the last node step, read by the pending items
      int node = -1, action = 0, fp = 0, pinc = 0, pexc = 0;
      bool split = false;
      V4<R> entry  = mk4<R>(0, 0, 0, 0);
      float ent_d2 = 0.0f;  // squared distance of the entry from the group box
      while(true)
        {
          const int queued = L.na + L.nb + L.nn;
          const bool flush = (t_next < t_end || q0 < ptot) ? list_full(L)
                                                           : (sp > 0 ? (queued >= Cap<R>::eval || L.nn >= Cap<R>::near_at)
                                                                     : queued > 0);
          if(flush)
            {
              WALK_STAT(0, queued);
              WALK_STAT(10, 1);
              evaluate<R, PERIODIC, POT, TPL, EWALD>(L, T, dsum, w);
              __syncwarp();
            }
          if(t_next < t_end)
            {
              // MULTIPLE_NODE_SOFTENING: one entry per softening type with that type's mass and softening
              // (forcetree_walk.c:382-401); for a target whose own softening exceeds the node's largest
              // this equals the single entry, the kernel being linear in the mass
              const int t    = t_next++;
              const float mt = (action == 1 && split) ? w.mpt[(int64_t)node * w.nsoft + t] : 0.0f;
              push<R, PERIODIC>(L, mt != 0.0f, mk4<R>(entry.x, entry.y, entry.z, mt), (R)w.soft[t], ent_d2,
                                fmaxf(h_grp, w.soft[t]), ex, ey, ez, w, lt_mask);
              continue;
            }
          if(q0 < ptot)
            {
              // particles of opened nodes -> list, one particle per lane per round; particles beyond
              // Rcut of the whole group are dropped
              const int q = q0 + lane;
              q0 += 32;
              WALK_STAT(9, 1);
              int owner = 0;  // owner lane: number of lanes whose inclusive prefix is <= q
#pragma unroll
              for(int s = 16; s >= 1; s >>= 1)
                {
                  const int v = __shfl_sync(0xffffffffu, pinc, owner + s - 1);
                  if(v <= q)
                    owner += s;
                }
              owner          = owner < 31 ? owner : 31;
              const int ofp  = __shfl_sync(0xffffffffu, fp, owner);
              const int oexc = __shfl_sync(0xffffffffu, pexc, owner);
              bool keep      = false;
              V4<R> pe       = mk4<R>(0, 0, 0, 0);
              float ph = 0, pd2 = 0;
              if(q < ptot)
                {
                  const int pi     = ofp + (q - oexc);
                  const double4 pp = g_pm[pi];
                  pe   = mk4<R>(wrapd(pp.x - gx, w), wrapd(pp.y - gy, w), wrapd(pp.z - gz, w), pp.w);
                  ph   = w.soft[g_pst[pi]];
                  keep = pp.w != 0.0;
                  const float dmx = fmaxf(fabsf((float)pe.x) - ex, 0.0f), dmy = fmaxf(fabsf((float)pe.y) - ey, 0.0f),
                              dmz = fmaxf(fabsf((float)pe.z) - ez, 0.0f);
                  pd2 = dmx * dmx + dmy * dmy + dmz * dmz;
                  if(PERIODIC)
                    keep = keep && pd2 < w.rcut2;
                }
              push<R, PERIODIC>(L, keep, pe, (R)ph, pd2, fmaxf(h_grp, ph), ex, ey, ez, w, lt_mask);
              continue;
            }
          if(sp == 0)
            break;

          // ---- node step: up to 32 stack nodes, one per lane ----
          const int take = sp < 32 ? sp : 32;
          sp -= take;
          WALK_STAT(1, take);
          WALK_STAT(6, 1);
          node = -1;
          if(lane < take)
            node = stack[sp + lane];
          __syncwarp();

          action = 0;  // 1 accept, 2 open
          entry  = mk4<R>(0, 0, 0, 0);
          ent_d2 = 0.0f;
          split  = false;  // MULTIPLE_NODE_SOFTENING: accepted node listed per type
          float hj = 0;
          int fc = 0, nc = 0, np = 0;
          fp = 0;
          bool vote = false, vote_keep = false;  // per-target vote pending; entry kept if accepted
          float4 vrel = make_float4(0, 0, 0, 0);   // centre - CoM, side of a voting node
          if(node >= 0)
            {
              // the three records of the node are fetched together (one memory round trip)
              const double4 sm = g_sm[node];
              const float4 rel = g_rel[node];
              const int4 kd    = g_kids[node];
              if(sm.w != 0.0)
                {
                  const double dsx = wrapd(sm.x - gx, w), dsy = wrapd(sm.y - gy, w), dsz = wrapd(sm.z - gz, w);
                  const float sx = (float)dsx, sy = (float)dsy, sz = (float)dsz;
                  const float cx = sx + rel.x, cy = sy + rel.y, cz = sz + rel.z;
                  const float L  = rel.w;
                  const float m  = (float)sm.w;
                  hj             = w.soft[kd.w];
                  bool prune     = false;
                  if(PERIODIC)
                    {
                      const float eff = w.rcut + 0.5f * L;
                      prune = (fabsf(cx) - ex > eff) || (fabsf(cy) - ey > eff) || (fabsf(cz) - ez > eff);
                    }
                  if(!prune)
                    {
                      const float dmx = fmaxf(fabsf(sx) - ex, 0.0f), dmy = fmaxf(fabsf(sy) - ey, 0.0f),
                                  dmz = fmaxf(fabsf(sz) - ez, 0.0f);
                      const float rmin2 = dmx * dmx + dmy * dmy + dmz * dmz;
                      const float L2    = L * L;
                      bool open;
                      if(bh)
                        open = L2 > rmin2 * w.theta2;
                      else
                        // with ACTIVATE_MINIMUM_OPENING_ANGLE the mass test also needs the node to span more than
                        // 0.4 radian from the nearest point of the box (conservative for every target)
                        open = (L2 > rmin2 * 1.44f) ||
                               (m * L2 > rmin2 * rmin2 * aold_min && (!w.minangle || L2 > rmin2 * 0.16f)) ||
                               (fabsf(cx) < 0.6f * L + ex && fabsf(cy) < 0.6f * L + ey && fabsf(cz) < 0.6f * L + ez);
                      if(!open && hj > h_min)
                        {
                          // a target's softening is below the node's largest: open inside that
                          // softening, or (MULTIPLE_NODE_SOFTENING) use the node per softening type
                          if(w.mns)
                            split = true;
                          else if(rmin2 < hj * hj)
                            open = true;
                        }
                      if(open)
                        {
                          action = 2;
                          fc     = kd.x;
                          fp     = kd.y;
                          nc     = kd.z & 15;
                          np     = (kd.z >> 4) & 15;
                          if(L2 < vote_r2 && rmin2 < vote_r2)
                            {
                              vote      = true;
                              vote_keep = !PERIODIC || rmin2 < w.rcut2;
                              vrel      = rel;
                              entry     = mk4<R>(dsx, dsy, dsz, sm.w);
                              ent_d2    = rmin2;
                            }
                        }
                      else if(!PERIODIC || rmin2 < w.rcut2)
                        {
                          // accepted; a node whose CoM is beyond Rcut of every target contributes nothing
                          action = 1;
                          entry  = mk4<R>(dsx, dsy, dsz, sm.w);
                          ent_d2 = rmin2;
                        }
                    }
                }
            }
          // per-target vote: the node stays open only if some target's own criterion opens it
          if(const unsigned vm = __ballot_sync(0xffffffffu, vote))
            {
              WALK_STAT(7, 1);
              WALK_STAT(8, __popc(vm));
              bool need    = false;
              const float L = vrel.w, L2 = L * L;
#pragma unroll
              for(int k = 0; k < TPL; k++)
                for(int i = 0; i < 32; i++)
                  {
                    const float tx = (float)__shfl_sync(0xffffffffu, T[k].x, i), ty = (float)__shfl_sync(0xffffffffu, T[k].y, i),
                                tz = (float)__shfl_sync(0xffffffffu, T[k].z, i), th = (float)__shfl_sync(0xffffffffu, T[k].h, i),
                                ta = aold_sh[warp][i + 32 * k];
                    if(vote && !need && i + 32 * k < cnt)
                      {
                        const float enx = (float)entry.x, eny = (float)entry.y, enz = (float)entry.z;
                        const float dx = enx - tx, dy = eny - ty, dz = enz - tz;
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        bool o;
                        if(bh)
                          o = L2 > r2 * w.theta2;
                        else
                          o = (L2 > r2 * 1.44f) || ((float)entry.w * L2 > r2 * r2 * ta && (!w.minangle || L2 > r2 * 0.16f)) ||
                              (fabsf(enx + vrel.x - tx) < 0.6f * L && fabsf(eny + vrel.y - ty) < 0.6f * L &&
                               fabsf(enz + vrel.z - tz) < 0.6f * L);
                        if(!o && !w.mns && hj > th && r2 < hj * hj)
                          o = true;
                        need = o;
                      }
                  }
              if(vote && !need)
                {
                  action = vote_keep ? 1 : 0;
                  split  = w.mns && hj > h_min;
                  nc = np = 0;
                }
            }
          // accepted nodes -> list (the list holds fewer than Cap::eval entries, so 32 more fit);
          // nodes used per softening type follow as pending items
          push<R, PERIODIC>(L, action == 1 && !split, entry, (R)hj, ent_d2, fmaxf(h_grp, hj), ex, ey, ez, w, lt_mask);
          t_next = 0;
          t_end  = __ballot_sync(0xffffffffu, action == 1 && split) ? w.nsoft : 0;
          // particles (pending rounds) and node children of opened nodes: one scan of both counts
          // (each below 16, particles in the low half-word)
          const int npx  = (action == 2) ? np : 0;
          const int ncx  = (action == 2) ? nc : 0;
          const int both = wscan_incl(npx | (ncx << 16), lane);
          const int tot  = __shfl_sync(0xffffffffu, both, 31);
          pinc           = both & 0xffff;
          ptot           = tot & 0xffff;
          pexc           = pinc - npx;
          q0             = 0;
          WALK_STAT(2, ptot);
          // node children of opened nodes -> stack (contiguous in breadth-first order)
          const int cinc = both >> 16;
          const int ctot = tot >> 16;
          if(sp + ctot <= kStackCap)
            {
              const int cb = sp + cinc - ncx;
              for(int q = 0; q < ncx; q++)
                stack[cb + q] = fc + q;
              sp += ctot;
            }
          else if(lane == 0)
            atomicOr(err, 16);  // stack too small: the walk of this group is incomplete
          __syncwarp();
        }
#pragma unroll
      for(int k = 0; k < TPL; k++)
        {
          const int s = lane + 32 * k;
          if(s < cnt)
            {
              const int64_t t    = tlist ? (int64_t)tlist[t0 + s] : t0 + s;
              acc_out[3 * t + 0] = dsum[(4 * k + 0) * 32];
              acc_out[3 * t + 1] = dsum[(4 * k + 1) * 32];
              acc_out[3 * t + 2] = dsum[(4 * k + 2) * 32];
              if(POT)
                pot_out[t] = dsum[(4 * k + 3) * 32];
              nint_out[t] = T[k].ni;
            }
        }
      // the group's interactions (idle slots count none)
      unsigned long long gtot = 0;
#pragma unroll
      for(int k = 0; k < TPL; k++)
        gtot += lane + 32 * k < cnt ? (unsigned long long)T[k].ni : 0ull;
      for(int o = 16; o > 0; o >>= 1)
        gtot += __shfl_xor_sync(0xffffffffu, gtot, o);
      if(lane == 0)
        total_sh[warp] += gtot;
      __syncwarp();
    }
  if(lane == 0 && total_sh[warp])
    atomicAdd(total, total_sh[warp]);
}

// ---- walk groups -------------------------------------------------------------------------
// A group is up to `cap` consecutive targets in Peano-Hilbert order, never spanning two systems.
// cd[i] is the depth of the deepest cell holding particles i and i+1 (-1 across systems and after
// the last particle).  Optionally (slack < 64) groups are also cut between tree cells: pd[i] is the
// depth of the deepest cell around particle i that holds more than cap particles (-1: its whole
// system fits in one group), and consecutive particles stay in one group only while each lies
// inside the other's pd cell (up to `slack` levels above it).  Cell cuts bound a group's box by a
// tree cell at the price of partly filled warps; the per-target vote of the walk already removes
// the cost of loose groups, and plain key-order groups are faster on the measured workloads.
// depth of the deepest cell around sorted particle i that holds more than cap particles (-1: its whole
// system fits in one group), by widening [l, r] one cell at a time along the pair depths
__device__ __forceinline__ int cap_cell_depth(int64_t i, const int8_t *__restrict__ cd, int cap)
{
  int64_t l = i, r = i;  // current cell [l, r]
  while(true)
    {
      const int dl = l > 0 ? cd[l - 1] : -1;
      const int dr = cd[r];
      const int d  = dl > dr ? dl : dr;  // depth of the next larger cell
      if(d < 0)
        return -1;
      while(l > 0 && cd[l - 1] >= d)
        if(r - --l + 1 > cap)
          return d;
      while(cd[r] >= d)
        if(++r - l + 1 > cap)
          return d;
    }
}

__global__ void k_grp_pd(int64_t n, const int8_t *__restrict__ cd, int cap, int8_t *__restrict__ pd)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    pd[i] = (int8_t)cap_cell_depth(i, cd, cap);
}

// The same for an active list (targets at sorted positions tpos, in key order): the cell depth at each
// target, and the depth of the deepest cell holding consecutive targets k and k + 1 (-1 after the last)
__global__ void k_grp_pd_at(int64_t nt, const int32_t *__restrict__ tpos, const int8_t *__restrict__ cd, int cap,
                            int8_t *__restrict__ apd)
{
  for(int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nt; k += (int64_t)gridDim.x * blockDim.x)
    apd[k] = (int8_t)cap_cell_depth(tpos[k], cd, cap);
}
__global__ void k_active_cd(int64_t nt, const int32_t *__restrict__ tpos, const uint64_t *__restrict__ ix,
                            const uint64_t *__restrict__ iy, const uint64_t *__restrict__ iz, int8_t *__restrict__ acd)
{
  for(int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nt; k += (int64_t)gridDim.x * blockDim.x)
    {
      int d = -1;
      if(k + 1 < nt)
        {
          const int64_t a = tpos[k], b = tpos[k + 1];
          d               = common_depth(ix[a], iy[a], iz[a], ix[b], iy[b], iz[b]);
        }
      acd[k] = (int8_t)d;
    }
}

// segment start candidates: i where a group must begin (system start or a cut before i)
__global__ void k_grp_cut(int64_t n, const int8_t *__restrict__ cd, const int8_t *__restrict__ pd, int slack,
                          int32_t *__restrict__ segv)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      bool cut = (i == 0);
      if(!cut)
        {
          const int c = cd[i - 1];
          cut         = c < 0;
          if(pd && !cut)
            {
              const int p = pd[i - 1] > pd[i] ? pd[i - 1] : pd[i];
              cut         = c < p - slack;
            }
        }
      segv[i] = cut ? (int32_t)i : 0;
    }
}

__global__ void k_grp_start(int64_t n, const int32_t *__restrict__ seg, int cap, int32_t *__restrict__ flag)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = ((i - seg[i]) % cap == 0) ? 1 : 0;
}

// group table: (first target, count, root node, -1 = criterion of the walk constants)
__global__ void k_grp_fill(int64_t n, const int32_t *__restrict__ flag, const int32_t *__restrict__ gid, int cap,
                           const int32_t *__restrict__ sys, int4 *__restrict__ groups, int *__restrict__ ngroups)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      if(flag[i])
        {
          int cnt = 1;
          while(cnt < cap && i + cnt < n && !flag[i + cnt])
            cnt++;
          groups[gid[i]] = make_int4((int)i, cnt, sys ? sys[i] : 0, -1);
        }
      if(i == n - 1)
        *ngroups = gid[i] + flag[i];
    }
}

// outputs (sorted order) of the targets outside this slice set to zero; the slice's target range
// is [start of group g_begin, start of group g_end) with the FP32 group table, else n*s/ns..
__global__ void k_slice_mask(int64_t n, int slice, int nslices, const int4 *__restrict__ groups, const int *__restrict__ ngroups,
                             const int64_t *__restrict__ slice_rng, double *__restrict__ acc, double *__restrict__ pot,
                             int32_t *__restrict__ nint)
{
  int64_t t_begin, t_end;
  if(slice_rng)
    {
      t_begin = slice_rng[2];
      t_end   = slice_rng[3];
    }
  else if(groups)
    {
      const int64_t ng = *ngroups;
      const int64_t gb = ng * slice / nslices, ge = ng * (slice + 1) / nslices;
      t_begin          = gb < ng ? groups[gb].x : n;
      t_end            = ge < ng ? groups[ge].x : n;
    }
  else
    {
      t_begin = n * slice / nslices;
      t_end   = n * (slice + 1) / nslices;
    }
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if(i < t_begin || i >= t_end)
      {
        acc[3 * i] = acc[3 * i + 1] = acc[3 * i + 2] = 0.0;
        if(pot)
          pot[i] = 0.0;
        nint[i] = 0;
      }
}

struct MaxOp32
{
  __device__ __forceinline__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

int grid_for(int64_t n, int threads)
{
  int64_t b = (n + threads - 1) / threads;
  if(b > 148 * 16)
    b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

void make_w32(const WalkConst &wc, W32Const *w)
{
  memset(w, 0, sizeof(*w));
  w->box       = wc.box;
  w->half_box  = wc.half_box;
  w->rcut      = (float)wc.rcut;
  w->rcut2     = (float)wc.rcut2;
  // margin for the rounding of the FP32 separations and the box extents (relative ~1e-6)
  w->rcut2_all = (float)(wc.rcut2 * (1.0 - 1.0 / 4096.0));
  w->asmthfac  = (float)wc.asmthfac;
  const double finv = wc.pm ? wc.asmthinv2 : 1.0;
  w->theta2    = (float)(wc.theta * wc.theta);
  w->erracc    = (float)wc.erracc;
  w->periodic  = wc.periodic;
  w->bh        = wc.bh;
  w->ewd_fac   = (float)wc.ewd_fac_intp;
  w->mns       = wc.mns;
  w->minangle  = wc.minangle;
  w->nsoft     = wc.nsoft;
  for(int i = 0; i <= GPUGRAV_MAX_SOFTTYPES; i++)
    w->soft[i] = (float)wc.soft[i];
  for(int i = 0; i <= kNtab; i++)
    {
      float f0 = (float)(finv * wc.tab_force[i]), f1 = (float)(finv * ((i < kNtab) ? wc.tab_force[i + 1] : wc.tab_force[i]));
      float p0 = wc.tab_pot[i], p1 = (i < kNtab) ? wc.tab_pot[i + 1] : wc.tab_pot[i];
      w->tab[i] = make_float4(f0, f1 - f0, p0, p1 - p0);
      // FP64 walk: the reference's float table entries, scaled and differenced in double
      const double d0 = finv * wc.tab_force[i], d1 = finv * ((i < kNtab) ? wc.tab_force[i + 1] : wc.tab_force[i]);
      const double q0 = wc.tab_pot[i], q1 = (i < kNtab) ? wc.tab_pot[i + 1] : wc.tab_pot[i];
      w->tab64[i]     = make_double4(d0, d1 - d0, q0, q1 - q0);
    }
  w->rcut2_d    = wc.rcut2;
  w->asmthfac_d = wc.asmthfac;
}
}  // namespace

// buffers of the FP32 walk layout and group table for n particles and nn nodes
cudaError_t layout32_buffers(gpugrav_ctx *c, int64_t n, int64_t nn)
{
  GG_TRY(c->g_key.ensure(nn * 8));
  GG_TRY(c->g_key_alt.ensure(nn * 8));
  GG_TRY(c->g_val.ensure(nn * 4));
  GG_TRY(c->g_val_alt.ensure(nn * 4));
  GG_TRY(c->g_bfs.ensure(nn * 4));
  GG_TRY(c->g_np.ensure((nn + 1) * 4));
  GG_TRY(c->g_poff.ensure((nn + 1) * 4));
  GG_TRY(c->g_sm.ensure(nn * sizeof(double4)));
  GG_TRY(c->g_rel.ensure(nn * sizeof(float4)));
  GG_TRY(c->g_kids.ensure(nn * sizeof(int4)));
  GG_TRY(c->g_pm.ensure(n * sizeof(double4)));
  GG_TRY(c->g_pst.ensure(n + 16));
  GG_TRY(c->g_groups.ensure(n * sizeof(int4)));
  GG_TRY(c->g_ngroups.ensure(16));
  GG_TRY(c->g_gpd.ensure(n + 16));
  GG_TRY(c->g_gseg.ensure(n * 4));
  GG_TRY(c->g_gflag.ensure(n * 4));
  GG_TRY(c->g_gid.ensure(n * 4));
  return cudaSuccess;
}

// layout32_stage's buffers and temporary storage sized once for n particles and nn nodes
cudaError_t layout32_reserve(gpugrav_ctx *c, int64_t n, int64_t nn)
{
  GG_TRY(layout32_buffers(c, n, nn));
  size_t tb = 0, t2 = 0;
  GG_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, c->g_key.as<uint64_t>(), c->g_key_alt.as<uint64_t>(),
                                         c->g_val.as<int32_t>(), c->g_val_alt.as<int32_t>(), (int)nn, 0, 40, c->stream));
  GG_TRY(cub::DeviceScan::InclusiveScan(nullptr, t2, c->g_gflag.as<int32_t>(), c->g_gseg.as<int32_t>(), MaxOp32(), (int)n,
                                        c->stream));
  tb = t2 > tb ? t2 : tb;
  GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t2, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), (int)n, c->stream));
  tb = t2 > tb ? t2 : tb;
  return c->sort_tmp.ensure(tb);
}

// walk group table of the current tree (see k_grp_pd); the group count stays on the device
cudaError_t groups_stage(gpugrav_ctx *c)
{
  const int64_t n = c->n;
  cudaStream_t st = c->stream;
  const bool ewald = c->prm.periodic && !(c->prm.asmth > 0);  // the Ewald variant walks one target per lane
  const int cap    = 32 * walk32_tpl(c);
  GG_TRY(cudaMemsetAsync(c->g_ngroups.p, 0, sizeof(int), st));
  if(n == 0)
    return cudaSuccess;
  const bool cells = c->group_slack < 64;  // otherwise: cut at system starts only
  if(cells)
    k_grp_pd<<<grid_for(n, 256), 256, 0, st>>>(n, c->s_cd.as<int8_t>(), cap, c->g_gpd.as<int8_t>());
  k_grp_cut<<<grid_for(n, 256), 256, 0, st>>>(n, c->s_cd.as<int8_t>(), cells ? c->g_gpd.as<int8_t>() : nullptr,
                                               c->group_slack, c->g_gflag.as<int32_t>());
  size_t tb = 0;
  GG_TRY(cub::DeviceScan::InclusiveScan(nullptr, tb, c->g_gflag.as<int32_t>(), c->g_gseg.as<int32_t>(), MaxOp32(), (int)n, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::InclusiveScan(c->sort_tmp.p, tb, c->g_gflag.as<int32_t>(), c->g_gseg.as<int32_t>(), MaxOp32(), (int)n,
                                        st));
  k_grp_start<<<grid_for(n, 256), 256, 0, st>>>(n, c->g_gseg.as<int32_t>(), cap, c->g_gflag.as<int32_t>());
  tb = 0;
  GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), (int)n, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), (int)n, st));
  k_grp_fill<<<grid_for(n, 256), 256, 0, st>>>(n, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), cap,
                                                c->multi ? c->m_sys.as<int32_t>() : nullptr, c->g_groups.as<int4>(),
                                                c->g_ngroups.as<int>());
  return cudaGetLastError();
}

// walk group table of an active list (gravity_tree(timebin)'s TargetList, sorted positions in key
// order in tpos): up to cap consecutive active targets, also cut where two consecutive targets share
// only a cell more than active_slack levels above the cells of cap particles around them -- active
// targets that follow each other in key order can lie far apart (the background particles on both
// sides of a dense core), and one group box spanning the core would open it for every target.  On the
// zoom box at N = 2^24 the walk of the 2^23 background particles alone takes 55 ms with slack 2
// against 259 ms without cuts; the Plummer particles alone are within 0.6 %.
cudaError_t groups_active_stage(gpugrav_ctx *c, int64_t nt, int cap)
{
  cudaStream_t st = c->stream;
  GG_TRY(c->g_groups.ensure((size_t)(nt + 1) * sizeof(int4)));
  GG_TRY(c->g_ngroups.ensure(16));
  GG_TRY(cudaMemsetAsync(c->g_ngroups.p, 0, sizeof(int), st));
  if(nt == 0)
    return cudaSuccess;
  GG_TRY(c->t_cd.ensure(nt + 16));
  GG_TRY(c->t_pd.ensure(nt + 16));
  GG_TRY(c->g_gseg.ensure(nt * 4));
  GG_TRY(c->g_gflag.ensure(nt * 4));
  GG_TRY(c->g_gid.ensure(nt * 4));
  const int32_t *tpos = c->t_pos_alt.as<int32_t>();
  // every particle active: consecutive targets are neighbours, plain chunks as in the full walk's table
  const bool cells = c->active_slack < 64 && nt < c->n;
  k_active_cd<<<grid_for(nt, 256), 256, 0, st>>>(nt, tpos, c->s_ix.as<uint64_t>(), c->s_iy.as<uint64_t>(), c->s_iz.as<uint64_t>(),
                                                  c->t_cd.as<int8_t>());
  if(cells)
    k_grp_pd_at<<<grid_for(nt, 256), 256, 0, st>>>(nt, tpos, c->s_cd.as<int8_t>(), cap, c->t_pd.as<int8_t>());
  k_grp_cut<<<grid_for(nt, 256), 256, 0, st>>>(nt, c->t_cd.as<int8_t>(), cells ? c->t_pd.as<int8_t>() : nullptr,
                                                c->active_slack, c->g_gflag.as<int32_t>());
  size_t tb = 0;
  GG_TRY(cub::DeviceScan::InclusiveScan(nullptr, tb, c->g_gflag.as<int32_t>(), c->g_gseg.as<int32_t>(), MaxOp32(), (int)nt, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::InclusiveScan(c->sort_tmp.p, tb, c->g_gflag.as<int32_t>(), c->g_gseg.as<int32_t>(), MaxOp32(), (int)nt,
                                        st));
  k_grp_start<<<grid_for(nt, 256), 256, 0, st>>>(nt, c->g_gseg.as<int32_t>(), cap, c->g_gflag.as<int32_t>());
  tb = 0;
  GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), (int)nt, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), (int)nt, st));
  k_grp_fill<<<grid_for(nt, 256), 256, 0, st>>>(nt, c->g_gflag.as<int32_t>(), c->g_gid.as<int32_t>(), cap, nullptr,
                                                 c->g_groups.as<int4>(), c->g_ngroups.as<int>());
  return cudaGetLastError();
}

// breadth-first node layout + particles grouped by parent (built once per tree)
cudaError_t layout32_stage(gpugrav_ctx *c)
{
  c->mark(nullptr);
  const int64_t n = c->n, nn = c->num_nodes;
  cudaStream_t st = c->stream;
  GG_TRY(layout32_buffers(c, n, nn));
  const bool mns = (c->prm.flags & GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING) != 0;
  if(mns)
    GG_TRY(c->g_mpt.ensure((size_t)(nn + 16) * c->prm.nsofttypes * sizeof(float)));
  k_g_keys<<<grid_for(nn, 256), 256, 0, st>>>(nn, c->n_depth.as<uint8_t>(), c->n_dfs.as<int32_t>(), c->g_key.as<uint64_t>(),
                                               c->g_val.as<int32_t>());
  size_t tb = 0;
  GG_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, c->g_key.as<uint64_t>(), c->g_key_alt.as<uint64_t>(),
                                         c->g_val.as<int32_t>(), c->g_val_alt.as<int32_t>(), (int)nn, 0, 40, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceRadixSort::SortPairs(c->sort_tmp.p, tb, c->g_key.as<uint64_t>(), c->g_key_alt.as<uint64_t>(),
                                         c->g_val.as<int32_t>(), c->g_val_alt.as<int32_t>(), (int)nn, 0, 40, st));
  k_g_rank<<<grid_for(nn, 256), 256, 0, st>>>(nn, n, c->g_val_alt.as<int32_t>(), c->n_suns.as<int32_t>(), c->g_bfs.as<int32_t>(),
                                               c->g_np.as<int32_t>());
  tb = 0;
  GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->g_np.as<int32_t>(), c->g_poff.as<int32_t>(), (int)nn, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, c->g_np.as<int32_t>(), c->g_poff.as<int32_t>(), (int)nn, st));
  int *err = c->counters.as<int>() + 13;
  GG_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
  k_g_fill<<<grid_for(nn, 256), 256, 0, st>>>(nn, n, c->g_val_alt.as<int32_t>(), c->n_suns.as<int32_t>(), c->g_bfs.as<int32_t>(),
                                               c->g_poff.as<int32_t>(), c->n_sm.as<double4>(), c->n_cl.as<double4>(),
                                               c->n_maxsoft.as<uint8_t>(), c->s_pm.as<double4>(), c->s_st.as<uint8_t>(),
                                               c->g_sm.as<double4>(), c->g_rel.as<float4>(), c->g_kids.as<int4>(),
                                               c->g_pm.as<double4>(), c->g_pst.as<uint8_t>(), err,
                                               mns ? c->n_mpt.as<double>() : nullptr, c->prm.nsofttypes,
                                               mns ? c->g_mpt.as<float>() : nullptr);
  GG_TRY(cudaGetLastError());
  int e = 0;
  GG_TRY(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  GG_TRY(cudaStreamSynchronize(st));
  if(e)
    return cudaErrorUnknown;
  c->mark("l1 layout32");
  GG_TRY(groups_stage(c));
  c->mark("l2 groups");
  c->layout32_valid = true;
  c->groups_active  = false;
  return cudaSuccess;
}

typedef decltype(&k_walk32<true, true, 1>) Walk32Kernel;

// Everything that must happen before the walk launch and may not be captured in a graph
// (layout, constants upload from host memory, stack allocation, launch shape).
cudaError_t walk32_prepare(gpugrav_ctx *c, const WalkConst &wc)
{
  if(!c->layout32_valid)
    GG_TRY(layout32_stage(c));
  cudaStream_t st = c->stream;
  W32Const w;
  make_w32(wc, &w);
  if(wc.ewald)
    {
      GG_TRY(ewald_ensure(c));
      w.ewd = c->ewd32.as<float4>();
    }
  if(wc.mns)
    w.mpt = c->g_mpt.as<float>();
  GG_TRY(c->scratch.ensure(sizeof(W32Const) + 256));
  GG_TRY(cudaMemcpyAsync(c->scratch.p, &w, sizeof(w), cudaMemcpyHostToDevice, st));
  GG_TRY(cudaStreamSynchronize(st));  // `w` lives on this stack frame
  int dev = 0, sms = 0, per_sm = 0;
  GG_TRY(cudaGetDevice(&dev));
  GG_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const bool periodic = wc.pm != 0;  // TreePM split (Rcut, erfc table)
  const bool pot      = c->want_pot;
  const int tpl       = walk32_tpl(c);
  // the group walk in FP64 arithmetic (precision ablation): TreePM and isolated, one target per lane
  const bool fp64     = c->prm.precision == GPUGRAV_PREC_FP64_GROUP;
  if(fp64 && wc.ewald)
    return cudaErrorNotSupported;
  Walk32Kernel kern = fp64 ? (tpl == 2 ? (periodic ? (pot ? k_walk32<true, true, 2, false, double> : k_walk32<true, false, 2, false, double>)
                                                    : (pot ? k_walk32<false, true, 2, false, double> : k_walk32<false, false, 2, false, double>))
                                      : (periodic ? (pot ? k_walk32<true, true, 1, false, double> : k_walk32<true, false, 1, false, double>)
                                                  : (pot ? k_walk32<false, true, 1, false, double> : k_walk32<false, false, 1, false, double>)))
                    : wc.ewald ? (pot ? k_walk32<false, true, 1, true> : k_walk32<false, false, 1, true>)
                      : tpl == 2 ? (periodic ? (pot ? k_walk32<true, true, 2> : k_walk32<true, false, 2>)
                                             : (pot ? k_walk32<false, true, 2> : k_walk32<false, false, 2>))
                                 : (periodic ? (pot ? k_walk32<true, true, 1> : k_walk32<true, false, 1>)
                                             : (pot ? k_walk32<false, true, 1> : k_walk32<false, false, 1>));
  GG_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kWarps, 0));
  if(per_sm < 1)
    per_sm = 1;
  c->w32_kernel = (void *)kern;
  c->w32_blocks = sms * per_sm;
  GG_TRY(c->g_stack.ensure((size_t)c->w32_blocks * kWarps * kStackCap * sizeof(int)));
  return cudaSuccess;
}

// The walk itself: counter reset + one persistent launch (capturable).  The group table and
// its count live in device memory, so a captured launch serves every tree of the same buffers.
cudaError_t walk32_launch(gpugrav_ctx *c)
{
  cudaStream_t st = c->stream;
  int *work       = c->counters.as<int>() + 20;
  int *err        = c->counters.as<int>() + 14;
  GG_TRY(cudaMemsetAsync(work, 0, sizeof(int), st));
  Walk32Kernel kern = (Walk32Kernel)c->w32_kernel;
  kern<<<c->w32_blocks, 32 * kWarps, 0, st>>>(c->g_sm.as<double4>(), c->g_rel.as<float4>(), c->g_kids.as<int4>(),
                                              c->g_pm.as<double4>(), c->g_pst.as<uint8_t>(), c->s_pm.as<double4>(),
                                              c->s_st.as<uint8_t>(), c->oldacc_s.as<float>(), c->g_ngroups.as<int>(),
                                              c->g_groups.as<int4>(), c->w_tlist, c->slice, c->nslices,
                                              c->slice_rng_on ? c->slice_rng.as<int64_t>() : nullptr,
                                              (const W32Const *)c->scratch.p,
                                              c->g_stack.as<int>(), work, c->acc_s.as<double>(), c->pot_s.as<double>(),
                                              c->nint_s.as<int32_t>(), (unsigned long long *)(c->counters.as<int>() + 32), err);
  return cudaGetLastError();
}

// ---- cost-balanced target slices ----
// Cost of every walk group (FP32) or target (FP64) in key order, from the caller's per-particle cost
// (the previous step's interaction counts, as force_assign_cost_values feeds the reference's domain
// decomposition, src/gravity/forcetree.c:945-1010).
__global__ void k_unit_cost(int64_t nu, int64_t n, const int4 *__restrict__ groups, const uint32_t *__restrict__ perm,
                            const float *__restrict__ cost, double *__restrict__ ucost)
{
  for(int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < nu; u += (int64_t)gridDim.x * blockDim.x)
    {
      if(groups)
        {
          const int4 g = groups[u];
          double s     = 0;
          for(int k = 0; k < g.y; k++)
            s += cost[perm[g.x + k]];
          ucost[u] = s;
        }
      else
        ucost[u] = cost[perm[u]];
    }
}

// units [b(s), b(s+1)) with b(s) the first unit whose exclusive cost prefix reaches s/ns of the total
// (equal unit counts when the total is 0); rng = (first group, end group, first target, end target)
__global__ void k_slice_bounds(int64_t nu, int64_t n, const int4 *__restrict__ groups, const double *__restrict__ incl, int slice,
                               int nslices, int64_t *__restrict__ rng)
{
  if(blockIdx.x || threadIdx.x)
    return;
  const double total = nu > 0 ? incl[nu - 1] : 0.0;
  int64_t b[2];
  for(int e = 0; e < 2; e++)
    {
      const int s = slice + e;
      if(s == 0 || nu == 0)
        b[e] = 0;
      else if(s == nslices)
        b[e] = nu;
      else if(!(total > 0))
        b[e] = nu * s / nslices;
      else
        {
          const double want = total * s / nslices;
          int64_t lo = 0, hi = nu;  // first u with exclusive prefix (incl[u-1]) >= want
          while(lo < hi)
            {
              const int64_t mid = (lo + hi) / 2;
              const double ex   = mid > 0 ? incl[mid - 1] : 0.0;
              if(ex >= want)
                hi = mid;
              else
                lo = mid + 1;
            }
          b[e] = lo;
        }
    }
  if(groups)
    {
      rng[0] = b[0];
      rng[1] = b[1];
      rng[2] = b[0] < nu ? groups[b[0]].x : n;
      rng[3] = b[1] < nu ? groups[b[1]].x : n;
    }
  else
    {
      rng[0] = rng[1] = 0;
      rng[2] = b[0];
      rng[3] = b[1];
    }
}

// device-side slice range from the caller's costs (gpugrav_set_target_slice_cost); FP32: in walk
// groups (the group count is read on the host once, here), FP64: in targets
cudaError_t slice_cost_stage(gpugrav_ctx *c, bool fp32)
{
  c->slice_rng_on = false;
  if(c->nslices <= 1 || !c->cost_set)
    return cudaSuccess;
  cudaStream_t st = c->stream;
  int64_t nu      = c->n;
  if(fp32)
    {
      int ng = 0;
      GG_TRY(cudaMemcpyAsync(&ng, c->g_ngroups.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      GG_TRY(cudaStreamSynchronize(st));
      nu = ng;
    }
  GG_TRY(c->slice_rng.ensure(4 * sizeof(int64_t)));
  GG_TRY(c->cost_u.ensure((nu + 1) * sizeof(double)));
  GG_TRY(c->cost_p.ensure((nu + 1) * sizeof(double)));
  const int4 *groups = fp32 ? c->g_groups.as<int4>() : nullptr;
  k_unit_cost<<<grid_for(nu, 256), 256, 0, st>>>(nu, c->n, groups, c->perm.as<uint32_t>(), c->cost_in.as<float>(),
                                                 c->cost_u.as<double>());
  size_t tb = 0;
  GG_TRY(cub::DeviceScan::InclusiveSum(nullptr, tb, c->cost_u.as<double>(), c->cost_p.as<double>(), (int)nu, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::InclusiveSum(c->sort_tmp.p, tb, c->cost_u.as<double>(), c->cost_p.as<double>(), (int)nu, st));
  k_slice_bounds<<<1, 32, 0, st>>>(nu, c->n, groups, c->cost_p.as<double>(), c->slice, c->nslices, c->slice_rng.as<int64_t>());
  GG_TRY(cudaGetLastError());
  c->slice_rng_on = true;
  return cudaSuccess;
}

// zero the outputs of the targets outside the current target slice (no-op without slicing)
cudaError_t slice_mask_stage(gpugrav_ctx *c, bool fp32)
{
  if(c->nslices <= 1)
    return cudaSuccess;
  k_slice_mask<<<grid_for(c->n, 256), 256, 0, c->stream>>>(c->n, c->slice, c->nslices, fp32 ? c->g_groups.as<int4>() : nullptr,
                                                           fp32 ? c->g_ngroups.as<int>() : nullptr,
                                                           c->slice_rng_on ? c->slice_rng.as<int64_t>() : nullptr, c->acc_s.as<double>(),
                                                           c->want_pot ? c->pot_s.as<double>() : nullptr, c->nint_s.as<int32_t>());
  return cudaGetLastError();
}

cudaError_t walk32_stage(gpugrav_ctx *c, const WalkConst &wc)
{
  GG_TRY(walk32_prepare(c, wc));
  return walk32_launch(c);
}
}  // namespace gg

#ifdef GG_WALK32_STATS
// measurement build only: read and reset the walk statistics of the current device
extern "C" int gpugrav_walk_stats(unsigned long long *out)
{
  if(cudaMemcpyFromSymbol(out, gg::g_walk_stats, sizeof(unsigned long long) * gg::kWalkStats) != cudaSuccess)
    return -1;
  unsigned long long z[gg::kWalkStats] = {};
  return cudaMemcpyToSymbol(gg::g_walk_stats, z, sizeof(z)) == cudaSuccess ? 0 : -1;
}
#endif
