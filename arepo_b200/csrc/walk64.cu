// walk64.cu -- FP64 parity walk.  Compiled with -fmad=false.
//
// force_treeevaluate (src/gravity/forcetree_walk.c:115-514) for every target,
// with the reference's arithmetic operation for operation.  The tree is laid
// out in the reference's traversal order (depth first, slots 0..7), so that
// "nextnode" of an entry is the next entry and "sibling" is the entry after its
// subtree (w_link.x).  A warp takes 32 consecutive targets in key order; each
// lane keeps its own position in its own traversal, and the warp always serves
// the smallest position among its lanes: the entry is loaded once for the warp
// and evaluated by exactly the lanes that are at it.  Every lane therefore sees
// the same interaction sequence, in the same order, as the reference walk for
// its target -- the per-target results are bit-identical to the reference.
#include "internal.h"

namespace gg
{
namespace
{
// cubic-spline softening coefficients, src/main/allvars.h:557-573
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

__device__ __forceinline__ double nearest(double x, const WalkConst &w)
{
  // GRAVITY_NEAREST_X, src/main/allvars.h:602-608
  if(!w.periodic)
    return x;
  return (x > w.half_box) ? (x - w.box) : ((x < -w.half_box) ? (x + w.box) : x);
}

constexpr int kWarps = 4;

// EWALD (pure periodic tree) and MNS (MULTIPLE_NODE_SOFTENING) are compiled in only where used: the
// TreePM and isolated walks keep the register budget of a kernel without them.  The walk is
// latency-bound (lanes wait on the entry the warp serves), so occupancy beats spill-free code: on
// the zoom box 12 blocks per SM (48 warps) walk 1.18x faster than 6 and 1.3x faster than 5.
template <bool EWALD, bool MNS>
__global__ void __launch_bounds__(32 * kWarps, 12) k_walk64(const double4 *__restrict__ w_sm, const double4 *__restrict__ w_cl,
                                                        const int2 *__restrict__ w_link, uint32_t n_entries,
                                                        const double4 *__restrict__ tpm, const uint8_t *__restrict__ tst,
                                                        const float *__restrict__ oldacc, int64_t t_begin, int64_t t_end,
                                                        const int32_t *__restrict__ tlist, const WalkConst *__restrict__ wcp,
                                                        double *__restrict__ acc_out, double *__restrict__ pot_out,
                                                        int32_t *__restrict__ nint_out, unsigned long long *__restrict__ total)
{
  __shared__ WalkConst w;
  for(int t = threadIdx.x; t < (int)(sizeof(WalkConst) / 4); t += blockDim.x)
    ((int *)&w)[t] = ((const int *)wcp)[t];
  __syncthreads();

  const int lane  = threadIdx.x & 31;
  // position in the walk's target range; the target itself (sorted particle index) is the same
  // position, or its entry in the list of active targets
  const int64_t slot = t_begin + ((int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5)) * 32 + lane;
  const bool valid   = slot < t_end;
  const int64_t tgt  = valid && tlist ? (int64_t)tlist[slot] : slot;

  double pos_x = 0, pos_y = 0, pos_z = 0, aold = 0, h_i = 0;
  if(valid)
    {
      double4 p = tpm[tgt];
      pos_x     = p.x;
      pos_y     = p.y;
      pos_z     = p.z;
      aold      = w.erracc * (double)oldacc[tgt];
      h_i       = w.soft[tst[tgt]];
    }
  double acc_x = 0, acc_y = 0, acc_z = 0, pot = 0;
  int ninteractions = 0;
  uint32_t next     = valid ? 0u : n_entries;  // entry 0 is the root (Tree_MaxPart)

  while(true)
    {
      const uint32_t i = __reduce_min_sync(0xffffffffu, next);
      if(i >= n_entries)
        break;
      const int2 link  = w_link[i];
      const double4 sm = w_sm[i];
      const bool node  = (link.y & kNodeFlag) != 0;
      double4 cl       = make_double4(0, 0, 0, 0);
      if(node)
        cl = w_cl[i];
      if(next != i)
        continue;

      double dx, dy, dz, r2, mass, hmax;
      bool split = false;  // MULTIPLE_NODE_SOFTENING: node used per softening type
      if(!node)
        {
          // single particle, src/gravity/forcetree_walk.c:178-195
          dx         = nearest(sm.x - pos_x, w);
          dy         = nearest(sm.y - pos_y, w);
          dz         = nearest(sm.z - pos_z, w);
          r2         = dx * dx + dy * dy + dz * dz;
          mass       = sm.w;
          double h_j = w.soft[link.y & 0xff];
          hmax       = (h_j > h_i) ? h_j : h_i;
          next       = i + 1;
        }
      else
        {
          // internal node, src/gravity/forcetree_walk.c:196-330
          mass = sm.w;
          dx   = nearest(sm.x - pos_x, w);
          dy   = nearest(sm.y - pos_y, w);
          dz   = nearest(sm.z - pos_z, w);
          r2   = dx * dx + dy * dy + dz * dz;
          const double len = cl.w;
          if(w.pm && r2 > w.rcut2)
            {
              double eff_dist = w.rcut + 0.5 * len;
              double dist     = nearest(cl.x - pos_x, w);
              bool out        = (dist < -eff_dist || dist > eff_dist);
              if(!out)
                {
                  dist = nearest(cl.y - pos_y, w);
                  out  = (dist < -eff_dist || dist > eff_dist);
                }
              if(!out)
                {
                  dist = nearest(cl.z - pos_z, w);
                  out  = (dist < -eff_dist || dist > eff_dist);
                }
              if(out)
                {
                  next = (uint32_t)link.x;
                  continue;
                }
            }
          if(w.bh)
            {
              if(len * len > r2 * w.theta * w.theta)
                {
                  next = i + 1;
                  continue;
                }
            }
          else
            {
              double len2 = len * len;
              if(len2 > r2 * (1.2 * 1.2))
                {
                  next = i + 1;
                  continue;
                }
              // ACTIVATE_MINIMUM_OPENING_ANGLE adds a minimum angle to the mass test (forcetree_walk.c:266-271)
              if(mass * len2 > r2 * r2 * aold && (!w.minangle || len2 > r2 * (0.4 * 0.4)))
                {
                  next = i + 1;
                  continue;
                }
              if(fabs(nearest(cl.x - pos_x, w)) < 0.60 * len && fabs(nearest(cl.y - pos_y, w)) < 0.60 * len &&
                 fabs(nearest(cl.z - pos_z, w)) < 0.60 * len)
                {
                  next = i + 1;
                  continue;
                }
            }
          double h_j = w.soft[link.y & 0xff];
          if(h_j > h_i)
            {
              if(MNS)
                split = true;  // src/gravity/forcetree_walk.c:296-308
              else if(r2 < h_j * h_j)
                {
                  next = i + 1;
                  continue;
                }
              hmax = h_j;
            }
          else
            hmax = h_i;
          next = (uint32_t)link.x;
        }

      // multipole (monopole) interaction, src/gravity/forcetree_walk.c:363-488
      if(mass)
        {
          double r            = sqrt(r2);
          double factor_force = 0, factor_pot = 0;
          if(w.pm)
            {
              double tabentry = w.asmthfac * r;
              int tabindex    = (int)tabentry;
              if(!(tabindex < kNtab))
                continue;
              double tabweight = tabentry - tabindex;
              factor_force     = (1.0 - tabweight) * w.tab_force[tabindex] + tabweight * w.tab_force[tabindex + 1];
              factor_pot       = (1.0 - tabweight) * w.tab_pot[tabindex] + tabweight * w.tab_pot[tabindex + 1];
            }
          // per softening type under MULTIPLE_NODE_SOFTENING (forcetree_walk.c:382-401), else once
          const int t0 = (MNS && split) ? 0 : -1, t1 = (MNS && split) ? w.nsoft : 0;
          for(int type = t0; type < t1; type++)
            {
              if(type >= 0)
                {
                  mass             = w.w_mpt[(int64_t)i * w.nsoft + type];
                  const double hjt = w.soft[type];
                  hmax             = (hjt > h_i) ? hjt : h_i;
                }
              if(!mass)
                continue;
              double fac, wp;
              if(r >= hmax)
                {
                  double rinv  = 1.0 / r;
                  double rinv3 = rinv * rinv * rinv;
                  if(w.pm)
                    {
                      fac = rinv3 + rinv * factor_force * w.asmthinv2;
                      wp  = rinv * factor_pot;
                    }
                  else
                    {
                      fac = rinv3;
                      wp  = -rinv;
                    }
                }
              else
                {
                  double h_inv  = 1.0 / hmax;
                  double h3_inv = h_inv * h_inv * h_inv;
                  double u      = r * h_inv;
                  if(u < 0.5)
                    {
                      double u2 = u * u;
                      fac       = h3_inv * (SF1 + u2 * (SF2 * u + SF3));
                      wp        = h_inv * (SF4 + u2 * (SF5 + u2 * (SF6 * u + SF7)));
                    }
                  else
                    {
                      double u2 = u * u;
                      double u3 = u2 * u;
                      fac       = h3_inv * (SF8 + SF9 * u + SF10 * u2 + SF11 * u3 + SF12 / u3);
                      wp        = h_inv * (SF13 + SF14 / u + u2 * (SF1 + u * (SF15 + u * (SF16 + SF17 * u))));
                    }
                  if(w.pm && r > 0)
                    {
                      double rinv = 1.0 / r;
                      fac += rinv * factor_force * w.asmthinv2;
                      wp += rinv * (factor_pot + 1.0);
                    }
                }
              pot += mass * wp;
              fac *= mass;
              acc_x += dx * fac;
              acc_y += dy * fac;
              acc_z += dz * fac;
              if(EWALD)
                {
                  // all further periodic images, src/gravity/forcetree_walk.c:469-477
                  double fcorr[3], pcorr;
                  ewald_corr(dx, dy, dz, w, fcorr, pcorr);
                  acc_x += mass * fcorr[0];
                  acc_y += mass * fcorr[1];
                  acc_z += mass * fcorr[2];
                  pot += mass * pcorr;
                }
            }
          ninteractions++;
        }
    }

  if(valid)
    {
      acc_out[3 * tgt + 0] = acc_x;
      acc_out[3 * tgt + 1] = acc_y;
      acc_out[3 * tgt + 2] = acc_z;
      pot_out[tgt]         = pot;
      nint_out[tgt]        = ninteractions;
    }
  // interaction total for the timing report
  unsigned long long v = valid ? (unsigned long long)ninteractions : 0ull;
  for(int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  if(lane == 0 && v)
    atomicAdd(total, v);
}
}  // namespace

cudaError_t walk64_stage(gpugrav_ctx *c, const WalkConst &wc)
{
  // targets: every particle, or the active list (gpugrav_walk_targets); the slice's range from the
  // device when it is balanced by cost
  const int64_t n = c->w_tlist ? c->w_ntargets : c->n;
  int64_t t_begin = n * c->slice / c->nslices, t_end = n * (c->slice + 1) / c->nslices;
  if(c->slice_rng_on && !c->w_tlist)
    {
      int64_t rng[4];
      GG_TRY(cudaMemcpyAsync(rng, c->slice_rng.p, sizeof(rng), cudaMemcpyDeviceToHost, c->stream));
      GG_TRY(cudaStreamSynchronize(c->stream));
      t_begin = rng[2];
      t_end   = rng[3];
    }
  const int64_t warps   = (t_end - t_begin + 31) / 32;
  const int64_t blocks  = warps > 0 ? (warps + kWarps - 1) / kWarps : 1;
  auto kern = wc.ewald ? (wc.mns ? k_walk64<true, true> : k_walk64<true, false>)
                       : (wc.mns ? k_walk64<false, true> : k_walk64<false, false>);
  kern<<<(unsigned)blocks, 32 * kWarps, 0, c->stream>>>(
      c->w_sm.as<double4>(), c->w_cl.as<double4>(), c->w_link.as<int2>(), (uint32_t)c->n_entries, c->s_pm.as<double4>(),
      c->s_st.as<uint8_t>(), c->oldacc_s.as<float>(), t_begin, t_end, c->w_tlist, c->wconst.as<WalkConst>(),
      c->acc_s.as<double>(), c->pot_s.as<double>(),
      c->nint_s.as<int32_t>(), (unsigned long long *)(c->counters.as<int>() + 32));
  return cudaGetLastError();
}
}  // namespace gg
