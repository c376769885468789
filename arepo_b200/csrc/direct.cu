// direct.cu -- FP64 direct summation over all loaded particles for a set of
// targets: the accuracy instrument of gravity_forcetest_evaluate
// (src/gravity/gravtree_forcetest.c:483-601) without the Ewald terms.  For a
// periodic TreePM run it returns the short-range force with the exact erfc
// factor (u = r / (2 Asmth)); for an isolated run the Newtonian force.  Both
// with the cubic-spline softening of the walk.  Sources are split in chunks;
// partial sums are reduced in a fixed order (deterministic).
#include "internal.h"

namespace gg
{
namespace
{
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

constexpr int kTile   = 128;  // targets per block (one per thread)
constexpr int kChunks = 64;   // source chunks

__global__ void __launch_bounds__(kTile) k_direct(const double4 *__restrict__ pm, const uint8_t *__restrict__ st, int64_t n,
                                                  const int64_t *__restrict__ targets_sorted, int64_t nt,
                                                  const WalkConst *__restrict__ wcp, int cut, double4 *__restrict__ partial)
{
  __shared__ double4 src[kTile];
  __shared__ double hsrc[kTile];
  const WalkConst &w = *wcp;
  const int64_t t    = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int chunk    = blockIdx.y;
  const int64_t per  = (n + kChunks - 1) / kChunks;
  const int64_t j0 = chunk * per, j1 = (j0 + per < n) ? j0 + per : n;
  double4 me = make_double4(0, 0, 0, 0);
  double h_i = 0;
  if(t < nt)
    {
      int64_t i = targets_sorted[t];
      me        = pm[i];
      h_i       = w.soft[st[i]];
    }
  const double asmth = (w.pm) ? (0.5 / sqrt(w.asmthinv2)) : 0.0;
  double ax = 0, ay = 0, az = 0, pt = 0;
  for(int64_t jb = j0; jb < j1; jb += kTile)
    {
      __syncthreads();
      int64_t j = jb + threadIdx.x;
      if(j < j1)
        {
          src[threadIdx.x]  = pm[j];
          hsrc[threadIdx.x] = w.soft[st[j]];
        }
      __syncthreads();
      int cnt = (int)((j1 - jb) < kTile ? (j1 - jb) : kTile);
      if(t < nt)
        for(int q = 0; q < cnt; q++)
          {
            double4 s   = src[q];
            double dx   = s.x - me.x, dy = s.y - me.y, dz = s.z - me.z;
            if(w.periodic)
              {
                dx = (dx > w.half_box) ? dx - w.box : ((dx < -w.half_box) ? dx + w.box : dx);
                dy = (dy > w.half_box) ? dy - w.box : ((dy < -w.half_box) ? dy + w.box : dy);
                dz = (dz > w.half_box) ? dz - w.box : ((dz < -w.half_box) ? dz + w.box : dz);
              }
            double r2 = dx * dx + dy * dy + dz * dz;
            if(cut && w.pm && !(r2 < w.rcut2))
              continue;  // beyond Rcut: the part of the force left to the PM mesh
            double r  = sqrt(r2);
            double m  = s.w;
            double h_j  = hsrc[q];
            double hmax = (h_j > h_i) ? h_j : h_i;
            double fac_newton = 0, wp_newton = 0, fac, wp;
            if(r > 0)
              {
                fac_newton = m / (r2 * r);
                wp_newton  = -m / r;
              }
            if(r >= hmax)
              {
                fac = fac_newton;
                wp  = wp_newton;
              }
            else
              {
                double h_inv = 1.0 / hmax, h3_inv = h_inv * h_inv * h_inv, u = r * h_inv;
                if(u < 0.5)
                  {
                    double u2 = u * u;
                    fac       = m * h3_inv * (SF1 + u2 * (SF2 * u + SF3));
                    wp        = m * h_inv * (SF4 + u2 * (SF5 + u2 * (SF6 * u + SF7)));
                  }
                else
                  {
                    double u2 = u * u, u3 = u2 * u;
                    fac = m * h3_inv * (SF8 + SF9 * u + SF10 * u2 + SF11 * u3 + SF12 / u3);
                    wp  = m * h_inv * (SF13 + SF14 / u + u2 * (SF1 + u * (SF15 + u * (SF16 + SF17 * u))));
                  }
              }
            if(w.pm)
              {
                double u            = 0.5 / asmth * r;
                double factor_force = (erfc(u) + 2.0 * u / sqrt(M_PI) * exp(-u * u) - 1.0);
                double factor_pot   = erfc(u);
                fac += fac_newton * factor_force;
                wp += wp_newton * (factor_pot - 1.0);
              }
            ax += dx * fac;
            ay += dy * fac;
            az += dz * fac;
            pt += wp;
            if(w.ewald)
              {
                // pure periodic tree: every image through the Ewald correction
                double fcorr[3], pcorr;
                ewald_corr(dx, dy, dz, w, fcorr, pcorr);
                ax += m * fcorr[0];
                ay += m * fcorr[1];
                az += m * fcorr[2];
                pt += m * pcorr;
              }
          }
    }
  if(t < nt)
    partial[(int64_t)chunk * nt + t] = make_double4(ax, ay, az, pt);
}

__global__ void k_direct_reduce(const double4 *__restrict__ partial, int64_t nt, double *__restrict__ acc, double *__restrict__ pot)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= nt)
    return;
  double ax = 0, ay = 0, az = 0, pt = 0;
  for(int c = 0; c < kChunks; c++)
    {
      double4 p = partial[(int64_t)c * nt + t];
      ax += p.x;
      ay += p.y;
      az += p.z;
      pt += p.w;
    }
  acc[3 * t + 0] = ax;
  acc[3 * t + 1] = ay;
  acc[3 * t + 2] = az;
  pot[t]         = pt;
}

// caller index -> sorted index
__global__ void k_invert(const uint32_t *__restrict__ perm, int64_t n, int32_t *__restrict__ inv)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    inv[perm[i]] = (int32_t)i;
}

__global__ void k_map_targets(const int64_t *__restrict__ tg, int64_t nt, const int32_t *__restrict__ inv, int64_t *__restrict__ out)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(t < nt)
    out[t] = inv[tg[t]];
}
// gravity_direct (src/gravity/gravdirect.c:61-257) with force_evaluate_direct's pair arithmetic
// (src/gravity/forcetree_walk.c:557-708): the n particles are targets and sources; every thread sums
// all sources in their order with the reference's operations (FP64, no contraction), so the result is
// bit-identical.  Flag bit 1: a softening type >= nsofttypes.
__global__ void __launch_bounds__(kTile) k_gravity_direct(const double *__restrict__ pos, const double *__restrict__ mass,
                                                          const uint8_t *__restrict__ st, int64_t n,
                                                          const WalkConst *__restrict__ wcp, double *__restrict__ acc,
                                                          double *__restrict__ pot, int *__restrict__ flag)
{
  __shared__ double4 src[kTile];
  __shared__ double hsrc[kTile];
  const WalkConst &w = *wcp;
  const int64_t i    = (int64_t)blockIdx.x * kTile + threadIdx.x;
  double pos_x = 0, pos_y = 0, pos_z = 0, h_i = 0;
  if(i < n)
    {
      pos_x = pos[3 * i + 0];
      pos_y = pos[3 * i + 1];
      pos_z = pos[3 * i + 2];
      if(st[i] >= w.nsoft)
        atomicOr(flag, 1);
      h_i = w.soft[st[i] < w.nsoft ? st[i] : 0];
    }
  double acc_x = 0, acc_y = 0, acc_z = 0, pt = 0;
  for(int64_t jb = 0; jb < n && n > 1; jb += kTile)
    {
      __syncthreads();
      const int64_t j = jb + threadIdx.x;
      if(j < n)
        {
          src[threadIdx.x]  = make_double4(pos[3 * j + 0], pos[3 * j + 1], pos[3 * j + 2], mass[j]);
          hsrc[threadIdx.x] = w.soft[st[j] < w.nsoft ? st[j] : 0];
        }
      __syncthreads();
      const int cnt = (int)((n - jb) < kTile ? (n - jb) : kTile);
      if(i < n)
        for(int q = 0; q < cnt; q++)
          {
            const double4 s  = src[q];
            const double h_j = hsrc[q];
            double hmax      = (h_j > h_i) ? h_j : h_i;
            double dx = s.x - pos_x, dy = s.y - pos_y, dz = s.z - pos_z;
            if(w.periodic)
              {
                dx = (dx > w.half_box) ? (dx - w.box) : ((dx < -w.half_box) ? (dx + w.box) : dx);
                dy = (dy > w.half_box) ? (dy - w.box) : ((dy < -w.half_box) ? (dy + w.box) : dy);
                dz = (dz > w.half_box) ? (dz - w.box) : ((dz < -w.half_box) ? (dz + w.box) : dz);
              }
            double r2 = dx * dx + dy * dy + dz * dz;
            double m  = s.w;
            double r  = sqrt(r2);
            double factor_force = 0, factor_pot = 0;
            if(w.pm)
              {
                double tabentry = w.asmthfac * r;
                int tabindex    = (int)tabentry;
                if(tabindex >= kNtab)
                  continue;
                double tabweight = tabentry - tabindex;
                factor_force     = (1.0 - tabweight) * w.tab_force[tabindex] + tabweight * w.tab_force[tabindex + 1];
                factor_pot       = (1.0 - tabweight) * w.tab_pot[tabindex] + tabweight * w.tab_pot[tabindex + 1];
              }
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
            pt += m * wp;
            fac *= m;
            acc_x += dx * fac;
            acc_y += dy * fac;
            acc_z += dz * fac;
            if(w.ewald)
              {
                double fcorr[3], pcorr;
                ewald_corr(dx, dy, dz, w, fcorr, pcorr);
                acc_x += m * fcorr[0];
                acc_y += m * fcorr[1];
                acc_z += m * fcorr[2];
                pt += m * pcorr;
              }
          }
    }
  if(i < n)
    {
      acc[3 * i + 0] = acc_x;
      acc[3 * i + 1] = acc_y;
      acc[3 * i + 2] = acc_z;
      if(pot)
        pot[i] = pt;
    }
}

__global__ void k_fill_i32(int32_t *__restrict__ a, int64_t n, int32_t v)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}
}  // namespace

cudaError_t gravity_direct_stage(gpugrav_ctx *c, int64_t n, const double *d_pos, const double *d_mass, const uint8_t *d_st,
                                 double *d_acc, double *d_pot, int32_t *d_nint, int *d_flag)
{
  k_gravity_direct<<<(unsigned)((n + kTile - 1) / kTile), kTile, 0, c->stream>>>(d_pos, d_mass, d_st, n, c->wconst.as<WalkConst>(),
                                                                                   d_acc, d_pot, d_flag);
  if(d_nint)
    k_fill_i32<<<(unsigned)((n + 255) / 256 < 2368 ? (n + 255) / 256 : 2368), 256, 0, c->stream>>>(d_nint, n, (int32_t)n);
  return cudaGetLastError();
}

cudaError_t direct_stage(gpugrav_ctx *c, const WalkConst &wc, int64_t nt, const int64_t *d_targets, int cut, double *d_acc,
                         double *d_pot)
{
  (void)wc;
  if(nt == 0)
    return cudaSuccess;
  cudaError_t e;
  DevBuf inv, ts, part;
  if((e = inv.ensure(c->n * sizeof(int32_t))) != cudaSuccess || (e = ts.ensure(nt * sizeof(int64_t))) != cudaSuccess ||
     (e = part.ensure((size_t)kChunks * nt * sizeof(double4))) != cudaSuccess)
    return e;
  k_invert<<<(unsigned)((c->n + 255) / 256 < 2368 ? (c->n + 255) / 256 : 2368), 256, 0, c->stream>>>(c->perm.as<uint32_t>(), c->n,
                                                                                                       inv.as<int32_t>());
  k_map_targets<<<(unsigned)((nt + 255) / 256), 256, 0, c->stream>>>(d_targets, nt, inv.as<int32_t>(), ts.as<int64_t>());
  dim3 grid((unsigned)((nt + kTile - 1) / kTile), kChunks);
  k_direct<<<grid, kTile, 0, c->stream>>>(c->s_pm.as<double4>(), c->s_st.as<uint8_t>(), c->n, ts.as<int64_t>(), nt,
                                         c->wconst.as<WalkConst>(), cut, part.as<double4>());
  k_direct_reduce<<<(unsigned)((nt + 255) / 256), 256, 0, c->stream>>>(part.as<double4>(), nt, d_acc, d_pot);
  e = cudaGetLastError();
  cudaStreamSynchronize(c->stream);
  inv.release();
  ts.release();
  part.release();
  return e;
}
}  // namespace gg
