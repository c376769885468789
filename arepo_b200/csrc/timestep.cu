// timestep.cu -- gravity time steps and time bins on the device.  Compiled with -fmad=false.
//
// get_timestep_gravity (src/time_integration/timestep.c:284-353) with the same operations in the same
// order (bit-identical integer steps), the bin assignment of timebins_get_bin_and_do_validity_checks
// (timestep.c:725-770), and the compaction of the active particles of the synchronized bins (the
// TimeBinsGravity.ActiveParticleList that gravity_tree's TargetList is made from).
#include <cub/cub.cuh>

#include "internal.h"

namespace gg
{
namespace
{
struct TsConst
{
  gpugrav_timestep_params p;
  double soft[GPUGRAV_MAX_SOFTTYPES + 1];
  int32_t nsoft;
};

// error codes (first failing particle kept in fail[1]): 1 below MinSizeTimestep, 2 integer step out
// of (0, TIMEBASE), 3 integer step 1, 4 beyond the end of the timeline, 5 softening type >= nsofttypes
__device__ __forceinline__ void ts_fail(int *fail, unsigned long long *first, int code, int64_t i)
{
  atomicCAS(fail, 0, code);
  atomicMin(first, (unsigned long long)i);
}

__global__ void k_timestep_gravity(const TsConst *__restrict__ cp, int64_t n, const double *__restrict__ acc,
                                   const double *__restrict__ pm, const double *__restrict__ mass, const uint64_t *__restrict__ ids,
                                   const uint8_t *__restrict__ st, const int8_t *__restrict__ bin_old, int64_t *__restrict__ ti_out,
                                   int8_t *__restrict__ bin_out, int *__restrict__ fail, unsigned long long *__restrict__ first)
{
  const TsConst &c              = *cp;
  const gpugrav_timestep_params &t = c.p;
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      if(st[i] >= c.nsoft)
        {
          ts_fail(fail, first, 5, i);
          continue;
        }
      double ax = t.cf_a2inv * acc[3 * i + 0];
      double ay = t.cf_a2inv * acc[3 * i + 1];
      double az = t.cf_a2inv * acc[3 * i + 2];
      if(pm)
        {
          ax += t.cf_a2inv * pm[3 * i + 0];
          ay += t.cf_a2inv * pm[3 * i + 1];
          az += t.cf_a2inv * pm[3 * i + 2];
        }
      double ac = sqrt(ax * ax + ay * ay + az * az);
      if(ac == 0)
        ac = 1.0e-30;
      double dt = sqrt(2 * t.err_tol_int_accuracy * t.cf_atime * c.soft[st[i]] / 2.8 / ac);
      dt *= t.cf_hubble_a;
      if(mass[i] == 0 && ids && ids[i] == 0)
        dt = t.max_size_timestep;
      if(dt >= t.max_size_timestep)
        dt = t.max_size_timestep;
      if(dt < t.min_size_timestep)
        {
          if(t.nostop_below_min)
            dt = t.min_size_timestep;
          else
            ts_fail(fail, first, 1, i);
        }
      if(t.dt_displacement > 0 && dt >= t.dt_displacement)
        dt = t.dt_displacement;
      // integertime of the build: int (TIMEBINS 29) or long long
      const int64_t ti_step = t.timebase <= ((int64_t)1 << 30) ? (int64_t)(int)(dt / t.timebase_interval)
                                                                 : (int64_t)(dt / t.timebase_interval);
      if(!(ti_step > 0 && ti_step < t.timebase))
        ts_fail(fail, first, 2, i);
      ti_out[i] = ti_step;
      // the bin: power-of-two subdivision, only synchronized bins for a longer step
      int64_t ti_min = t.timebase;
      while(ti_min > ti_step)
        ti_min >>= 1;
      int64_t ts = ti_min;
      int bin    = -1;
      if(ts == 0)
        bin = 0;
      if(ts == 1)
        ts_fail(fail, first, 3, i);
      while(ts)
        {
          bin++;
          ts >>= 1;
        }
      // (ts is 0 here, as the reference's ti_step after its bit loop; only a raised step is checked below)
      const int bo = bin_old[i];
      if(bin > bo)
        {
          while(bin > bo && !t.synchronized[bin])
            bin--;
          ts = bin ? ((int64_t)1 << bin) : 0;
        }
      if(t.ti_current >= t.timebase)
        {
          ts  = 0;
          bin = 0;
        }
      if(t.timebase - t.ti_current < ts)
        ts_fail(fail, first, 4, i);
      bin_out[i] = (int8_t)bin;
    }
}

__global__ void k_active_flags(int64_t n, const int8_t *__restrict__ bin, const uint8_t *__restrict__ sync, int32_t *__restrict__ flag)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      const int b = bin[i];
      flag[i]     = (b >= 0 && b < 64 && sync[b]) ? 1 : 0;
    }
}

__global__ void k_active_scatter(int64_t n, const int32_t *__restrict__ flag, const int32_t *__restrict__ pos, int32_t *__restrict__ list,
                                 int64_t *__restrict__ count)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      if(flag[i])
        list[pos[i]] = (int32_t)i;
      if(i == n - 1)
        *count = (int64_t)pos[i] + flag[i];
    }
}

int grid_for(int64_t n)
{
  int64_t b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}
}  // namespace

cudaError_t timestep_stage(gpugrav_ctx *c, const gpugrav_timestep_params *tp, int64_t n, const double *acc, const double *pm,
                           const double *mass, const uint64_t *ids, const uint8_t *st, const int8_t *bin_old, int64_t *ti,
                           int8_t *bin, int *fail_code, int64_t *first)
{
  TsConst h;
  memset(&h, 0, sizeof(h));
  h.p     = *tp;
  h.nsoft = c->prm.nsofttypes;
  for(int i = 0; i <= GPUGRAV_MAX_SOFTTYPES; i++)
    h.soft[i] = c->prm.force_softening[i];
  GG_TRY(c->scratch.ensure(sizeof(TsConst) + 256));
  char *sp = c->scratch.as<char>();
  int *d_fail = (int *)(sp + sizeof(TsConst) + 16);
  unsigned long long *d_first = (unsigned long long *)(sp + sizeof(TsConst) + 32);
  GG_TRY(cudaMemcpyAsync(sp, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  GG_TRY(cudaMemsetAsync(d_fail, 0, sizeof(int), c->stream));
  GG_TRY(cudaMemsetAsync(d_first, 0xff, sizeof(unsigned long long), c->stream));
  k_timestep_gravity<<<grid_for(n), 256, 0, c->stream>>>((const TsConst *)sp, n, acc, pm, mass, ids, st, bin_old, ti, bin, d_fail,
                                                         d_first);
  GG_TRY(cudaGetLastError());
  unsigned long long f = 0;
  GG_TRY(cudaMemcpyAsync(fail_code, d_fail, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GG_TRY(cudaMemcpyAsync(&f, d_first, sizeof(f), cudaMemcpyDeviceToHost, c->stream));
  GG_TRY(cudaStreamSynchronize(c->stream));  // `h` lives on this stack frame
  *first = (int64_t)f;
  return cudaSuccess;
}

cudaError_t active_stage(gpugrav_ctx *c, int64_t n, const int8_t *bin, const uint8_t *d_sync, int32_t *list, int64_t *d_count)
{
  GG_TRY(c->cnt.ensure(n * sizeof(int32_t) + 16));
  GG_TRY(c->base.ensure(n * sizeof(int32_t) + 16));
  k_active_flags<<<grid_for(n), 256, 0, c->stream>>>(n, bin, d_sync, c->cnt.as<int32_t>());
  size_t tb = 0;
  GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->cnt.as<int32_t>(), c->base.as<int32_t>(), (int)n, c->stream));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, c->cnt.as<int32_t>(), c->base.as<int32_t>(), (int)n, c->stream));
  k_active_scatter<<<grid_for(n), 256, 0, c->stream>>>(n, c->cnt.as<int32_t>(), c->base.as<int32_t>(), list, d_count);
  return cudaGetLastError();
}
}  // namespace gg
