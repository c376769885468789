// targets.cu -- walks of an active subset of the particles.
//
// gravity_tree(timebin) walks only the particles of the current gravity time bin: it builds
// TargetList from TimeBinsGravity.ActiveParticleList (src/gravity/gravtree.c:494-520) while the
// tree holds every particle.  Here the caller's list of active particles (caller indices, any order)
// becomes a list of sorted particle positions in Peano-Hilbert order, so that the FP64 walk's warps
// and the FP32 walk's groups take spatially close active targets together; results go back in the
// order of the caller's list.
#include <cub/cub.cuh>

#include "internal.h"

namespace gg
{
namespace
{
int grid_for(int64_t n, int threads)
{
  int64_t b = (n + threads - 1) / threads;
  if(b > 148 * 16)
    b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

// iperm[caller index] = sorted position
__global__ void k_inv_perm(int64_t n, const uint32_t *__restrict__ perm, uint32_t *__restrict__ iperm)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    iperm[perm[i]] = (uint32_t)i;
}

// sorted position of every listed target (flag bit 1: index out of range)
__global__ void k_target_pos(int64_t nt, const int32_t *__restrict__ targets, int64_t n, const uint32_t *__restrict__ iperm,
                             uint32_t *__restrict__ pos, uint32_t *__restrict__ idx, int *__restrict__ flag)
{
  for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nt; j += (int64_t)gridDim.x * blockDim.x)
    {
      const int32_t t = targets[j];
      if(t < 0 || t >= n)
        {
          atomicOr(flag, 1);
          pos[j] = 0;
        }
      else
        pos[j] = iperm[t];
      idx[j] = (uint32_t)j;
    }
}

// flag bit 2: a particle listed twice
__global__ void k_target_dups(int64_t nt, const uint32_t *__restrict__ pos, int *__restrict__ flag)
{
  for(int64_t j = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nt; j += (int64_t)gridDim.x * blockDim.x)
    if(pos[j] == pos[j - 1])
      atomicOr(flag, 2);
}

// results of the active list back to the caller's list order; entries outside [a, b) of the
// active list (another rank's target slice) are written as zero
__global__ void k_scatter_targets(int64_t nt, const uint32_t *__restrict__ tpos, const uint32_t *__restrict__ tidx, int64_t a,
                                  int64_t b, const double *__restrict__ acc_s, const double *__restrict__ pot_s,
                                  const int32_t *__restrict__ nint_s, double *__restrict__ acc, double *__restrict__ pot,
                                  int32_t *__restrict__ nint)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nt; i += (int64_t)gridDim.x * blockDim.x)
    {
      const int64_t o = tidx[i], s = tpos[i];
      const bool in   = i >= a && i < b;
      acc[3 * o + 0]  = in ? acc_s[3 * s + 0] : 0.0;
      acc[3 * o + 1]  = in ? acc_s[3 * s + 1] : 0.0;
      acc[3 * o + 2]  = in ? acc_s[3 * s + 2] : 0.0;
      if(pot)
        pot[o] = in ? pot_s[s] : 0.0;
      if(nint)
        nint[o] = in ? nint_s[s] : 0;
    }
}
}  // namespace

// Sorted positions of the caller's active list in key order (t_pos_alt) and their places in the
// list (t_idx_alt); flags: bit 1 an index outside [0, n), bit 2 a particle listed twice.
cudaError_t targets_stage(gpugrav_ctx *c, int64_t nt, const int32_t *d_targets, int *flags)
{
  cudaStream_t st = c->stream;
  const int64_t n = c->n;
  GG_TRY(c->iperm.ensure(n * sizeof(uint32_t)));
  GG_TRY(c->t_pos.ensure(nt * sizeof(uint32_t) + 16));
  GG_TRY(c->t_pos_alt.ensure(nt * sizeof(uint32_t) + 16));
  GG_TRY(c->t_idx.ensure(nt * sizeof(uint32_t) + 16));
  GG_TRY(c->t_idx_alt.ensure(nt * sizeof(uint32_t) + 16));
  int *flag = c->counters.as<int>() + 16;
  GG_TRY(cudaMemsetAsync(flag, 0, sizeof(int), st));
  k_inv_perm<<<grid_for(n, 256), 256, 0, st>>>(n, c->perm.as<uint32_t>(), c->iperm.as<uint32_t>());
  k_target_pos<<<grid_for(nt, 256), 256, 0, st>>>(nt, d_targets, n, c->iperm.as<uint32_t>(), c->t_pos.as<uint32_t>(),
                                                  c->t_idx.as<uint32_t>(), flag);
  int bits = 1;
  while(bits < 32 && ((int64_t)1 << bits) < n)
    bits++;
  size_t tb = 0;
  GG_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, c->t_pos.as<uint32_t>(), c->t_pos_alt.as<uint32_t>(),
                                         c->t_idx.as<uint32_t>(), c->t_idx_alt.as<uint32_t>(), (int)nt, 0, bits, st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(cub::DeviceRadixSort::SortPairs(c->sort_tmp.p, tb, c->t_pos.as<uint32_t>(), c->t_pos_alt.as<uint32_t>(),
                                         c->t_idx.as<uint32_t>(), c->t_idx_alt.as<uint32_t>(), (int)nt, 0, bits, st));
  k_target_dups<<<grid_for(nt, 256), 256, 0, st>>>(nt, c->t_pos_alt.as<uint32_t>(), flag);
  GG_TRY(cudaGetLastError());
  GG_TRY(cudaMemcpyAsync(flags, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  GG_TRY(cudaStreamSynchronize(st));
  return cudaSuccess;
}

cudaError_t targets_scatter(gpugrav_ctx *c, int64_t nt, int64_t a, int64_t b, double *acc, double *pot, int32_t *nint)
{
  k_scatter_targets<<<grid_for(nt, 256), 256, 0, c->stream>>>(nt, c->t_pos_alt.as<uint32_t>(), c->t_idx_alt.as<uint32_t>(), a, b,
                                                             c->acc_s.as<double>(), c->pot_s.as<double>(),
                                                             c->nint_s.as<int32_t>(), acc, pot, nint);
  return cudaGetLastError();
}
}  // namespace gg
