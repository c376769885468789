// domain.cu -- domain stage: periodic wrap, extent, Peano-Hilbert keys, stable
// key sort, gather into the sorted structure-of-arrays.  Compiled with
// -fmad=false: every double operation rounds like the reference's C.
//
//   wrap      do_box_wrapping          src/domain/domain_box.c:259-300
//   extent    domain_findExtent        src/domain/domain_box.c:107-197
//   keys      domain_double_to_int + peano_hilbert_key
//                                      src/domain/domain.c:361-370, src/domain/peano.c:374-390
//   sort      peano_hilbert_order      src/domain/peano.c:74-133 (stable: radix sort)
#include <cub/cub.cuh>

#include "internal.h"
#include "ph.cuh"

namespace gg
{
namespace
{
__constant__ PhTable c_ph;
bool g_ph_ready = false;

__device__ __forceinline__ uint64_t mant52(double d) { return (uint64_t)__double_as_longlong(d) & 0xFFFFFFFFFFFFFull; }

// do_box_wrapping: repeated +/- box until inside [0, box); bounded, reports failure
__device__ __forceinline__ bool wrap_coord(double &x, double box)
{
  int it = 0;
  while(x < 0 && it < 64)
    {
      x = __dadd_rn(x, box);
      it++;
    }
  while(x >= box && it < 128)
    {
      x = __dsub_rn(x, box);
      it++;
    }
  return x >= 0 && x < box;
}

__device__ __forceinline__ uint64_t to_int52(double x, double corner, double inv_len)
{
  return mant52(__dadd_rn(__dmul_rn(__dsub_rn(x, corner), inv_len), 1.0));
}

struct MinOp
{
  __device__ double operator()(double u, double v) const { return fmin(u, v); }
};
struct MaxOp
{
  __device__ double operator()(double u, double v) const { return fmax(u, v); }
};

// ---- extent: per-block min/max, then a single-block finalisation ----
constexpr int kExtBlocks  = 296;
constexpr int kExtThreads = 256;

__global__ void k_extent_partial(const double *__restrict__ pos, int64_t n, int periodic, double box, double *partial,
                                 int *flags)
{
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  int bad      = 0;
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      for(int j = 0; j < 3; j++)
        {
          double x = pos[3 * i + j];
          if(!isfinite(x))
            {
              bad = 1;
              continue;
            }
          if(periodic && !wrap_coord(x, box))
            bad = 1;
          mn[j] = fmin(mn[j], x);
          mx[j] = fmax(mx[j], x);
        }
    }
  typedef cub::BlockReduce<double, kExtThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  for(int j = 0; j < 3; j++)
    {
      double a = BR(tmp).Reduce(mn[j], MinOp());
      __syncthreads();
      double b = BR(tmp).Reduce(mx[j], MaxOp());
      __syncthreads();
      if(threadIdx.x == 0)
        {
          partial[blockIdx.x * 6 + j]     = a;
          partial[blockIdx.x * 6 + 3 + j] = b;
        }
    }
  if(bad)
    atomicOr(flags, 2);
}

__global__ void k_extent_final(const double *partial, int nblocks, BuildConst *bc)
{
  if(threadIdx.x != 0 || blockIdx.x != 0)
    return;
  double xmin[3], xmax[3];
  for(int j = 0; j < 3; j++)
    {
      // preset to the simulation box (src/domain/domain_box.c:113-118)
      xmin[j] = 0;
      xmax[j] = bc->box;
    }
  for(int b = 0; b < nblocks; b++)
    for(int j = 0; j < 3; j++)
      {
        if(xmin[j] > partial[b * 6 + j])
          xmin[j] = partial[b * 6 + j];
        if(xmax[j] < partial[b * 6 + 3 + j])
          xmax[j] = partial[b * 6 + 3 + j];
      }
  double len = 0;
  for(int j = 0; j < 3; j++)
    if(__dsub_rn(xmax[j], xmin[j]) > len)
      len = __dsub_rn(xmax[j], xmin[j]);
  len = __dmul_rn(len, bc->periodic ? 1.00001 : 1.2);
  for(int j = 0; j < 3; j++)
    {
      bc->dom.center[j] = __dmul_rn(0.5, __dadd_rn(xmin[j], xmax[j]));
      bc->dom.corner[j] = __dsub_rn(__dmul_rn(0.5, __dadd_rn(xmin[j], xmax[j])), __dmul_rn(0.5, len));
    }
  bc->dom.len         = len;
  bc->dom.inverse_len = __ddiv_rn(1.0, len);
  bc->dom.big_fac     = __ddiv_rn(len, 4503599627370496.0); /* 2^52 */
}

// ---- keys ----
__global__ void k_keys(const double *__restrict__ pos, int64_t n, const BuildConst *__restrict__ bc, u128 *__restrict__ key,
                       uint32_t *__restrict__ idx, int *flags)
{
  __shared__ uint16_t tab[48 * 8];
  for(int t = threadIdx.x; t < 48 * 8; t += blockDim.x)
    tab[t] = c_ph.e[t];
  __syncthreads();
  const int periodic = bc->periodic;
  const double box   = bc->box;
  const double inv   = bc->dom.inverse_len;
  const double len   = bc->dom.len;
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      uint64_t ip[3];
      int bad = 0;
      for(int j = 0; j < 3; j++)
        {
          double x = pos[3 * i + j];
          if(periodic)
            wrap_coord(x, box);
          double c = bc->dom.corner[j];
          // particle must lie in [DomainCorner, DomainCorner + DomainLen) (src/gravity/forcetree.c:411-415)
          if(!(x >= c && x < __dadd_rn(c, len)))
            bad = 1;
          ip[j] = to_int52(x, c, inv);
        }
      if(bad)
        atomicOr(flags, 1);
      key[i] = ph_key_dev(tab, ip[0] >> (52 - kBits), ip[1] >> (52 - kBits), ip[2] >> (52 - kBits), kBits);
      idx[i] = (uint32_t)i;
    }
}

// ---- gather into sorted SoA ----
__global__ void k_gather(const double *__restrict__ pos, const double *__restrict__ mass, const uint8_t *__restrict__ st,
                         const uint32_t *__restrict__ perm, int64_t n, const BuildConst *__restrict__ bc,
                         double4 *__restrict__ s_pm, uint64_t *__restrict__ s_ix, uint64_t *__restrict__ s_iy,
                         uint64_t *__restrict__ s_iz, uint8_t *__restrict__ s_st, int *flags)
{
  const int nsoft    = bc->nsoft;
  const int periodic = bc->periodic;
  const double box   = bc->box;
  const double inv   = bc->dom.inverse_len;
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      uint32_t o = perm[i];
      double x = pos[3 * (int64_t)o + 0], y = pos[3 * (int64_t)o + 1], z = pos[3 * (int64_t)o + 2];
      if(periodic)
        {
          wrap_coord(x, box);
          wrap_coord(y, box);
          wrap_coord(z, box);
        }
      s_pm[i] = make_double4(x, y, z, mass[o]);
      s_ix[i] = to_int52(x, bc->dom.corner[0], inv);
      s_iy[i] = to_int52(y, bc->dom.corner[1], inv);
      s_iz[i] = to_int52(z, bc->dom.corner[2], inv);
      uint8_t t = st[o];
      s_st[i]   = t;
      // a softening type must index ForceSoftening[0 .. nsofttypes-1]
      if(t >= nsoft)
        atomicOr(flags, 4);
    }
}

int grid_for(int64_t n, int threads)
{
  int64_t b = (n + threads - 1) / threads;
  if(b > 148 * 16)
    b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}
}  // namespace

cudaError_t domain_stage(gpugrav_ctx *c, bool compute_extent, int *status_flags)
{
  cudaError_t e;
  if(!g_ph_ready)
    {
      PhTable t = ph_make_table();
      if((e = cudaMemcpyToSymbol(c_ph, &t, sizeof(t))) != cudaSuccess)
        return e;
      g_ph_ready = true;
    }
  const int64_t n = c->n;
  if((e = c->scratch.ensure(kExtBlocks * 6 * sizeof(double) + 64)) != cudaSuccess)
    return e;
  if((e = c->counters.ensure(64 * sizeof(int))) != cudaSuccess)
    return e;
  if((e = c->key.ensure(n * sizeof(u128))) != cudaSuccess || (e = c->key_alt.ensure(n * sizeof(u128))) != cudaSuccess ||
     (e = c->idx.ensure(n * sizeof(uint32_t))) != cudaSuccess || (e = c->perm.ensure(n * sizeof(uint32_t))) != cudaSuccess)
    return e;
  int *flags = c->counters.as<int>();
  cudaMemsetAsync(flags, 0, sizeof(int), c->stream);
  BuildConst *bc = c->bconst.as<BuildConst>();
  if(compute_extent)
    {
      k_extent_partial<<<kExtBlocks, kExtThreads, 0, c->stream>>>(c->pos_in.as<double>(), n, c->prm.periodic, c->prm.box_size,
                                                                  c->scratch.as<double>(), flags);
      k_extent_final<<<1, 32, 0, c->stream>>>(c->scratch.as<double>(), kExtBlocks, bc);
    }
  k_keys<<<grid_for(n, 256), 256, 0, c->stream>>>(c->pos_in.as<double>(), n, bc, c->key.as<u128>(), c->idx.as<uint32_t>(), flags);
  if((e = cudaGetLastError()) != cudaSuccess)
    return e;
  if((e = cudaMemcpyAsync(status_flags, flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess)
    return e;
  return cudaStreamSynchronize(c->stream);
}

cudaError_t sort_stage(gpugrav_ctx *c)
{
  const int64_t n = c->n;
  cudaError_t e;
  size_t tmp_bytes = 0;
  e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, c->key.as<u128>(), c->key_alt.as<u128>(), c->idx.as<uint32_t>(),
                                      c->perm.as<uint32_t>(), (int)n, 0, 3 * kBits, c->stream);
  if(e != cudaSuccess)
    return e;
  if((e = c->sort_tmp.ensure(tmp_bytes)) != cudaSuccess)
    return e;
  // stable LSD radix sort over the 126 key bits: equal keys keep the caller order,
  // as the merge sort of peano_hilbert_order does
  e = cub::DeviceRadixSort::SortPairs(c->sort_tmp.p, tmp_bytes, c->key.as<u128>(), c->key_alt.as<u128>(), c->idx.as<uint32_t>(),
                                      c->perm.as<uint32_t>(), (int)n, 0, 3 * kBits, c->stream);
  return e;
}

cudaError_t gather_stage(gpugrav_ctx *c)
{
  const int64_t n = c->n;
  cudaError_t e;
  if((e = c->s_pm.ensure(n * sizeof(double4))) != cudaSuccess || (e = c->s_ix.ensure(n * 8)) != cudaSuccess ||
     (e = c->s_iy.ensure(n * 8)) != cudaSuccess || (e = c->s_iz.ensure(n * 8)) != cudaSuccess ||
     (e = c->s_st.ensure(n + 16)) != cudaSuccess)
    return e;
  k_gather<<<grid_for(n, 256), 256, 0, c->stream>>>(c->pos_in.as<double>(), c->mass_in.as<double>(), c->st_in.as<uint8_t>(),
                                                   c->perm.as<uint32_t>(), n, c->bconst.as<BuildConst>(), c->s_pm.as<double4>(),
                                                   c->s_ix.as<uint64_t>(), c->s_iy.as<uint64_t>(), c->s_iz.as<uint64_t>(),
                                                   c->s_st.as<uint8_t>(), c->counters.as<int>());
  return cudaGetLastError();
}
}  // namespace gg
