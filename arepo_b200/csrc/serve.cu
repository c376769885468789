// serve.cu -- continuous-batching serving loop for many independent isolated
// N-body systems (each: a Barnes-Hut force pass, a relative-criterion pass, then
// K kick-drift-kick leapfrog steps, as compute_grav_accelerations / the KDK step
// of the reference do: src/gravity/accel.c:58-80, src/time_integration/
// do_gravity_hydro.c:63-83, src/time_integration/predict.c:357-425).
//
// Requests are admitted at tick boundaries while slots, the particle pool and the
// device-memory budget allow.  Every tick advances all admitted systems by one
// force evaluation: one batched build over all of them (keys carry the system's
// slot in their top bits, so each system gets its own root and canonical octree on
// its own domain grid) and one persistent FP32 walk over per-system target groups.
// A system's arithmetic never depends on which other systems share the tick:
// its keys, order, tree, traversal and sums are the same alone and in the mix.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "internal.h"
#include "ph.cuh"

namespace gg
{
namespace
{
__constant__ PhTable c_ph_srv;
int g_ph_srv_ready[64] = {0};

enum
{
  ST_NEW  = 0,  // this tick: Barnes-Hut force at the initial positions
  ST_INIT = 1,  // this tick: relative-criterion force at the initial positions
  ST_STEP = 2,  // this tick: kick + drift, force, kick
  ST_DONE = 3
};

// per system of the current tick (device copy)
struct SysDev
{
  int64_t pool_off;  // first particle in the pool
  int64_t coff;      // first particle in tick-compact (and sorted) order
  int32_t n;
  int32_t state;
  double dt;
};

__device__ __forceinline__ int find_sys(const int64_t *__restrict__ starts, int nsys, int64_t i)
{
  int lo = 0, hi = nsys - 1;
  while(lo < hi)
    {
      int m = (lo + hi + 1) >> 1;
      if(starts[m] <= i)
        lo = m;
      else
        hi = m - 1;
    }
  return lo;
}

__device__ __forceinline__ uint64_t mant52(double d) { return (uint64_t)__double_as_longlong(d) & 0xFFFFFFFFFFFFFull; }

// compact index -> pool index and system
__global__ void k_srv_expand(int64_t ntot, int nsys, const SysDev *__restrict__ sys, const int64_t *__restrict__ cstart,
                             int64_t *__restrict__ c2p, int32_t *__restrict__ csys)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ntot; i += (int64_t)gridDim.x * blockDim.x)
    {
      int s   = find_sys(cstart, nsys, i);
      c2p[i]  = sys[s].pool_off + (i - sys[s].coff);
      csys[i] = s;
    }
}

// kick + drift of the systems that are stepping (before their force)
__global__ void k_srv_pre(int64_t ntot, const SysDev *__restrict__ sys, const int64_t *__restrict__ c2p,
                          const int32_t *__restrict__ csys, double4 *__restrict__ pos, double4 *__restrict__ vel,
                          const double4 *__restrict__ acc)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ntot; i += (int64_t)gridDim.x * blockDim.x)
    {
      const SysDev &S = sys[csys[i]];
      if(S.state != ST_STEP)
        continue;
      int64_t p = c2p[i];
      double4 v = vel[p], a = acc[p], x = pos[p];
      const double h = 0.5 * S.dt;
      v.x += a.x * h;
      v.y += a.y * h;
      v.z += a.z * h;
      x.x += v.x * S.dt;
      x.y += v.y * S.dt;
      x.z += v.z * S.dt;
      vel[p] = v;
      pos[p] = x;
    }
}

// Order-preserving map of a double onto an unsigned integer (for atomic min / max).
__device__ __forceinline__ unsigned long long ord64(double x)
{
  const unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord64(unsigned long long u)
{
  return __longlong_as_double((long long)((u >> 63) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u));
}

// Extent of every system: blockIdx.y strides over the system's particles; partial boxes are
// combined with atomics on ord64 values (ext: per system 3 minima then 3 maxima, preset by the host
// to all-ones and zero).
__global__ void k_srv_extent(int nsys, const SysDev *__restrict__ sys, const int64_t *__restrict__ c2p,
                             const double4 *__restrict__ pos, unsigned long long *__restrict__ ext)
{
  const int s = blockIdx.x;
  if(s >= nsys)
    return;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  const int64_t n = sys[s].n, coff = sys[s].coff;
  for(int64_t i = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.y * blockDim.x)
    {
      const double4 x = pos[c2p[coff + i]];
      mn[0] = fmin(mn[0], x.x), mx[0] = fmax(mx[0], x.x);
      mn[1] = fmin(mn[1], x.y), mx[1] = fmax(mx[1], x.y);
      mn[2] = fmin(mn[2], x.z), mx[2] = fmax(mx[2], x.z);
    }
  for(int j = 0; j < 3; j++)
    for(int o = 16; o > 0; o >>= 1)
      {
        mn[j] = fmin(mn[j], __shfl_xor_sync(0xffffffffu, mn[j], o));
        mx[j] = fmax(mx[j], __shfl_xor_sync(0xffffffffu, mx[j], o));
      }
  if((threadIdx.x & 31) == 0 && (int64_t)blockIdx.y * blockDim.x + threadIdx.x < n)
    for(int j = 0; j < 3; j++)
      {
        atomicMin(&ext[6 * s + j], ord64(mn[j]));
        atomicMax(&ext[6 * s + 3 + j], ord64(mx[j]));
      }
}

// domain of every system: cube of 1.2 times the largest extent around the box centre
__global__ void k_srv_domains(int nsys, const unsigned long long *__restrict__ ext, gpugrav_domain *__restrict__ doms)
{
  for(int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x)
    {
      double lo[3], hi[3], len = 0;
      for(int j = 0; j < 3; j++)
        {
          lo[j] = unord64(ext[6 * s + j]);
          hi[j] = unord64(ext[6 * s + 3 + j]);
          len   = fmax(len, hi[j] - lo[j]);
        }
      len = 1.2 * (len > 0 ? len : 1.0);
      gpugrav_domain d;
      for(int j = 0; j < 3; j++)
        {
          d.center[j] = 0.5 * (lo[j] + hi[j]);
          d.corner[j] = d.center[j] - 0.5 * len;
        }
      d.len         = len;
      d.inverse_len = 1.0 / len;
      d.big_fac     = len / 4503599627370496.0;
      doms[s]       = d;
    }
}

// admitted system: submitted arrays pos (3n) | vel (3n) | mass (n), softening types -> pool
__global__ void k_srv_unpack(int64_t n, int64_t off, const double *__restrict__ in, const uint8_t *__restrict__ st,
                             double4 *__restrict__ pos, double4 *__restrict__ vel, uint8_t *__restrict__ stype)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      pos[off + i]   = make_double4(in[3 * i], in[3 * i + 1], in[3 * i + 2], in[6 * n + i]);
      vel[off + i]   = make_double4(in[3 * (n + i)], in[3 * (n + i) + 1], in[3 * (n + i) + 2], 0.0);
      stype[off + i] = st[i];
    }
}

// finished systems: pool (double4) -> packed pos | vel | acc (3n doubles each) for one download
__global__ void k_srv_pack(int64_t n, int64_t off, const double4 *__restrict__ pos, const double4 *__restrict__ vel,
                           const double4 *__restrict__ acc, double *__restrict__ out)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      const double4 p = pos[off + i], v = vel[off + i], a = acc[off + i];
      out[3 * i + 0] = p.x, out[3 * i + 1] = p.y, out[3 * i + 2] = p.z;
      out[3 * (n + i) + 0] = v.x, out[3 * (n + i) + 1] = v.y, out[3 * (n + i) + 2] = v.z;
      out[3 * (2 * n + i) + 0] = a.x, out[3 * (2 * n + i) + 1] = a.y, out[3 * (2 * n + i) + 2] = a.z;
    }
}

__device__ __forceinline__ uint64_t to52(double x, double corner, double inv) { return mant52((x - corner) * inv + 1.0); }

// key = slot of the system in the top bits, then the system's 126-bit Peano-Hilbert key
__global__ void k_srv_keys(int64_t ntot, const int32_t *__restrict__ csys, const int64_t *__restrict__ c2p,
                           const double4 *__restrict__ pos, const gpugrav_domain *__restrict__ doms, u128 *__restrict__ key,
                           uint32_t *__restrict__ idx)
{
  __shared__ uint16_t tab[48 * 8];
  for(int t = threadIdx.x; t < 48 * 8; t += blockDim.x)
    tab[t] = c_ph_srv.e[t];
  __syncthreads();
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ntot; i += (int64_t)gridDim.x * blockDim.x)
    {
      const int s              = csys[i];
      const gpugrav_domain &d  = doms[s];
      const double4 x          = pos[c2p[i]];
      uint64_t ix = to52(x.x, d.corner[0], d.inverse_len), iy = to52(x.y, d.corner[1], d.inverse_len),
               iz = to52(x.z, d.corner[2], d.inverse_len);
      u128 k = ph_key_dev(tab, ix >> 10, iy >> 10, iz >> 10, kBits);
      key[i] = ((u128)(uint32_t)s << 114) | (k >> 12);
      idx[i] = (uint32_t)i;
    }
}

__global__ void k_srv_gather(int64_t ntot, const uint32_t *__restrict__ sorted_idx, const int32_t *__restrict__ csys,
                             const int64_t *__restrict__ c2p, const double4 *__restrict__ pos, const uint8_t *__restrict__ st,
                             const float *__restrict__ oldacc, const gpugrav_domain *__restrict__ doms,
                             double4 *__restrict__ s_pm, uint64_t *__restrict__ s_ix, uint64_t *__restrict__ s_iy,
                             uint64_t *__restrict__ s_iz, uint8_t *__restrict__ s_st, int32_t *__restrict__ m_sys,
                             int64_t *__restrict__ s2p, float *__restrict__ s_old)
{
  for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ntot; j += (int64_t)gridDim.x * blockDim.x)
    {
      const uint32_t i        = sorted_idx[j];
      const int s             = csys[i];
      const int64_t p         = c2p[i];
      const gpugrav_domain &d = doms[s];
      const double4 x         = pos[p];
      s_pm[j]  = x;
      s_ix[j]  = to52(x.x, d.corner[0], d.inverse_len);
      s_iy[j]  = to52(x.y, d.corner[1], d.inverse_len);
      s_iz[j]  = to52(x.z, d.corner[2], d.inverse_len);
      s_st[j]  = st[p];
      m_sys[j] = s;
      s2p[j]   = p;
      s_old[j] = oldacc[p];
    }
}

// criterion per group: Barnes-Hut for systems on their first force evaluation
__global__ void k_srv_bh(const int *__restrict__ ngroups, const SysDev *__restrict__ sys, int4 *__restrict__ groups)
{
  const int ng = *ngroups;
  for(int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x)
    groups[g].w = sys[groups[g].z].state == ST_NEW ? 1 : 0;
}

// store forces, kick the stepping systems, OldAcc = |a| for the next relative pass
__global__ void k_srv_post(const int64_t *__restrict__ dntot, const int32_t *__restrict__ m_sys, const SysDev *__restrict__ sys,
                           const int64_t *__restrict__ s2p, const double *__restrict__ acc_s, double4 *__restrict__ vel,
                           double4 *__restrict__ acc, float *__restrict__ oldacc)
{
  const int64_t ntot = *dntot;
  for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ntot; j += (int64_t)gridDim.x * blockDim.x)
    {
      const int64_t p  = s2p[j];
      const SysDev &S  = sys[m_sys[j]];
      double4 a        = make_double4(acc_s[3 * j + 0], acc_s[3 * j + 1], acc_s[3 * j + 2], 0.0);
      acc[p]           = a;
      oldacc[p]        = (float)sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
      if(S.state == ST_STEP)
        {
          double4 v     = vel[p];
          const double h = 0.5 * S.dt;
          v.x += a.x * h;
          v.y += a.y * h;
          v.z += a.z * h;
          vel[p] = v;
        }
    }
}

int grid_for(int64_t n, int threads)
{
  int64_t b = (n + threads - 1) / threads;
  if(b > 148 * 16)
    b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace
}  // namespace gg

using namespace gg;

struct gpugrav_serve
{
  gpugrav_ctx *ctx = nullptr;  // build + walk machinery (several-systems mode)
  gpugrav_params prm{};
  gpugrav_serve_config cfg{};
  int device = 0;
  cudaStream_t st = nullptr;

  struct Req
  {
    int64_t id = 0;
    int64_t n  = 0;
    int32_t nsteps = 0;
    double dt      = 0;
    std::unique_ptr<double[]> in;  // pos (3n) | vel (3n) | mass (n), until admitted (not resident)
    std::unique_ptr<uint8_t[]> st;
    bool resident = false;         // particles already in the pool (placed at submission)
    // running
    int32_t state = ST_NEW, steps_done = 0;
    int64_t pool_off = -1;
    double t_submit = 0, t_admit = 0, t_done = 0;
    // result
  };
  std::deque<Req *> queue;       // waiting for admission (arrival order)
  std::vector<Req *> active;     // admitted, in admission order
  std::deque<Req *> finished;    // results waiting to be polled
  std::map<int64_t, int64_t> free_ranges;  // pool offset -> length
  int64_t pool_cap = 0;
  int64_t bytes_per_particle = 0;

  gg::DevBuf pos, vel, acc, oldacc, stype;  // particle pool
  gg::DevBuf sysdev, cstart, c2p, csys, s2p, ntot_dev, ext, up, dl;
  gg::PinnedBuf staging;

  // captured walk + store/kick graph; re-captured when a buffer it names moves
  cudaGraphExec_t graph = nullptr;
  std::vector<const void *> graph_key;
  int64_t graph_captures = 0, graph_replays = 0;

  gpugrav_serve_stats stats{};
  std::string err;
};

namespace
{
int sfail(gpugrav_serve *s, int status, const char *what, cudaError_t e = cudaSuccess)
{
  char buf[512];
  if(e != cudaSuccess)
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
  else
    snprintf(buf, sizeof(buf), "%s", what);
  if(s)
    s->err = buf;
  return status;
}
#define SCK(call, what)                                \
  do                                                   \
    {                                                  \
      cudaError_t _e = (call);                         \
      if(_e != cudaSuccess)                            \
        return sfail(s, GPUGRAV_ERR_CUDA, what, _e);   \
    }                                                  \
  while(0)

bool pool_alloc(gpugrav_serve *s, int64_t n, int64_t *off)
{
  for(auto it = s->free_ranges.begin(); it != s->free_ranges.end(); ++it)
    if(it->second >= n)
      {
        *off         = it->first;
        int64_t rest = it->second - n, start = it->first + n;
        s->free_ranges.erase(it);
        if(rest > 0)
          s->free_ranges[start] = rest;
        return true;
      }
  return false;
}

void pool_free(gpugrav_serve *s, int64_t off, int64_t n)
{
  auto it = s->free_ranges.emplace(off, n).first;
  auto nx = std::next(it);
  if(nx != s->free_ranges.end() && it->first + it->second == nx->first)
    {
      it->second += nx->second;
      s->free_ranges.erase(nx);
    }
  if(it != s->free_ranges.begin())
    {
      auto pv = std::prev(it);
      if(pv->first + pv->second == it->first)
        {
          pv->second += it->second;
          s->free_ranges.erase(it);
        }
    }
}

cudaError_t serve_reserve(gpugrav_serve *s)
{
  gpugrav_ctx *c  = s->ctx;
  const int64_t n = s->pool_cap;
  const int nsys  = s->cfg.max_systems;
  GG_TRY(c->m_doms.ensure((size_t)nsys * sizeof(gpugrav_domain)));
  GG_TRY(c->key.ensure(n * sizeof(u128)));
  GG_TRY(c->key_alt.ensure(n * sizeof(u128)));
  GG_TRY(c->idx.ensure(n * 4));
  GG_TRY(c->perm.ensure(n * 4));
  GG_TRY(c->s_pm.ensure(n * sizeof(double4)));
  GG_TRY(c->s_ix.ensure(n * 8));
  GG_TRY(c->s_iy.ensure(n * 8));
  GG_TRY(c->s_iz.ensure(n * 8));
  GG_TRY(c->s_st.ensure(n + 16));
  GG_TRY(c->m_sys.ensure(n * 4));
  GG_TRY(c->oldacc_s.ensure(n * 4));
  GG_TRY(c->acc_s.ensure(n * 24));
  GG_TRY(c->pot_s.ensure(n * 8));
  GG_TRY(c->nint_s.ensure(n * 4));
  size_t tb = 0;
  GG_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tb, c->key.as<u128>(), c->key_alt.as<u128>(), c->idx.as<uint32_t>(),
                                         c->perm.as<uint32_t>(), (int)n, 0, 128, s->st));
  GG_TRY(c->sort_tmp.ensure(tb));
  GG_TRY(gg::build_reserve(c, n, n, nsys));
  GG_TRY(gg::layout32_reserve(c, n, n));
  GG_TRY(s->up.ensure((size_t)n * (7 * sizeof(double) + 1)));
  // pinned staging of the result downloads: requests up to 2^20 particles without a later allocation
  GG_TRY(s->staging.ensure((size_t)(n < (1 << 20) ? n : (1 << 20)) * 9 * sizeof(double)));
  return s->dl.ensure((size_t)n * 9 * sizeof(double));
}

// Host copy between the caller's (pageable) arrays and pinned staging.  One thread moves only a
// few GB/s through pageable memory, so copies of several MB are split over up to 8 threads.
void host_copy(void *dst, const void *src, size_t bytes)
{
  constexpr size_t kMinPerThread = 4u << 20;
  unsigned t = std::thread::hardware_concurrency();
  t          = t > 8 ? 8 : t;
  if(bytes < 2 * kMinPerThread || t < 2)
    {
      memcpy(dst, src, bytes);
      return;
    }
  if((size_t)t > bytes / kMinPerThread)
    t = (unsigned)(bytes / kMinPerThread);
  const size_t per = ((bytes + t - 1) / t + 4095) & ~(size_t)4095;
  std::vector<std::thread> pool;
  size_t done = per;  // the first piece is copied by this thread
  try
    {
      for(; done < bytes; done += per)
        {
          const size_t len = bytes - done < per ? bytes - done : per;
          pool.emplace_back([=] { memcpy((char *)dst + done, (const char *)src + done, len); });
        }
    }
  catch(...)
    {
      // no thread to be had: copy the rest here
      memcpy((char *)dst + done, (const char *)src + done, bytes - done);
    }
  memcpy(dst, src, per < bytes ? per : bytes);
  for(auto &th : pool)
    th.join();
}

// caller arrays -> pool at off, through the upload buffer: (x, y, z, m), (vx, vy, vz, 0), types.
// When the pinned staging (reserved at creation) holds the request, the arrays are packed there and
// sent in one DMA; the call then waits for it, since the staging serves the next copy too.
cudaError_t upload(gpugrav_serve *s, int64_t off, int64_t n, const double *pos, const double *vel, const double *mass,
                   const uint8_t *st)
{
  cudaStream_t q = s->st;
  GG_TRY(s->up.ensure((size_t)n * (7 * sizeof(double) + 1)));
  double *din  = s->up.as<double>();
  uint8_t *dst = (uint8_t *)(din + 7 * n);
  const size_t bytes = (size_t)n * (7 * sizeof(double) + 1);
  if(bytes <= s->staging.cap)
    {
      double *h = (double *)s->staging.p;
      host_copy(h, pos, (size_t)n * 3 * sizeof(double));
      host_copy(h + 3 * n, vel, (size_t)n * 3 * sizeof(double));
      host_copy(h + 6 * n, mass, (size_t)n * sizeof(double));
      memcpy(h + 7 * n, st, n);
      GG_TRY(cudaMemcpyAsync(din, h, bytes, cudaMemcpyHostToDevice, q));
      GG_TRY(cudaStreamSynchronize(q));
    }
  else
    {
      GG_TRY(cudaMemcpyAsync(din, pos, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, q));
      GG_TRY(cudaMemcpyAsync(din + 3 * n, vel, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, q));
      GG_TRY(cudaMemcpyAsync(din + 6 * n, mass, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, q));
      GG_TRY(cudaMemcpyAsync(dst, st, n, cudaMemcpyHostToDevice, q));
    }
  k_srv_unpack<<<grid_for(n, 256), 256, 0, q>>>(n, off, din, dst, s->pos.as<double4>(), s->vel.as<double4>(),
                                                s->stype.as<uint8_t>());
  return cudaGetLastError();
}

int64_t in_flight(const gpugrav_serve *s)
{
  int64_t t = 0;
  for(auto *r : s->active)
    t += r->n;
  for(auto *r : s->finished)  // results stay in the pool until polled
    t += r->n;
  return t;
}
}  // namespace

extern "C" {

int32_t gpugrav_serve_create(gpugrav_serve **out, int32_t device, const gpugrav_params *params, const gpugrav_serve_config *cfg)
{
  if(!out || !params || !cfg || cfg->abi_version != GPUGRAV_ABI_VERSION || cfg->max_systems < 1 || cfg->max_particles < 64)
    return GPUGRAV_ERR_INVALID;
  if(params->periodic)
    return GPUGRAV_ERR_UNSUPPORTED;  // the serving loop runs isolated systems
  gpugrav_params p = *params;
  p.precision      = GPUGRAV_PREC_FP32;
  *out             = nullptr;
  gpugrav_ctx *ctx = nullptr;
  int r            = gpugrav_create(&ctx, device, &p);
  if(r != GPUGRAV_OK)
    return r;
  gpugrav_serve *s = new gpugrav_serve();
  s->ctx           = ctx;
  s->prm           = p;
  s->cfg           = *cfg;
  s->device        = device;
  s->st            = ctx->stream;
  ctx->multi       = true;
  int prev         = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  if(device < 64 && !g_ph_srv_ready[device])
    {
      PhTable t = ph_make_table();
      cudaMemcpyToSymbol(c_ph_srv, &t, sizeof(t));
      g_ph_srv_ready[device] = 1;
    }
  // particle pool sized by max_particles; admission also keeps the estimated device
  // footprint of the particles in flight under the budget
  s->pool_cap           = cfg->max_particles;
  s->bytes_per_particle = 700;  // pool + sorted arrays + tree + walk layout, measured upper estimate
  bool ok = s->pos.ensure(s->pool_cap * sizeof(double4)) == cudaSuccess &&
            s->vel.ensure(s->pool_cap * sizeof(double4)) == cudaSuccess &&
            s->acc.ensure(s->pool_cap * sizeof(double4)) == cudaSuccess &&
            s->oldacc.ensure(s->pool_cap * sizeof(float)) == cudaSuccess &&
            s->stype.ensure(s->pool_cap + 16) == cudaSuccess &&
            s->sysdev.ensure((size_t)cfg->max_systems * sizeof(SysDev)) == cudaSuccess &&
            s->cstart.ensure((size_t)(cfg->max_systems + 1) * 8) == cudaSuccess &&
            s->c2p.ensure(s->pool_cap * 8) == cudaSuccess && s->csys.ensure(s->pool_cap * 4) == cudaSuccess &&
            s->s2p.ensure(s->pool_cap * 8) == cudaSuccess && s->ntot_dev.ensure(64) == cudaSuccess &&
            s->ext.ensure((size_t)cfg->max_systems * 6 * 8) == cudaSuccess;
  // the build context's constants (isolated, softening table)
  if(ok)
    {
      BuildConst bc;
      memset(&bc, 0, sizeof(bc));
      bc.periodic = 0;
      bc.nsoft    = p.nsofttypes;
      bc.box      = p.box_size;
      for(int i = 0; i <= p.nsofttypes; i++)
        bc.soft[i] = p.force_softening[i];
      ok = cudaMemcpy(ctx->bconst.p, &bc, sizeof(bc), cudaMemcpyHostToDevice) == cudaSuccess;
    }
  // working memory of a tick over a full pool, allocated once here instead of during the first
  // large ticks (one node per particle: the trees of these systems need about half that)
  ok = ok && serve_reserve(s) == cudaSuccess;
  cudaSetDevice(prev);
  if(!ok)
    {
      gpugrav_serve_destroy(s);
      return GPUGRAV_ERR_OOM;
    }
  s->free_ranges[0] = s->pool_cap;
  *out              = s;
  return GPUGRAV_OK;
}

int32_t gpugrav_serve_destroy(gpugrav_serve *s)
{
  if(!s)
    return GPUGRAV_ERR_INVALID;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  if(s->graph)
    cudaGraphExecDestroy(s->graph);
  for(auto *r : s->queue)
    delete r;
  for(auto *r : s->active)
    delete r;
  for(auto *r : s->finished)
    delete r;
  gg::DevBuf *bufs[] = {&s->pos, &s->vel, &s->acc, &s->oldacc, &s->stype, &s->sysdev, &s->cstart,
                        &s->ext, &s->up, &s->dl, &s->c2p, &s->csys, &s->s2p, &s->ntot_dev};
  for(auto *b : bufs)
    b->release();
  s->staging.release();
  if(s->ctx)
    gpugrav_destroy(s->ctx);
  cudaSetDevice(prev);
  delete s;
  return GPUGRAV_OK;
}

const char *gpugrav_serve_last_error(gpugrav_serve *s) { return s ? s->err.c_str() : "no server"; }

int32_t gpugrav_serve_submit(gpugrav_serve *s, int64_t id, int64_t n, const double *pos, const double *vel, const double *mass,
                             const uint8_t *softtype, int32_t nsteps, double dt)
{
  if(!s || id < 0 || n < 2 || !pos || !vel || !mass || !softtype || nsteps < 0 || !(dt >= 0) || !std::isfinite(dt))
    return GPUGRAV_ERR_INVALID;
  if(n > s->pool_cap || n > (int64_t)1 << 30)
    return sfail(s, GPUGRAV_ERR_TOO_LARGE, "request larger than the particle pool");
  for(int64_t i = 0; i < 3 * n; i++)
    if(!std::isfinite(pos[i]) || !std::isfinite(vel[i]))
      return sfail(s, GPUGRAV_ERR_INVALID, "non-finite position or velocity");
  for(int64_t i = 0; i < n; i++)
    if(softtype[i] >= s->prm.nsofttypes)
      return sfail(s, GPUGRAV_ERR_INVALID, "softening type >= nsofttypes");
  auto *r   = new gpugrav_serve::Req();
  r->id     = id;
  r->n      = n;
  r->nsteps = nsteps;
  r->dt     = dt;
  // Straight into the pool when it has room and everything queued is resident too (pool ranges
  // then follow the admission order, so a resident request never holds memory that a request
  // ahead of it waits for); otherwise a host copy, uploaded at admission.
  bool all_resident = true;
  for(auto *q : s->queue)
    all_resident = all_resident && q->resident;
  int64_t off = -1;
  if(all_resident && pool_alloc(s, n, &off))
    {
      int prev = 0;
      cudaGetDevice(&prev);
      if(prev != s->device)
        cudaSetDevice(s->device);
      cudaError_t e = upload(s, off, n, pos, vel, mass, softtype);
      if(e == cudaSuccess)
        e = cudaStreamSynchronize(s->st);  // the caller's arrays may change after return
      cudaSetDevice(prev);
      if(e != cudaSuccess)
        {
          pool_free(s, off, n);
          delete r;
          return sfail(s, GPUGRAV_ERR_CUDA, "upload", e);
        }
      r->resident = true;
      r->pool_off = off;
    }
  else
    {
      r->in.reset(new(std::nothrow) double[7 * n]);
      r->st.reset(new(std::nothrow) uint8_t[n]);
      if(!r->in || !r->st)
        {
          delete r;
          return sfail(s, GPUGRAV_ERR_OOM, "request copy");
        }
      host_copy(r->in.get(), pos, 3 * n * sizeof(double));
      host_copy(r->in.get() + 3 * n, vel, 3 * n * sizeof(double));
      host_copy(r->in.get() + 6 * n, mass, n * sizeof(double));
      memcpy(r->st.get(), softtype, n);
    }
  r->t_submit = now_s();
  s->queue.push_back(r);
  s->stats.submitted++;
  return GPUGRAV_OK;
}

int32_t gpugrav_serve_cancel(gpugrav_serve *s, int64_t id)
{
  if(!s)
    return GPUGRAV_ERR_INVALID;
  for(auto it = s->queue.begin(); it != s->queue.end(); ++it)
    if((*it)->id == id)
      {
        if((*it)->resident)
          pool_free(s, (*it)->pool_off, (*it)->n);
        delete *it;
        s->queue.erase(it);
        s->stats.cancelled++;
        return GPUGRAV_OK;
      }
  for(auto it = s->active.begin(); it != s->active.end(); ++it)
    if((*it)->id == id)
      {
        pool_free(s, (*it)->pool_off, (*it)->n);
        delete *it;
        s->active.erase(it);
        s->stats.cancelled++;
        return GPUGRAV_OK;
      }
  return sfail(s, GPUGRAV_ERR_INVALID, "no such request waiting or running");
}

int32_t gpugrav_serve_tick(gpugrav_serve *s, int32_t *n_active)
{
  if(!s)
    return GPUGRAV_ERR_INVALID;
  int prev = 0;
  cudaGetDevice(&prev);
  if(prev != s->device)
    cudaSetDevice(s->device);
  struct Restore
  {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  gpugrav_ctx *c  = s->ctx;
  cudaStream_t st = s->st;
  const double t_tick = now_s();

  // ---- admission (arrival order) ----
  std::vector<gpugrav_serve::Req *> admitted;
  while(!s->queue.empty() && (int)s->active.size() < s->cfg.max_systems)
    {
      gpugrav_serve::Req *r = s->queue.front();
      int64_t fl            = in_flight(s);
      if(s->cfg.memory_budget_bytes > 0 && (fl + r->n) * s->bytes_per_particle > s->cfg.memory_budget_bytes)
        break;
      if(!r->resident)
        {
          int64_t off;
          if(!pool_alloc(s, r->n, &off))
            break;
          r->pool_off = off;
          const double *in = r->in.get();
          SCK(upload(s, off, r->n, in, in + 3 * r->n, in + 6 * r->n, r->st.get()), "upload");
          admitted.push_back(r);  // the next copy into `up` follows this unpack in stream order
        }
      s->queue.pop_front();
      r->state   = ST_NEW;
      r->t_admit = t_tick;
      s->active.push_back(r);
      s->stats.admitted++;
    }
  if(!admitted.empty())
    {
      SCK(cudaStreamSynchronize(st), "upload");  // host copies of the inputs are no longer needed
      for(auto *r : admitted)
        r->in.reset(), r->st.reset();
    }
  const double t_admitted = now_s();
  s->stats.admit_s += t_admitted - t_tick;
  const int nsys = (int)s->active.size();
  if(n_active)
    *n_active = nsys;
  if(nsys == 0)
    return GPUGRAV_OK;

  // ---- system table ----
  std::vector<SysDev> sd(nsys);
  std::vector<int64_t> cst(nsys);
  int64_t ntot = 0;
  for(int k = 0; k < nsys; k++)
    {
      auto *r       = s->active[k];
      sd[k].pool_off = r->pool_off;
      sd[k].coff     = ntot;
      sd[k].n        = (int32_t)r->n;
      sd[k].state    = r->state;
      sd[k].dt       = r->dt;
      cst[k]         = ntot;
      ntot += r->n;
    }
  SCK(cudaMemcpyAsync(s->sysdev.p, sd.data(), nsys * sizeof(SysDev), cudaMemcpyHostToDevice, st), "system table");
  SCK(cudaMemcpyAsync(s->cstart.p, cst.data(), nsys * 8, cudaMemcpyHostToDevice, st), "system table");
  SCK(cudaMemcpyAsync(s->ntot_dev.p, &ntot, sizeof(ntot), cudaMemcpyHostToDevice, st), "system table");  // read by store/kick

  // ---- kick + drift, keys, sort, gather ----
  const SysDev *dsys = s->sysdev.as<SysDev>();
  cudaEventRecord(c->ev[12], st);
  c->mark(nullptr);
  k_srv_expand<<<grid_for(ntot, 256), 256, 0, st>>>(ntot, nsys, dsys, s->cstart.as<int64_t>(), s->c2p.as<int64_t>(),
                                                    s->csys.as<int32_t>());
  k_srv_pre<<<grid_for(ntot, 256), 256, 0, st>>>(ntot, dsys, s->c2p.as<int64_t>(), s->csys.as<int32_t>(), s->pos.as<double4>(),
                                                 s->vel.as<double4>(), s->acc.as<double4>());
  if(c->m_doms.ensure((size_t)nsys * sizeof(gpugrav_domain)) != cudaSuccess || c->key.ensure(ntot * sizeof(u128)) != cudaSuccess ||
     c->key_alt.ensure(ntot * sizeof(u128)) != cudaSuccess || c->idx.ensure(ntot * 4) != cudaSuccess ||
     c->perm.ensure(ntot * 4) != cudaSuccess || c->s_pm.ensure(ntot * sizeof(double4)) != cudaSuccess ||
     c->s_ix.ensure(ntot * 8) != cudaSuccess || c->s_iy.ensure(ntot * 8) != cudaSuccess || c->s_iz.ensure(ntot * 8) != cudaSuccess ||
     c->s_st.ensure(ntot + 16) != cudaSuccess || c->m_sys.ensure(ntot * 4) != cudaSuccess ||
     c->oldacc_s.ensure(ntot * 4) != cudaSuccess || c->acc_s.ensure(ntot * 24) != cudaSuccess ||
     c->pot_s.ensure(ntot * 8) != cudaSuccess || c->nint_s.ensure(ntot * 4) != cudaSuccess)
    return sfail(s, GPUGRAV_ERR_OOM, "tick buffers");
  SCK(cudaMemsetAsync(s->ext.p, 0xFF, (size_t)nsys * 6 * 8, st), "extent");
  SCK(cudaMemset2DAsync(s->ext.as<unsigned long long>() + 3, 6 * 8, 0, 3 * 8, nsys, st), "extent");
  k_srv_extent<<<dim3(nsys, 32), 256, 0, st>>>(nsys, dsys, s->c2p.as<int64_t>(), s->pos.as<double4>(),
                                               s->ext.as<unsigned long long>());
  k_srv_domains<<<grid_for(nsys, 128), 128, 0, st>>>(nsys, s->ext.as<unsigned long long>(), c->m_doms.as<gpugrav_domain>());
  k_srv_keys<<<grid_for(ntot, 256), 256, 0, st>>>(ntot, s->csys.as<int32_t>(), s->c2p.as<int64_t>(), s->pos.as<double4>(),
                                                  c->m_doms.as<gpugrav_domain>(), c->key.as<u128>(), c->idx.as<uint32_t>());
  size_t tb = 0;
  SCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, c->key.as<u128>(), c->key_alt.as<u128>(), c->idx.as<uint32_t>(),
                                      c->perm.as<uint32_t>(), (int)ntot, 0, 128, st),
      "sort");
  if(c->sort_tmp.ensure(tb) != cudaSuccess)
    return sfail(s, GPUGRAV_ERR_OOM, "sort");
  SCK(cub::DeviceRadixSort::SortPairs(c->sort_tmp.p, tb, c->key.as<u128>(), c->key_alt.as<u128>(), c->idx.as<uint32_t>(),
                                      c->perm.as<uint32_t>(), (int)ntot, 0, 128, st),
      "sort");
  k_srv_gather<<<grid_for(ntot, 256), 256, 0, st>>>(ntot, c->perm.as<uint32_t>(), s->csys.as<int32_t>(), s->c2p.as<int64_t>(),
                                                    s->pos.as<double4>(), s->stype.as<uint8_t>(), s->oldacc.as<float>(),
                                                    c->m_doms.as<gpugrav_domain>(), c->s_pm.as<double4>(),
                                                    c->s_ix.as<uint64_t>(), c->s_iy.as<uint64_t>(), c->s_iz.as<uint64_t>(),
                                                    c->s_st.as<uint8_t>(), c->m_sys.as<int32_t>(), s->s2p.as<int64_t>(),
                                                    c->oldacc_s.as<float>());
  SCK(cudaGetLastError(), "tick kernels");

  // ---- batched build over all systems ----
  c->n          = ntot;
  c->ntop       = nsys;
  c->built      = false;
  c->layout32_valid = false;
  int bstat = 0;
  c->mark("s1 pre+extent+keys+sort+gather");
  cudaEventRecord(c->ev[16], st);
  SCK(gg::build_stage(c, &bstat), "build");
  cudaEventRecord(c->ev[17], st);
  if(bstat != GPUGRAV_OK)
    return sfail(s, bstat, "build failed");
  SCK(gg::layout32_stage(c), "layout");

  // ---- walk + store/kick (captured graph, replayed while no buffer moved) ----
  WalkConst wc;
  make_walk_const(s->prm, &wc);
  c->want_pot = false;
  cudaEventRecord(c->ev[13], st);
  SCK(gg::walk32_prepare(c, wc), "walk");
  // Every pointer and launch parameter the captured nodes hold; the counts they depend on
  // (particles, groups) are read from device memory, so one graph serves every tick
  // until a buffer is reallocated.
  const std::vector<const void *> key = {c->g_sm.p,     c->g_rel.p,    c->g_kids.p,   c->g_pm.p,          c->g_pst.p,
                                         c->s_pm.p,     c->s_st.p,     c->oldacc_s.p, c->g_groups.p,      c->g_stack.p,
                                         c->acc_s.p,    c->pot_s.p,    c->nint_s.p,   c->scratch.p,       c->counters.p,
                                         c->m_sys.p,    s->s2p.p,      s->sysdev.p,   s->ntot_dev.p,      s->vel.p,
                                         s->acc.p,      s->oldacc.p,   c->g_ngroups.p, c->w32_kernel,
                                         (const void *)(intptr_t)c->w32_blocks};
  if(!s->graph || key != s->graph_key)
    {
      if(s->graph)
        {
          cudaGraphExecDestroy(s->graph);
          s->graph = nullptr;
        }
      cudaGraph_t g = nullptr;
      SCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
      cudaError_t e1 = cudaMemsetAsync(c->counters.as<int>() + 14, 0, 4, st);
      k_srv_bh<<<148 * 4, 256, 0, st>>>(c->g_ngroups.as<int>(), dsys, c->g_groups.as<int4>());
      cudaError_t e2 = gg::walk32_launch(c);
      k_srv_post<<<148 * 8, 256, 0, st>>>(s->ntot_dev.as<int64_t>(), c->m_sys.as<int32_t>(), dsys, s->s2p.as<int64_t>(),
                                          c->acc_s.as<double>(), s->vel.as<double4>(), s->acc.as<double4>(), s->oldacc.as<float>());
      cudaError_t e3 = cudaGetLastError();
      cudaError_t e4 = cudaStreamEndCapture(st, &g);
      SCK(e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3 != cudaSuccess ? e3 : e4, "capture");
      cudaError_t e5 = cudaGraphInstantiate(&s->graph, g, 0);
      cudaGraphDestroy(g);
      if(e5 != cudaSuccess)
        s->graph = nullptr;
      SCK(e5, "graph instantiate");
      s->graph_key = key;
      s->graph_captures++;
    }
  c->mark("s2 walk prepare+capture");
  cudaEventRecord(c->ev[14], st);
  SCK(cudaGraphLaunch(s->graph, st), "walk graph");
  cudaEventRecord(c->ev[15], st);
  s->graph_replays++;
  int walk_err                = 0;
  unsigned long long inter    = 0;
  SCK(cudaMemcpyAsync(&walk_err, c->counters.as<int>() + 14, 4, cudaMemcpyDeviceToHost, st), "walk flags");
  SCK(cudaMemcpyAsync(&inter, c->counters.as<int>() + 32, 8, cudaMemcpyDeviceToHost, st), "walk flags");
  SCK(cudaMemsetAsync(c->counters.as<int>() + 32, 0, 8, st), "walk flags");
  SCK(cudaStreamSynchronize(st), "tick");
  c->mark("s3 walk graph");
  if(walk_err)
    return sfail(s, GPUGRAV_ERR_DEEP_TREE, "walk stack exhausted");

  // ---- state machine, completion ----
  const double t_end = now_s();
  {
    float b = 0, w = 0, k = 0, t = 0;
    cudaEventElapsedTime(&b, c->ev[12], c->ev[13]);
    cudaEventElapsedTime(&w, c->ev[14], c->ev[15]);
    cudaEventElapsedTime(&k, c->ev[12], c->ev[16]);
    cudaEventElapsedTime(&t, c->ev[16], c->ev[17]);
    s->stats.build_s += 1e-3 * b;
    s->stats.keys_s += 1e-3 * k;
    s->stats.tree_s += 1e-3 * t;
    s->stats.walk_s += 1e-3 * w;
    s->stats.interactions += (int64_t)inter;
  }
  std::vector<gpugrav_serve::Req *> keep, done_now;
  for(auto *r : s->active)
    {
      bool done = false;
      if(r->state == ST_NEW)
        r->state = ST_INIT;
      else if(r->state == ST_INIT)
        {
          r->state = ST_STEP;
          done     = (r->nsteps == 0);
        }
      else if(r->state == ST_STEP)
        {
          r->steps_done++;
          done = r->steps_done >= r->nsteps;
        }
      s->stats.particle_steps += r->n;
      if(!done)
        {
          keep.push_back(r);
          continue;
        }
      done_now.push_back(r);
    }
  // finished: results stay in the pool until polled (copied straight into the caller's arrays)
  for(auto *r : done_now)
    {
      r->t_done = now_s();
      s->finished.push_back(r);
      s->stats.completed++;
    }
  s->active.swap(keep);
  s->stats.finish_s += now_s() - t_end;
  s->stats.ticks++;
  s->stats.last_tick_s      = t_end - t_tick;
  s->stats.last_tick_particles = ntot;
  s->stats.last_tick_systems   = nsys;
  s->stats.graph_captures      = s->graph_captures;
  s->stats.graph_replays       = s->graph_replays;
  return GPUGRAV_OK;
}

int32_t gpugrav_serve_poll(gpugrav_serve *s, int64_t *id, int64_t *n, double *pos, double *vel, double *acc, int64_t capacity,
                           double *times)
{
  if(!s || !id || !n)
    return GPUGRAV_ERR_INVALID;
  if(s->finished.empty())
    {
      *id = -1;
      *n  = 0;
      return GPUGRAV_OK;
    }
  gpugrav_serve::Req *r = s->finished.front();
  *id                   = r->id;
  *n                    = r->n;
  if(capacity < r->n)
    return GPUGRAV_OK;  // size reported; call again with room for n particles
  if(pos || vel || acc)
    {
      int prev = 0;
      cudaGetDevice(&prev);
      if(prev != s->device)
        cudaSetDevice(s->device);
      struct Restore
      {
        int d;
        ~Restore() { cudaSetDevice(d); }
      } restore{prev};
      cudaStream_t st = s->st;
      if(s->dl.ensure((size_t)r->n * 9 * sizeof(double)) != cudaSuccess)
        return sfail(s, GPUGRAV_ERR_OOM, "download buffer");
      const double *d = s->dl.as<double>();
      k_srv_pack<<<grid_for(r->n, 256), 256, 0, st>>>(r->n, r->pool_off, s->pos.as<double4>(), s->vel.as<double4>(),
                                                      s->acc.as<double4>(), s->dl.as<double>());
      const size_t b = (size_t)r->n * 3 * sizeof(double);
      SCK(cudaGetLastError(), "download");
      // one DMA into pinned staging, then host copies (a device-to-pageable copy is several times slower)
      if(s->staging.ensure(3 * b) != cudaSuccess)
        return sfail(s, GPUGRAV_ERR_OOM, "download staging");
      SCK(cudaMemcpyAsync(s->staging.p, d, 3 * b, cudaMemcpyDeviceToHost, st), "download");
      SCK(cudaStreamSynchronize(st), "download");
      const char *h = (const char *)s->staging.p;
      if(pos)
        host_copy(pos, h, b);
      if(vel)
        host_copy(vel, h + b, b);
      if(acc)
        host_copy(acc, h + 2 * b, b);
    }
  pool_free(s, r->pool_off, r->n);
  if(times)
    {
      times[0] = r->t_submit;
      times[1] = r->t_admit;
      times[2] = r->t_done;
    }
  s->finished.pop_front();
  delete r;
  return GPUGRAV_OK;
}

int32_t gpugrav_serve_get_stats(gpugrav_serve *s, gpugrav_serve_stats *out)
{
  if(!s || !out)
    return GPUGRAV_ERR_INVALID;
  *out            = s->stats;
  out->waiting    = (int64_t)s->queue.size();
  out->running    = (int64_t)s->active.size();
  out->in_flight_particles = in_flight(s);
  return GPUGRAV_OK;
}

}  // extern "C"
