// direct_noalloc.cu -- FP64 direct summation that allocates nothing.
//
// gpugrav_direct needs a context, which owns device memory that the library
// allocates (particle copies, the sorted arrays, a scratch buffer of partial
// sums).  Some callers cannot allocate device memory at the point where they
// want the accuracy check: a code that has handed the whole GPU memory to its
// own pool allocator at start-up (a PyTorch caching allocator, an AREPO run that
// reserves the device once), or one that cannot accept the device-wide
// synchronisation that cudaMalloc/cudaFree imply in the middle of a time step.
// gpugrav_direct_noalloc takes the caller's device arrays as they are and keeps
// its only scratch (partial sums per source chunk) in a fixed file-scope device
// array, so it calls no cudaMalloc, cudaFree or any other allocating routine.
//
// Limits and sharing:
//  * at most kMaxTargets (4096) targets per call; larger requests are rejected
//    with GPUGRAV_ERR_TOO_LARGE before any launch;
//  * the scratch array (4 MiB) exists on every GPU that loads the library and is
//    held until the process exits;
//  * every call on a device uses the same array.  A call writes each partial sum
//    it reads before reading it, so nothing has to start at zero and no state
//    carries over, but two calls whose kernels overlap on the GPU (different
//    streams, or host threads) race on the array: serialise them;
//  * the first call in a CUDA context looks up the array's device address in that
//    context (cudaGetSymbolAddress, with the device current); make that first
//    call before any stream capture.  The address is kept per context: a caller
//    that drives the device through its own (non-primary) context gets that
//    context's copy of the array;
//  * softening types must lie in [0, nsofttypes): a target of another type gets
//    NaN outputs, and a source of another type makes the outputs of every target
//    it interacts with NaN (no softening length exists for it).
#include <mutex>

#include "internal.h"

namespace
{
constexpr int kMaxTargets = 4096;
constexpr int kChunks     = 32;
constexpr int kTile       = 128;

// partial sums (acc.x, acc.y, acc.z, pot) per (source chunk, target)
static __device__ __align__(256) double4 g_noalloc_partial[kChunks * kMaxTargets];

// device address of g_noalloc_partial per CUDA context (looked up once per context)
struct ScratchAddr
{
  void *ctx;
  double4 *addr;
};
constexpr int kMaxContexts = 64;
ScratchAddr g_scratch_addr[kMaxContexts];
int g_scratch_n = 0;
std::mutex g_scratch_mu;

// cuCtxGetCurrent through the runtime's driver entry point (no link dependency on libcuda)
typedef int (*CtxGetCurrentFn)(void **);
CtxGetCurrentFn ctx_get_current()
{
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrentFn)f;
  });
  return fn;
}

// softening length of type t, NaN for a type without one (t >= nsofttypes)
__device__ __forceinline__ double soft_of(const gg::WalkConst &w, unsigned t)
{
  return t < (unsigned)w.nsoft ? w.soft[t] : __longlong_as_double(0x7ff8000000000000ll);
}

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

// same pair arithmetic as k_direct (direct.cu); sources read from the caller's arrays
__global__ void __launch_bounds__(kTile) k_direct_noalloc(const double *__restrict__ pos, const double *__restrict__ mass,
                                                          const uint8_t *__restrict__ st, int64_t n,
                                                          const double *__restrict__ tpos, const uint8_t *__restrict__ tst,
                                                          int64_t nt, const gg::WalkConst w, int cut, double4 *__restrict__ partial)
{
  __shared__ double4 src[kTile];
  __shared__ double hsrc[kTile];
  const int64_t t   = (int64_t)blockIdx.x * kTile + threadIdx.x;
  const int chunk   = blockIdx.y;
  const int64_t per = (n + kChunks - 1) / kChunks;
  const int64_t j0 = chunk * per, j1 = (j0 + per < n) ? j0 + per : n;
  double mx = 0, my = 0, mz = 0, h_i = 0;
  if(t < nt)
    {
      mx  = tpos[3 * t + 0];
      my  = tpos[3 * t + 1];
      mz  = tpos[3 * t + 2];
      h_i = soft_of(w, tst[t]);
    }
  const double asmth = w.periodic ? (0.5 / sqrt(w.asmthinv2)) : 0.0;
  double ax = 0, ay = 0, az = 0, pt = 0;
  for(int64_t jb = j0; jb < j1; jb += kTile)
    {
      __syncthreads();
      int64_t j = jb + threadIdx.x;
      if(j < j1)
        {
          // a source without a softening length gets a NaN mass: every pair it enters is NaN
          const double hj   = soft_of(w, st[j]);
          src[threadIdx.x]  = make_double4(pos[3 * j + 0], pos[3 * j + 1], pos[3 * j + 2], hj == hj ? mass[j] : hj);
          hsrc[threadIdx.x] = hj;
        }
      __syncthreads();
      int cnt = (int)((j1 - jb) < kTile ? (j1 - jb) : kTile);
      if(t < nt)
        for(int q = 0; q < cnt; q++)
          {
            double4 s = src[q];
            double dx = s.x - mx, dy = s.y - my, dz = s.z - mz;
            if(w.periodic)
              {
                dx = (dx > w.half_box) ? dx - w.box : ((dx < -w.half_box) ? dx + w.box : dx);
                dy = (dy > w.half_box) ? dy - w.box : ((dy < -w.half_box) ? dy + w.box : dy);
                dz = (dz > w.half_box) ? dz - w.box : ((dz < -w.half_box) ? dz + w.box : dz);
              }
            double r2 = dx * dx + dy * dy + dz * dz;
            if(cut && w.periodic && !(r2 < w.rcut2))
              continue;
            double r    = sqrt(r2);
            double m    = s.w;
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
            if(w.periodic)
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
          }
    }
  // every (chunk, target) slot read by the reduction below is written here in the same call
  if(t < nt)
    partial[(int64_t)chunk * kMaxTargets + t] = make_double4(ax, ay, az, pt);
}

__global__ void k_direct_noalloc_reduce(const double4 *__restrict__ partial, int64_t nt, double *__restrict__ acc,
                                        double *__restrict__ pot)
{
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= nt)
    return;
  double ax = 0, ay = 0, az = 0, pt = 0;
  for(int c = 0; c < kChunks; c++)
    {
      double4 p = partial[(int64_t)c * kMaxTargets + t];
      ax += p.x;
      ay += p.y;
      az += p.z;
      pt += p.w;
    }
  acc[3 * t + 0] = ax;
  acc[3 * t + 1] = ay;
  acc[3 * t + 2] = az;
  if(pot)
    pot[t] = pt;
}
}  // namespace

extern "C" int32_t gpugrav_direct_noalloc(int32_t device, const gpugrav_params *params, int64_t n, const double *pos,
                                          const double *mass, const uint8_t *softtype, int64_t ntargets,
                                          const double *target_pos, const uint8_t *target_softtype, int32_t mode,
                                          double *acc, double *pot, void *stream)
{
  if(gg::validate_params(params) != GPUGRAV_OK)
    return GPUGRAV_ERR_INVALID;
  if(params->periodic && !(params->asmth > 0))  // the Ewald tables would need an allocation
    return GPUGRAV_ERR_INVALID;
  if(mode != GPUGRAV_DIRECT_FULL && mode != GPUGRAV_DIRECT_CUT)
    return GPUGRAV_ERR_INVALID;
  if(n < 1 || ntargets < 0 || !pos || !mass || !softtype || (ntargets > 0 && (!target_pos || !target_softtype || !acc)))
    return GPUGRAV_ERR_INVALID;
  if(ntargets > kMaxTargets)
    return GPUGRAV_ERR_TOO_LARGE;
  if(device < 0)
    return GPUGRAV_ERR_INVALID;
  if(ntargets == 0)
    return GPUGRAV_OK;

  int prev = -1;
  if(cudaGetDevice(&prev) != cudaSuccess)
    return GPUGRAV_ERR_CUDA;
  if(prev != device && cudaSetDevice(device) != cudaSuccess)
    return GPUGRAV_ERR_CUDA;
  int32_t status = GPUGRAV_OK;
  // set-up, once per CUDA context with the device current: the device address of the scratch array
  double4 *scratch = nullptr;
  {
    CtxGetCurrentFn get = ctx_get_current();
    void *ctx           = nullptr;
    if(!get || get(&ctx) != 0)
      status = GPUGRAV_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    for(int i = 0; status == GPUGRAV_OK && i < g_scratch_n; i++)
      if(g_scratch_addr[i].ctx == ctx)
        scratch = g_scratch_addr[i].addr;
    if(status == GPUGRAV_OK && !scratch)
      {
        void *p = nullptr;
        if(g_scratch_n >= kMaxContexts || cudaGetSymbolAddress(&p, g_noalloc_partial) != cudaSuccess || !p)
          status = GPUGRAV_ERR_CUDA;
        else
          {
            g_scratch_addr[g_scratch_n++] = ScratchAddr{ctx, (double4 *)p};
            scratch                       = (double4 *)p;
          }
      }
  }
  if(status == GPUGRAV_OK)
    {
      gg::WalkConst wc;
      gg::make_walk_const(*params, &wc);
      cudaStream_t st = (cudaStream_t)stream;
      dim3 grid((unsigned)((ntargets + kTile - 1) / kTile), kChunks);
      k_direct_noalloc<<<grid, kTile, 0, st>>>(pos, mass, softtype, n, target_pos, target_softtype, ntargets, wc,
                                               mode == GPUGRAV_DIRECT_CUT, scratch);
      k_direct_noalloc_reduce<<<(unsigned)((ntargets + 255) / 256), 256, 0, st>>>(scratch, ntargets, acc, pot);
      if(cudaGetLastError() != cudaSuccess)
        status = GPUGRAV_ERR_CUDA;
    }
  if(prev != device)
    cudaSetDevice(prev);
  return status;
}
