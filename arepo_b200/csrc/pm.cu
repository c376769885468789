// pm.cu -- periodic particle-mesh long-range force on the GPU.
//
// Replaces pmforce_periodic(0, NULL) (src/gravity/pm/pm_periodic.c:1572-1936, the uniform data
// path of pmforce_uniform_optimized_prepare_density / _readout_forces_or_potential, :720-1538):
//   1. CIC mass assignment onto a PMGRID^3 mesh (node-based: cell (int)(PMGRID/L x), weights
//      1-dx and dx, periodic, :1090-1165), FP64 atomics;
//   2. real-to-complex FFT (cuFFT, FP64);
//   3. Green's function -exp(-k^2 Asmth^2) / k^2 times the CIC deconvolution
//      (sin(k d/2) / (k d/2))^-4 per axis, zero mode cleared (:1620-1704); both factors separate
//      into per-axis tables;
//   4. complex-to-real FFT: the potential mesh (unnormalised, as the FFTW backward transform);
//   5. per component, the force mesh: the 4-point finite difference of the potential,
//      fac ((4/3)(phi[-1] - phi[+1]) - (1/6)(phi[-2] - phi[+2])), fac = 4 pi G / L^3 / (2 d)
//      (:1735-1800), written into the complex buffer (free after the inverse transform), then
//      read at the 8 CIC nodes of every particle and CIC-weighted (:1322-1538); the potential is
//      read the same way from the potential mesh with 4 pi G / L^3.  One coalesced pass over the
//      mesh per component keeps the particle reads at 8 per component instead of 13 per node.
// G = 1 (accelerations without the factor G, like the tree walk).  The mesh is FP64 (the reference's
// default fft_real is float; FP64 costs little here next to the tree walk).

#include <cufft.h>

#include <cmath>
#include <vector>

#include "internal.h"

namespace gg
{
namespace
{
// (int)(f x) and its offset as in the reference; cells wrapped into the mesh.  A position that is
// not finite or absurdly far outside the box sets *bad and is placed at cell 0 with weight 0, so
// that no index ever leaves the mesh.
__device__ __forceinline__ void cic_axis(double x, double f, int n, int &c0, int &c1, double &w, int *bad)
{
  const double xs = f * x;
  if(!(xs > -1.0e15 && xs < 1.0e15))
    {
      atomicOr(bad, 1);
      c0 = 0;
      c1 = 1 % n;
      w  = 0.0;
      return;
    }
  const double s = floor(xs);  // positions in [0, L): the reference's (int) truncation
  w              = xs - s;
  int c          = (int)(s - (double)n * floor(s / n));  // in [0, n)
  c              = c < 0 ? 0 : (c >= n ? n - 1 : c);
  c0             = c;
  c1             = c0 + 1 == n ? 0 : c0 + 1;
}

__global__ void k_pm_deposit(int64_t np, const double *__restrict__ pos, const double *__restrict__ mass, int n, double f,
                             double *__restrict__ rho, int *bad)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x)
    {
      int x0, x1, y0, y1, z0, z1;
      double dx, dy, dz;
      cic_axis(pos[3 * i + 0], f, n, x0, x1, dx, bad);
      cic_axis(pos[3 * i + 1], f, n, y0, y1, dy, bad);
      cic_axis(pos[3 * i + 2], f, n, z0, z1, dz, bad);
      const double m = mass[i];
      const int64_t N = n;
      atomicAdd(&rho[(x0 * N + y0) * N + z0], m * (1.0 - dx) * (1.0 - dy) * (1.0 - dz));
      atomicAdd(&rho[(x0 * N + y0) * N + z1], m * (1.0 - dx) * (1.0 - dy) * dz);
      atomicAdd(&rho[(x0 * N + y1) * N + z0], m * (1.0 - dx) * dy * (1.0 - dz));
      atomicAdd(&rho[(x0 * N + y1) * N + z1], m * (1.0 - dx) * dy * dz);
      atomicAdd(&rho[(x1 * N + y0) * N + z0], m * dx * (1.0 - dy) * (1.0 - dz));
      atomicAdd(&rho[(x1 * N + y0) * N + z1], m * dx * (1.0 - dy) * dz);
      atomicAdd(&rho[(x1 * N + y1) * N + z0], m * dx * dy * (1.0 - dz));
      atomicAdd(&rho[(x1 * N + y1) * N + z1], m * dx * dy * dz);
    }
}


// mesh of the forward transform: n x n x (n/2 + 1), last index fastest.  The Gaussian and the CIC
// deconvolution factor per axis: tab[i] = (exp(-k_i^2 Asmth^2), 1 / sinc(k_i d / 2)^4) for the wave
// number k_i of mesh index i, so that an entry costs one product and one division.
__global__ void k_pm_green(int n, double kfac, const double2 *__restrict__ tab, cufftDoubleComplex *__restrict__ rk)
{
  const int nz      = n / 2 + 1;
  const int64_t tot = (int64_t)n * n * nz;
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x)
    {
      const int z = (int)(i % nz);
      const int y = (int)((i / nz) % n);
      const int x = (int)(i / ((int64_t)nz * n));
      const int xx = x >= n / 2 ? x - n : x, yy = y >= n / 2 ? y - n : y, zz = z >= n / 2 ? z - n : z;
      const double kx = kfac * xx, ky = kfac * yy, kz = kfac * zz;
      const double k2 = kx * kx + ky * ky + kz * kz;
      double g        = 0.0;  // the zero mode carries the mean density: no force
      if(k2 > 0)
        {
          const double2 a = tab[x], b = tab[y], c = tab[z];
          g               = -(a.x * b.x * c.x) * (a.y * b.y * c.y) / k2;
        }
      rk[i].x *= g;
      rk[i].y *= g;
    }
}

// one component of the force mesh: the 4-point difference of the potential along `dim`.  One block
// per mesh row (x, y), threads along z: coordinates without a per-point division, coalesced rows.
__global__ void k_pm_fd(int n, int dim, double fac, const double *__restrict__ phi, double *__restrict__ force)
{
  const int64_t N = n;
  auto wrap       = [n](int q) { return q < 0 ? q + n : (q >= n ? q - n : q); };
  for(int64_t row = blockIdx.x; row < N * N; row += gridDim.x)
    {
      const int x = (int)(row / N), y = (int)(row % N);
      const double *r0 = phi + row * N;
      // the rows (dim 0: x +- 1, 2; dim 1: y +- 1, 2) or this row (dim 2) holding the four neighbours
      const double *rm1 = r0, *rp1 = r0, *rm2 = r0, *rp2 = r0;
      if(dim == 0)
        {
          rm1 = phi + (wrap(x - 1) * N + y) * N;
          rp1 = phi + (wrap(x + 1) * N + y) * N;
          rm2 = phi + (wrap(x - 2) * N + y) * N;
          rp2 = phi + (wrap(x + 2) * N + y) * N;
        }
      else if(dim == 1)
        {
          rm1 = phi + (x * N + wrap(y - 1)) * N;
          rp1 = phi + (x * N + wrap(y + 1)) * N;
          rm2 = phi + (x * N + wrap(y - 2)) * N;
          rp2 = phi + (x * N + wrap(y + 2)) * N;
        }
      for(int z = threadIdx.x; z < n; z += blockDim.x)
        {
          const int zm1 = dim == 2 ? wrap(z - 1) : z, zp1 = dim == 2 ? wrap(z + 1) : z;
          const int zm2 = dim == 2 ? wrap(z - 2) : z, zp2 = dim == 2 ? wrap(z + 2) : z;
          force[row * N + z] = fac * ((4.0 / 3) * (rm1[zm1] - rp1[zp1]) - (1.0 / 6) * (rm2[zm2] - rp2[zp2]));
        }
    }
}

// CIC readout of one mesh at every particle: out[ostride * i + ooff] = scale * sum_nodes w mesh
__global__ void k_pm_cic_read(int64_t np, const double *__restrict__ pos, int n, double f, const double *__restrict__ mesh,
                              double scale, double *__restrict__ out, int ostride, int ooff, int *bad)
{
  const int64_t N = n;
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x)
    {
      int c[3][2];
      double w[3][2];
      for(int a = 0; a < 3; a++)
        {
          double d;
          cic_axis(pos[3 * i + a], f, n, c[a][0], c[a][1], d, bad);
          w[a][0] = 1.0 - d;
          w[a][1] = d;
        }
      double v = 0;
      for(int ix = 0; ix < 2; ix++)
        for(int iy = 0; iy < 2; iy++)
          for(int iz = 0; iz < 2; iz++)
            v += mesh[(c[0][ix] * N + c[1][iy]) * N + c[2][iz]] * (w[0][ix] * w[1][iy] * w[2][iz]);
      out[ostride * i + ooff] = v * scale;
    }
}

int blocks_for(int64_t n)
{
  int64_t b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 32 ? 148 * 32 : b));
}
}  // namespace

// PM force for np particles (device arrays pos n*3, mass n) into acc (n*3) and pot (n, may be null)
cudaError_t pm_stage(gpugrav_ctx *c, int pmgrid, int64_t np, const double *pos, const double *mass, double *acc, double *pot,
                     int *cufft_status)
{
  cudaStream_t st  = c->stream;
  const int n      = pmgrid;
  const int64_t N3 = (int64_t)n * n * n, NC = (int64_t)n * n * (n / 2 + 1);
  *cufft_status    = CUFFT_SUCCESS;
  if(c->pm_grid != n)
    {
      if(c->pm_grid > 0)
        {
          cufftDestroy((cufftHandle)c->pm_plan_f);
          cufftDestroy((cufftHandle)c->pm_plan_b);
          c->pm_grid = 0;
        }
      cufftHandle pf, pb;
      cufftResult r = cufftPlan3d(&pf, n, n, n, CUFFT_D2Z);
      if(r != CUFFT_SUCCESS)
        {
          *cufft_status = r;
          return cudaSuccess;
        }
      r = cufftPlan3d(&pb, n, n, n, CUFFT_Z2D);
      if(r != CUFFT_SUCCESS)
        {
          cufftDestroy(pf);
          *cufft_status = r;
          return cudaSuccess;
        }
      c->pm_plan_f = (int)pf;
      c->pm_plan_b = (int)pb;
      c->pm_grid   = n;
    }
  GG_TRY(c->pm_rho.ensure(N3 * sizeof(double)));
  GG_TRY(c->pm_rhok.ensure(NC * sizeof(cufftDoubleComplex)));
  {
    // per-axis factors of the Green's function (host, n entries)
    const double bx = c->prm.box_size, dd = bx / n, kf = 2.0 * M_PI / bx, a2 = c->prm.asmth * c->prm.asmth;
    std::vector<double2> tab(n);
    for(int i = 0; i < n; i++)
      {
        const int ii   = i >= n / 2 ? i - n : i;
        const double k = kf * ii;
        double s       = 1.0;
        if(ii != 0)
          {
            const double a = k * 0.5 * dd;
            s              = sin(a) / a;
          }
        const double f = 1.0 / s;
        tab[i]         = make_double2(exp(-k * k * a2), f * f * f * f);
      }
    GG_TRY(c->pm_tab.ensure(n * sizeof(double2)));
    GG_TRY(cudaMemcpyAsync(c->pm_tab.p, tab.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
    GG_TRY(cudaStreamSynchronize(st));  // `tab` lives on this stack frame
  }
  cufftSetStream((cufftHandle)c->pm_plan_f, st);
  cufftSetStream((cufftHandle)c->pm_plan_b, st);
  const double box = c->prm.box_size, d = box / n, f = n / box;
  GG_TRY(cudaMemsetAsync(c->pm_rho.p, 0, N3 * sizeof(double), st));
  int *bad = c->counters.as<int>() + 15;
  GG_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
  k_pm_deposit<<<blocks_for(np), 256, 0, st>>>(np, pos, mass, n, f, c->pm_rho.as<double>(), bad);
  GG_TRY(cudaGetLastError());
  cufftResult r = cufftExecD2Z((cufftHandle)c->pm_plan_f, c->pm_rho.as<double>(), c->pm_rhok.as<cufftDoubleComplex>());
  if(r == CUFFT_SUCCESS)
    {
      k_pm_green<<<blocks_for(NC), 256, 0, st>>>(n, 2.0 * M_PI / box, c->pm_tab.as<double2>(),
                                                  c->pm_rhok.as<cufftDoubleComplex>());
      GG_TRY(cudaGetLastError());
      r = cufftExecZ2D((cufftHandle)c->pm_plan_b, c->pm_rhok.as<cufftDoubleComplex>(), c->pm_rho.as<double>());
    }
  if(r != CUFFT_SUCCESS)
    {
      *cufft_status = r;
      return cudaSuccess;
    }
  const double fac_pot = 4.0 * M_PI / (box * box * box);
  double *force        = (double *)c->pm_rhok.p;  // n^2 (n/2+1) complex >= n^3 doubles
  for(int dim = 0; dim < 3; dim++)
    {
      const int64_t rows = (int64_t)n * n;
      k_pm_fd<<<(int)(rows < 148 * 16 ? rows : 148 * 16), 256, 0, st>>>(n, dim, fac_pot / (2.0 * d), c->pm_rho.as<double>(),
                                                                          force);
      k_pm_cic_read<<<blocks_for(np), 256, 0, st>>>(np, pos, n, f, force, 1.0, acc, 3, dim, bad);
    }
  if(pot)
    k_pm_cic_read<<<blocks_for(np), 256, 0, st>>>(np, pos, n, f, c->pm_rho.as<double>(), fac_pot, pot, 1, 0, bad);
  return cudaGetLastError();
}

void pm_release(gpugrav_ctx *c)
{
  if(c->pm_grid > 0)
    {
      cufftDestroy((cufftHandle)c->pm_plan_f);
      cufftDestroy((cufftHandle)c->pm_plan_b);
      c->pm_grid = 0;
    }
  c->pm_rho.release();
  c->pm_rhok.release();
  c->pm_tab.release();
}
}  // namespace gg
