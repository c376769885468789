// ewald.cu -- Ewald correction tables of the periodic pure-tree walk (periodic box without PM).
//
// ewald_init (src/gravity/forcetree_ewald.c:89-254) tabulates, for one octant of the unit box on a
// (EN+1)^3 grid (EN = 64, entry (i, j, k) at (i, j, k) / (2 EN)), the difference between the force
// (and potential) of a unit mass with all its periodic images and of the nearest image alone
// (ewald_force, :463-527, and ewald_psi, :393-461: real-space erfc sums over 9^3 images, Fourier
// sums over the reciprocal lattice), and scales them by 1/L^2 and 1/L.  The walk adds the
// trilinear interpolation of the table per interaction (ewald_corr, :268-342).
//
// The same sums are evaluated here on the host with the C library's erfc/exp/sin/cos, in the same
// order, so that the table is the reference's to the last bit (the FP64 walk is compared bit for
// bit with the reference); entries are independent and computed on all host threads, once per
// process.  A caller that already holds AREPO's tables passes them with gpugrav_set_ewald_table.

#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

#include "internal.h"

namespace gg
{
namespace
{
double ewald_psi(double x, double y, double z)
{
  double r = sqrt(x * x + y * y + z * z);
  if(r == 0)
    return 0;
  const double alpha = 3.0;
  const int nmax     = 4;
  double sum1        = 0;
  for(int nx = -nmax; nx <= nmax; nx++)
    for(int ny = -nmax; ny <= nmax; ny++)
      for(int nz = -nmax; nz <= nmax; nz++)
        {
          double dx = x - nx, dy = y - ny, dz = z - nz;
          double rr = sqrt(dx * dx + dy * dy + dz * dz);
          sum1 += erfc(alpha * rr) / rr;
        }
  const double alpha2 = alpha * alpha;
  const int kmax      = (int)(2 * alpha + 0.5);
  double sum2         = 0.0;
  for(int nx = -kmax; nx <= kmax; nx++)
    for(int ny = -kmax; ny <= kmax; ny++)
      for(int nz = -kmax; nz <= kmax; nz++)
        {
          double kx = (2.0 * M_PI) * nx, ky = (2.0 * M_PI) * ny, kz = (2.0 * M_PI) * nz;
          double k2 = kx * kx + ky * ky + kz * kz;
          if(k2 > 0)
            {
              double kdotx = (x * kx + y * ky + z * kz);
              sum2 += 4.0 * M_PI / k2 * exp(-k2 / (4.0 * alpha2)) * cos(kdotx);
            }
        }
  return M_PI / (alpha * alpha) - sum1 - sum2 + 1.0 / r;
}

void ewald_force(double x, double y, double z, double force[3])
{
  for(int i = 0; i < 3; i++)
    force[i] = 0;
  double r2 = x * x + y * y + z * z;
  if(r2 == 0)
    return;
  const double alpha  = 2.0;
  const double alpha2 = alpha * alpha;
  double r3inv        = 1.0 / (r2 * sqrt(r2));
  force[0] += r3inv * x;
  force[1] += r3inv * y;
  force[2] += r3inv * z;
  const int nmax = 4;
  for(int nx = -nmax; nx <= nmax; nx++)
    for(int ny = -nmax; ny <= nmax; ny++)
      for(int nz = -nmax; nz <= nmax; nz++)
        {
          double dx   = x - nx, dy = y - ny, dz = z - nz;
          double rr2  = dx * dx + dy * dy + dz * dz;
          double r    = sqrt(rr2);
          double val  = erfc(alpha * r) + 2.0 * alpha * r / sqrt(M_PI) * exp(-alpha2 * rr2);
          double val2 = val / (rr2 * r);
          force[0] -= dx * val2;
          force[1] -= dy * val2;
          force[2] -= dz * val2;
        }
  const int hmax = (int)(2 * alpha + 0.5);
  for(int hx = -hmax; hx <= hmax; hx++)
    for(int hy = -hmax; hy <= hmax; hy++)
      for(int hz = -hmax; hz <= hmax; hz++)
        {
          double h2 = hx * hx + hy * hy + hz * hz;
          if(h2 > 0)
            {
              double hdotx = x * hx + y * hy + z * hz;
              double val   = 2.0 / h2 * exp(-M_PI * M_PI * h2 / alpha2) * sin(2.0 * M_PI * hdotx);
              force[0] -= hx * val;
              force[1] -= hy * val;
              force[2] -= hz * val;
            }
        }
}

std::once_flag g_table_once;
std::vector<double> g_table;  // fx | fy | fz | pot, unscaled, (EN+1)^3 each, k fastest
}  // namespace

const std::vector<double> &ewald_unit_table()
{
  std::call_once(g_table_once, [] {
    const int m = kEwaldN + 1, total = m * m * m;
    g_table.assign(4 * (size_t)total, 0.0);
    unsigned nt = std::thread::hardware_concurrency();
    nt          = nt < 1 ? 1 : (nt > 64 ? 64 : nt);
    std::vector<std::thread> th;
    for(unsigned t = 0; t < nt; t++)
      th.emplace_back([t, nt, m, total] {
        for(int n = (int)t; n < total; n += (int)nt)
          {
            int i = n / (m * m), j = (n - i * m * m) / m, k = n - i * m * m - j * m;
            double xx = 0.5 * ((double)i) / kEwaldN, yy = 0.5 * ((double)j) / kEwaldN, zz = 0.5 * ((double)k) / kEwaldN;
            double f[3];
            g_table[3 * (size_t)total + n] = ewald_psi(xx, yy, zz);
            ewald_force(xx, yy, zz, f);
            g_table[n]                     = f[0];
            g_table[(size_t)total + n]     = f[1];
            g_table[2 * (size_t)total + n] = f[2];
          }
      });
    for(auto &x : th)
      x.join();
  });
  return g_table;
}

// tables of the context scaled to its box (fcorr / L^2, potcorr / L, forcetree_ewald.c:239-251):
// FP64 (fx | fy | fz | pot) for the FP64 walk and the direct sum, float4 (fx, fy, fz, pot) per entry
// for the FP32 walk.  `user` (may be null): the caller's already scaled tables.
cudaError_t ewald_upload(gpugrav_ctx *c, const double *user)
{
  const int m = kEwaldN + 1;
  const size_t total = (size_t)m * m * m;
  std::vector<double> t(4 * total);
  if(user)
    t.assign(user, user + 4 * total);
  else
    {
      const std::vector<double> &u = ewald_unit_table();
      const double L = c->prm.box_size;
      for(size_t q = 0; q < 3 * total; q++)
        t[q] = u[q] / (L * L);
      for(size_t q = 3 * total; q < 4 * total; q++)
        t[q] = u[q] / L;
    }
  std::vector<float4> t32(total);
  for(size_t q = 0; q < total; q++)
    t32[q] = make_float4((float)t[q], (float)t[total + q], (float)t[2 * total + q], (float)t[3 * total + q]);
  GG_TRY(c->ewd.ensure(4 * total * sizeof(double)));
  GG_TRY(c->ewd32.ensure(total * sizeof(float4)));
  GG_TRY(cudaMemcpy(c->ewd.p, t.data(), 4 * total * sizeof(double), cudaMemcpyHostToDevice));
  GG_TRY(cudaMemcpy(c->ewd32.p, t32.data(), total * sizeof(float4), cudaMemcpyHostToDevice));
  c->ewd_box  = user ? -1.0 : c->prm.box_size;
  c->ewd_user = user != nullptr;
  return cudaSuccess;
}

// tables of the current box on the device (computed or scaled only when the box changed)
cudaError_t ewald_ensure(gpugrav_ctx *c)
{
  if(c->ewd_user || (c->ewd.p && c->ewd_box == c->prm.box_size))
    return cudaSuccess;
  return ewald_upload(c, nullptr);
}
}  // namespace gg
