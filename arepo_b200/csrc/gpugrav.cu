// gpugrav.cu -- C ABI of libarepo_gpugrav: context, call sequencing, transfers.
//
// The call sequence mirrors gravity() (src/gravity/accel.c:94-192) on one rank:
//   gpugrav_load   ~ do_box_wrapping + domain_findExtent + keys + peano_hilbert_order
//   gpugrav_build  ~ construct_forcetree(0, ...)
//   gpugrav_walk   ~ gravity_tree(timebin)
// Errors are returned as status codes (negative codes mirror force_treebuild_construct's);
// nothing in the library exits.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "internal.h"

using namespace gg;

// ------------------------------------------------------------------------------
// buffers
// ------------------------------------------------------------------------------
void gpugrav_ctx::mark(const char *what)
{
  if(!profile)
    return;
  cudaStreamSynchronize(stream);
  const double t = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  if(what && prof_t > 0)
    prof[what] += t - prof_t;
  prof_t = t;
}

cudaError_t gg::DevBuf::ensure(size_t bytes)
{
  if(bytes <= cap && p)
    return cudaSuccess;
  // a buffer that has to grow gets 25% headroom: sizes that drift upward from call to call (node
  // counts of successive trees) would otherwise reallocate, and synchronise the device, every call
  const bool regrow = p != nullptr;
  if(p)
    cudaFree(p);
  p   = nullptr;
  cap = 0;
  size_t want = bytes < 256 ? 256 : bytes;
  if(regrow)
    want += want / 4;
  want        = (want + 255) & ~(size_t)255;
  cudaError_t e = cudaMalloc(&p, want);
  if(e != cudaSuccess)
    {
      p = nullptr;
      return e;
    }
  cap = want;
  return cudaSuccess;
}

void gg::DevBuf::release()
{
  if(p)
    cudaFree(p);
  p   = nullptr;
  cap = 0;
}

cudaError_t gg::PinnedBuf::ensure(size_t bytes)
{
  if(bytes <= cap && p)
    return cudaSuccess;
  if(p)
    cudaFreeHost(p);
  p             = nullptr;
  cap           = 0;
  cudaError_t e = cudaMallocHost(&p, bytes);
  if(e != cudaSuccess)
    {
      p = nullptr;
      return e;
    }
  cap = bytes;
  return cudaSuccess;
}

void gg::PinnedBuf::release()
{
  if(p)
    cudaFreeHost(p);
  p   = nullptr;
  cap = 0;
}

// ------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------
namespace
{
int fail(gpugrav_ctx *c, int status, const char *what, cudaError_t e = cudaSuccess)
{
  if(c)
    {
      char buf[512];
      if(e != cudaSuccess)
        snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
      else
        snprintf(buf, sizeof(buf), "%s", what);
      c->err = buf;
    }
  return status;
}

#define CK(call, what)                                 \
  do                                                   \
    {                                                  \
      cudaError_t _e = (call);                         \
      if(_e != cudaSuccess)                            \
        return fail(c, GPUGRAV_ERR_CUDA, what, _e);    \
    }                                                  \
  while(0)

__global__ void k_gather_f32(const float *__restrict__ in, const uint32_t *__restrict__ perm, int64_t n, float *__restrict__ out)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in ? in[perm[i]] : 0.0f;
}

__global__ void k_scatter_out(const double *__restrict__ acc_s, const double *__restrict__ pot_s, const int32_t *__restrict__ nint_s,
                              const uint32_t *__restrict__ perm, int64_t n, double *__restrict__ acc, double *__restrict__ pot,
                              int32_t *__restrict__ nint)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      int64_t o      = perm[i];
      acc[3 * o + 0] = acc_s[3 * i + 0];
      acc[3 * o + 1] = acc_s[3 * i + 1];
      acc[3 * o + 2] = acc_s[3 * i + 2];
      if(pot)
        pot[o] = pot_s[i];
      if(nint)
        nint[o] = nint_s[i];
    }
}

int grid_for(int64_t n, int threads)
{
  int64_t b = (n + threads - 1) / threads;
  if(b > 148 * 16)
    b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

struct DeviceGuard
{
  int prev = -1;
  explicit DeviceGuard(int dev)
  {
    cudaGetDevice(&prev);
    if(prev != dev)
      cudaSetDevice(dev);
  }
  ~DeviceGuard()
  {
    if(prev >= 0)
      cudaSetDevice(prev);
  }
};

float elapsed(cudaEvent_t a, cudaEvent_t b)
{
  float ms = 0;
  if(cudaEventElapsedTime(&ms, a, b) != cudaSuccess)
    return 0;
  return ms;
}
}  // namespace

// Parameter checks shared by every entry point that takes a gpugrav_params.
int gg::validate_params(const gpugrav_params *p)
{
  if(!p || p->abi_version != GPUGRAV_ABI_VERSION)
    return GPUGRAV_ERR_INVALID;
  if(p->nsofttypes < 1 || p->nsofttypes > GPUGRAV_MAX_SOFTTYPES)
    return GPUGRAV_ERR_INVALID;
  if(p->force_softening[p->nsofttypes] != 0.0)
    return GPUGRAV_ERR_INVALID;
  for(int i = 0; i < p->nsofttypes; i++)
    if(!(p->force_softening[i] >= 0.0) || !std::isfinite(p->force_softening[i]))
      return GPUGRAV_ERR_INVALID;
  if(!(p->box_size > 0) || !std::isfinite(p->box_size))
    return GPUGRAV_ERR_INVALID;
  if(p->periodic && p->asmth != 0.0)
    {
      // TreePM split; asmth == 0 selects the pure periodic tree with Ewald correction
      if(!(p->asmth > 0) || !(p->rcut > 0) || !(p->rcut_cells > 0))
        return GPUGRAV_ERR_INVALID;
    }
  if(!(p->err_tol_theta >= 0) || !(p->err_tol_force_acc >= 0))
    return GPUGRAV_ERR_INVALID;
  if(p->precision != GPUGRAV_PREC_FP64 && p->precision != GPUGRAV_PREC_FP32 && p->precision != GPUGRAV_PREC_FP64_GROUP)
    return GPUGRAV_ERR_INVALID;
  if(p->multiple_domains < 1 || p->multiple_domains > 512 || !(p->top_node_factor > 0))
    return GPUGRAV_ERR_INVALID;
  if((p->flags & ~(GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING | GPUGRAV_FLAG_MINIMUM_OPENING_ANGLE | GPUGRAV_FLAG_ALLOW_DIRECT_SUMMATION)) != 0 ||
     p->reserved != 0)
    return GPUGRAV_ERR_INVALID;
  return GPUGRAV_OK;
}

// short-range table exactly as force_short_range_init (src/gravity/forcetree_walk.c:72-85)
void gg::make_walk_const(const gpugrav_params &p, WalkConst *w)
{
  memset(w, 0, sizeof(*w));
  w->periodic = p.periodic;
  w->mns      = (p.flags & GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING) ? 1 : 0;
  w->minangle = (p.flags & GPUGRAV_FLAG_MINIMUM_OPENING_ANGLE) ? 1 : 0;
  w->nsoft    = p.nsofttypes;
  w->pm       = p.periodic && p.asmth > 0;
  w->ewald    = p.periodic && !(p.asmth > 0);
  if(w->ewald)
    w->ewd_fac_intp = 2.0 * gg::kEwaldN / p.box_size;
  w->bh       = p.err_tol_theta > 0 ? 1 : 0;
  w->box      = p.box_size;
  w->half_box = 0.5 * p.box_size;
  w->theta    = p.err_tol_theta;
  w->erracc   = p.err_tol_force_acc;
  for(int i = 0; i <= p.nsofttypes; i++)
    w->soft[i] = p.force_softening[i];
  if(w->pm)
    {
      double rcut     = p.rcut;
      double asmth    = p.asmth;
      double asmthinv = 0.5 / asmth;
      w->rcut         = rcut;
      w->rcut2        = rcut * rcut;
      w->asmthinv2    = asmthinv * asmthinv;
      w->asmthfac     = asmthinv * (kNtab / (p.rcut_cells / 2.0));
      for(int i = 0; i <= kNtab; i++)
        {
          double u          = ((p.rcut_cells / 2.0) / kNtab) * i;
          w->tab_pot[i]     = (float)(-erfc(u));
          w->tab_force[i]   = (u > 0) ? (float)((erfc(u) + 2.0 * u / sqrt(M_PI) * exp(-u * u) - 1.0) / (u * u)) : 0.0f;
        }
    }
}

// ------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------
extern "C" {

int32_t gpugrav_abi_version(void) { return GPUGRAV_ABI_VERSION; }

const char *gpugrav_status_string(int32_t s)
{
  switch(s)
    {
      case GPUGRAV_OK:
        return "ok";
      case GPUGRAV_ERR_TREE_FULL:
        return "tree storage exhausted (-1)";
      case GPUGRAV_ERR_TOPNODES:
        return "top-level nodes invalid or do not fit (-2)";
      case GPUGRAV_ERR_OUT_OF_BOX:
        return "particle outside the domain box (-3): redo the domain decomposition";
      case GPUGRAV_ERR_INVALID:
        return "invalid argument";
      case GPUGRAV_ERR_OOM:
        return "out of memory";
      case GPUGRAV_ERR_CUDA:
        return "CUDA error";
      case GPUGRAV_ERR_TIMEOUT:
        return "bounded wait timed out";
      case GPUGRAV_ERR_STATE:
        return "call order violated";
      case GPUGRAV_ERR_DEEP_TREE:
        return "tree deeper than supported";
      case GPUGRAV_ERR_UNSUPPORTED:
        return "unsupported option";
      case GPUGRAV_ERR_TOO_LARGE:
        return "request exceeds a fixed capacity (gpugrav_direct_noalloc: at most 4096 targets per call)";
      default:
        return "unknown status";
    }
}

const char *gpugrav_last_error(gpugrav_ctx *c) { return c ? c->err.c_str() : "no context"; }

int32_t gpugrav_create(gpugrav_ctx **out, int32_t device, const gpugrav_params *p)
{
  if(!out)
    return GPUGRAV_ERR_INVALID;
  *out  = nullptr;
  int v = validate_params(p);
  if(v != GPUGRAV_OK)
    return v;
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    {
      cudaGetLastError();
      return GPUGRAV_ERR_CUDA;
    }
  gpugrav_ctx *c = new(std::nothrow) gpugrav_ctx();
  if(!c)
    return GPUGRAV_ERR_OOM;
  c->device = device;
  c->prm    = *p;
  if(const char *e = getenv("GPUGRAV_WALK32_TPL"))
    c->walk32_tpl = atoi(e) == 1 ? 1 : atoi(e) == 2 ? 2 : 0;
  if(const char *e = getenv("GPUGRAV_GROUP_SLACK"))
    c->group_slack = atoi(e);
  if(const char *e = getenv("GPUGRAV_ACTIVE_GROUP_SLACK"))
    c->active_slack = atoi(e);
  if(const char *e = getenv("GPUGRAV_PROFILE"))
    c->profile = atoi(e) != 0;
  DeviceGuard g(device);
  if(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    {
      delete c;
      return GPUGRAV_ERR_CUDA;
    }
  c->own_stream = true;
  for(auto &e : c->ev)
    if(cudaEventCreate(&e) != cudaSuccess)
      {
        delete c;
        return GPUGRAV_ERR_CUDA;
      }
  if(c->bconst.ensure(sizeof(BuildConst)) != cudaSuccess || c->wconst.ensure(sizeof(WalkConst)) != cudaSuccess ||
     c->counters.ensure(64 * sizeof(int)) != cudaSuccess)
    {
      delete c;
      return GPUGRAV_ERR_OOM;
    }
  *out = c;
  return GPUGRAV_OK;
}

int32_t gpugrav_destroy(gpugrav_ctx *c)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(c->profile)
    for(auto &kv : c->prof)
      fprintf(stderr, "gpugrav profile %-24s %10.3f ms\n", kv.first.c_str(), 1e3 * kv.second);
  DeviceGuard g(c->device);
  cudaStreamSynchronize(c->stream);
  gg::DevBuf *bufs[] = {&c->bconst, &c->wconst, &c->pos_in, &c->mass_in, &c->st_in, &c->key, &c->key_alt, &c->idx, &c->perm,
                        &c->sort_tmp, &c->s_pm, &c->s_ix, &c->s_iy, &c->s_iz, &c->s_st, &c->s_cd, &c->s_tl, &c->s_tlnode,
                        &c->cnt, &c->base, &c->hcnt, &c->hack_list, &c->hack_scratch, &c->counters, &c->top, &c->skel,
                        &c->n_suns, &c->n_depth, &c->n_cl, &c->n_sm, &c->n_maxsoft, &c->n_size, &c->n_father, &c->n_sibling,
                        &c->n_next, &c->n_dfs, &c->n_first, &c->p_next, &c->p_father, &c->p_dfs, &c->depth_hist,
                        &c->depth_order, &c->w_sm, &c->w_cl, &c->w_link, &c->g_key, &c->g_key_alt, &c->g_val, &c->g_val_alt, &c->g_bfs, &c->g_np, &c->g_poff, &c->g_sm, &c->g_rel, &c->g_kids, &c->g_pm, &c->g_pst, &c->g_stack, &c->acc_s, &c->pot_s,
                        &c->nint_s, &c->oldacc_s, &c->oldacc_in, &c->out_acc, &c->out_pot, &c->out_nint, &c->scratch,
                        &c->g_groups, &c->g_ngroups, &c->g_gpd, &c->g_gseg, &c->g_gflag, &c->g_gid, &c->t_cd, &c->t_pd, &c->m_sys, &c->m_doms,
                        &c->pm_pos, &c->pm_mass, &c->pm_acc, &c->pm_pot, &c->ewd, &c->ewd32, &c->n_mpt, &c->w_mpt,
                        &c->g_mpt, &c->iperm, &c->t_in, &c->t_pos, &c->t_pos_alt, &c->t_idx, &c->t_idx_alt,
                        &c->cost_in, &c->cost_u, &c->cost_p, &c->slice_rng};
  gg::pm_release(c);
  for(auto *b : bufs)
    b->release();
  c->pinned.release();
  for(auto &e : c->ev)
    if(e)
      cudaEventDestroy(e);
  if(c->own_stream && c->stream)
    cudaStreamDestroy(c->stream);
  delete c;
  return GPUGRAV_OK;
}

int32_t gpugrav_set_params(gpugrav_ctx *c, const gpugrav_params *p)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  int v = validate_params(p);
  if(v != GPUGRAV_OK)
    return fail(c, v, "invalid parameters");
  bool geometry_changed = (p->periodic != c->prm.periodic) || (p->box_size != c->prm.box_size) ||
                          (p->nsofttypes != c->prm.nsofttypes) ||
                          memcmp(p->force_softening, c->prm.force_softening, sizeof(p->force_softening)) != 0;
  c->prm = *p;
  if(geometry_changed)
    {
      c->loaded = false;
      c->built  = false;
    }
  return GPUGRAV_OK;
}

int32_t gpugrav_set_stream(gpugrav_ctx *c, void *stream)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  DeviceGuard g(c->device);
  cudaStreamSynchronize(c->stream);
  if(c->own_stream && c->stream)
    cudaStreamDestroy(c->stream);
  if(stream)
    {
      c->stream     = (cudaStream_t)stream;
      c->own_stream = false;
    }
  else
    {
      if(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(c, GPUGRAV_ERR_CUDA, "stream creation");
      c->own_stream = true;
    }
  return GPUGRAV_OK;
}

int32_t gpugrav_synchronize(gpugrav_ctx *c)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  DeviceGuard g(c->device);
  CK(cudaStreamSynchronize(c->stream), "synchronize");
  return GPUGRAV_OK;
}

int32_t gpugrav_load(gpugrav_ctx *c, int64_t n, const double *pos, const double *mass, const uint8_t *softtype, int32_t mem,
                     const gpugrav_domain *dom)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(n < 2 || n >= (int64_t)1 << 30 || !pos || !mass || !softtype || (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_load: need n >= 2, n < 2^30 and non-null arrays");
  DeviceGuard g(c->device);
  c->loaded = false;
  c->built  = false;
  c->n      = n;
  cudaStream_t st = c->stream;
  cudaEventRecord(c->ev[0], st);
  if(c->pos_in.ensure(n * 3 * sizeof(double)) != cudaSuccess || c->mass_in.ensure(n * sizeof(double)) != cudaSuccess ||
     c->st_in.ensure(n + 16) != cudaSuccess)
    return fail(c, GPUGRAV_ERR_OOM, "gpugrav_load: device allocation");
  cudaMemcpyKind kind = (mem == GPUGRAV_MEM_HOST) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  CK(cudaMemcpyAsync(c->pos_in.p, pos, n * 3 * sizeof(double), kind, st), "upload positions");
  CK(cudaMemcpyAsync(c->mass_in.p, mass, n * sizeof(double), kind, st), "upload masses");
  CK(cudaMemcpyAsync(c->st_in.p, softtype, n, kind, st), "upload softening types");
  cudaEventRecord(c->ev[1], st);

  // softening types must index ForceSoftening[0..nsofttypes-1]: validated on the host copy when given
  BuildConst bc;
  memset(&bc, 0, sizeof(bc));
  bc.n        = n;
  bc.periodic = c->prm.periodic;
  bc.nsoft    = c->prm.nsofttypes;
  bc.mns      = (c->prm.flags & GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING) ? 1 : 0;
  bc.box      = c->prm.box_size;
  for(int i = 0; i <= c->prm.nsofttypes; i++)
    bc.soft[i] = c->prm.force_softening[i];
  if(dom)
    {
      if(!(dom->len > 0) || !std::isfinite(dom->len))
        return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_load: invalid domain");
      bc.dom = *dom;
    }
  CK(cudaMemcpyAsync(c->bconst.p, &bc, sizeof(bc), cudaMemcpyHostToDevice, st), "upload constants");

  int flags = 0;
  CK(gg::domain_stage(c, dom == nullptr, &flags), "domain stage");
  if(flags & 2)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_load: non-finite particle position");
  if(flags & 1)
    return fail(c, GPUGRAV_ERR_OUT_OF_BOX, "gpugrav_load: particle outside the domain box");
  cudaEventRecord(c->ev[2], st);
  CK(gg::sort_stage(c), "key sort");
  cudaEventRecord(c->ev[3], st);
  CK(gg::gather_stage(c), "gather");
  CK(cudaMemcpyAsync(&bc, c->bconst.p, sizeof(bc), cudaMemcpyDeviceToHost, st), "download domain");
  CK(cudaMemcpyAsync(&flags, c->counters.p, sizeof(int), cudaMemcpyDeviceToHost, st), "download flags");
  CK(cudaStreamSynchronize(st), "domain stage");
  c->dom = bc.dom;
  if(flags & 4)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_load: softening type >= nsofttypes");
  c->timings.upload_ms = elapsed(c->ev[0], c->ev[1]);
  c->timings.domain_ms = elapsed(c->ev[1], c->ev[2]);
  c->timings.sort_ms   = elapsed(c->ev[2], c->ev[3]);
  c->loaded            = true;
  return GPUGRAV_OK;
}

int32_t gpugrav_build(gpugrav_ctx *c, const gpugrav_topnode *top, int32_t ntop)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(!c->loaded)
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_build before gpugrav_load");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  c->built        = false;
  c->layout32_valid = false;
  cudaEventRecord(c->ev[4], st);
  if(top)
    {
      if(ntop < 1 || ntop > kMaxTop)
        return fail(c, GPUGRAV_ERR_TOPNODES, "gpugrav_build: top node count out of range");
      if(c->top.ensure(kMaxTop * sizeof(gpugrav_topnode)) != cudaSuccess)
        return fail(c, GPUGRAV_ERR_OOM, "top nodes");
      c->top_host.assign(top, top + ntop);
      CK(cudaMemcpyAsync(c->top.p, top, ntop * sizeof(gpugrav_topnode), cudaMemcpyHostToDevice, st), "upload top nodes");
      c->ntop = ntop;
    }
  else
    {
      int s = 0;
      CK(gg::toptree_stage(c, &s), "top tree");
      if(s != GPUGRAV_OK)
        return fail(c, s, "gpugrav_build: top-level tree could not be refined (PEANOGRID too coarse)");
    }
  cudaEventRecord(c->ev[5], st);
  int s = 0;
  CK(gg::build_stage(c, &s), "tree build");
  if(s != GPUGRAV_OK)
    return fail(c, s, s == GPUGRAV_ERR_TOPNODES ? "gpugrav_build: invalid top-level tree"
                                                : "gpugrav_build: tree build self-check failed");
  cudaEventRecord(c->ev[6], st);
  CK(cudaStreamSynchronize(st), "tree build");
  c->timings.toptree_ms = elapsed(c->ev[4], c->ev[5]);
  c->timings.build_ms   = elapsed(c->ev[5], c->ev[6]);
  c->built              = true;
  return GPUGRAV_OK;
}

int32_t gpugrav_pm_periodic(gpugrav_ctx *c, int32_t pmgrid, int64_t n, const double *pos, const double *mass, double *acc,
                            double *pot, int32_t mem)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(pmgrid < 8 || pmgrid > 2048 || n < 0 || (n > 0 && (!pos || !mass || !acc)) ||
     (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_pm_periodic: need 8 <= pmgrid <= 2048 and pos, mass, acc");
  if(!c->prm.periodic || !(c->prm.box_size > 0) || !(c->prm.asmth > 0))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_pm_periodic: needs a periodic context with box_size > 0 and asmth > 0");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const double *d_pos = pos, *d_mass = mass;
  double *d_acc = acc, *d_pot = pot;
  if(mem == GPUGRAV_MEM_HOST)
    {
      if(c->pm_pos.ensure(n * 24 + 16) != cudaSuccess || c->pm_mass.ensure(n * 8 + 16) != cudaSuccess ||
         c->pm_acc.ensure(n * 24 + 16) != cudaSuccess || (pot && c->pm_pot.ensure(n * 8 + 16) != cudaSuccess))
        return fail(c, GPUGRAV_ERR_OOM, "gpugrav_pm_periodic: device allocation");
      CK(cudaMemcpyAsync(c->pm_pos.p, pos, n * 24, cudaMemcpyHostToDevice, st), "upload positions");
      CK(cudaMemcpyAsync(c->pm_mass.p, mass, n * 8, cudaMemcpyHostToDevice, st), "upload masses");
      d_pos  = c->pm_pos.as<double>();
      d_mass = c->pm_mass.as<double>();
      d_acc  = c->pm_acc.as<double>();
      d_pot  = pot ? c->pm_pot.as<double>() : nullptr;
    }
  cudaEventRecord(c->ev[18], st);
  int fft_status = 0;
  CK(gg::pm_stage(c, pmgrid, n, d_pos, d_mass, d_acc, d_pot, &fft_status), "pm");
  cudaEventRecord(c->ev[19], st);
  if(fft_status != 0)
    {
      const std::string m = "gpugrav_pm_periodic: cuFFT error " + std::to_string(fft_status);
      return fail(c, GPUGRAV_ERR_CUDA, m.c_str());
    }
  if(mem == GPUGRAV_MEM_HOST)
    {
      CK(cudaMemcpyAsync(acc, d_acc, n * 24, cudaMemcpyDeviceToHost, st), "download acc");
      if(pot)
        CK(cudaMemcpyAsync(pot, d_pot, n * 8, cudaMemcpyDeviceToHost, st), "download pot");
    }
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, c->counters.as<int>() + 15, 4, cudaMemcpyDeviceToHost, st), "pm flags");
  CK(cudaStreamSynchronize(st), "pm");
  c->timings.pm_ms = elapsed(c->ev[18], c->ev[19]);
  if(bad)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_pm_periodic: non-finite position or position far outside the box");
  return GPUGRAV_OK;
}

int32_t gpugrav_export_mass_per_type(gpugrav_ctx *c, double *out)
{
  if(!c || !out)
    return GPUGRAV_ERR_INVALID;
  if(!c->built)
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_export_mass_per_type before gpugrav_build");
  if(!(c->prm.flags & GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING))
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_export_mass_per_type: built without MULTIPLE_NODE_SOFTENING");
  DeviceGuard g(c->device);
  CK(cudaMemcpyAsync(out, c->n_mpt.p, (size_t)c->num_nodes * c->prm.nsofttypes * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream),
     "download per-type masses");
  CK(cudaStreamSynchronize(c->stream), "download per-type masses");
  return GPUGRAV_OK;
}

int32_t gpugrav_set_ewald_table(gpugrav_ctx *c, int32_t en, const double *fx, const double *fy, const double *fz,
                                const double *pot)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(en != gg::kEwaldN || !fx || !fy || !fz || !pot)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_set_ewald_table: needs en = 64 and four tables");
  const size_t m = (size_t)(en + 1) * (en + 1) * (en + 1);
  std::vector<double> t(4 * m);
  memcpy(t.data(), fx, m * sizeof(double));
  memcpy(t.data() + m, fy, m * sizeof(double));
  memcpy(t.data() + 2 * m, fz, m * sizeof(double));
  memcpy(t.data() + 3 * m, pot, m * sizeof(double));
  DeviceGuard g(c->device);
  CK(cudaStreamSynchronize(c->stream), "Ewald tables");  // no walk may read the old tables
  CK(gg::ewald_upload(c, t.data()), "Ewald tables");
  return GPUGRAV_OK;
}

int32_t gpugrav_set_target_slice_cost(gpugrav_ctx *c, int32_t slice, int32_t nslices, int64_t n, const float *cost, int32_t mem)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(nslices < 1 || slice < 0 || slice >= nslices || (cost && n < 1) || (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_set_target_slice_cost: need 0 <= slice < nslices and n >= 1");
  c->slice    = slice;
  c->nslices  = nslices;
  c->cost_set = false;
  if(!cost)
    return GPUGRAV_OK;
  DeviceGuard g(c->device);
  if(c->cost_in.ensure(n * sizeof(float) + 16) != cudaSuccess)
    return fail(c, GPUGRAV_ERR_OOM, "gpugrav_set_target_slice_cost: device allocation");
  CK(cudaMemcpyAsync(c->cost_in.p, cost, n * sizeof(float),
                     mem == GPUGRAV_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream),
     "upload costs");
  if(mem == GPUGRAV_MEM_HOST)
    CK(cudaStreamSynchronize(c->stream), "upload costs");  // the caller may reuse its array
  c->cost_n   = n;
  c->cost_set = true;
  return GPUGRAV_OK;
}

int32_t gpugrav_set_target_slice(gpugrav_ctx *c, int32_t slice, int32_t nslices)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(nslices < 1 || slice < 0 || slice >= nslices)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_set_target_slice: need 0 <= slice < nslices");
  c->slice    = slice;
  c->nslices  = nslices;
  c->cost_set = false;  // equal shares of the targets
  return GPUGRAV_OK;
}

}  // extern "C"

namespace
{
// gravity_tree for every loaded particle (targets == nullptr) or for the caller's list of active
// particles (caller indices); outputs in caller order or in the order of the list
int walk_impl(gpugrav_ctx *c, int64_t nt, const int32_t *targets, const float *oldacc, double *acc, double *pot,
              int32_t *ninter, int32_t mem)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(!c->built)
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_walk before gpugrav_build");
  const bool active = targets != nullptr;
  if(!active && c->cost_set && c->nslices > 1 && c->cost_n != c->n)
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_walk: slice costs were set for another particle count");
  if((!acc && !(active && nt == 0)) || (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_walk: acc must be non-null");
  if(active && (nt < 0 || nt > c->n))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_walk_targets: need 0 <= ntargets <= n");
  if(active && nt == 0)
    return GPUGRAV_OK;
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const int64_t n    = c->n;
  const int64_t nout = active ? nt : n;
  if(c->acc_s.ensure(n * 3 * sizeof(double)) != cudaSuccess || c->pot_s.ensure(n * sizeof(double)) != cudaSuccess ||
     c->nint_s.ensure(n * sizeof(int32_t)) != cudaSuccess || c->oldacc_s.ensure(n * sizeof(float)) != cudaSuccess ||
     c->oldacc_in.ensure(n * sizeof(float)) != cudaSuccess || (active && c->t_in.ensure(nt * sizeof(int32_t) + 16) != cudaSuccess))
    return fail(c, GPUGRAV_ERR_OOM, "gpugrav_walk: device allocation");
  WalkConst wc;
  make_walk_const(c->prm, &wc);
  if(wc.ewald)
    {
      CK(gg::ewald_ensure(c), "Ewald tables");
      wc.ewd = c->ewd.as<double>();
    }
  if(wc.mns)
    wc.w_mpt = c->w_mpt.as<double>();
  c->want_pot = (pot != nullptr);
  CK(cudaMemcpyAsync(c->wconst.p, &wc, sizeof(wc), cudaMemcpyHostToDevice, st), "walk constants");
  cudaEventRecord(c->ev[7], st);
  const float *old_dev = nullptr;
  if(oldacc)
    {
      if(mem == GPUGRAV_MEM_HOST)
        {
          CK(cudaMemcpyAsync(c->oldacc_in.p, oldacc, n * sizeof(float), cudaMemcpyHostToDevice, st), "upload OldAcc");
          old_dev = c->oldacc_in.as<float>();
        }
      else
        old_dev = oldacc;
    }
  k_gather_f32<<<grid_for(n, 256), 256, 0, st>>>(old_dev, c->perm.as<uint32_t>(), n, c->oldacc_s.as<float>());
  // active list: sorted positions in key order (targets_stage checks range and duplicates)
  const bool fp32 = c->prm.precision != GPUGRAV_PREC_FP64;  // the group walk (FP32, or its FP64 form)
  const int cap   = 32 * gg::walk32_tpl(c);                    // group size
  int64_t a = 0, b = nout;  // this call's target slice of the active list
  c->w_tlist    = nullptr;
  c->w_ntargets = 0;
  if(active)
    {
      const int32_t *d_t = targets;
      if(mem == GPUGRAV_MEM_HOST)
        {
          CK(cudaMemcpyAsync(c->t_in.p, targets, nt * sizeof(int32_t), cudaMemcpyHostToDevice, st), "upload targets");
          d_t = c->t_in.as<int32_t>();
        }
      int flags = 0;
      CK(gg::targets_stage(c, nt, d_t, &flags), "active targets");
      if(flags & 1)
        return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_walk_targets: target index outside [0, n)");
      if(flags & 2)
        return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_walk_targets: a particle is listed twice");
      if(fp32)
        {
          const int64_t ng = (nt + cap - 1) / cap, gb = ng * c->slice / c->nslices, ge = ng * (c->slice + 1) / c->nslices;
          a = gb * cap;
          b = ge * cap < nt ? ge * cap : nt;
        }
      else
        {
          a = nt * c->slice / c->nslices;
          b = nt * (c->slice + 1) / c->nslices;
        }
    }
  CK(cudaMemsetAsync(c->counters.as<int>() + 32, 0, 8, st), "reset counters");
  CK(cudaMemsetAsync(c->counters.as<int>() + 14, 0, 4, st), "reset counters");
  cudaEventRecord(c->ev[8], st);
  cudaError_t we = cudaSuccess;
  if(fp32)
    {
      we = gg::walk32_prepare(c, wc);
      if(we == cudaSuccess)
        {
          if(active)
            {
              we               = gg::groups_active_stage(c, nt, cap);
              c->groups_active = true;
            }
          else if(c->groups_active)
            {
              we               = gg::groups_stage(c);  // the table of every particle again
              c->groups_active = false;
            }
        }
      c->slice_rng_on = false;
      if(!active && we == cudaSuccess)
        we = gg::slice_cost_stage(c, true);  // cost-balanced slice range, if costs are set
      if(active)
        {
          c->w_tlist    = c->t_pos_alt.as<int32_t>();
          c->w_ntargets = nt;
        }
      if(we == cudaSuccess)
        we = gg::walk32_launch(c);
    }
  else
    {
      c->slice_rng_on = false;
      if(active)
        {
          c->w_tlist    = c->t_pos_alt.as<int32_t>();
          c->w_ntargets = nt;
        }
      else
        we = gg::slice_cost_stage(c, false);
      if(we == cudaSuccess)
        we = gg::walk64_stage(c, wc);
    }
  c->w_tlist    = nullptr;
  c->w_ntargets = 0;
  CK(we, fp32 ? "fp32 walk" : "fp64 walk");
  if(!active)
    CK(gg::slice_mask_stage(c, fp32), "target slice");
  cudaEventRecord(c->ev[9], st);
  double *d_acc = acc, *d_pot = pot;
  int32_t *d_nint = ninter;
  if(mem == GPUGRAV_MEM_HOST)
    {
      if(c->out_acc.ensure(nout * 3 * sizeof(double)) != cudaSuccess || c->out_pot.ensure(nout * sizeof(double)) != cudaSuccess ||
         c->out_nint.ensure(nout * sizeof(int32_t)) != cudaSuccess)
        return fail(c, GPUGRAV_ERR_OOM, "gpugrav_walk: output staging");
      d_acc  = c->out_acc.as<double>();
      d_pot  = pot ? c->out_pot.as<double>() : nullptr;
      d_nint = ninter ? c->out_nint.as<int32_t>() : nullptr;
    }
  if(active)
    CK(gg::targets_scatter(c, nt, a, b, d_acc, d_pot, d_nint), "scatter");
  else
    {
      k_scatter_out<<<grid_for(n, 256), 256, 0, st>>>(c->acc_s.as<double>(), c->pot_s.as<double>(), c->nint_s.as<int32_t>(),
                                                      c->perm.as<uint32_t>(), n, d_acc, d_pot, d_nint);
      CK(cudaGetLastError(), "scatter");
    }
  if(mem == GPUGRAV_MEM_HOST)
    {
      CK(cudaMemcpyAsync(acc, d_acc, nout * 3 * sizeof(double), cudaMemcpyDeviceToHost, st), "download acc");
      if(pot)
        CK(cudaMemcpyAsync(pot, d_pot, nout * sizeof(double), cudaMemcpyDeviceToHost, st), "download pot");
      if(ninter)
        CK(cudaMemcpyAsync(ninter, d_nint, nout * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "download interactions");
    }
  unsigned long long tot = 0;
  int walk_err = 0;
  CK(cudaMemcpyAsync(&tot, c->counters.as<int>() + 32, 8, cudaMemcpyDeviceToHost, st), "interaction total");
  CK(cudaMemcpyAsync(&walk_err, c->counters.as<int>() + 14, 4, cudaMemcpyDeviceToHost, st), "walk flags");
  cudaEventRecord(c->ev[10], st);
  CK(cudaStreamSynchronize(st), "walk");
  if(walk_err)
    return fail(c, GPUGRAV_ERR_DEEP_TREE, "gpugrav_walk: traversal stack of the FP32 walk exhausted");
  c->timings.walk_ms              = elapsed(c->ev[8], c->ev[9]);
  c->timings.download_ms          = elapsed(c->ev[9], c->ev[10]);
  c->timings.interactions         = (int64_t)tot;
  c->timings.walk_kernel_launches = 1;
  return GPUGRAV_OK;
}

// gravity_direct for n particles (targets = sources), outputs in the given order
int gravity_direct_impl(gpugrav_ctx *c, int64_t n, const double *pos, const double *mass, const uint8_t *softtype, double *acc,
                        double *pot, int32_t *ninter, int32_t mem)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(n < 1 || n >= (int64_t)1 << 30 || !pos || !mass || !softtype || !acc || (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_gravity_direct: need n >= 1 and pos, mass, softtype, acc");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  c->loaded = c->built = false;  // the particle buffers are reused
  WalkConst wc;
  make_walk_const(c->prm, &wc);
  if(wc.ewald)
    {
      CK(gg::ewald_ensure(c), "Ewald tables");
      wc.ewd = c->ewd.as<double>();
    }
  CK(cudaMemcpyAsync(c->wconst.p, &wc, sizeof(wc), cudaMemcpyHostToDevice, st), "walk constants");
  const double *d_pos = pos, *d_mass = mass;
  const uint8_t *d_st = softtype;
  double *d_acc = acc, *d_pot = pot;
  int32_t *d_nint = ninter;
  if(mem == GPUGRAV_MEM_HOST)
    {
      if(c->pos_in.ensure(n * 24) != cudaSuccess || c->mass_in.ensure(n * 8) != cudaSuccess || c->st_in.ensure(n + 16) != cudaSuccess ||
         c->out_acc.ensure(n * 24) != cudaSuccess || c->out_pot.ensure(n * 8) != cudaSuccess ||
         c->out_nint.ensure(n * 4) != cudaSuccess)
        return fail(c, GPUGRAV_ERR_OOM, "gpugrav_gravity_direct: device allocation");
      CK(cudaMemcpyAsync(c->pos_in.p, pos, n * 24, cudaMemcpyHostToDevice, st), "upload positions");
      CK(cudaMemcpyAsync(c->mass_in.p, mass, n * 8, cudaMemcpyHostToDevice, st), "upload masses");
      CK(cudaMemcpyAsync(c->st_in.p, softtype, n, cudaMemcpyHostToDevice, st), "upload softening types");
      d_pos  = c->pos_in.as<double>();
      d_mass = c->mass_in.as<double>();
      d_st   = c->st_in.as<uint8_t>();
      d_acc  = c->out_acc.as<double>();
      d_pot  = pot ? c->out_pot.as<double>() : nullptr;
      d_nint = ninter ? c->out_nint.as<int32_t>() : nullptr;
    }
  int *flag = c->counters.as<int>() + 17;
  CK(cudaMemsetAsync(flag, 0, sizeof(int), st), "reset flag");
  cudaEventRecord(c->ev[8], st);
  CK(gg::gravity_direct_stage(c, n, d_pos, d_mass, d_st, d_acc, d_pot, d_nint, flag), "direct summation");
  cudaEventRecord(c->ev[9], st);
  if(mem == GPUGRAV_MEM_HOST)
    {
      CK(cudaMemcpyAsync(acc, d_acc, n * 24, cudaMemcpyDeviceToHost, st), "download acc");
      if(pot)
        CK(cudaMemcpyAsync(pot, d_pot, n * 8, cudaMemcpyDeviceToHost, st), "download pot");
      if(ninter)
        CK(cudaMemcpyAsync(ninter, d_nint, n * 4, cudaMemcpyDeviceToHost, st), "download interactions");
    }
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, st), "flags");
  CK(cudaStreamSynchronize(st), "direct summation");
  if(bad)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_gravity_direct: softening type >= nsofttypes");
  c->timings.walk_ms              = elapsed(c->ev[8], c->ev[9]);
  c->timings.interactions         = n * n;
  c->timings.walk_kernel_launches = 1;
  return GPUGRAV_OK;
}
}  // namespace

extern "C" {

int32_t gpugrav_walk(gpugrav_ctx *c, const float *oldacc, double *acc, double *pot, int32_t *ninter, int32_t mem)
{
  return walk_impl(c, 0, nullptr, oldacc, acc, pot, ninter, mem);
}

int32_t gpugrav_walk_targets(gpugrav_ctx *c, int64_t ntargets, const int32_t *targets, const float *oldacc, double *acc,
                             double *pot, int32_t *ninter, int32_t mem)
{
  if(!targets && ntargets != 0)
    return c ? fail(c, GPUGRAV_ERR_INVALID, "gpugrav_walk_targets: targets is null") : GPUGRAV_ERR_INVALID;
  static const int32_t none = 0;
  return walk_impl(c, ntargets, targets ? targets : &none, oldacc, acc, pot, ninter, mem);
}

int32_t gpugrav_timestep_gravity(gpugrav_ctx *c, const gpugrav_timestep_params *tp, int64_t n, const double *grav_accel,
                                 const double *grav_pm, const double *mass, const uint64_t *ids, const uint8_t *softtype,
                                 const int8_t *bin_old, int64_t *ti_step, int8_t *bin, int64_t *failed, int32_t mem)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(!tp || n < 1 || !grav_accel || !mass || !softtype || !bin_old || !ti_step || !bin || !(tp->timebase_interval > 0) ||
     tp->timebase < 2 || (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_timestep_gravity: invalid arguments");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  const double *d_acc = grav_accel, *d_pm = grav_pm, *d_mass = mass;
  const uint64_t *d_ids = ids;
  const uint8_t *d_st = softtype;
  const int8_t *d_bo  = bin_old;
  int64_t *d_ti       = ti_step;
  int8_t *d_bin       = bin;
  gg::DevBuf tmp;
  if(mem == GPUGRAV_MEM_HOST)
    {
      // one staging block: acc | pm | mass | ids | ti | softtype | bin_old | bin
      const size_t need = n * (24 + (grav_pm ? 24 : 0) + 8 + (ids ? 8 : 0) + 8 + 3) + 256;
      if(tmp.ensure(need) != cudaSuccess)
        return fail(c, GPUGRAV_ERR_OOM, "gpugrav_timestep_gravity: device allocation");
      char *q = tmp.as<char>();
      auto take = [&](size_t b) { char *r = q; q += (b + 15) & ~(size_t)15; return r; };
      double *a = (double *)take(n * 24), *pm = grav_pm ? (double *)take(n * 24) : nullptr, *m = (double *)take(n * 8);
      uint64_t *id = ids ? (uint64_t *)take(n * 8) : nullptr;
      d_ti         = (int64_t *)take(n * 8);
      uint8_t *s   = (uint8_t *)take(n);
      int8_t *bo = (int8_t *)take(n), *bn = (int8_t *)take(n);
      CK(cudaMemcpyAsync(a, grav_accel, n * 24, cudaMemcpyHostToDevice, st), "upload");
      if(pm)
        CK(cudaMemcpyAsync(pm, grav_pm, n * 24, cudaMemcpyHostToDevice, st), "upload");
      CK(cudaMemcpyAsync(m, mass, n * 8, cudaMemcpyHostToDevice, st), "upload");
      if(id)
        CK(cudaMemcpyAsync(id, ids, n * 8, cudaMemcpyHostToDevice, st), "upload");
      CK(cudaMemcpyAsync(s, softtype, n, cudaMemcpyHostToDevice, st), "upload");
      CK(cudaMemcpyAsync(bo, bin_old, n, cudaMemcpyHostToDevice, st), "upload");
      d_acc = a, d_pm = pm, d_mass = m, d_ids = id, d_st = s, d_bo = bo, d_bin = bn;
    }
  int code = 0;
  int64_t first = -1;
  CK(gg::timestep_stage(c, tp, n, d_acc, d_pm, d_mass, d_ids, d_st, d_bo, d_ti, d_bin, &code, &first), "time steps");
  if(mem == GPUGRAV_MEM_HOST)
    {
      CK(cudaMemcpyAsync(ti_step, d_ti, n * 8, cudaMemcpyDeviceToHost, st), "download");
      CK(cudaMemcpyAsync(bin, d_bin, n, cudaMemcpyDeviceToHost, st), "download");
      CK(cudaStreamSynchronize(st), "time steps");
    }
  tmp.release();
  if(failed)
    *failed = code ? first : -1;
  static const char *what[] = {"", "time step below MinSizeTimestep", "integer time step outside (0, TIMEBASE)",
                               "time step of integer size 1", "time step beyond the end of the timeline",
                               "softening type >= nsofttypes"};
  if(code)
    return fail(c, GPUGRAV_ERR_INVALID, what[code < 6 ? code : 0]);
  return GPUGRAV_OK;
}

int32_t gpugrav_active_particles(gpugrav_ctx *c, int64_t n, const int8_t *bin, const uint8_t *synchronized, int32_t *list,
                                 int64_t *count, int32_t mem)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(n < 1 || n >= (int64_t)1 << 31 || !bin || !synchronized || !list || !count || (mem != GPUGRAV_MEM_HOST && mem != GPUGRAV_MEM_DEVICE))
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_active_particles: invalid arguments");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  gg::DevBuf tmp;
  const size_t need = n * 5 + 256;
  if(tmp.ensure(need) != cudaSuccess)
    return fail(c, GPUGRAV_ERR_OOM, "gpugrav_active_particles: device allocation");
  uint8_t *d_sync  = tmp.as<uint8_t>();
  int64_t *d_count = (int64_t *)(tmp.as<char>() + 64);
  const int8_t *d_bin = bin;
  int32_t *d_list     = list;
  if(mem == GPUGRAV_MEM_HOST)
    {
      int8_t *b = (int8_t *)(tmp.as<char>() + 128);
      d_list    = (int32_t *)(tmp.as<char>() + 128 + ((n + 15) & ~(int64_t)15));
      CK(cudaMemcpyAsync(b, bin, n, cudaMemcpyHostToDevice, st), "upload bins");
      d_bin = b;
    }
  CK(cudaMemcpyAsync(d_sync, synchronized, 64, cudaMemcpyHostToDevice, st), "upload synchronized bins");
  CK(cudaMemsetAsync(d_count, 0, 8, st), "reset count");
  CK(gg::active_stage(c, n, d_bin, d_sync, d_list, d_count), "active particles");
  int64_t cnt = 0;
  CK(cudaMemcpyAsync(&cnt, d_count, 8, cudaMemcpyDeviceToHost, st), "download count");
  CK(cudaStreamSynchronize(st), "active particles");
  if(mem == GPUGRAV_MEM_HOST && cnt > 0)
    {
      CK(cudaMemcpyAsync(list, d_list, cnt * 4, cudaMemcpyDeviceToHost, st), "download list");
      CK(cudaStreamSynchronize(st), "active particles");
    }
  tmp.release();
  *count = cnt;
  return GPUGRAV_OK;
}

int32_t gpugrav_gravity_direct(gpugrav_ctx *c, int64_t n, const double *pos, const double *mass, const uint8_t *softtype,
                               double *acc, double *pot, int32_t mem)
{
  return gravity_direct_impl(c, n, pos, mass, softtype, acc, pot, nullptr, mem);
}

int32_t gpugrav_compute(gpugrav_ctx *c, int64_t n, const double *pos, const double *mass, const uint8_t *softtype,
                        const float *oldacc, const gpugrav_domain *dom, const gpugrav_topnode *top, int32_t ntop, double *acc,
                        double *pot, int32_t *ninter, int32_t mem)
{
  if(c && (c->prm.flags & GPUGRAV_FLAG_ALLOW_DIRECT_SUMMATION) && n < GPUGRAV_DIRECT_SUMMATION_THRESHOLD)
    return gravity_direct_impl(c, n, pos, mass, softtype, acc, pot, ninter, mem);  // gravity(), accel.c:103-110
  int s = gpugrav_load(c, n, pos, mass, softtype, mem, dom);
  if(s != GPUGRAV_OK)
    return s;
  s = gpugrav_build(c, top, ntop);
  if(s != GPUGRAV_OK)
    return s;
  return gpugrav_walk(c, oldacc, acc, pot, ninter, mem);
}

int32_t gpugrav_get_domain(gpugrav_ctx *c, gpugrav_domain *dom)
{
  if(!c || !dom)
    return GPUGRAV_ERR_INVALID;
  if(!c->loaded)
    return fail(c, GPUGRAV_ERR_STATE, "no particles loaded");
  *dom = c->dom;
  return GPUGRAV_OK;
}

int32_t gpugrav_get_order(gpugrav_ctx *c, int64_t *order)
{
  if(!c || !order)
    return GPUGRAV_ERR_INVALID;
  if(!c->loaded)
    return fail(c, GPUGRAV_ERR_STATE, "no particles loaded");
  DeviceGuard g(c->device);
  std::vector<uint32_t> tmp(c->n);
  CK(cudaMemcpyAsync(tmp.data(), c->perm.p, c->n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream), "download order");
  CK(cudaStreamSynchronize(c->stream), "download order");
  for(int64_t i = 0; i < c->n; i++)
    order[i] = tmp[i];
  return GPUGRAV_OK;
}

int32_t gpugrav_get_keys(gpugrav_ctx *c, uint64_t *hi, uint64_t *lo)
{
  if(!c || !hi || !lo)
    return GPUGRAV_ERR_INVALID;
  if(!c->loaded)
    return fail(c, GPUGRAV_ERR_STATE, "no particles loaded");
  DeviceGuard g(c->device);
  std::vector<u128> tmp(c->n);
  CK(cudaMemcpyAsync(tmp.data(), c->key_alt.p, c->n * sizeof(u128), cudaMemcpyDeviceToHost, c->stream), "download keys");
  CK(cudaStreamSynchronize(c->stream), "download keys");
  for(int64_t i = 0; i < c->n; i++)
    {
      hi[i] = (uint64_t)(tmp[i] >> 64);
      lo[i] = (uint64_t)tmp[i];
    }
  return GPUGRAV_OK;
}

int32_t gpugrav_get_topnodes(gpugrav_ctx *c, gpugrav_topnode *top, int32_t capacity, int32_t *ntop)
{
  if(!c || !ntop)
    return GPUGRAV_ERR_INVALID;
  if(!c->built)
    return fail(c, GPUGRAV_ERR_STATE, "no tree built");
  *ntop = (int32_t)c->top_host.size();
  if(top)
    {
      if(capacity < *ntop)
        return fail(c, GPUGRAV_ERR_INVALID, "top node buffer too small");
      memcpy(top, c->top_host.data(), c->top_host.size() * sizeof(gpugrav_topnode));
    }
  return GPUGRAV_OK;
}

int32_t gpugrav_get_tree_info(gpugrav_ctx *c, gpugrav_tree_info *info)
{
  if(!c || !info)
    return GPUGRAV_ERR_INVALID;
  if(!c->built)
    return fail(c, GPUGRAV_ERR_STATE, "no tree built");
  info->num_particles    = c->n;
  info->max_part         = c->n;
  info->num_nodes        = c->num_nodes;
  info->first_non_top    = c->n + c->ntop;
  info->num_topnodes     = c->ntop;
  info->num_topleaves    = c->nleaves;
  info->max_depth        = c->max_depth;
  info->coincident_cells = c->hack_cells;
  return GPUGRAV_OK;
}

int32_t gpugrav_export_tree(gpugrav_ctx *c, double *center, double *len, double *s, double *mass, int32_t *sibling,
                            int32_t *nextnode, int32_t *father, uint8_t *maxsofttype, int32_t *p_next, int32_t *p_father)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  if(!c->built)
    return fail(c, GPUGRAV_ERR_STATE, "no tree built");
  DeviceGuard g(c->device);
  const int64_t nn = c->num_nodes, n = c->n;
  cudaStream_t st  = c->stream;
  std::vector<double4> cl, sm;
  if(center || len)
    {
      cl.resize(nn);
      CK(cudaMemcpyAsync(cl.data(), c->n_cl.p, nn * sizeof(double4), cudaMemcpyDeviceToHost, st), "export");
    }
  if(s || mass)
    {
      sm.resize(nn);
      CK(cudaMemcpyAsync(sm.data(), c->n_sm.p, nn * sizeof(double4), cudaMemcpyDeviceToHost, st), "export");
    }
  if(sibling)
    CK(cudaMemcpyAsync(sibling, c->n_sibling.p, nn * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "export");
  if(nextnode)
    CK(cudaMemcpyAsync(nextnode, c->n_next.p, nn * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "export");
  if(father)
    CK(cudaMemcpyAsync(father, c->n_father.p, nn * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "export");
  if(maxsofttype)
    CK(cudaMemcpyAsync(maxsofttype, c->n_maxsoft.p, nn, cudaMemcpyDeviceToHost, st), "export");
  if(p_next)
    CK(cudaMemcpyAsync(p_next, c->p_next.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "export");
  if(p_father)
    CK(cudaMemcpyAsync(p_father, c->p_father.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "export");
  CK(cudaStreamSynchronize(st), "export");
  for(int64_t k = 0; k < nn; k++)
    {
      if(center)
        {
          center[3 * k + 0] = cl[k].x;
          center[3 * k + 1] = cl[k].y;
          center[3 * k + 2] = cl[k].z;
        }
      if(len)
        len[k] = cl[k].w;
      if(s)
        {
          s[3 * k + 0] = sm[k].x;
          s[3 * k + 1] = sm[k].y;
          s[3 * k + 2] = sm[k].z;
        }
      if(mass)
        mass[k] = sm[k].w;
    }
  return GPUGRAV_OK;
}

int32_t gpugrav_get_timings(gpugrav_ctx *c, gpugrav_timings *t)
{
  if(!c || !t)
    return GPUGRAV_ERR_INVALID;
  *t = c->timings;
  return GPUGRAV_OK;
}

int32_t gpugrav_direct_split(gpugrav_ctx *c, int64_t ntargets, const int64_t *targets, double *acc_total, double *pot_total,
                             double *acc_short, double *pot_short)
{
  if(!c)
    return GPUGRAV_ERR_INVALID;
  const bool treepm = c->prm.periodic && c->prm.asmth > 0;
  if((acc_short || pot_short) && !treepm)
    return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_direct_split: the short-range part needs a TreePM context");
  if(!c->loaded)
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_direct_split before gpugrav_load");
  std::vector<double> a, p;
  if(acc_short || pot_short)
    {
      a.resize(3 * ntargets + 3);
      p.resize(ntargets + 1);
      int s = gpugrav_direct(c, ntargets, targets, GPUGRAV_DIRECT_FULL, a.data(), p.data());
      if(s != GPUGRAV_OK)
        return s;
      // the reference adds mass pi / (Asmth^2 V) per source to the short-range potential
      std::vector<double> m(c->n);
      CK(cudaMemcpyAsync(m.data(), c->mass_in.p, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "masses");
      CK(cudaStreamSynchronize(c->stream), "masses");
      const double box = c->prm.box_size, as = c->prm.asmth;
      double add = 0;
      for(int64_t j = 0; j < c->n; j++)
        add += m[j] * M_PI / (as * as * box * box * box);
      if(acc_short)
        memcpy(acc_short, a.data(), 3 * ntargets * sizeof(double));
      if(pot_short)
        for(int64_t t = 0; t < ntargets; t++)
          pot_short[t] = p[t] + add;
    }
  if(acc_total || pot_total)
    {
      // Newtonian pairs; in a periodic box with the Ewald correction: the direct sum of a context
      // without the TreePM split
      a.assign(3 * ntargets + 3, 0.0);
      p.assign(ntargets + 1, 0.0);
      const gpugrav_params keep = c->prm;
      if(treepm)
        {
          c->prm.asmth = 0.0;
          c->prm.rcut  = 0.0;
        }
      int s = gpugrav_direct(c, ntargets, targets, GPUGRAV_DIRECT_FULL, a.data(), p.data());
      c->prm = keep;
      if(s != GPUGRAV_OK)
        return s;
      if(acc_total)
        memcpy(acc_total, a.data(), 3 * ntargets * sizeof(double));
      if(pot_total)
        memcpy(pot_total, p.data(), ntargets * sizeof(double));
    }
  return GPUGRAV_OK;
}

int32_t gpugrav_direct(gpugrav_ctx *c, int64_t ntargets, const int64_t *targets, int32_t mode, double *acc, double *pot)
{
  if(!c || ntargets < 0 || (ntargets > 0 && (!targets || !acc)) || (mode != GPUGRAV_DIRECT_FULL && mode != GPUGRAV_DIRECT_CUT))
    return GPUGRAV_ERR_INVALID;
  if(!c->loaded)
    return fail(c, GPUGRAV_ERR_STATE, "gpugrav_direct before gpugrav_load");
  DeviceGuard g(c->device);
  cudaStream_t st = c->stream;
  for(int64_t i = 0; i < ntargets; i++)
    if(targets[i] < 0 || targets[i] >= c->n)
      return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_direct: target index out of range");
  gg::DevBuf dt, da, dp;
  if(dt.ensure(ntargets * 8 + 8) != cudaSuccess || da.ensure(ntargets * 24 + 8) != cudaSuccess ||
     dp.ensure(ntargets * 8 + 8) != cudaSuccess)
    return fail(c, GPUGRAV_ERR_OOM, "gpugrav_direct: allocation");
  WalkConst wc;
  make_walk_const(c->prm, &wc);
  if(wc.ewald)
    {
      if(mode == GPUGRAV_DIRECT_CUT)
        return fail(c, GPUGRAV_ERR_INVALID, "gpugrav_direct: no Rcut without the TreePM split (asmth == 0)");
      CK(gg::ewald_ensure(c), "Ewald tables");
      wc.ewd = c->ewd.as<double>();
    }
  CK(cudaMemcpyAsync(c->wconst.p, &wc, sizeof(wc), cudaMemcpyHostToDevice, st), "walk constants");
  CK(cudaMemcpyAsync(dt.p, targets, ntargets * 8, cudaMemcpyHostToDevice, st), "targets");
  CK(gg::direct_stage(c, wc, ntargets, dt.as<int64_t>(), mode == GPUGRAV_DIRECT_CUT, da.as<double>(), dp.as<double>()),
     "direct summation");
  CK(cudaMemcpyAsync(acc, da.p, ntargets * 24, cudaMemcpyDeviceToHost, st), "download");
  if(pot)
    CK(cudaMemcpyAsync(pot, dp.p, ntargets * 8, cudaMemcpyDeviceToHost, st), "download");
  CK(cudaStreamSynchronize(st), "direct summation");
  dt.release();
  da.release();
  dp.release();
  return GPUGRAV_OK;
}

}  // extern "C"
