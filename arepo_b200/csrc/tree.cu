// tree.cu -- top-level tree, octree build, multipole moments, threading and the
// depth-first walk layout.  Compiled with -fmad=false (bit-exact doubles).
//
// The reference inserts particles one at a time in Peano-Hilbert order
// (force_treebuild_insert_single_point, src/gravity/forcetree.c:835-938).  The
// resulting octree is canonical: below the top-level skeleton, a node exists for
// every cell that holds at least two particles (down to MAX_TREE_LEVEL), and the
// node for a cell is created while inserting the second particle of that cell.
// Because the particles of any cell are contiguous in key order, that particle is
// (first particle of the cell) + 1, and the reference's node numbering is the
// order of (inserting particle, depth).  Here every adjacent pair (j-1, j) of the
// sorted particles contributes the nodes for the cells holding both j-1 and j that
// are deeper than the cells holding j-2 and j-1: counted, prefix-summed and filled
// in parallel.  Cells at MAX_TREE_LEVEL that hold several particles follow the
// reference's slot-shifting rule (src/gravity/forcetree.c:861-877), which depends
// on insertion order: those cells are replayed sequentially, one thread each.
//
// Moments (force_update_node_recursive, src/gravity/forcetree.c:1217-1429) are
// accumulated bottom-up one depth level at a time, each node summing its eight
// slots in order 0..7 exactly as the recursion does; the nextnode/sibling
// threading and depth-first positions are filled top-down.
#include <cub/cub.cuh>

#include "internal.h"
#include "ph.cuh"

namespace gg
{
namespace
{
__constant__ PhTable c_ph_tree;
int g_ph_tree_ready[64] = {0};

struct SkelInfo
{
  int32_t ntop_nodes;  // nodes created (NTopnodes)
  int32_t nleaves;
  int32_t status;      // 0 ok, <0 invalid top tree
  int32_t max_top_depth;
};

__device__ __forceinline__ int morton_slot(uint64_t x, uint64_t y, uint64_t z, int depth)
{
  // child index inside a node of depth (depth-1): bits 52-depth, x | y<<1 | z<<2 (src/gravity/forcetree.c:854-855)
  int b = 52 - depth;
  return (int)(((x >> b) & 1) | (((y >> b) & 1) << 1) | (((z >> b) & 1) << 2));
}

struct TreeArgs
{
  int64_t n;
  int32_t ntop;
  const double4 *pm;
  const uint64_t *ix, *iy, *iz;
  const uint8_t *st;
  const int8_t *cd;      // n entries, cd[n-1] = -1
  const uint8_t *tl;     // top-leaf depth
  const int32_t *tlnode; // top-leaf node (relative index)
  const int32_t *base;   // n+1
  const gpugrav_domain *dom;
  const int32_t *sys;           // several independent systems: system of each sorted particle (else null)
  const gpugrav_domain *doms;   // ... and the domain of each system
  int64_t nn;            // node capacity (known after the numbering scan; 0 before)
  int *err;              // self-check flag: set instead of writing out of bounds
};

// domain whose integer grid particle j lives on
__device__ __forceinline__ const gpugrav_domain *dom_of(const TreeArgs &a, int64_t j) { return a.sys ? &a.doms[a.sys[j]] : a.dom; }

// node index self-check: every computed node index must lie in [0, nn)
__device__ __forceinline__ bool node_ok(const TreeArgs &a, int64_t k)
{
  if(k >= 0 && k < a.nn)
    return true;
  atomicOr(a.err, 1);
  return false;
}

__device__ __forceinline__ int CD(const TreeArgs &a, int64_t i) { return (i < 0 || i >= a.n - 1) ? -1 : (int)a.cd[i]; }
__device__ __forceinline__ int cap30(int d) { return d < kMaxTreeLevel ? d : kMaxTreeLevel; }

// first depth of the canonical nodes created while inserting particle j (pair j-1, j)
__device__ __forceinline__ int dstart_of(const TreeArgs &a, int64_t j)
{
  int t = a.tl[j - 1], p = cap30(CD(a, j - 2));
  return (t > p ? t : p) + 1;
}
__device__ __forceinline__ int canon_count(const TreeArgs &a, int64_t j)
{
  if(j <= 0)
    return 0;
  int c = cap30(CD(a, j - 1)) - dstart_of(a, j) + 1;
  return c > 0 ? c : 0;
}
__device__ __forceinline__ int delta(const TreeArgs &a, int64_t p, int64_t q)
{
  if(a.sys && a.sys[p] != a.sys[q])
    return -1;  // different systems share no cell
  return common_depth(a.ix[p], a.iy[p], a.iz[p], a.ix[q], a.iy[q], a.iz[q]);
}
// smallest s <= i with delta(s, i) >= d  (start of the depth-d cell containing i)
__device__ int64_t cell_start(const TreeArgs &a, int64_t i, int d)
{
  int64_t lo_ok = i, step = 1, lo_bad = -1;
  while(true)
    {
      int64_t c = i - step;
      if(c < 0)
        {
          lo_bad = -1;
          break;
        }
      if(delta(a, c, i) >= d)
        {
          lo_ok = c;
          step <<= 1;
        }
      else
        {
          lo_bad = c;
          break;
        }
    }
  // answer in (lo_bad, lo_ok]
  while(lo_ok - lo_bad > 1)
    {
      int64_t m = lo_bad + (lo_ok - lo_bad) / 2;
      if(delta(a, m, i) >= d)
        lo_ok = m;
      else
        lo_bad = m;
    }
  return lo_ok;
}
// largest e >= s with delta(s, e) >= d
__device__ int64_t cell_end(const TreeArgs &a, int64_t s, int d)
{
  int64_t hi_ok = s, step = 1, hi_bad = a.n;
  while(true)
    {
      int64_t c = s + step;
      if(c >= a.n)
        {
          hi_bad = a.n;
          break;
        }
      if(delta(a, s, c) >= d)
        {
          hi_ok = c;
          step <<= 1;
        }
      else
        {
          hi_bad = c;
          break;
        }
    }
  while(hi_bad - hi_ok > 1)
    {
      int64_t m = hi_ok + (hi_bad - hi_ok) / 2;
      if(delta(a, s, m) >= d)
        hi_ok = m;
      else
        hi_bad = m;
    }
  return hi_ok;
}
// relative index of the canonical node of depth d whose cell starts at particle s
__device__ __forceinline__ int64_t node_of(const TreeArgs &a, int64_t s, int d)
{
  return (int64_t)a.ntop + a.base[s + 1] + (d - dstart_of(a, s + 1));
}

// ------------------------------------------------------------------------------
// Top-level tree for one rank (domain_determineTopTree, src/domain/domain_toplevel.c:111-269,
// domain_do_local_refine :280-368, domain_walktoptree :381-393), work load = count / N.
// One thread; particle counts of key ranges by binary search in the sorted keys.
// ------------------------------------------------------------------------------
struct TopTmp
{
  u128 size, start;
  int64_t count, pindex;
  int32_t daughter, leaf;
  double work;
};

__device__ int64_t lower_bound_key(const u128 *keys, int64_t lo, int64_t hi, u128 k)
{
  while(lo < hi)
    {
      int64_t m = lo + (hi - lo) / 2;
      if(keys[m] < k)
        lo = m + 1;
      else
        hi = m;
    }
  return lo;
}

__device__ bool top_less(const TopTmp *T, int a, int b)
{
  if(T[a].work > T[b].work)
    return true;
  if(T[a].work < T[b].work)
    return false;
  return a < b;
}

__global__ void k_toptree(const u128 *__restrict__ keys, int64_t n, double tnf, int mdom, TopTmp *T, int *queue, int *list,
                          gpugrav_topnode *out, int max_top, int *result)
{
  if(threadIdx.x != 0 || blockIdx.x != 0)
    return;
  const int ntask = 1;
  int a = 1 + (ntask / 7 + 1) * 8, b = (int)(tnf * mdom * ntask);
  int limit_ntop = 2 * (a > b ? a : b);
  if(limit_ntop + 8 > max_top)
    {
      *result = -1;
      return;
    }
  double limit = 1.0 / (tnf * mdom * ntask);
  int nq = 0, ntop = 1, nleaves = 1;
  T[0].daughter = -1;
  T[0].size     = (u128)1 << (3 * kBits);
  T[0].start    = 0;
  T[0].pindex   = 0;
  T[0].count    = n;
  T[0].work     = 1.0;
  queue[nq++]   = 0;
  int count;
  do
    {
      for(int i = 1; i < nq; i++)
        for(int j = i; j > 0 && top_less(T, queue[j], queue[j - 1]); j--)
          {
            int t        = queue[j];
            queue[j]     = queue[j - 1];
            queue[j - 1] = t;
          }
      count                 = 0;
      double first_workload = 0;
      for(int q = 0; q < nq; q++)
        if(T[queue[q]].size >= 8)
          {
            first_workload = T[queue[q]].work;
            break;
          }
      for(int q = 0; q < nq; q++)
        {
          int np = queue[q];
          if(T[np].work < 0.125 * first_workload)
            break;
          if(ntop + 8 * (count + 1) >= limit_ntop)
            break;
          if(T[np].work > limit || (nleaves < mdom * ntask && count == 0))
            {
              if(T[np].size < 8)
                {
                  *result = -2;  // the reference stops here: PEANOGRID not fine enough
                  return;
                }
              list[count++] = np;
            }
        }
      if(count > 0)
        {
          for(int k = 0; k < count; k++)
            {
              int i         = list[k];
              T[i].daughter = ntop;
              ntop += 8;
              nleaves += 7;
              int64_t lo = T[i].pindex, hi = T[i].pindex + T[i].count;
              int64_t first[9];
              for(int j = 0; j < 8; j++)
                {
                  int sub         = T[i].daughter + j;
                  T[sub].daughter = -1;
                  T[sub].size     = T[i].size >> 3;
                  T[sub].start    = T[i].start + (u128)j * T[sub].size;
                  first[j]        = lower_bound_key(keys, lo, hi, T[sub].start);
                }
              first[8] = hi;
              for(int j = 0; j < 8; j++)
                {
                  int sub       = T[i].daughter + j;
                  T[sub].pindex = first[j];
                  T[sub].count  = first[j + 1] - first[j];
                  T[sub].work   = (double)T[sub].count / (double)n;
                }
            }
          int w = 0;
          for(int q = 0; q < nq; q++)
            if(T[queue[q]].daughter < 0)
              queue[w++] = queue[q];
          nq = w;
          for(int k = 0; k < count; k++)
            for(int j = 0; j < 8; j++)
              queue[nq++] = T[list[k]].daughter + j;
        }
    }
  while(count > 0);

  // leaf numbering in Peano-Hilbert order (domain_walktoptree): iterative DFS
  int stack[3 * kBits + 8], sp = 0, leaves = 0;
  int child[3 * kBits + 8];
  stack[sp] = 0;
  child[sp] = 0;
  if(T[0].daughter < 0)
    T[0].leaf = leaves++;
  else
    {
      sp = 1;
      while(sp > 0)
        {
          int nd = stack[sp - 1];
          if(child[sp - 1] == 8)
            {
              sp--;
              continue;
            }
          int c = T[nd].daughter + child[sp - 1]++;
          if(T[c].daughter < 0)
            T[c].leaf = leaves++;
          else
            {
              stack[sp] = c;
              child[sp] = 0;
              sp++;
            }
        }
    }
  if(T[0].daughter >= 0)
    {
      // the DFS above started with stack[0] = root
    }

  for(int i = 0; i < ntop; i++)
    {
      out[i].start_key_hi = (uint64_t)(T[i].start >> 64);
      out[i].start_key_lo = (uint64_t)T[i].start;
      out[i].size_hi      = (uint64_t)(T[i].size >> 64);
      out[i].size_lo      = (uint64_t)T[i].size;
      out[i].daughter     = T[i].daughter;
      out[i].leaf         = T[i].daughter < 0 ? T[i].leaf : 0;
      // MortonToPeanoSubnode: Hilbert state after the node's key digits, then digit per octant
      int levels = 0;
      u128 s     = T[i].size;
      while(s < ((u128)1 << (3 * kBits)))
        {
          s <<= 3;
          levels++;
        }
      unsigned state = 0;
      for(int l = 0; l < levels; l++)
        {
          unsigned digit = (unsigned)((T[i].start >> (3 * (kBits - 1 - l))) & 7);
          unsigned oct   = 0;
          while(oct < 8 && (c_ph_tree.e[state * 8 + oct] & 7) != digit)
            oct++;
          state = c_ph_tree.e[state * 8 + (oct & 7)] >> 3;
        }
      for(unsigned oct = 0; oct < 8; oct++)
        {
          unsigned morton             = ((oct >> 2) & 1) | (((oct >> 1) & 1) << 1) | ((oct & 1) << 2);
          out[i].morton_to_peano[morton] = (uint8_t)(c_ph_tree.e[state * 8 + oct] & 7);
        }
    }
  *result = ntop;
}

// ------------------------------------------------------------------------------
// Skeleton: force_create_empty_nodes (src/gravity/forcetree.c:1131-1180), iteratively,
// creating nodes in the same order (i, j, k loops, depth first).  One thread.
// Relative node 0 is the root (len DomainLen, centre DomainCenter).
// ------------------------------------------------------------------------------
__global__ void k_skeleton(const gpugrav_topnode *__restrict__ top, int ntop, const BuildConst *__restrict__ bc,
                           int32_t *__restrict__ suns, double4 *__restrict__ cl, uint8_t *__restrict__ depth,
                           int32_t *__restrict__ leafnode, int32_t *__restrict__ nodetop, SkelInfo *info)
{
  if(threadIdx.x != 0 || blockIdx.x != 0)
    return;
  info->status = 0;
  int nleaves  = 0;
  for(int t = 0; t < ntop; t++)
    {
      if(top[t].daughter >= 0)
        {
          if(top[t].daughter <= t || top[t].daughter + 8 > ntop)
            {
              info->status = -2;
              return;
            }
        }
      else
        {
          nleaves++;
        }
    }
  for(int t = 0; t < ntop; t++)
    if(top[t].daughter < 0 && (top[t].leaf < 0 || top[t].leaf >= nleaves))
      {
        info->status = -2;
        return;
      }
  for(int l = 0; l < nleaves; l++)
    leafnode[l] = -1;

  const gpugrav_domain &dom = bc->dom;
  for(int j = 0; j < 8; j++)
    suns[j] = -1;
  cl[0]    = make_double4(dom.center[0], dom.center[1], dom.center[2], dom.len);
  depth[0] = 0;
  nodetop[0] = 0;
  int numnodes = 1;
  if(top[0].daughter < 0)
    leafnode[top[0].leaf] = 0;

  struct Frame
  {
    int no, topnode, bits, ijk;
    uint64_t x, y, z;
  };
  Frame st[3 * kBits + 8];
  int sp      = 0;
  st[sp++]    = Frame{0, 0, 1, 0, 0, 0, 0};
  int maxd    = 0;
  while(sp > 0)
    {
      Frame &f = st[sp - 1];
      if(top[f.topnode].daughter < 0 || f.ijk == 8)
        {
          sp--;
          continue;
        }
      int i = (f.ijk >> 2) & 1, j = (f.ijk >> 1) & 1, k = f.ijk & 1;
      f.ijk++;
      if(numnodes >= ntop)
        {
          info->status = -2;
          return;
        }
      int sub   = ph_last_digit_dev(c_ph_tree.e, (f.x << 1) + i, (f.y << 1) + j, (f.z << 1) + k, f.bits);
      int count = i + 2 * j + 4 * k;
      int nf    = numnodes++;
      suns[8 * f.no + count] = (int32_t)(nf + bc->n);  // slots hold global indices: nodes start at n
      double4 p      = cl[f.no];
      double lenhalf = __dmul_rn(0.25, p.w);
      cl[nf] = make_double4(__dadd_rn(p.x, __dmul_rn((double)(2 * i - 1), lenhalf)),
                            __dadd_rn(p.y, __dmul_rn((double)(2 * j - 1), lenhalf)),
                            __dadd_rn(p.z, __dmul_rn((double)(2 * k - 1), lenhalf)), __dmul_rn(0.5, p.w));
      for(int q = 0; q < 8; q++)
        suns[8 * nf + q] = -1;
      depth[nf] = (uint8_t)(depth[f.no] + 1);
      if(depth[nf] > maxd)
        maxd = depth[nf];
      int d = top[f.topnode].daughter + sub;
      nodetop[nf] = d;
      if(top[d].daughter == -1)
        leafnode[top[d].leaf] = nf;
      if(sp >= 3 * kBits + 8)
        {
          info->status = -2;
          return;
        }
      st[sp++] = Frame{nf, d, f.bits + 1, 0, 2 * f.x + i, 2 * f.y + j, 2 * f.z + k};
    }
  for(int l = 0; l < nleaves; l++)
    if(leafnode[l] < 0)
      {
        info->status = -2;
        return;
      }
  info->ntop_nodes    = numnodes;
  info->nleaves       = nleaves;
  info->max_top_depth = maxd;
}

// top leaf of every sorted particle: walk TopNodes with MortonToPeanoSubnode
// (src/gravity/forcetree.c:507-522)
__global__ void k_topleaf(const gpugrav_topnode *__restrict__ top, const int32_t *__restrict__ leafnode, int64_t n,
                          const uint64_t *__restrict__ ix, const uint64_t *__restrict__ iy, const uint64_t *__restrict__ iz,
                          uint8_t *__restrict__ tl, int32_t *__restrict__ tlnode)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      uint64_t x = ix[i], y = iy[i], z = iz[i];
      int no = 0, levels = 0;
      while(top[no].daughter >= 0 && levels < 52)
        {
          int b      = 51 - levels;
          int sub    = (int)(((x >> b) & 1) | (((y >> b) & 1) << 1) | (((z >> b) & 1) << 2));
          levels++;
          no = top[no].daughter + top[no].morton_to_peano[sub];
        }
      tl[i]     = (uint8_t)levels;
      tlnode[i] = leafnode[top[no].leaf];
    }
}

__global__ void k_pairdepth(int64_t n, const uint64_t *__restrict__ ix, const uint64_t *__restrict__ iy,
                            const uint64_t *__restrict__ iz, const int32_t *__restrict__ sys, int8_t *__restrict__ cd)
{
  // particles of different systems share no cell
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    cd[i] = (i + 1 < n && (!sys || sys[i] == sys[i + 1]))
                ? (int8_t)common_depth(ix[i], iy[i], iz[i], ix[i + 1], iy[i + 1], iz[i + 1])
                : (int8_t)-1;
}

// several systems: node s is the root of system s (len DomainLen, centre DomainCenter of that system)
__global__ void k_roots(int nsys, const gpugrav_domain *__restrict__ doms, int32_t *__restrict__ suns, double4 *__restrict__ cl,
                        uint8_t *__restrict__ depth)
{
  for(int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x)
    {
      for(int q = 0; q < 8; q++)
        suns[8 * (int64_t)s + q] = -1;
      cl[s]    = make_double4(doms[s].center[0], doms[s].center[1], doms[s].center[2], doms[s].len);
      depth[s] = 0;
    }
}

// several systems: every particle's "top leaf" is its system's root, at depth 0
__global__ void k_tl_roots(int64_t n, const int32_t *__restrict__ sys, uint8_t *__restrict__ tl, int32_t *__restrict__ tlnode)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
      tl[i]     = 0;
      tlnode[i] = sys[i];
    }
}

// canonical node count per inserting particle + detection of replayed (coincident) cells
__global__ void k_count(TreeArgs a, int32_t *__restrict__ cnt, int32_t *__restrict__ hack_start, int *counters)
{
  for(int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= a.n; j += (int64_t)gridDim.x * blockDim.x)
    {
      if(j == a.n)
        {
          cnt[j] = 0;
          continue;
        }
      cnt[j] = canon_count(a, j);
      // cell at MAX_TREE_LEVEL with >= 2 particles starting at j (below a shallower top leaf) ...
      bool h = (a.tl[j] < kMaxTreeLevel) && (CD(a, j) >= kMaxTreeLevel) && (CD(a, j - 1) < kMaxTreeLevel);
      // ... or a top leaf at or below MAX_TREE_LEVEL (its first particle)
      h = h || (a.tl[j] >= kMaxTreeLevel && (j == 0 || a.tlnode[j - 1] != a.tlnode[j]));
      if(h)
        {
          int slot = atomicAdd(&counters[1], 1);
          hack_start[slot] = (int32_t)j;
        }
    }
}

// ---- replay of cells where the MAX_TREE_LEVEL rule applies ----
struct HackCell
{
  int64_t s, e;      // particle range (sorted indices, inclusive)
  int64_t scratch;   // offset into the scratch node pool (count pass)
  int32_t level;     // depth of the cell's node
  int32_t top_leaf;  // 1: the cell is a top leaf
};

__global__ void k_hack_range(TreeArgs a, const int32_t *__restrict__ hack_start, int nh, HackCell *cells, int64_t *sizes)
{
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if(h >= nh)
    return;
  int64_t s = hack_start[h];
  HackCell c;
  c.s = s;
  if(a.tl[s] >= kMaxTreeLevel)
    {
      int64_t e = s;
      while(e + 1 < a.n && a.tlnode[e + 1] == a.tlnode[s])
        e++;
      c.e        = e;
      c.level    = a.tl[s];
      c.top_leaf = 1;
    }
  else
    {
      c.e        = cell_end(a, s, kMaxTreeLevel);
      c.level    = kMaxTreeLevel;
      c.top_leaf = 0;
    }
  c.scratch = 0;
  cells[h]  = c;
  sizes[h]  = c.e - c.s + 1;
}

template <bool FILL>
__device__ void replay_cell(const TreeArgs &a, const HackCell &c, int32_t *suns, int32_t *scratch_suns, int32_t *cnt,
                            double4 *cl, uint8_t *depth, int32_t *father)
{
  // node storage: FILL -> the real node arrays (relative indices); count pass -> a local pool
  // whose entry 0 is the cell node itself
  const int64_t n = a.n;
  int64_t cellnode;
  if(FILL)
    cellnode = c.top_leaf ? (int64_t)a.tlnode[c.s] : node_of(a, c.s, kMaxTreeLevel);
  else
    cellnode = 0;
  int32_t *S    = FILL ? suns : scratch_suns;
  int64_t local = 1;
  // node storage capacity: the whole node array, or one pool entry per particle of the cell
  // (each insertion below MAX_TREE_LEVEL creates at most one node)
  const int64_t cap = FILL ? a.nn : (c.e - c.s + 1);
  if(cellnode < 0 || cellnode >= cap)
    {
      atomicOr(a.err, 2);
      return;
    }
  auto SUN = [&](int64_t node, int slot) -> int32_t & { return S[8 * node + slot]; };
  if(!FILL)
    for(int q = 0; q < 8; q++)
      SUN(0, q) = -1;

  // the first particle takes its natural slot (node creation, src/gravity/forcetree.c:921-924,
  // or the first insertion into an empty top leaf)
  SUN(cellnode, morton_slot(a.ix[c.s], a.iy[c.s], a.iz[c.s], c.level + 1)) = (int32_t)c.s;

  for(int64_t q = c.s + 1; q <= c.e; q++)
    {
      const uint64_t xxb = a.ix[q], yyb = a.iy[q], zzb = a.iz[q];
      int levels         = c.level;
      uint64_t mask      = 1ull << (51 - levels);
      int shiftx = 51 - levels, shifty = 50 - levels, shiftz = 49 - levels;
      int64_t centermask = (int64_t)0xFFF0000000000000ull;
      centermask >>= levels;
      int64_t th = cellnode + n;  // node handle: >= n is a node
      int64_t parent = -1;
      int subnode    = 0;
      int created    = 0;
      int64_t fbase  = FILL ? ((int64_t)a.ntop + a.base[q] + canon_count(a, q)) : 0;
      auto shr = [](uint64_t v, int s) -> uint64_t { return (s < 0 || s > 63) ? 0 : (v >> s); };
      for(int guard = 0; guard < 4096; guard++)
        {
          if(th >= n)
            {
              int64_t nd = th - n;
              subnode    = (int)(shr(xxb & mask, shiftx) | shr(yyb & mask, shifty) | shr(zzb & mask, shiftz));
              shiftx--;
              shifty--;
              shiftz--;
              centermask >>= 1;
              mask >>= 1;
              levels++;
              if(levels > kMaxTreeLevel)
                {
                  for(int jj = 0; jj < 8; jj++)
                    {
                      if(SUN(nd, subnode) < 0)
                        break;
                      subnode++;
                      if(subnode >= 8)
                        subnode = 7;
                    }
                }
              int32_t nn = SUN(nd, subnode);
              if(nn >= 0)
                {
                  parent = nd;
                  th     = nn;
                }
              else
                {
                  SUN(nd, subnode) = (int32_t)q;
                  break;
                }
            }
          else
            {
              int64_t nf = FILL ? (fbase + created) : (local++);
              if(nf < 0 || nf >= cap || th < 0 || th >= n)
                {
                  atomicOr(a.err, 2);
                  return;
                }
              SUN(parent, subnode) = (int32_t)(nf + n);
              if(FILL)
                {
                  const gpugrav_domain *dm = dom_of(a, q);
                  const double bf          = dm->big_fac;
                  double len               = __dmul_rn((double)(mask << 1), bf);
                  double cx = __dadd_rn(__dmul_rn((double)((xxb & (uint64_t)centermask) | mask), bf), dm->corner[0]);
                  double cy = __dadd_rn(__dmul_rn((double)((yyb & (uint64_t)centermask) | mask), bf), dm->corner[1]);
                  double cz = __dadd_rn(__dmul_rn((double)((zzb & (uint64_t)centermask) | mask), bf), dm->corner[2]);
                  cl[nf]     = make_double4(cx, cy, cz, len);
                  depth[nf]  = (uint8_t)(levels > 255 ? 255 : levels);
                  father[nf] = (int32_t)parent;
                }
              for(int jj = 0; jj < 8; jj++)
                SUN(nf, jj) = -1;
              int sub2 = (int)(shr(a.ix[th] & mask, shiftx) | shr(a.iy[th] & mask, shifty) | shr(a.iz[th] & mask, shiftz));
              SUN(nf, sub2) = (int32_t)th;
              th            = nf + n;
              created++;
            }
        }
      if(!FILL)
        cnt[q] += created;
    }
}

__global__ void k_hack_count(TreeArgs a, const HackCell *cells, const int64_t *offsets, int nh, int32_t *scratch, int32_t *cnt)
{
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if(h >= nh)
    return;
  HackCell c = cells[h];
  replay_cell<false>(a, c, nullptr, scratch + 8 * offsets[h], cnt, nullptr, nullptr, nullptr);
}

__global__ void k_hack_fill(TreeArgs a, const HackCell *cells, int nh, int32_t *suns, double4 *cl, uint8_t *depth,
                            int32_t *father)
{
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if(h >= nh)
    return;
  HackCell c = cells[h];
  replay_cell<true>(a, c, suns, nullptr, nullptr, cl, depth, father);
}

// ---- canonical nodes: centre/len (src/gravity/forcetree.c:903-911), parent slot ----
__global__ void k_nodes(TreeArgs a, int32_t *__restrict__ suns, double4 *__restrict__ cl, uint8_t *__restrict__ depth,
                        int32_t *__restrict__ first)
{
  for(int64_t j = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * blockDim.x)
    {
      int cnt = canon_count(a, j);
      if(cnt <= 0)
        continue;
      int d0          = dstart_of(a, j);
      int64_t k0      = (int64_t)a.ntop + a.base[j];
      uint64_t x = a.ix[j], y = a.iy[j], z = a.iz[j];
      const gpugrav_domain *dm = dom_of(a, j);
      const double bf          = dm->big_fac;
      for(int t = 0; t < cnt; t++)
        {
          int d      = d0 + t;
          int64_t k  = k0 + t;
          uint64_t m = 1ull << (51 - d);
          uint64_t keep = ~((1ull << (52 - d)) - 1ull);
          double len = __dmul_rn((double)(m << 1), bf);
          double cx  = __dadd_rn(__dmul_rn((double)((x & keep) | m), bf), dm->corner[0]);
          double cy  = __dadd_rn(__dmul_rn((double)((y & keep) | m), bf), dm->corner[1]);
          double cz  = __dadd_rn(__dmul_rn((double)((z & keep) | m), bf), dm->corner[2]);
          cl[k]      = make_double4(cx, cy, cz, len);
          depth[k]   = (uint8_t)d;
          first[k]   = (int32_t)(j - 1);
          for(int q = 0; q < 8; q++)
            suns[8 * k + q] = -1;
        }
    }
}

// link canonical nodes into their parents' slots
__global__ void k_link_nodes(TreeArgs a, int32_t *__restrict__ suns)
{
  for(int64_t j = 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < a.n; j += (int64_t)gridDim.x * blockDim.x)
    {
      int cnt = canon_count(a, j);
      if(cnt <= 0)
        continue;
      int d0     = dstart_of(a, j);
      int64_t k0 = (int64_t)a.ntop + a.base[j];
      uint64_t x = a.ix[j], y = a.iy[j], z = a.iz[j];
      // first node: parent is the top leaf or a canonical node of an earlier particle
      int pd = d0 - 1;
      int64_t parent;
      if(pd == a.tl[j - 1])
        parent = a.tlnode[j - 1];
      else
        parent = node_of(a, cell_start(a, j - 1, pd), pd);
      if(!node_ok(a, parent) || !node_ok(a, k0 + cnt - 1))
        continue;
      suns[8 * parent + morton_slot(x, y, z, d0)] = (int32_t)(k0 + a.n);
      for(int t = 1; t < cnt; t++)
        suns[8 * (k0 + t - 1) + morton_slot(x, y, z, d0 + t)] = (int32_t)(k0 + t + a.n);
    }
}

// particles into the slot of their deepest node
__global__ void k_leaves(TreeArgs a, int32_t *__restrict__ suns)
{
  for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.n; i += (int64_t)gridDim.x * blockDim.x)
    {
      int tl = a.tl[i];
      if(tl >= kMaxTreeLevel)
        continue;  // replayed
      int dp = cap30(CD(a, i - 1)), dn = cap30(CD(a, i));
      int D  = dp > dn ? dp : dn;
      int64_t parent;
      if(D <= tl)
        {
          parent = a.tlnode[i];
          D      = tl;
        }
      else if(D >= kMaxTreeLevel)
        continue;  // replayed
      else if(dn == D && CD(a, i - 1) < D)
        parent = node_of(a, i, D);
      else
        parent = node_of(a, cell_start(a, i, D), D);
      if(!node_ok(a, parent))
        continue;
      suns[8 * parent + morton_slot(a.ix[i], a.iy[i], a.iz[i], D + 1)] = (int32_t)i;
    }
}

// ---- depth buckets ----
__global__ void k_depth_hist(const uint8_t *__restrict__ depth, int64_t nn, int *hist)
{
  __shared__ int h[256];
  for(int t = threadIdx.x; t < 256; t += blockDim.x)
    h[t] = 0;
  __syncthreads();
  for(int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nn; k += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&h[depth[k]], 1);
  __syncthreads();
  for(int t = threadIdx.x; t < 256; t += blockDim.x)
    if(h[t])
      atomicAdd(&hist[t], h[t]);
}

// Nodes into depth buckets.  The order inside a bucket is free (every node of a level is
// processed independently), so the lanes of a warp that share a depth take one atomic together.
__global__ void k_depth_scatter(const uint8_t *__restrict__ depth, int64_t nn, int *cursor, int32_t *order)
{
  const int lane = threadIdx.x & 31;
  for(int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nn; k += (int64_t)gridDim.x * blockDim.x)
    {
      const unsigned act   = __activemask();
      const int d          = depth[k];
      const unsigned peers = __match_any_sync(act, d);
      const int leader     = __ffs(peers) - 1;
      int base             = 0;
      if(lane == leader)
        base = atomicAdd(&cursor[d], __popc(peers));
      base = __shfl_sync(peers, base, leader);
      order[base + __popc(peers & ((1u << lane) - 1u))] = (int32_t)k;
    }
}

// ---- moments of one depth level (force_update_node_recursive, src/gravity/forcetree.c:1266-1392) ----
__global__ void k_moments(const int32_t *__restrict__ order, int count, int64_t n, const int32_t *__restrict__ suns,
                          const double4 *__restrict__ pm, const uint8_t *__restrict__ st, const double4 *__restrict__ cl,
                          double4 *__restrict__ sm, uint8_t *__restrict__ maxsoft, int32_t *__restrict__ size,
                          const BuildConst *__restrict__ bc, double *__restrict__ mpt)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= count)
    return;
  int64_t k = order[t];
  if(mpt)
    {
      // ExtNodes[].mass_per_type (MULTIPLE_NODE_SOFTENING, src/gravity/forcetree.c:1256-1308): per type,
      // the particle masses and the child sums of slots 0..7 in order
      const int ns = bc->nsoft;
      double acc[GPUGRAV_MAX_SOFTTYPES];
      for(int q = 0; q < ns; q++)
        acc[q] = 0.0;
      for(int q = 0; q < 8; q++)
        {
          int32_t c = suns[8 * k + q];
          if(c < 0)
            continue;
          if(c < n)
            {
              const int s = st[c];
              acc[s]      = __dadd_rn(acc[s], pm[c].w);
            }
          else
            for(int u = 0; u < ns; u++)
              acc[u] = __dadd_rn(acc[u], mpt[(c - n) * ns + u]);
        }
      for(int q = 0; q < ns; q++)
        mpt[k * ns + q] = acc[q];
    }
  double mass = 0, sx = 0, sy = 0, sz = 0;
  int ms      = bc->nsoft;  // NSOFTTYPES + NSOFTTYPES_HYDRO: the entry whose softening is 0
  int sz_     = 1;
  for(int q = 0; q < 8; q++)
    {
      int32_t c = suns[8 * k + q];
      if(c < 0)
        continue;
      if(c < n)
        {
          double4 p = pm[c];
          mass      = __dadd_rn(mass, p.w);
          sx        = __dadd_rn(sx, __dmul_rn(p.w, p.x));
          sy        = __dadd_rn(sy, __dmul_rn(p.w, p.y));
          sz        = __dadd_rn(sz, __dmul_rn(p.w, p.z));
          int s     = st[c];
          if(bc->soft[ms] < bc->soft[s])
            ms = s;
          sz_ += 1;
        }
      else
        {
          int64_t kk = c - n;
          double4 p  = sm[kk];
          mass       = __dadd_rn(mass, p.w);
          sx         = __dadd_rn(sx, __dmul_rn(p.w, p.x));
          sy         = __dadd_rn(sy, __dmul_rn(p.w, p.y));
          sz         = __dadd_rn(sz, __dmul_rn(p.w, p.z));
          int s      = maxsoft[kk];
          if(bc->soft[ms] < bc->soft[s])
            ms = s;
          sz_ += size[kk];
        }
    }
  if(mass != 0)
    {
      sx = __ddiv_rn(sx, mass);
      sy = __ddiv_rn(sy, mass);
      sz = __ddiv_rn(sz, mass);
    }
  else
    {
      double4 c = cl[k];
      sx        = c.x;
      sy        = c.y;
      sz        = c.z;
    }
  sm[k]      = make_double4(sx, sy, sz, mass);
  maxsoft[k] = (uint8_t)ms;
  size[k]    = sz_;
}

// ---- threading and depth-first positions of one level (top-down) ----
__global__ void k_dfs(const int32_t *__restrict__ order, int count, int64_t n, const int32_t *__restrict__ suns,
                      const int32_t *__restrict__ size, int32_t *__restrict__ ndfs, int32_t *__restrict__ nsib,
                      int32_t *__restrict__ nnext, int32_t *__restrict__ nfather, int32_t *__restrict__ pdfs,
                      int32_t *__restrict__ pnext, int32_t *__restrict__ pfather)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= count)
    return;
  int64_t k   = order[t];
  int32_t P   = ndfs[k];
  int32_t SIB = nsib[k];
  int32_t c[8];
  int m = 0;
  for(int q = 0; q < 8; q++)
    {
      int32_t v = suns[8 * k + q];
      if(v >= 0)
        c[m++] = v;
    }
  int32_t off = P + 1;
  for(int i = 0; i < m; i++)
    {
      int32_t v   = c[i];
      int32_t nxt = (i + 1 < m) ? c[i + 1] : SIB;
      if(v < n)
        {
          pdfs[v]    = off;
          pnext[v]   = nxt;
          pfather[v] = (int32_t)(k + n);
          off += 1;
        }
      else
        {
          int64_t kk  = v - n;
          ndfs[kk]    = off;
          nsib[kk]    = nxt;
          nfather[kk] = (int32_t)(k + n);
          off += size[kk];
        }
    }
  nnext[k] = (m > 0) ? c[0] : SIB;
}

// several systems: traversal positions of the roots (exclusive prefix of their subtree sizes, in ndfs)
__global__ void k_roots_finish(int nsys, int32_t *nsib, int32_t *nfather)
{
  for(int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x)
    {
      nsib[s]    = -1;
      nfather[s] = -1;
    }
}

__global__ void k_root_init(int32_t *ndfs, int32_t *nsib, int32_t *nfather)
{
  ndfs[0]    = 0;
  nsib[0]    = -1;
  nfather[0] = -1;
}

// ---- walk layout in depth-first order ----
__global__ void k_layout(int64_t n, int64_t nn, const double4 *__restrict__ pm, const uint8_t *__restrict__ st,
                         const int32_t *__restrict__ pdfs, const double4 *__restrict__ sm, const double4 *__restrict__ cl,
                         const uint8_t *__restrict__ maxsoft, const int32_t *__restrict__ size,
                         const int32_t *__restrict__ ndfs, double4 *__restrict__ w_sm, double4 *__restrict__ w_cl,
                         int2 *__restrict__ w_link, int *err, const double *__restrict__ mpt, int nsoft,
                         double *__restrict__ w_mpt)
{
  const int64_t ne = n + nn;
  for(int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n + nn; t += (int64_t)gridDim.x * blockDim.x)
    {
      if(t < n)
        {
          int32_t e = pdfs[t];
          if(e < 0 || e >= ne)
            {
              atomicOr(err, 4);
              continue;
            }
          w_sm[e]   = pm[t];
          w_cl[e]   = make_double4(0, 0, 0, 0);
          w_link[e] = make_int2(e + 1, (int)st[t]);
        }
      else
        {
          int64_t k = t - n;
          int32_t e = ndfs[k];
          if(e < 0 || e >= ne || e + size[k] > ne)
            {
              atomicOr(err, 4);
              continue;
            }
          w_sm[e]   = sm[k];
          w_cl[e]   = cl[k];
          w_link[e] = make_int2(e + size[k], (int)maxsoft[k] | kNodeFlag);
          if(w_mpt)
            for(int q = 0; q < nsoft; q++)
              w_mpt[(int64_t)e * nsoft + q] = mpt[k * nsoft + q];
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

cudaError_t ensure_ph(int device)
{
  if(device >= 0 && device < 64 && g_ph_tree_ready[device])
    return cudaSuccess;
  PhTable t     = ph_make_table();
  cudaError_t e = cudaMemcpyToSymbol(c_ph_tree, &t, sizeof(t));
  if(e == cudaSuccess && device >= 0 && device < 64)
    g_ph_tree_ready[device] = 1;
  return e;
}
}  // namespace

cudaError_t toptree_stage(gpugrav_ctx *c, int *status)
{
  GG_TRY(ensure_ph(c->device));
  const int max_top = kMaxTop;
  GG_TRY(c->top.ensure(max_top * sizeof(gpugrav_topnode)));
  GG_TRY(c->scratch.ensure(max_top * (sizeof(TopTmp) + 2 * sizeof(int)) + 256));
  GG_TRY(c->counters.ensure(64 * sizeof(int)));
  char *s     = (char *)c->scratch.p;
  TopTmp *T   = (TopTmp *)s;
  int *queue  = (int *)(s + max_top * sizeof(TopTmp));
  int *list   = queue + max_top;
  int *result = c->counters.as<int>() + 8;
  k_toptree<<<1, 32, 0, c->stream>>>(c->key_alt.as<u128>(), c->n, c->prm.top_node_factor, c->prm.multiple_domains, T, queue,
                                      list, c->top.as<gpugrav_topnode>(), max_top, result);
  GG_TRY(cudaGetLastError());
  int r = 0;
  GG_TRY(cudaMemcpyAsync(&r, result, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  GG_TRY(cudaStreamSynchronize(c->stream));
  if(r < 0)
    {
      *status = GPUGRAV_ERR_TOPNODES;
      return cudaSuccess;
    }
  c->ntop = r;
  c->top_host.resize(r);
  GG_TRY(cudaMemcpyAsync(c->top_host.data(), c->top.p, r * sizeof(gpugrav_topnode), cudaMemcpyDeviceToHost, c->stream));
  GG_TRY(cudaStreamSynchronize(c->stream));
  *status = GPUGRAV_OK;
  return cudaSuccess;
}

// Builds the whole tree: skeleton, nodes, moments, threading, walk layout.
// node arrays for nn nodes
cudaError_t node_arrays(gpugrav_ctx *c, int64_t nn)
{
  cudaError_t e;
  if((e = c->n_suns.ensure(nn * 8 * sizeof(int32_t))) != cudaSuccess)
    return e;
  if((e = c->n_depth.ensure(nn + 16)) != cudaSuccess)
    return e;
  if((e = c->n_cl.ensure(nn * sizeof(double4))) != cudaSuccess)
    return e;
  if((e = c->n_sm.ensure(nn * sizeof(double4))) != cudaSuccess)
    return e;
  if((e = c->n_maxsoft.ensure(nn + 16)) != cudaSuccess)
    return e;
  if((e = c->n_size.ensure(nn * sizeof(int32_t))) != cudaSuccess)
    return e;
  if((e = c->n_father.ensure(nn * sizeof(int32_t))) != cudaSuccess)
    return e;
  if((e = c->n_sibling.ensure(nn * sizeof(int32_t))) != cudaSuccess)
    return e;
  if((e = c->n_next.ensure(nn * sizeof(int32_t))) != cudaSuccess)
    return e;
  if((e = c->n_dfs.ensure(nn * sizeof(int32_t))) != cudaSuccess)
    return e;
  if((e = c->n_first.ensure(nn * sizeof(int32_t))) != cudaSuccess)
    return e;
  return cudaSuccess;
}

// every buffer of build_stage sized for n particles, nn nodes and ntop top nodes (or systems), so
// that a long-lived caller allocates once
cudaError_t build_reserve(gpugrav_ctx *c, int64_t n, int64_t nn, int32_t ntop)
{
  GG_TRY(c->s_cd.ensure(n + 16));
  GG_TRY(c->s_tl.ensure(n + 16));
  GG_TRY(c->s_tlnode.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->cnt.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->base.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->hack_list.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->counters.ensure(64 * sizeof(int)));
  GG_TRY(c->skel.ensure(sizeof(SkelInfo) + (size_t)(ntop + 8) * 2 * sizeof(int32_t)));
  GG_TRY(node_arrays(c, nn + 16));
  GG_TRY(c->depth_hist.ensure(2 * 256 * sizeof(int)));
  GG_TRY(c->depth_order.ensure((nn + 16) * sizeof(int32_t)));
  GG_TRY(c->p_next.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->p_father.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->p_dfs.ensure((n + 16) * sizeof(int32_t)));
  size_t tb = 0;
  GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->cnt.as<int32_t>(), c->base.as<int32_t>(), (int)(n + 1), c->stream));
  return c->sort_tmp.ensure(tb);
}

cudaError_t build_stage(gpugrav_ctx *c, int *status)
{
  GG_TRY(ensure_ph(c->device));
  const int64_t n    = c->n;
  const int32_t ntop = c->ntop;
  cudaStream_t st    = c->stream;
  int launches       = 0;
  *status            = GPUGRAV_OK;
  c->mark(nullptr);

  GG_TRY(c->s_cd.ensure(n + 16));
  GG_TRY(c->s_tl.ensure(n + 16));
  GG_TRY(c->s_tlnode.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->cnt.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->base.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->hack_list.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->counters.ensure(64 * sizeof(int)));
  GG_TRY(c->skel.ensure(sizeof(SkelInfo) + (size_t)(ntop + 8) * 2 * sizeof(int32_t)));
  int *counters     = c->counters.as<int>();
  SkelInfo *sinfo   = (SkelInfo *)c->skel.p;
  int32_t *leafnode = (int32_t *)((char *)c->skel.p + sizeof(SkelInfo));
  int32_t *nodetop  = leafnode + ntop + 4;

  // skeleton needs node storage for the first ntop nodes; size node arrays for ntop now, grow later
  auto ensure_nodes = [&](int64_t nn) { return node_arrays(c, nn); };

  // 1. per-particle top leaf, pair depths (skeleton first: it validates the top tree and maps leaves to nodes)
  const int32_t *msys            = c->multi ? c->m_sys.as<int32_t>() : nullptr;
  const gpugrav_domain *mdoms    = c->multi ? c->m_doms.as<gpugrav_domain>() : nullptr;
  GG_TRY(ensure_nodes(ntop + 16));
  if(c->multi)
    {
      // independent systems: one root per system, no top-level skeleton below it
      k_roots<<<grid_for(ntop, 128), 128, 0, st>>>(ntop, mdoms, c->n_suns.as<int32_t>(), c->n_cl.as<double4>(),
                                                    c->n_depth.as<uint8_t>());
      k_tl_roots<<<grid_for(n, 256), 256, 0, st>>>(n, msys, c->s_tl.as<uint8_t>(), c->s_tlnode.as<int32_t>());
      c->nleaves = ntop;
      launches += 2;
    }
  else
    {
      k_skeleton<<<1, 32, 0, st>>>(c->top.as<gpugrav_topnode>(), ntop, c->bconst.as<BuildConst>(), c->n_suns.as<int32_t>(),
                                    c->n_cl.as<double4>(), c->n_depth.as<uint8_t>(), leafnode, nodetop, sinfo);
      launches++;
      SkelInfo si;
      GG_TRY(cudaMemcpyAsync(&si, sinfo, sizeof(si), cudaMemcpyDeviceToHost, st));
      GG_TRY(cudaStreamSynchronize(st));
      if(si.status < 0 || si.ntop_nodes != ntop)
        {
          *status = GPUGRAV_ERR_TOPNODES;
          return cudaSuccess;
        }
      c->nleaves = si.nleaves;
      k_topleaf<<<grid_for(n, 256), 256, 0, st>>>(c->top.as<gpugrav_topnode>(), leafnode, n, c->s_ix.as<uint64_t>(),
                                                   c->s_iy.as<uint64_t>(), c->s_iz.as<uint64_t>(), c->s_tl.as<uint8_t>(),
                                                   c->s_tlnode.as<int32_t>());
      launches++;
    }
  k_pairdepth<<<grid_for(n, 256), 256, 0, st>>>(n, c->s_ix.as<uint64_t>(), c->s_iy.as<uint64_t>(), c->s_iz.as<uint64_t>(), msys,
                                                 c->s_cd.as<int8_t>());
  launches++;

  TreeArgs a;
  a.n      = n;
  a.ntop   = ntop;
  a.pm     = c->s_pm.as<double4>();
  a.ix     = c->s_ix.as<uint64_t>();
  a.iy     = c->s_iy.as<uint64_t>();
  a.iz     = c->s_iz.as<uint64_t>();
  a.st     = c->s_st.as<uint8_t>();
  a.cd     = c->s_cd.as<int8_t>();
  a.tl     = c->s_tl.as<uint8_t>();
  a.tlnode = c->s_tlnode.as<int32_t>();
  a.base   = c->base.as<int32_t>();
  a.dom    = &c->bconst.as<BuildConst>()->dom;
  a.sys    = msys;
  a.doms   = mdoms;
  a.nn     = 0;
  a.err    = counters + 12;

  c->mark("b1 roots+pairdepth");
  // 2. node counts per inserting particle, replayed cells
  GG_TRY(cudaMemsetAsync(counters, 0, 16 * sizeof(int), st));
  k_count<<<grid_for(n + 1, 256), 256, 0, st>>>(a, c->cnt.as<int32_t>(), c->hack_list.as<int32_t>(), counters);
  launches++;
  int hc[2];
  GG_TRY(cudaMemcpyAsync(hc, counters, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  GG_TRY(cudaStreamSynchronize(st));
  const int nh  = hc[1];
  c->hack_cells = nh;
  HackCell *cells = nullptr;
  if(nh > 0)
    {
      GG_TRY(c->hcnt.ensure((size_t)nh * (sizeof(HackCell) + 2 * sizeof(int64_t)) + 64));
      cells            = (HackCell *)c->hcnt.p;
      int64_t *sizes   = (int64_t *)(cells + nh);
      int64_t *offsets = sizes + nh;
      k_hack_range<<<(nh + 127) / 128, 128, 0, st>>>(a, c->hack_list.as<int32_t>(), nh, cells, sizes);
      size_t tb = 0;
      GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, sizes, offsets, nh, st));
      GG_TRY(c->sort_tmp.ensure(tb));
      GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, sizes, offsets, nh, st));
      int64_t last[2];
      GG_TRY(cudaMemcpyAsync(&last[0], sizes + nh - 1, 8, cudaMemcpyDeviceToHost, st));
      GG_TRY(cudaMemcpyAsync(&last[1], offsets + nh - 1, 8, cudaMemcpyDeviceToHost, st));
      GG_TRY(cudaStreamSynchronize(st));
      int64_t pool = last[0] + last[1];
      GG_TRY(c->hack_scratch.ensure((size_t)pool * 8 * sizeof(int32_t) + 64));
      k_hack_count<<<(nh + 127) / 128, 128, 0, st>>>(a, cells, offsets, nh, c->hack_scratch.as<int32_t>(), c->cnt.as<int32_t>());
      launches += 2;
    }

  c->mark("b2 count+hack");
  // 3. numbering: exclusive scan of per-particle node counts
  {
    size_t tb = 0;
    GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->cnt.as<int32_t>(), c->base.as<int32_t>(), (int)(n + 1), st));
    GG_TRY(c->sort_tmp.ensure(tb));
    GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, c->cnt.as<int32_t>(), c->base.as<int32_t>(), (int)(n + 1), st));
    launches++;
  }
  int32_t mdyn = 0;
  GG_TRY(cudaMemcpyAsync(&mdyn, c->base.as<int32_t>() + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  GG_TRY(cudaStreamSynchronize(st));
  const int64_t nn = (int64_t)ntop + mdyn;
  if(n + nn >= (int64_t)INT32_MAX)
    {
      *status = GPUGRAV_ERR_TREE_FULL;
      return cudaSuccess;
    }
  c->num_nodes = nn;
  c->n_entries = n + nn;
  a.nn         = nn;

  c->mark("b3 scan");
  // grow node arrays, keeping the skeleton written by k_skeleton
  if((size_t)nn * 8 * sizeof(int32_t) > c->n_suns.cap || (size_t)nn * sizeof(double4) > c->n_cl.cap ||
     (size_t)nn + 16 > c->n_depth.cap)
    {
      // the skeleton is cheap: re-create after growth
      gg::DevBuf *bufs[] = {&c->n_suns, &c->n_depth, &c->n_cl, &c->n_sm, &c->n_maxsoft, &c->n_size,
                            &c->n_father, &c->n_sibling, &c->n_next, &c->n_dfs, &c->n_first};
      for(auto *b : bufs)
        b->release();
      GG_TRY(ensure_nodes(nn + 16));
      if(c->multi)
        k_roots<<<grid_for(ntop, 128), 128, 0, st>>>(ntop, mdoms, c->n_suns.as<int32_t>(), c->n_cl.as<double4>(),
                                                      c->n_depth.as<uint8_t>());
      else
        k_skeleton<<<1, 32, 0, st>>>(c->top.as<gpugrav_topnode>(), ntop, c->bconst.as<BuildConst>(), c->n_suns.as<int32_t>(),
                                      c->n_cl.as<double4>(), c->n_depth.as<uint8_t>(), leafnode, nodetop, sinfo);
      launches++;
    }

  c->mark("b3b grow");
  // 4. fill canonical nodes, link, place particles, replay coincident cells
  k_nodes<<<grid_for(n, 256), 256, 0, st>>>(a, c->n_suns.as<int32_t>(), c->n_cl.as<double4>(), c->n_depth.as<uint8_t>(),
                                             c->n_first.as<int32_t>());
  k_link_nodes<<<grid_for(n, 256), 256, 0, st>>>(a, c->n_suns.as<int32_t>());
  k_leaves<<<grid_for(n, 256), 256, 0, st>>>(a, c->n_suns.as<int32_t>());
  launches += 3;
  if(nh > 0)
    {
      k_hack_fill<<<(nh + 127) / 128, 128, 0, st>>>(a, cells, nh, c->n_suns.as<int32_t>(), c->n_cl.as<double4>(),
                                                     c->n_depth.as<uint8_t>(), c->n_father.as<int32_t>());
      launches++;
    }
  GG_TRY(cudaGetLastError());

  c->mark("b4 nodes+link+leaves");
  // 5. depth buckets
  GG_TRY(c->depth_hist.ensure(2 * 256 * sizeof(int)));
  GG_TRY(c->depth_order.ensure((nn + 16) * sizeof(int32_t)));
  int *hist = c->depth_hist.as<int>();
  GG_TRY(cudaMemsetAsync(hist, 0, 256 * sizeof(int), st));
  k_depth_hist<<<grid_for(nn, 256), 256, 0, st>>>(c->n_depth.as<uint8_t>(), nn, hist);
  int h_hist[256];
  GG_TRY(cudaMemcpyAsync(h_hist, hist, sizeof(h_hist), cudaMemcpyDeviceToHost, st));
  GG_TRY(cudaStreamSynchronize(st));
  int h_off[257];
  h_off[0] = 0;
  int maxd = 0;
  for(int d = 0; d < 256; d++)
    {
      h_off[d + 1] = h_off[d] + h_hist[d];
      if(h_hist[d])
        maxd = d;
    }
  c->max_depth = maxd;
  int *cursor  = hist + 256;
  GG_TRY(cudaMemcpyAsync(cursor, h_off, 256 * sizeof(int), cudaMemcpyHostToDevice, st));
  k_depth_scatter<<<grid_for(nn, 256), 256, 0, st>>>(c->n_depth.as<uint8_t>(), nn, cursor, c->depth_order.as<int32_t>());
  launches += 2;

  c->mark("b5 depth buckets");
  // 6. moments bottom-up (with MULTIPLE_NODE_SOFTENING also the per-type masses)
  const int32_t *order = c->depth_order.as<int32_t>();
  const bool mns       = (c->prm.flags & GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING) != 0;
  const int nsoft      = c->prm.nsofttypes;
  if(mns)
    GG_TRY(c->n_mpt.ensure((size_t)(nn + 16) * nsoft * sizeof(double)));
  for(int d = maxd; d >= 0; d--)
    {
      int cnt = h_hist[d];
      if(!cnt)
        continue;
      k_moments<<<(cnt + 127) / 128, 128, 0, st>>>(order + h_off[d], cnt, n, c->n_suns.as<int32_t>(), c->s_pm.as<double4>(),
                                                   c->s_st.as<uint8_t>(), c->n_cl.as<double4>(), c->n_sm.as<double4>(),
                                                   c->n_maxsoft.as<uint8_t>(), c->n_size.as<int32_t>(),
                                                   c->bconst.as<BuildConst>(), mns ? c->n_mpt.as<double>() : nullptr);
      launches++;
    }
  c->mark("b6 moments");
  // 7. threading top-down
  GG_TRY(c->p_next.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->p_father.ensure((n + 16) * sizeof(int32_t)));
  GG_TRY(c->p_dfs.ensure((n + 16) * sizeof(int32_t)));
  if(c->multi)
    {
      // each system's traversal follows the previous one's: roots at the prefix sums of the subtree sizes
      size_t tb = 0;
      GG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tb, c->n_size.as<int32_t>(), c->n_dfs.as<int32_t>(), ntop, st));
      GG_TRY(c->sort_tmp.ensure(tb));
      GG_TRY(cub::DeviceScan::ExclusiveSum(c->sort_tmp.p, tb, c->n_size.as<int32_t>(), c->n_dfs.as<int32_t>(), ntop, st));
      k_roots_finish<<<grid_for(ntop, 128), 128, 0, st>>>(ntop, c->n_sibling.as<int32_t>(), c->n_father.as<int32_t>());
    }
  else
    k_root_init<<<1, 1, 0, st>>>(c->n_dfs.as<int32_t>(), c->n_sibling.as<int32_t>(), c->n_father.as<int32_t>());
  launches++;
  for(int d = 0; d <= maxd; d++)
    {
      int cnt = h_hist[d];
      if(!cnt)
        continue;
      k_dfs<<<(cnt + 127) / 128, 128, 0, st>>>(order + h_off[d], cnt, n, c->n_suns.as<int32_t>(), c->n_size.as<int32_t>(),
                                               c->n_dfs.as<int32_t>(), c->n_sibling.as<int32_t>(), c->n_next.as<int32_t>(),
                                               c->n_father.as<int32_t>(), c->p_dfs.as<int32_t>(), c->p_next.as<int32_t>(),
                                               c->p_father.as<int32_t>());
      launches++;
    }
  c->mark("b7 threading");
  // 8. walk layout of the FP64 walk (several systems are walked by the FP32 group walk only)
  if(!c->multi)
    {
      const int64_t ne = n + nn;
      GG_TRY(c->w_sm.ensure(ne * sizeof(double4)));
      GG_TRY(c->w_cl.ensure(ne * sizeof(double4)));
      GG_TRY(c->w_link.ensure(ne * sizeof(int2)));
      if(mns)
        GG_TRY(c->w_mpt.ensure((size_t)ne * nsoft * sizeof(double)));
      k_layout<<<grid_for(ne, 256), 256, 0, st>>>(n, nn, c->s_pm.as<double4>(), c->s_st.as<uint8_t>(), c->p_dfs.as<int32_t>(),
                                                   c->n_sm.as<double4>(), c->n_cl.as<double4>(), c->n_maxsoft.as<uint8_t>(),
                                                   c->n_size.as<int32_t>(), c->n_dfs.as<int32_t>(), c->w_sm.as<double4>(),
                                                   c->w_cl.as<double4>(), c->w_link.as<int2>(), a.err,
                                                   mns ? c->n_mpt.as<double>() : nullptr, nsoft,
                                                   mns ? c->w_mpt.as<double>() : nullptr);
      launches++;
    }
  c->mark("b8 layout64");
  c->timings.build_kernel_launches = launches;
  GG_TRY(cudaGetLastError());
  int err = 0;
  GG_TRY(cudaMemcpyAsync(&err, a.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  GG_TRY(cudaStreamSynchronize(st));
  if(err)
    {
      c->err  = "tree build self-check failed (flags " + std::to_string(err) + ")";
      *status = GPUGRAV_ERR_TREE_FULL;
    }
  return cudaSuccess;
}
}  // namespace gg
