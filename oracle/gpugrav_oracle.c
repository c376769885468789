/*
 * gpugrav_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the reference's short-range
 * tree-gravity path.  It is the checker for the CUDA library: only tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py may load it.
 * Every function cites the reference code it restates (paths relative to the
 * reference project root).  Floating point follows the reference operation
 * by operation (plain IEEE double, no fused multiply-add), so that its
 * results are bit-identical to the reference build in oracle/ref.
 *
 * Pipeline (one rank, DOUBLEPRECISION=1 storage):
 *   or_extent    domain_findExtent            src/domain/domain_box.c:107-197
 *   or_keys      domain_double_to_int +        src/domain/domain.c:361-370
 *                peano_hilbert_key             src/domain/peano.c:334-390
 *   or_sort      stable merge sort by key      src/domain/peano.c:74-133, 508-544
 *   or_toptree   domain_determineTopTree       src/domain/domain_toplevel.c:111-393
 *                (count-only work load, see below) and
 *                domain_preserve_relevant_topnode_data  src/domain/domain.c:246-272
 *   or_build     force_treebuild_construct,    src/gravity/forcetree.c:320-823
 *                force_create_empty_nodes,     src/gravity/forcetree.c:1131-1180
 *                force_treebuild_insert_single_point  :835-938
 *                force_update_node_recursive   :1217-1429
 *   or_walk      force_treeevaluate (mode 0)   src/gravity/forcetree_walk.c:115-514
 *   or_direct    gravity_forcetest_evaluate    src/gravity/gravtree_forcetest.c:421-648
 *                (direct FP64 summation, exact erfc; Ewald terms omitted)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define OR_NTAB 127
#define OR_MAX_TREE_LEVEL 30
#define OR_BITS 42

/* Cubic-spline softening coefficients, src/main/allvars.h:557-573 (same literals). */
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

/* ------------------------------------------------------------------------ */
/* Parameters (mirrors the fields of All.* used on the path)                 */
/* ------------------------------------------------------------------------ */
typedef struct
{
  int periodic;      /* 1: periodic: TreePM (PMGRID build) if asmth > 0, else pure tree with Ewald
                        correction (periodic build without PMGRID); 0: isolated (GRAVITY_NOT_PERIODIC) */
  int nsoft;         /* NSOFTTYPES; ForceSoftening has nsoft+1 entries, the last one 0 */
  double box;        /* All.BoxSize */
  double asmth;      /* All.Asmth[0] */
  double rcut;       /* All.Rcut[0] */
  double rcut_cells; /* RCUT, extent of the tabulated short-range factor */
  double theta;      /* All.ErrTolTheta; > 0 selects the Barnes-Hut criterion */
  double erracc;     /* All.ErrTolForceAcc */
  double tnf;        /* All.TopNodeFactor */
  int mdom;          /* All.MultipleDomains */
  int flags;         /* bit 0: MULTIPLE_NODE_SOFTENING, bit 1: ACTIVATE_MINIMUM_OPENING_ANGLE */
  double soft[16];   /* All.ForceSoftening[] */
} or_params;

typedef struct
{
  double corner[3], center[3], len, inverse_len, big_fac;
} or_domain;

/* ------------------------------------------------------------------------ */
/* Peano-Hilbert curve: 48-state tables of src/domain/peano.c:334-362        */
/* (data must be identical for bit-exact keys)                              */
/* ------------------------------------------------------------------------ */
static const unsigned char or_rot[48][8] = {
    {36, 28, 25, 27, 10, 10, 25, 27}, {29, 11, 24, 24, 37, 11, 26, 26}, {8, 8, 25, 27, 30, 38, 25, 27},
    {9, 39, 24, 24, 9, 31, 26, 26},   {40, 24, 44, 32, 40, 6, 44, 6},   {25, 7, 33, 7, 41, 41, 45, 45},
    {4, 42, 4, 46, 26, 42, 34, 46},   {43, 43, 47, 47, 5, 27, 5, 35},   {33, 35, 36, 28, 33, 35, 2, 2},
    {32, 32, 29, 3, 34, 34, 37, 3},   {33, 35, 0, 0, 33, 35, 30, 38},   {32, 32, 1, 39, 34, 34, 1, 31},
    {24, 42, 32, 46, 14, 42, 14, 46}, {43, 43, 47, 47, 25, 15, 33, 15}, {40, 12, 44, 12, 40, 26, 44, 34},
    {13, 27, 13, 35, 41, 41, 45, 45}, {28, 41, 28, 22, 38, 43, 38, 22}, {42, 40, 23, 23, 29, 39, 29, 39},
    {41, 36, 20, 36, 43, 30, 20, 30}, {37, 31, 37, 31, 42, 40, 21, 21}, {28, 18, 28, 45, 38, 18, 38, 47},
    {19, 19, 46, 44, 29, 39, 29, 39}, {16, 36, 45, 36, 16, 30, 47, 30}, {37, 31, 37, 31, 17, 17, 46, 44},
    {12, 4, 1, 3, 34, 34, 1, 3},      {5, 35, 0, 0, 13, 35, 2, 2},      {32, 32, 1, 3, 6, 14, 1, 3},
    {33, 15, 0, 0, 33, 7, 2, 2},      {16, 0, 20, 8, 16, 30, 20, 30},   {1, 31, 9, 31, 17, 17, 21, 21},
    {28, 18, 28, 22, 2, 18, 10, 22},  {19, 19, 23, 23, 29, 3, 29, 11},  {9, 11, 12, 4, 9, 11, 26, 26},
    {8, 8, 5, 27, 10, 10, 13, 27},    {9, 11, 24, 24, 9, 11, 6, 14},    {8, 8, 25, 15, 10, 10, 25, 7},
    {0, 18, 8, 22, 38, 18, 38, 22},   {19, 19, 23, 23, 1, 39, 9, 39},   {16, 36, 20, 36, 16, 2, 20, 10},
    {37, 3, 37, 11, 17, 17, 21, 21},  {4, 17, 4, 46, 14, 19, 14, 46},   {18, 16, 47, 47, 5, 15, 5, 15},
    {17, 12, 44, 12, 19, 6, 44, 6},   {13, 7, 13, 7, 18, 16, 45, 45},   {4, 42, 4, 21, 14, 42, 14, 23},
    {43, 43, 22, 20, 5, 15, 5, 15},   {40, 12, 21, 12, 40, 6, 23, 6},   {13, 7, 13, 7, 41, 41, 22, 20}};

static const unsigned char or_sub[48][8] = {
    {0, 7, 1, 6, 3, 4, 2, 5}, {7, 4, 6, 5, 0, 3, 1, 2}, {4, 3, 5, 2, 7, 0, 6, 1}, {3, 0, 2, 1, 4, 7, 5, 6}, {1, 0, 6, 7, 2, 3, 5, 4},
    {0, 3, 7, 4, 1, 2, 6, 5}, {3, 2, 4, 5, 0, 1, 7, 6}, {2, 1, 5, 6, 3, 0, 4, 7}, {6, 1, 7, 0, 5, 2, 4, 3}, {1, 2, 0, 3, 6, 5, 7, 4},
    {2, 5, 3, 4, 1, 6, 0, 7}, {5, 6, 4, 7, 2, 1, 3, 0}, {7, 6, 0, 1, 4, 5, 3, 2}, {6, 5, 1, 2, 7, 4, 0, 3}, {5, 4, 2, 3, 6, 7, 1, 0},
    {4, 7, 3, 0, 5, 6, 2, 1}, {6, 7, 5, 4, 1, 0, 2, 3}, {7, 0, 4, 3, 6, 1, 5, 2}, {0, 1, 3, 2, 7, 6, 4, 5}, {1, 6, 2, 5, 0, 7, 3, 4},
    {2, 3, 1, 0, 5, 4, 6, 7}, {3, 4, 0, 7, 2, 5, 1, 6}, {4, 5, 7, 6, 3, 2, 0, 1}, {5, 2, 6, 1, 4, 3, 7, 0}, {7, 0, 6, 1, 4, 3, 5, 2},
    {0, 3, 1, 2, 7, 4, 6, 5}, {3, 4, 2, 5, 0, 7, 1, 6}, {4, 7, 5, 6, 3, 0, 2, 1}, {6, 7, 1, 0, 5, 4, 2, 3}, {7, 4, 0, 3, 6, 5, 1, 2},
    {4, 5, 3, 2, 7, 6, 0, 1}, {5, 6, 2, 1, 4, 7, 3, 0}, {1, 6, 0, 7, 2, 5, 3, 4}, {6, 5, 7, 4, 1, 2, 0, 3}, {5, 2, 4, 3, 6, 1, 7, 0},
    {2, 1, 3, 0, 5, 6, 4, 7}, {0, 1, 7, 6, 3, 2, 4, 5}, {1, 2, 6, 5, 0, 3, 7, 4}, {2, 3, 5, 4, 1, 0, 6, 7}, {3, 0, 4, 7, 2, 1, 5, 6},
    {1, 0, 2, 3, 6, 7, 5, 4}, {0, 7, 3, 4, 1, 6, 2, 5}, {7, 6, 4, 5, 0, 1, 3, 2}, {6, 1, 5, 2, 7, 0, 4, 3}, {5, 4, 6, 7, 2, 3, 1, 0},
    {4, 3, 7, 0, 5, 2, 6, 1}, {3, 2, 0, 1, 4, 5, 7, 6}, {2, 5, 1, 6, 3, 4, 0, 7}};

/* 52-bit mantissa of a double in [1,2): force_double_to_int, src/gravity/forcetree.h:122-131 */
static inline uint64_t mant52(double d)
{
  uint64_t u;
  memcpy(&u, &d, 8);
  return u & 0xFFFFFFFFFFFFFull;
}

/* peano_hilbert_key, src/domain/peano.c:374-390 */
static u128 ph_key(uint64_t x, uint64_t y, uint64_t z, int bits)
{
  unsigned rot = 0;
  u128 key     = 0;
  for(uint64_t mask = 1ull << (bits - 1); mask > 0; mask >>= 1)
    {
      unsigned pix = ((x & mask) ? 4u : 0u) | ((y & mask) ? 2u : 0u) | ((z & mask) ? 1u : 0u);
      key          = (key << 3) | or_sub[rot][pix];
      rot          = or_rot[rot][pix];
    }
  return key;
}

/* ------------------------------------------------------------------------ */
/* Domain extent: src/domain/domain_box.c:107-197 (DO_NOT_RANDOMIZE_DOMAINCENTER) */
/* ------------------------------------------------------------------------ */
void or_extent(int64_t n, const double *pos, const or_params *p, or_domain *d)
{
  double xmin[3], xmax[3];
  for(int j = 0; j < 3; j++)
    {
      /* preset to the simulation box */
      xmin[j] = 0;
      xmax[j] = p->box;
    }
  for(int64_t i = 0; i < n; i++)
    for(int j = 0; j < 3; j++)
      {
        if(xmin[j] > pos[3 * i + j])
          xmin[j] = pos[3 * i + j];
        if(xmax[j] < pos[3 * i + j])
          xmax[j] = pos[3 * i + j];
      }
  double len = 0;
  for(int j = 0; j < 3; j++)
    if(xmax[j] - xmin[j] > len)
      len = xmax[j] - xmin[j];
  if(p->periodic)
    len *= 1.00001;
  else
    len *= 1.2;
  for(int j = 0; j < 3; j++)
    {
      d->center[j] = 0.5 * (xmin[j] + xmax[j]);
      d->corner[j] = 0.5 * (xmin[j] + xmax[j]) - 0.5 * len;
    }
  d->len         = len;
  d->inverse_len = 1.0 / len;
  d->big_fac     = len / (double)(1ll << 52);
}

/* periodic wrap of a coordinate into [0, box), src/gravity/forcetree.c:405-410 and
 * do_box_wrapping src/domain/domain_box.c:259-275 */
static inline double wrap_pos(double x, const or_params *p)
{
  if(!p->periodic)
    return x;
  if(x < 0)
    x += p->box;
  if(x >= p->box)
    x -= p->box;
  return x;
}

/* ------------------------------------------------------------------------ */
/* Keys: per particle 52-bit integer coordinates and the 126-bit PH key      */
/* src/domain/domain_toplevel.c:120-126, src/gravity/forcetree.c:493-495     */
/* ------------------------------------------------------------------------ */
void or_keys(int64_t n, const double *pos, const or_params *p, const or_domain *d, uint64_t *key_hi, uint64_t *key_lo,
             uint64_t *intpos)
{
  for(int64_t i = 0; i < n; i++)
    {
      uint64_t ip[3];
      for(int j = 0; j < 3; j++)
        ip[j] = mant52(((wrap_pos(pos[3 * i + j], p) - d->corner[j]) * d->inverse_len) + 1.0);
      u128 k = ph_key(ip[0] >> (52 - OR_BITS), ip[1] >> (52 - OR_BITS), ip[2] >> (52 - OR_BITS), OR_BITS);
      if(key_hi)
        {
          key_hi[i] = (uint64_t)(k >> 64);
          key_lo[i] = (uint64_t)k;
        }
      if(intpos)
        for(int j = 0; j < 3; j++)
          intpos[3 * i + j] = ip[j];
    }
}

/* ------------------------------------------------------------------------ */
/* Stable sort by key: msort_peano_with_tmp, src/domain/peano.c:508-544      */
/* ------------------------------------------------------------------------ */
typedef struct
{
  u128 key;
  int64_t index;
} or_kv;

static void msort_kv(or_kv *b, size_t n, or_kv *t)
{
  if(n <= 1)
    return;
  size_t n1 = n / 2, n2 = n - n1;
  or_kv *b1 = b, *b2 = b + n1;
  msort_kv(b1, n1, t);
  msort_kv(b2, n2, t);
  or_kv *tmp = t;
  while(n1 > 0 && n2 > 0)
    {
      if(b1->key <= b2->key)
        {
          --n1;
          *tmp++ = *b1++;
        }
      else
        {
          --n2;
          *tmp++ = *b2++;
        }
    }
  if(n1 > 0)
    memcpy(tmp, b1, n1 * sizeof(or_kv));
  memcpy(b, t, (n - n2) * sizeof(or_kv));
}

/* perm[i] = original index of the particle at sorted position i */
void or_sort(int64_t n, const uint64_t *key_hi, const uint64_t *key_lo, int64_t *perm)
{
  or_kv *a = malloc(sizeof(or_kv) * (n > 0 ? n : 1));
  or_kv *t = malloc(sizeof(or_kv) * (n > 0 ? n : 1));
  for(int64_t i = 0; i < n; i++)
    {
      a[i].key   = ((u128)key_hi[i] << 64) | key_lo[i];
      a[i].index = i;
    }
  msort_kv(a, (size_t)n, t);
  for(int64_t i = 0; i < n; i++)
    perm[i] = a[i].index;
  free(a);
  free(t);
}

/* ------------------------------------------------------------------------ */
/* Top-level tree: domain_determineTopTree for one rank                     */
/* src/domain/domain_toplevel.c:111-269, domain_do_local_refine :280-368,   */
/* domain_walktoptree :381-393.  The work load of a top node is its particle */
/* count divided by N (the reference weights gravity cost and particle count */
/* 1:1; with uniform per-particle cost both terms equal count/N).            */
/* ------------------------------------------------------------------------ */
typedef struct
{
  uint64_t start_hi, start_lo, size_hi, size_lo;
  int32_t daughter, leaf;
  uint8_t morton_to_peano[8];
} or_topnode; /* 48 bytes: the layout of the harness dump and of the library input */

typedef struct
{
  u128 size, start;
  int64_t count, pindex;
  int daughter, parent, leaf;
  double work;
} tn_t;

static int tn_less(const tn_t *T, int a, int b)
{
  /* queue order of mydata_cmp, src/domain/domain_toplevel.c:71-83: larger work first, then lower index */
  if(T[a].work > T[b].work)
    return 1;
  if(T[a].work < T[b].work)
    return 0;
  return a < b;
}

static void tn_walk(tn_t *T, int no, int *nleaves)
{
  if(T[no].daughter == -1)
    T[no].leaf = (*nleaves)++;
  else
    for(int i = 0; i < 8; i++)
      tn_walk(T, T[no].daughter + i, nleaves);
}

/* Morton child index -> PH child index for the children of a node whose key range
 * starts at `start` with size 8^level_count: the Hilbert state machine of
 * peano_hilbert_key run over the node's key digits; equivalent to the inverse-key
 * construction of domain_preserve_relevant_topnode_data, src/domain/domain.c:255-270 */
static void morton_to_peano(u128 start, u128 size, uint8_t *m2p)
{
  int levels_above = 0; /* number of key digits fixed by the node */
  u128 s           = size;
  while(s < ((u128)1 << (3 * OR_BITS)))
    {
      s <<= 3;
      levels_above++;
    }
  unsigned rot = 0;
  for(int l = 0; l < levels_above; l++)
    {
      unsigned digit = (unsigned)((start >> (3 * (OR_BITS - 1 - l))) & 7);
      unsigned pix   = 0;
      while(or_sub[rot][pix] != digit)
        pix++;
      rot = or_rot[rot][pix];
    }
  for(unsigned pix = 0; pix < 8; pix++)
    {
      unsigned morton = ((pix >> 2) & 1) | (((pix >> 1) & 1) << 1) | ((pix & 1) << 2);
      m2p[morton]     = or_sub[rot][pix];
    }
}

/* keys must be sorted; returns the number of top nodes written (<= max_top), or -1 */
int or_toptree(int64_t n, const uint64_t *key_hi, const uint64_t *key_lo, const or_params *p, or_topnode *out, int max_top)
{
  int ntask = 1;
  int a     = 1 + (ntask / 7 + 1) * 8;
  int b     = (int)(p->tnf * p->mdom * ntask);
  int limit_ntop = 2 * (a > b ? a : b);
  double limit   = 1.0 / (p->tnf * p->mdom * ntask);

  tn_t *T    = calloc(limit_ntop + 8, sizeof(tn_t));
  int *queue = malloc(sizeof(int) * (limit_ntop + 8));
  int *list  = malloc(sizeof(int) * (limit_ntop + 8));
  int nq = 0, ntop = 1, nleaves = 1;

  T[0].daughter = -1;
  T[0].parent   = -1;
  T[0].size     = (u128)1 << (3 * OR_BITS);
  T[0].start    = 0;
  T[0].pindex   = 0;
  T[0].count    = n;
  T[0].work     = 1.0;
  queue[nq++]   = 0;

  int count;
  do
    {
      /* keep the queue ordered (small: insertion sort) */
      for(int i = 1; i < nq; i++)
        for(int j = i; j > 0 && tn_less(T, queue[j], queue[j - 1]); j--)
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
          if(T[np].work > limit || (nleaves < p->mdom * ntask && count == 0))
            {
              if(T[np].size < 8)
                {
                  free(T);
                  free(queue);
                  free(list);
                  return -1; /* the reference terminates here (PEANOGRID not fine enough) */
                }
              list[count++] = np;
            }
        }
      if(count > 0)
        {
          for(int k = 0; k < count; k++)
            {
              int i       = list[k];
              T[i].daughter = ntop;
              ntop += 8;
              nleaves += 7;
              for(int j = 0; j < 8; j++)
                {
                  int sub        = T[i].daughter + j;
                  T[sub].daughter = -1;
                  T[sub].parent   = i;
                  T[sub].size     = T[i].size >> 3;
                  T[sub].start    = T[i].start + (u128)j * T[sub].size;
                  T[sub].pindex   = T[i].pindex;
                  T[sub].count    = 0;
                }
              int sub = T[i].daughter;
              for(int64_t q = T[i].pindex, j = 0; q < T[i].pindex + T[i].count; q++)
                {
                  u128 key = ((u128)key_hi[q] << 64) | key_lo[q];
                  if(j < 7)
                    while(key >= T[sub + 1].start)
                      {
                        j++;
                        sub++;
                        T[sub].pindex = q;
                        if(j >= 7)
                          break;
                      }
                  T[sub].count++;
                }
              for(int j = 0; j < 8; j++)
                T[T[i].daughter + j].work = (double)T[T[i].daughter + j].count / (double)n;
            }
          /* remove refined nodes from the queue, append their daughters */
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

  nleaves = 0;
  tn_walk(T, 0, &nleaves);

  if(ntop > max_top)
    {
      free(T);
      free(queue);
      free(list);
      return -1;
    }
  for(int i = 0; i < ntop; i++)
    {
      out[i].start_hi = (uint64_t)(T[i].start >> 64);
      out[i].start_lo = (uint64_t)T[i].start;
      out[i].size_hi  = (uint64_t)(T[i].size >> 64);
      out[i].size_lo  = (uint64_t)T[i].size;
      out[i].daughter = T[i].daughter;
      out[i].leaf     = T[i].daughter < 0 ? T[i].leaf : T[i].leaf;
      morton_to_peano(T[i].start, T[i].size, out[i].morton_to_peano);
    }
  free(T);
  free(queue);
  free(list);
  return ntop;
}

/* recompute MortonToPeanoSubnode for top nodes given by a caller */
void or_topnode_m2p(int ntop, or_topnode *tn)
{
  for(int i = 0; i < ntop; i++)
    morton_to_peano(((u128)tn[i].start_hi << 64) | tn[i].start_lo, ((u128)tn[i].size_hi << 64) | tn[i].size_lo,
                    tn[i].morton_to_peano);
}

/* ------------------------------------------------------------------------ */
/* Tree build + moments                                                     */
/* ------------------------------------------------------------------------ */
typedef struct
{
  /* particles in insertion (sorted) order */
  int64_t n;
  const double *pos; /* n*3, already wrapped */
  const double *mass;
  const uint8_t *stype;
  uint64_t *ip;      /* n*3 52-bit coordinates */
  /* nodes, index relative to max_part: node k lives at index max_part + k */
  int64_t max_part, max_nodes, num_nodes, first_non_top;
  int32_t *suns;     /* max_nodes*8 */
  double *center;    /* max_nodes*3 */
  double *len;
  double *s;         /* max_nodes*3 */
  double *nmass;
  int32_t *sibling, *nextnode, *father;
  uint8_t *maxsoft;
  int32_t *p_next;   /* Nextnode[] of particles */
  int32_t *p_father; /* Father[] of particles */
  const or_params *prm;
  const or_domain *dom;
  const or_topnode *top;
  int ntop;
  int32_t *domain_node_index; /* per top leaf */
} or_tree;

#define NODE(t, no) ((no) - (t)->max_part)

/* force_create_empty_nodes, src/gravity/forcetree.c:1131-1180 */
static int create_empty_nodes(or_tree *t, int64_t no, int topnode, int bits, int x, int y, int z)
{
  if(t->top[topnode].daughter >= 0)
    {
      for(int i = 0; i < 2; i++)
        for(int j = 0; j < 2; j++)
          for(int k = 0; k < 2; k++)
            {
              if(t->num_nodes >= t->max_nodes)
                return -1;
              int sub   = 7 & (int)ph_key((uint64_t)((x << 1) + i), (uint64_t)((y << 1) + j), (uint64_t)((z << 1) + k), bits);
              int count = i + 2 * j + 4 * k;
              int64_t nf = t->max_part + t->num_nodes;
              t->suns[8 * NODE(t, no) + count] = (int32_t)nf;
              double lenhalf                   = 0.25 * t->len[NODE(t, no)];
              t->len[NODE(t, nf)]              = 0.5 * t->len[NODE(t, no)];
              t->center[3 * NODE(t, nf) + 0]   = t->center[3 * NODE(t, no) + 0] + (2 * i - 1) * lenhalf;
              t->center[3 * NODE(t, nf) + 1]   = t->center[3 * NODE(t, no) + 1] + (2 * j - 1) * lenhalf;
              t->center[3 * NODE(t, nf) + 2]   = t->center[3 * NODE(t, no) + 2] + (2 * k - 1) * lenhalf;
              for(int q = 0; q < 8; q++)
                t->suns[8 * NODE(t, nf) + q] = -1;
              int d = t->top[topnode].daughter + sub;
              if(t->top[d].daughter == -1)
                t->domain_node_index[t->top[d].leaf] = (int32_t)nf;
              t->num_nodes++;
              if(create_empty_nodes(t, nf, d, bits + 1, 2 * x + i, 2 * y + j, 2 * z + k) < 0)
                return -1;
            }
    }
  return 0;
}

/* force_treebuild_insert_single_point, src/gravity/forcetree.c:835-938 */
static int insert_point(or_tree *t, int64_t i, int64_t th, int levels)
{
  int64_t parent      = -1;
  unsigned subnode    = 0;
  uint64_t xxb        = t->ip[3 * i + 0];
  uint64_t yyb        = t->ip[3 * i + 1];
  uint64_t zzb        = t->ip[3 * i + 2];
  uint64_t mask       = 1ull << ((52 - 1) - levels);
  int shiftx          = (52 - 1) - levels;
  int shifty          = (52 - 2) - levels;
  int shiftz          = (52 - 3) - levels;
  int64_t centermask  = (int64_t)0xFFF0000000000000ull;
  centermask >>= levels;

  while(1)
    {
      if(th >= t->max_part) /* internal node (single rank: no pseudo or imported points) */
        {
          subnode = (unsigned)(((xxb & mask) >> (shiftx--)) | ((yyb & mask) >> (shifty--)) | ((zzb & mask) >> (shiftz--)));
          centermask >>= 1;
          mask >>= 1;
          levels++;
          if(levels > OR_MAX_TREE_LEVEL)
            {
              /* coincident points: shift to the next free slot */
              for(int j = 0; j < 8; j++)
                {
                  if(t->suns[8 * NODE(t, th) + subnode] < 0)
                    break;
                  subnode++;
                  if(subnode >= 8)
                    subnode = 7;
                }
            }
          int64_t nn = t->suns[8 * NODE(t, th) + subnode];
          if(nn >= 0)
            {
              parent = th;
              th     = nn;
            }
          else
            {
              t->suns[8 * NODE(t, th) + subnode] = (int32_t)i;
              break;
            }
        }
      else
        {
          /* leaf occupied by a single particle: create a node */
          int64_t nf                             = t->max_part + t->num_nodes;
          t->suns[8 * NODE(t, parent) + subnode] = (int32_t)nf;
          double len = ((double)(mask << 1)) * t->dom->big_fac;
          double cx  = ((double)((xxb & (uint64_t)centermask) | mask)) * t->dom->big_fac + t->dom->corner[0];
          double cy  = ((double)((yyb & (uint64_t)centermask) | mask)) * t->dom->big_fac + t->dom->corner[1];
          double cz  = ((double)((zzb & (uint64_t)centermask) | mask)) * t->dom->big_fac + t->dom->corner[2];
          t->len[NODE(t, nf)]            = len;
          t->center[3 * NODE(t, nf) + 0] = cx;
          t->center[3 * NODE(t, nf) + 1] = cy;
          t->center[3 * NODE(t, nf) + 2] = cz;
          for(int j = 0; j < 8; j++)
            t->suns[8 * NODE(t, nf) + j] = -1;
          const uint64_t *q = &t->ip[3 * th];
          subnode = (unsigned)(((q[0] & mask) >> shiftx) | ((q[1] & mask) >> shifty) | ((q[2] & mask) >> shiftz));
          t->suns[8 * NODE(t, nf) + subnode] = (int32_t)th;
          th = nf;
          t->num_nodes++;
          if(t->num_nodes >= t->max_nodes)
            return -1;
        }
    }
  return 0;
}

/* force_update_node_recursive, src/gravity/forcetree.c:1217-1429 (single rank) */
static void update_node(or_tree *t, int64_t no, int64_t sib, int64_t father, int64_t *last)
{
  if(no >= t->max_part) /* internal node */
    {
      int32_t suns[8];
      for(int j = 0; j < 8; j++)
        suns[j] = t->suns[8 * NODE(t, no) + j];
      if(*last >= 0)
        {
          if(*last >= t->max_part)
            t->nextnode[NODE(t, *last)] = (int32_t)no;
          else
            t->p_next[*last] = (int32_t)no;
        }
      *last = no;

      double mass = 0, s[3] = {0, 0, 0};
      int maxsofttype = t->prm->nsoft; /* NSOFTTYPES + NSOFTTYPES_HYDRO: the entry with zero softening */
      for(int j = 0; j < 8; j++)
        {
          int64_t p = suns[j];
          if(p < 0)
            continue;
          int jj;
          int64_t pp = -1;
          for(jj = j + 1; jj < 8; jj++)
            if((pp = suns[jj]) >= 0)
              break;
          int64_t nextsib = (jj < 8) ? pp : sib;
          update_node(t, p, nextsib, no, last);
          if(p < t->max_part)
            {
              const double *pos = &t->pos[3 * p];
              mass += t->mass[p];
              s[0] += t->mass[p] * pos[0];
              s[1] += t->mass[p] * pos[1];
              s[2] += t->mass[p] * pos[2];
              if(t->prm->soft[maxsofttype] < t->prm->soft[t->stype[p]])
                maxsofttype = t->stype[p];
            }
          else
            {
              int64_t k = NODE(t, p);
              mass += t->nmass[k];
              s[0] += t->nmass[k] * t->s[3 * k + 0];
              s[1] += t->nmass[k] * t->s[3 * k + 1];
              s[2] += t->nmass[k] * t->s[3 * k + 2];
              if(t->prm->soft[maxsofttype] < t->prm->soft[t->maxsoft[k]])
                maxsofttype = t->maxsoft[k];
            }
        }
      int64_t k = NODE(t, no);
      if(mass)
        {
          s[0] /= mass;
          s[1] /= mass;
          s[2] /= mass;
        }
      else
        {
          s[0] = t->center[3 * k + 0];
          s[1] = t->center[3 * k + 1];
          s[2] = t->center[3 * k + 2];
        }
      t->nmass[k]      = mass;
      t->s[3 * k + 0]  = s[0];
      t->s[3 * k + 1]  = s[1];
      t->s[3 * k + 2]  = s[2];
      t->maxsoft[k]    = (uint8_t)maxsofttype;
      t->sibling[k]    = (int32_t)sib;
      t->father[k]     = (int32_t)father;
    }
  else
    {
      if(*last >= 0)
        {
          if(*last >= t->max_part)
            t->nextnode[NODE(t, *last)] = (int32_t)no;
          else
            t->p_next[*last] = (int32_t)no;
        }
      *last            = no;
      t->p_father[no] = (int32_t)father;
    }
}

/* ExtNodes[].mass_per_type of MULTIPLE_NODE_SOFTENING (force_update_node_recursive,
 * src/gravity/forcetree.c:1222-1308): per node and softening type, the masses of the particles in
 * slots 0..7 and the sums of the child nodes, in slot order.  Child nodes are created after their
 * parents (higher index), so one pass from the last node to the root sees every child first.
 * Returns 0, or -1 if that order does not hold. */
int or_mass_per_type(int64_t num_nodes, const int32_t *suns, int64_t max_part, const double *mass, const uint8_t *stype,
                     int nsoft, double *mpt)
{
  memset(mpt, 0, sizeof(double) * num_nodes * nsoft);
  for(int64_t k = num_nodes - 1; k >= 0; k--)
    for(int j = 0; j < 8; j++)
      {
        int64_t p = suns[8 * k + j];
        if(p < 0)
          continue;
        if(p < max_part)
          mpt[k * nsoft + stype[p]] += mass[p];
        else
          {
            int64_t q = p - max_part;
            if(q <= k)
              return -1;
            for(int t = 0; t < nsoft; t++)
              mpt[k * nsoft + t] += mpt[q * nsoft + t];
          }
      }
  return 0;
}

/*
 * Build the tree over particles given in insertion order.
 * max_part: index of the root (the reference uses All.MaxPart); max_nodes: capacity.
 * Output arrays are sized by the caller: node arrays max_nodes long.
 * Returns the number of nodes, or -1 (too many nodes), -2 (top nodes do not fit).
 */
int64_t or_build(int64_t n, const double *pos, const double *mass, const uint8_t *stype, const uint64_t *intpos, const or_params *p,
                 const or_domain *d, const or_topnode *top, int ntop, int64_t max_part, int64_t max_nodes, int32_t *suns_scratch,
                 double *center, double *len, double *s, double *nmass, int32_t *sibling, int32_t *nextnode, int32_t *father,
                 uint8_t *maxsoft, int32_t *p_next, int32_t *p_father, int64_t *first_non_top)
{
  or_tree t;
  memset(&t, 0, sizeof(t));
  t.n         = n;
  t.pos       = pos;
  t.mass      = mass;
  t.stype     = stype;
  t.ip        = (uint64_t *)intpos;
  t.max_part  = max_part;
  t.max_nodes = max_nodes;
  t.suns      = suns_scratch;
  t.center    = center;
  t.len       = len;
  t.s         = s;
  t.nmass     = nmass;
  t.sibling   = sibling;
  t.nextnode  = nextnode;
  t.father    = father;
  t.maxsoft   = maxsoft;
  t.p_next    = p_next;
  t.p_father  = p_father;
  t.prm       = p;
  t.dom       = d;
  t.top       = top;
  t.ntop      = ntop;
  int nleaves = 0;
  for(int i = 0; i < ntop; i++)
    if(top[i].daughter < 0)
      nleaves++;
  t.domain_node_index = malloc(sizeof(int32_t) * (nleaves > 0 ? nleaves : 1));

  /* root node, src/gravity/forcetree.c:338-350 */
  for(int j = 0; j < 8; j++)
    t.suns[j] = -1;
  t.len[0] = d->len;
  for(int j = 0; j < 3; j++)
    t.center[j] = d->center[j];
  t.num_nodes = 1;
  if(create_empty_nodes(&t, max_part, 0, 1, 0, 0, 0) < 0)
    {
      free(t.domain_node_index);
      return -2;
    }
  *first_non_top = max_part + t.num_nodes;
  if(ntop == 1)
    t.domain_node_index[0] = (int32_t)max_part;

  for(int64_t i = 0; i < n; i++)
    {
      /* walk down the top tree, src/gravity/forcetree.c:493-522 */
      uint64_t xxb = intpos[3 * i], yyb = intpos[3 * i + 1], zzb = intpos[3 * i + 2];
      uint64_t mask = 1ull << (52 - 1);
      int shiftx = 52 - 1, shifty = 52 - 2, shiftz = 52 - 3, levels = 0;
      int no = 0;
      while(top[no].daughter >= 0)
        {
          unsigned sub = (unsigned)(((xxb & mask) >> (shiftx--)) | ((yyb & mask) >> (shifty--)) | ((zzb & mask) >> (shiftz--)));
          mask >>= 1;
          levels++;
          no = top[no].daughter + top[no].morton_to_peano[sub];
        }
      int64_t th = t.domain_node_index[top[no].leaf];
      if(insert_point(&t, i, th, levels) < 0)
        {
          free(t.domain_node_index);
          return -1;
        }
    }

  int64_t last = -1;
  update_node(&t, max_part, -1, -1, &last);
  if(last >= max_part)
    t.nextnode[NODE(&t, last)] = -1;
  else
    t.p_next[last] = -1;
  free(t.domain_node_index);
  return t.num_nodes;
}

/* ------------------------------------------------------------------------ */
/* Short-range table: force_short_range_init, src/gravity/forcetree_walk.c:72-85 */
/* ------------------------------------------------------------------------ */
void or_shortrange_table(double rcut_cells, float *tab_force, float *tab_pot)
{
  for(int i = 0; i <= OR_NTAB; i++)
    {
      double u     = ((rcut_cells / 2.0) / OR_NTAB) * i;
      tab_pot[i]   = -erfc(u);
      tab_force[i] = (u > 0) ? (float)((erfc(u) + 2.0 * u / sqrt(M_PI) * exp(-u * u) - 1.0) / (u * u)) : 0.0f;
    }
}

/* ------------------------------------------------------------------------ */
/* Tree walk: force_treeevaluate mode 0, src/gravity/forcetree_walk.c:115-514 */
/* Particles and nodes as produced by or_build, targets are sorted indices.  */
/* ------------------------------------------------------------------------ */
static inline double nearest(double x, const or_params *p)
{
  if(!p->periodic)
    return x;
  double half = 0.5 * p->box;
  return (x > half) ? (x - p->box) : ((x < -half) ? (x + p->box) : x);
}

/* ------------------------------------------------------------------------ */
/* Ewald correction of the periodic pure-tree walk (no PMGRID):             */
/* src/gravity/forcetree_ewald.c                                            */
/* ------------------------------------------------------------------------ */
#define OR_EN 64

/* ewald_psi, forcetree_ewald.c:393-461 (cubic box, STRETCH = 1) */
static double or_ewald_psi(double x, double y, double z)
{
  double r = sqrt(x * x + y * y + z * z);
  if(r == 0)
    return 0;
  double alpha   = 3.0;
  const int nmax = 4;
  double sum1    = 0;
  for(int nx = -nmax; nx <= nmax; nx++)
    for(int ny = -nmax; ny <= nmax; ny++)
      for(int nz = -nmax; nz <= nmax; nz++)
        {
          double dx = x - nx, dy = y - ny, dz = z - nz;
          double rr = sqrt(dx * dx + dy * dy + dz * dz);
          sum1 += erfc(alpha * rr) / rr;
        }
  double alpha2 = alpha * alpha;
  int kmax      = (int)(2 * alpha + 0.5);
  double sum2   = 0.0;
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

/* ewald_force, forcetree_ewald.c:463-527 */
static void or_ewald_force(double x, double y, double z, double force[3])
{
  for(int i = 0; i < 3; i++)
    force[i] = 0;
  double r2 = x * x + y * y + z * z;
  if(r2 == 0)
    return;
  double alpha  = 2.0;
  double alpha2 = alpha * alpha;
  double r3inv  = 1.0 / (r2 * sqrt(r2));
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
  int hmax = (int)(2 * alpha + 0.5);
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

/* The unscaled tables of ewald_init (forcetree_ewald.c:154-185): one octant of the unit box, entry
 * (i, j, k) at (i, j, k) / (2 EN); (EN + 1)^3 values each, k fastest. */
void or_ewald_table(double *fx, double *fy, double *fz, double *pot)
{
  const int m = OR_EN + 1;
#pragma omp parallel for schedule(dynamic, 64)
  for(int n = 0; n < m * m * m; n++)
    {
      int i = n / (m * m), j = (n - i * m * m) / m, k = n - i * m * m - j * m;
      double xx = 0.5 * ((double)i) / OR_EN, yy = 0.5 * ((double)j) / OR_EN, zz = 0.5 * ((double)k) / OR_EN;
      double f[3];
      pot[n] = or_ewald_psi(xx, yy, zz);
      or_ewald_force(xx, yy, zz, f);
      fx[n] = f[0];
      fy[n] = f[1];
      fz[n] = f[2];
    }
}

static const double *or_ewd_fx, *or_ewd_fy, *or_ewd_fz, *or_ewd_pot; /* scaled to the box */
static double or_ewd_fac_intp;

/* the tables scaled to the box as at the end of ewald_init (forcetree_ewald.c:239-251); the caller
 * keeps the arrays alive */
void or_set_ewald_table(double box, const double *fx, const double *fy, const double *fz, const double *pot)
{
  or_ewd_fx = fx, or_ewd_fy = fy, or_ewd_fz = fz, or_ewd_pot = pot;
  or_ewd_fac_intp = 2 * OR_EN / box;
}

#define OR_EI(i, j, k) (((i) * (OR_EN + 1) + (j)) * (OR_EN + 1) + (k))

/* ewald_corr and ewald_pot_corr, forcetree_ewald.c:268-391 */
static void or_ewald_corr(double dx, double dy, double dz, double *fper, double *pcorr)
{
  int signx, signy, signz;
  if(dx < 0)
    {
      dx    = -dx;
      signx = +1;
    }
  else
    signx = -1;
  if(dy < 0)
    {
      dy    = -dy;
      signy = +1;
    }
  else
    signy = -1;
  if(dz < 0)
    {
      dz    = -dz;
      signz = +1;
    }
  else
    signz = -1;
  double u = dx * or_ewd_fac_intp;
  int i    = (int)u;
  if(i >= OR_EN)
    i = OR_EN - 1;
  u -= i;
  double v = dy * or_ewd_fac_intp;
  int j    = (int)v;
  if(j >= OR_EN)
    j = OR_EN - 1;
  v -= j;
  double w = dz * or_ewd_fac_intp;
  int k    = (int)w;
  if(k >= OR_EN)
    k = OR_EN - 1;
  w -= k;
  double f1 = (1 - u) * (1 - v) * (1 - w), f2 = (1 - u) * (1 - v) * (w), f3 = (1 - u) * (v) * (1 - w), f4 = (1 - u) * (v) * (w);
  double f5 = (u) * (1 - v) * (1 - w), f6 = (u) * (1 - v) * (w), f7 = (u) * (v) * (1 - w), f8 = (u) * (v) * (w);
  const double *t[4] = {or_ewd_fx, or_ewd_fy, or_ewd_fz, or_ewd_pot};
  double r[4];
  for(int c = 0; c < 4; c++)
    r[c] = t[c][OR_EI(i, j, k)] * f1 + t[c][OR_EI(i, j, k + 1)] * f2 + t[c][OR_EI(i, j + 1, k)] * f3 +
           t[c][OR_EI(i, j + 1, k + 1)] * f4 + t[c][OR_EI(i + 1, j, k)] * f5 + t[c][OR_EI(i + 1, j, k + 1)] * f6 +
           t[c][OR_EI(i + 1, j + 1, k)] * f7 + t[c][OR_EI(i + 1, j + 1, k + 1)] * f8;
  fper[0] = signx * r[0];
  fper[1] = signy * r[1];
  fper[2] = signz * r[2];
  *pcorr  = r[3];
}

void or_walk(int64_t ntargets, const int64_t *targets, const double *tpos, const float *oldacc, const uint8_t *tstype,
             const double *pos, const double *mass, const uint8_t *stype, const int32_t *p_next, int64_t max_part,
             int64_t num_nodes, const double *center, const double *len, const double *s, const double *nmass,
             const int32_t *sibling, const int32_t *nextnode, const uint8_t *maxsoft, const or_params *p, double *acc_out,
             double *pot_out, int32_t *ninter_out, const double *mpt)
{
  const int mns = (p->flags & 1) && mpt; /* MULTIPLE_NODE_SOFTENING */
  float tab_f[OR_NTAB + 1], tab_p[OR_NTAB + 1];
  const int pm    = p->periodic && p->asmth > 0;  /* TreePM split */
  const int ewald = p->periodic && !pm;           /* pure tree, Ewald-corrected */
  if(pm)
    or_shortrange_table(p->rcut_cells, tab_f, tab_p);
  const double rcut      = p->rcut;
  const double rcut2     = rcut * rcut;
  const double asmthinv  = pm ? 0.5 / p->asmth : 0.0;
  const double asmthinv2 = asmthinv * asmthinv;
  const double asmthfac  = asmthinv * (OR_NTAB / (p->rcut_cells / 2.0));

  for(int64_t q = 0; q < ntargets; q++)
    {
      int64_t tgt  = targets ? targets[q] : q;
      double pos_x = tpos[3 * tgt + 0], pos_y = tpos[3 * tgt + 1], pos_z = tpos[3 * tgt + 2];
      double aold  = p->erracc * oldacc[tgt];
      double h_i   = p->soft[tstype[tgt]];
      double acc_x = 0, acc_y = 0, acc_z = 0, pot = 0;
      int ninteractions = 0;
      int64_t no        = max_part;

      while(no >= 0)
        {
          double dx, dy, dz, r2, m, hmax;
          int64_t split = -1; /* node whose per-type masses are used (MULTIPLE_NODE_SOFTENING) */
          if(no < max_part)
            {
              dx = nearest(pos[3 * no + 0] - pos_x, p);
              dy = nearest(pos[3 * no + 1] - pos_y, p);
              dz = nearest(pos[3 * no + 2] - pos_z, p);
              r2 = dx * dx + dy * dy + dz * dz;
              m  = mass[no];
              double h_j = p->soft[stype[no]];
              hmax       = (h_j > h_i) ? h_j : h_i;
              no         = p_next[no];
            }
          else
            {
              int64_t k = no - max_part;
              m         = nmass[k];
              dx        = nearest(s[3 * k + 0] - pos_x, p);
              dy        = nearest(s[3 * k + 1] - pos_y, p);
              dz        = nearest(s[3 * k + 2] - pos_z, p);
              r2        = dx * dx + dy * dy + dz * dz;
              if(pm && r2 > rcut2)
                {
                  double eff_dist = rcut + 0.5 * len[k];
                  double dist     = nearest(center[3 * k + 0] - pos_x, p);
                  if(dist < -eff_dist || dist > eff_dist)
                    {
                      no = sibling[k];
                      continue;
                    }
                  dist = nearest(center[3 * k + 1] - pos_y, p);
                  if(dist < -eff_dist || dist > eff_dist)
                    {
                      no = sibling[k];
                      continue;
                    }
                  dist = nearest(center[3 * k + 2] - pos_z, p);
                  if(dist < -eff_dist || dist > eff_dist)
                    {
                      no = sibling[k];
                      continue;
                    }
                }
              if(p->theta)
                {
                  if(len[k] * len[k] > r2 * p->theta * p->theta)
                    {
                      no = nextnode[k];
                      continue;
                    }
                }
              else
                {
                  double len2 = len[k] * len[k];
                  if(len2 > r2 * (1.2 * 1.2))
                    {
                      no = nextnode[k];
                      continue;
                    }
                  /* ACTIVATE_MINIMUM_OPENING_ANGLE adds a minimum angle to the mass test (forcetree_walk.c:266-271) */
                  if(m * len2 > r2 * r2 * aold && (!(p->flags & 2) || len2 > r2 * (0.4 * 0.4)))
                    {
                      no = nextnode[k];
                      continue;
                    }
                  if(fabs(nearest(center[3 * k + 0] - pos_x, p)) < 0.60 * len[k])
                    if(fabs(nearest(center[3 * k + 1] - pos_y, p)) < 0.60 * len[k])
                      if(fabs(nearest(center[3 * k + 2] - pos_z, p)) < 0.60 * len[k])
                        {
                          no = nextnode[k];
                          continue;
                        }
                }
              double h_j = p->soft[maxsoft[k]];
              if(h_j > h_i)
                {
                  if(mns)
                    split = k; /* used per softening type instead of opened (forcetree_walk.c:296-308) */
                  else if(r2 < h_j * h_j)
                    {
                      no = nextnode[k];
                      continue;
                    }
                  hmax = h_j;
                }
              else
                hmax = h_i;
              no = sibling[k];
            }

          if(m)
            {
              double r = sqrt(r2);
              double factor_force = 0, factor_pot = 0;
              if(pm)
                {
                  double tabentry = asmthfac * r;
                  int tabindex    = (int)tabentry;
                  if(!(tabindex < OR_NTAB))
                    continue;
                  double tabweight = tabentry - tabindex;
                  factor_force     = (1.0 - tabweight) * tab_f[tabindex] + tabweight * tab_f[tabindex + 1];
                  factor_pot       = (1.0 - tabweight) * tab_p[tabindex] + tabweight * tab_p[tabindex + 1];
                }
              const int t0 = split >= 0 ? 0 : -1, t1 = split >= 0 ? p->nsoft : 0;
              for(int type = t0; type < t1; type++)
                {
              double mm = m;
              if(type >= 0)
                {
                  mm         = mpt[split * p->nsoft + type];
                  double hjt = p->soft[type];
                  hmax       = (hjt > h_i) ? hjt : h_i;
                }
              if(!mm)
                continue;
              double fac, wp;
              if(r >= hmax)
                {
                  double rinv  = 1.0 / r;
                  double rinv3 = rinv * rinv * rinv;
                  if(pm)
                    {
                      fac = rinv3 + rinv * factor_force * asmthinv2;
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
                  if(pm && r > 0)
                    {
                      double rinv = 1.0 / r;
                      fac += rinv * factor_force * asmthinv2;
                      wp += rinv * (factor_pot + 1.0);
                    }
                }
              pot += mm * wp;
              fac *= mm;
              acc_x += dx * fac;
              acc_y += dy * fac;
              acc_z += dz * fac;
              if(ewald)
                {
                  double fcorr[3], pcorr;
                  or_ewald_corr(dx, dy, dz, fcorr, &pcorr);
                  acc_x += mm * fcorr[0];
                  acc_y += mm * fcorr[1];
                  acc_z += mm * fcorr[2];
                  pot += mm * pcorr;
                }
                }
              ninteractions++;
            }
        }
      acc_out[3 * q + 0] = acc_x;
      acc_out[3 * q + 1] = acc_y;
      acc_out[3 * q + 2] = acc_z;
      if(pot_out)
        pot_out[q] = pot;
      if(ninter_out)
        ninter_out[q] = ninteractions;
    }
}

/* ------------------------------------------------------------------------ */
/* Direct FP64 summation with the exact short-range factor (TreePM) or plain */
/* Newtonian gravity (isolated): gravity_forcetest_evaluate,                */
/* src/gravity/gravtree_forcetest.c:483-601 (Ewald images omitted).          */
/* ------------------------------------------------------------------------ */
void or_direct(int64_t ntargets, const int64_t *targets, int64_t n, const double *pos, const double *mass, const uint8_t *stype,
               const or_params *p, double *acc_out, double *pot_out)
{
  for(int64_t q = 0; q < ntargets; q++)
    {
      int64_t i  = targets[q];
      double h_i = p->soft[stype[i]];
      double ax = 0, ay = 0, az = 0, pt = 0;
      for(int64_t j = 0; j < n; j++)
        {
          double dx = nearest(pos[3 * j + 0] - pos[3 * i + 0], p);
          double dy = nearest(pos[3 * j + 1] - pos[3 * i + 1], p);
          double dz = nearest(pos[3 * j + 2] - pos[3 * i + 2], p);
          double r2 = dx * dx + dy * dy + dz * dz;
          double r  = sqrt(r2);
          double m  = mass[j];
          double h_j  = p->soft[stype[j]];
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
              double h_inv  = 1.0 / hmax;
              double h3_inv = h_inv * h_inv * h_inv;
              double u      = r * h_inv;
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
          if(p->periodic && p->asmth > 0)
            {
              double u            = 0.5 / p->asmth * r;
              double factor_force = (erfc(u) + 2.0 * u / sqrt(M_PI) * exp(-u * u) - 1.0);
              double factor_pot   = erfc(u);
              fac += fac_newton * factor_force;
              wp += wp_newton * (factor_pot - 1.0);
            }
          ax += dx * fac;
          ay += dy * fac;
          az += dz * fac;
          pt += wp;
          if(p->periodic && !(p->asmth > 0))
            {
              /* pure periodic tree: all images through the Ewald correction (forcetest with Ewald) */
              double fcorr[3], pcorr;
              or_ewald_corr(dx, dy, dz, fcorr, &pcorr);
              ax += m * fcorr[0];
              ay += m * fcorr[1];
              az += m * fcorr[2];
              pt += m * pcorr;
            }
        }
      acc_out[3 * q + 0] = ax;
      acc_out[3 * q + 1] = ay;
      acc_out[3 * q + 2] = az;
      if(pot_out)
        pot_out[q] = pt;
    }
}

/* ------------------------------------------------------------------------ */
/* gravity_direct (src/gravity/gravdirect.c:61-257) with the pair arithmetic */
/* of force_evaluate_direct (src/gravity/forcetree_walk.c:557-708): the n    */
/* given (active) particles are both targets and sources, summed in order;  */
/* tabulated short-range factor (TreePM), Ewald correction (periodic tree),  */
/* spline softening.  One particle: zero force (gravdirect.c:65-81).         */
/* ------------------------------------------------------------------------ */
void or_gravity_direct(int64_t n, const double *pos, const double *mass, const uint8_t *stype, const or_params *p,
                       double *acc_out, double *pot_out)
{
  float tab_f[OR_NTAB + 1], tab_p[OR_NTAB + 1];
  const int pm    = p->periodic && p->asmth > 0;
  const int ewald = p->periodic && !pm;
  if(pm)
    or_shortrange_table(p->rcut_cells, tab_f, tab_p);
  const double asmthinv  = pm ? 0.5 / p->asmth : 0.0;
  const double asmthinv2 = asmthinv * asmthinv;
  const double asmthfac  = asmthinv * (OR_NTAB / (p->rcut_cells / 2.0));
  for(int64_t i = 0; i < n; i++)
    {
      double acc_x = 0, acc_y = 0, acc_z = 0, pot = 0;
      if(n > 1)
        {
          const double pos_x = pos[3 * i + 0], pos_y = pos[3 * i + 1], pos_z = pos[3 * i + 2];
          const double h_i   = p->soft[stype[i]];
          for(int64_t j = 0; j < n; j++)
            {
              double h_j  = p->soft[stype[j]];
              double hmax = (h_j > h_i) ? h_j : h_i;
              double dx   = nearest(pos[3 * j + 0] - pos_x, p);
              double dy   = nearest(pos[3 * j + 1] - pos_y, p);
              double dz   = nearest(pos[3 * j + 2] - pos_z, p);
              double r2   = dx * dx + dy * dy + dz * dz;
              double m    = mass[j];
              double r    = sqrt(r2);
              double factor_force = 0, factor_pot = 0;
              if(pm)
                {
                  double tabentry = asmthfac * r;
                  int tabindex    = (int)tabentry;
                  if(tabindex >= OR_NTAB)
                    continue;
                  double tabweight = tabentry - tabindex;
                  factor_force     = (1.0 - tabweight) * tab_f[tabindex] + tabweight * tab_f[tabindex + 1];
                  factor_pot       = (1.0 - tabweight) * tab_p[tabindex] + tabweight * tab_p[tabindex + 1];
                }
              double fac, wp;
              if(r >= hmax)
                {
                  double rinv  = 1.0 / r;
                  double rinv3 = rinv * rinv * rinv;
                  if(pm)
                    {
                      fac = rinv3 + rinv * factor_force * asmthinv2;
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
                  if(pm && r > 0)
                    {
                      double rinv = 1.0 / r;
                      fac += rinv * factor_force * asmthinv2;
                      wp += rinv * (factor_pot + 1.0);
                    }
                }
              pot += m * wp;
              fac *= m;
              acc_x += dx * fac;
              acc_y += dy * fac;
              acc_z += dz * fac;
              if(ewald)
                {
                  double fcorr[3], pcorr;
                  or_ewald_corr(dx, dy, dz, fcorr, &pcorr);
                  acc_x += m * fcorr[0];
                  acc_y += m * fcorr[1];
                  acc_z += m * fcorr[2];
                  pot += m * pcorr;
                }
            }
        }
      acc_out[3 * i + 0] = acc_x;
      acc_out[3 * i + 1] = acc_y;
      acc_out[3 * i + 2] = acc_z;
      if(pot_out)
        pot_out[i] = pot;
    }
}

/* ------------------------------------------------------------------------ */
/* get_timestep_gravity (src/time_integration/timestep.c:284-353) and the    */
/* bin of timebins_get_bin_and_do_validity_checks (timestep.c:725-770).      */
/* Returns 0, or the reference's stop: 1 below MinSizeTimestep, 2 integer    */
/* step outside (0, TIMEBASE), 3 integer step 1, 4 beyond the end of the     */
/* timeline.                                                                 */
/* ------------------------------------------------------------------------ */
typedef struct
{
  double eta, cf_atime, cf_a2inv, cf_hubble_a, dtmax, dtmin, dtdisp, timebase_interval;
  int64_t timebase, ti_current;
  int nostop;
  int pad;
  unsigned char sync[64];
} or_tsparams;

int or_timestep_gravity(int64_t n, const double *acc, const double *pm, const double *mass, const uint64_t *ids,
                        const uint8_t *stype, const or_params *p, const or_tsparams *t, const int8_t *bin_old, int64_t *ti_out,
                        int8_t *bin_out)
{
  int err = 0;
  for(int64_t i = 0; i < n; i++)
    {
      double ax = t->cf_a2inv * acc[3 * i + 0], ay = t->cf_a2inv * acc[3 * i + 1], az = t->cf_a2inv * acc[3 * i + 2];
      if(pm)
        {
          ax += t->cf_a2inv * pm[3 * i + 0];
          ay += t->cf_a2inv * pm[3 * i + 1];
          az += t->cf_a2inv * pm[3 * i + 2];
        }
      double ac = sqrt(ax * ax + ay * ay + az * az);
      if(ac == 0)
        ac = 1.0e-30;
      double dt = sqrt(2 * t->eta * t->cf_atime * p->soft[stype[i]] / 2.8 / ac);
      dt *= t->cf_hubble_a;
      if(mass[i] == 0 && ids && ids[i] == 0)
        dt = t->dtmax;
      if(dt >= t->dtmax)
        dt = t->dtmax;
      if(dt < t->dtmin)
        {
          if(t->nostop)
            dt = t->dtmin;
          else if(!err)
            err = 1;
        }
      if(t->dtdisp > 0 && dt >= t->dtdisp)
        dt = t->dtdisp;
      int64_t ti = t->timebase <= ((int64_t)1 << 30) ? (int64_t)(int)(dt / t->timebase_interval) : (int64_t)(dt / t->timebase_interval);
      if(!(ti > 0 && ti < t->timebase) && !err)
        err = 2;
      ti_out[i]      = ti;
      int64_t ti_min = t->timebase;
      while(ti_min > ti)
        ti_min >>= 1;
      int64_t ts = ti_min;
      int bin    = -1;
      if(ts == 0)
        bin = 0;
      if(ts == 1 && !err)
        err = 3;
      while(ts)
        {
          bin++;
          ts >>= 1;
        }
      if(bin > bin_old[i])
        {
          while(bin > bin_old[i] && !t->sync[bin])
            bin--;
          ts = bin ? ((int64_t)1 << bin) : 0;
        }
      if(t->ti_current >= t->timebase)
        {
          ts  = 0;
          bin = 0;
        }
      if(t->timebase - t->ti_current < ts && !err)
        err = 4;
      bin_out[i] = (int8_t)bin;
    }
  return err;
}
