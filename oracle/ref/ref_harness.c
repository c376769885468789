/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Drives the reference's own, unmodified gravity sources (compiled from the
 * reference tree by oracle/ref/Makefile against single-rank stub headers) for
 * one short-range force computation and dumps every intermediate that the
 * B200 library must reproduce:
 *
 *   domain_Decomposition()            domain/domain.c:78-185
 *     -> Peano-Hilbert keys + sort      domain/domain_toplevel.c:120-135, domain/peano.c:74-133
 *     -> top-level tree                 domain/domain_toplevel.c:111-269
 *   construct_forcetree(0, 1, 0, bin) gravity/forcetree.c:110-149     (as gravity/accel.c:127-132)
 *   force_treeevaluate() per target   gravity/forcetree_walk.c:115-514 (per-target acc, pot, interactions)
 *   gravity_tree(bin)                 gravity/gravtree.c:357-707       (cross-check of GravAccel)
 *   gravity_force_finalize(bin)       gravity/accel.c:204-347          (OldAcc for the relative pass)
 *
 * and then repeats build + walk with the relative opening criterion, exactly
 * as compute_grav_accelerations() does on the first step (gravity/accel.c:58-80).
 *
 * Usage: ref_harness <in.bin> <out.bin> [key=value ...]
 *   in.bin  : int64 N, then N*3 double positions, N double masses, N uint8 softening types
 *   keys    : box, asmth, rcut (periodic build only), theta, erracc, eps0, eps1 (Plummer
 *             softening per type), mdom (MultipleDomains), tnf (TopNodeFactor),
 *             passes (1 = BH only, 2 = BH then relative), dump (1 = write tree),
 *             stride (walk every stride-th particle in the timed loop), first, count
 *             (walk a contiguous slice of sorted targets; used for CPU timing),
 *             gt (1 = also run gravity_tree), tag (string printed with timings),
 *             procs (walk the selected targets with that many forked processes, which share
 *             the particles and the tree copy-on-write; targets dealt round-robin),
 *             reps (after the last pass, walk the selected targets that many more times and
 *             print each walk's wall time: the CPU timing of a bounded sample),
 *             lite (1 = write only the timing sections, not the per-particle arrays),
 *             active (k > 1: only every k-th particle, in P[] order, is in the active gravity time
 *             bin, so gravity_tree walks that TargetList), displace (f != 0: before the first
 *             pass, particle 0 is moved to DomainCorner + (1 + f) DomainLen in x, outside the domain
 *             box: the tree build's -3 recovery), gpu (harness builds with GPU_GRAVITY only: 1 or 2
 *             replaces construct_forcetree + gravity_tree by the library's FP64 or FP32 walk through
 *             gpu_gravity.c, the binding AREPO would use), direct (1 = gravity_direct, the
 *             direct summation gravity() runs below DIRECT_SUMMATION_THRESHOLD active particles,
 *             instead of the tree; builds with ALLOW_DIRECT_SUMMATION), tstep (1 = after the passes,
 *             get_timestep_gravity and the new gravity time bin of every particle, with eta
 *             (ErrTolIntAccuracy), dtmax, dtmin, dtdisp (DtDisplacement) and TimeMax = 1), pm (builds
 *             with the reference's periodic PM, ref_harness_pmfft: 1 = after the passes,
 *             pm_init_periodic + pmforce_periodic(0, NULL), dumping GravPM and PM_Potential)
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/time.h>
#include <sys/wait.h>
#include <unistd.h>

#include "allvars.h"
#include "proto.h"
#include "../domain/domain.h"

#ifdef GPU_GRAVITY
#include "gpugrav.h"
int gpu_gravity_tree(int timebin, int precision);
void gpu_gravity_free(void);
#endif

/* only every k-th particle active in the gravity time bin: gravity_tree's TargetList
 * (gravity/gravtree.c:494-520) is built from this list */
static void set_active_every(int k)
{
  int m = 0;
  for(int i = 0; i < NumPart; i += k)
    TimeBinsGravity.ActiveParticleList[m++] = i;
  TimeBinsGravity.NActiveParticles       = m;
  TimeBinsGravity.GlobalNActiveParticles = m;
}

static double wall(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static double arg_d(int argc, char **argv, const char *key, double def)
{
  size_t l = strlen(key);
  for(int i = 3; i < argc; i++)
    if(strncmp(argv[i], key, l) == 0 && argv[i][l] == '=')
      return atof(argv[i] + l + 1);
  return def;
}

static const char *arg_s(int argc, char **argv, const char *key, const char *def)
{
  size_t l = strlen(key);
  for(int i = 3; i < argc; i++)
    if(strncmp(argv[i], key, l) == 0 && argv[i][l] == '=')
      return argv[i] + l + 1;
  return def;
}

static void wr(FILE *f, const void *p, size_t sz, size_t n)
{
  if(n && fwrite(p, sz, n, f) != n)
    {
      fprintf(stderr, "ref_harness: short write\n");
      exit(2);
    }
}

static void wsec(FILE *f, const char *name, int64_t nbytes)
{
  char tag[16];
  memset(tag, 0, sizeof(tag));
  strncpy(tag, name, 15);
  wr(f, tag, 1, 16);
  wr(f, &nbytes, 8, 1);
}

static void split_key(peanokey k, uint64_t *hi, uint64_t *lo)
{
  unsigned __int128 u = (unsigned __int128)k;
  *lo                 = (uint64_t)u;
  *hi                 = (uint64_t)(u >> 64);
}

/* one sorted target with the reference's per-target routine */
static void walk_one(int i, double *acc, double *pot, int *ninter)
{
  gravdata_in in;
  gravdata_out out;
  for(int k = 0; k < 3; k++)
    in.Pos[k] = P[i].Pos[k];
  in.Type          = P[i].Type;
  in.SofteningType = P[i].SofteningType;
  in.OldAcc        = P[i].OldAcc;
  in.Firstnode     = 0;
  int n            = force_treeevaluate(&in, &out, i, 0, 0, 1, NULL, 0);
  for(int k = 0; k < 3; k++)
    acc[3 * i + k] = out.Acc[k];
  pot[i]    = out.Potential;
  ninter[i] = n;
}

/* walk the selected sorted targets; procs > 1: forked processes that share the particles and the
 * tree copy-on-write, each walking every procs-th selected target, results in shared memory */
static double walk_targets(int first, int count, int stride, int procs, double *acc, double *pot, int *ninter)
{
  double t0 = wall();
  if(procs <= 1)
    {
      for(int i = first; i < first + count; i += stride)
        walk_one(i, acc, pot, ninter);
      return wall() - t0;
    }
  size_t n     = (size_t)NumPart;
  size_t bytes = n * (3 * sizeof(double) + sizeof(double) + sizeof(int));
  char *sh     = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if(sh == MAP_FAILED)
    {
      fprintf(stderr, "ref_harness: mmap of the shared results failed\n");
      exit(3);
    }
  double *sacc = (double *)sh, *spot = sacc + 3 * n;
  int *snint   = (int *)(spot + n);
  fflush(stdout);
  fflush(stderr);
  pid_t *pids = malloc(sizeof(pid_t) * procs);
  for(int c = 0; c < procs; c++)
    {
      pids[c] = fork();
      if(pids[c] < 0)
        {
          fprintf(stderr, "ref_harness: fork failed\n");
          exit(3);
        }
      if(pids[c] == 0)
        {
          for(long i = first + (long)stride * c; i < first + count; i += (long)stride * procs)
            walk_one((int)i, sacc, spot, snint);
          _exit(0);
        }
    }
  int bad = 0;
  for(int c = 0; c < procs; c++)
    {
      int st = 0;
      if(waitpid(pids[c], &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0)
        bad = 1;
    }
  double t = wall() - t0;
  free(pids);
  if(bad)
    {
      fprintf(stderr, "ref_harness: a walk process failed\n");
      exit(3);
    }
  for(int i = first; i < first + count; i += stride)
    {
      for(int k = 0; k < 3; k++)
        acc[3 * i + k] = sacc[3 * i + k];
      pot[i]    = spot[i];
      ninter[i] = snint[i];
    }
  munmap(sh, bytes);
  return t;
}

static void dump_tree(FILE *f)
{
  int nn = Tree_NumNodes;
  wsec(f, "tree_meta", 6 * 8);
  int64_t meta[6] = {Tree_MaxPart, Tree_MaxNodes, nn, Tree_FirstNonTopLevelNode, NTopnodes, NTopleaves};
  wr(f, meta, 8, 6);
  /* nodes in index order [Tree_MaxPart, Tree_MaxPart + nn) */
  wsec(f, "node_f64", (int64_t)nn * 8 * 8);
  for(int no = Tree_MaxPart; no < Tree_MaxPart + nn; no++)
    {
      double v[8] = {Nodes[no].center[0], Nodes[no].center[1], Nodes[no].center[2], Nodes[no].len,
                     Nodes[no].u.d.s[0],  Nodes[no].u.d.s[1],  Nodes[no].u.d.s[2],  Nodes[no].u.d.mass};
      wr(f, v, 8, 8);
    }
  wsec(f, "node_i32", (int64_t)nn * 4 * 4);
  for(int no = Tree_MaxPart; no < Tree_MaxPart + nn; no++)
    {
      int32_t v[4] = {Nodes[no].u.d.sibling, Nodes[no].u.d.nextnode, Nodes[no].u.d.father, Nodes[no].u.d.maxsofttype};
      wr(f, v, 4, 4);
    }
#ifdef MULTIPLE_NODE_SOFTENING
  wsec(f, "node_mpt", (int64_t)nn * NSOFTTYPES * 8);
  for(int no = Tree_MaxPart; no < Tree_MaxPart + nn; no++)
    wr(f, ExtNodes[no].mass_per_type, 8, NSOFTTYPES);
#endif
  wsec(f, "nextnode", (int64_t)NumPart * 4);
  wr(f, Nextnode, 4, NumPart);
  wsec(f, "father", (int64_t)NumPart * 4);
  wr(f, Father, 4, NumPart);
}

static void free_tree(void)
{
  /* same release sequence as gravity() (gravity/accel.c:153-156) */
  myfree(Father);
  myfree(Nextnode);
  myfree(Tree_Points);
  force_treefree();
}

int main(int argc, char **argv)
{
  if(argc < 3)
    {
      fprintf(stderr, "usage: %s in.bin out.bin [key=value ...]\n", argv[0]);
      return 1;
    }

  ThisTask = 0;
  NTask    = 1;
  for(PTask = 0; NTask > (1 << PTask); PTask++)
    ;

  FILE *fi = fopen(argv[1], "rb");
  if(!fi)
    {
      fprintf(stderr, "cannot open %s\n", argv[1]);
      return 1;
    }
  int64_t n64;
  if(fread(&n64, 8, 1, fi) != 1)
    return 1;
  int n          = (int)n64;
  double *pos    = malloc(sizeof(double) * 3 * n);
  double *mass   = malloc(sizeof(double) * n);
  uint8_t *stype = malloc(n);
  if(fread(pos, 8, 3 * (size_t)n, fi) != 3 * (size_t)n || fread(mass, 8, n, fi) != (size_t)n || fread(stype, 1, n, fi) != (size_t)n)
    {
      fprintf(stderr, "short input\n");
      return 1;
    }
  fclose(fi);

  int passes = (int)arg_d(argc, argv, "passes", 2);
  int dump   = (int)arg_d(argc, argv, "dump", 1);
  int stride = (int)arg_d(argc, argv, "stride", 1);
  int first  = (int)arg_d(argc, argv, "first", 0);
  int count  = (int)arg_d(argc, argv, "count", n);
  int run_gt = (int)arg_d(argc, argv, "gt", 1);
  int procs  = (int)arg_d(argc, argv, "procs", 1);
  int reps   = (int)arg_d(argc, argv, "reps", 0);
  int lite   = (int)arg_d(argc, argv, "lite", 0);
  if(procs < 1)
    procs = 1;
  int active      = (int)arg_d(argc, argv, "active", 1);
  double displace = arg_d(argc, argv, "displace", 0.0);
  int use_gpu     = (int)arg_d(argc, argv, "gpu", 0);
  int use_direct  = (int)arg_d(argc, argv, "direct", 0);
  int use_tstep   = (int)arg_d(argc, argv, "tstep", 0);
  int use_pm      = (int)arg_d(argc, argv, "pm", 0);
#ifndef HARNESS_PM
  if(use_pm)
    {
      fprintf(stderr, "ref_harness: pm=1 needs the build with the periodic PM (ref_harness_pmfft)\n");
      return 1;
    }
#endif
#ifndef ALLOW_DIRECT_SUMMATION
  if(use_direct)
    {
      fprintf(stderr, "ref_harness: direct=1 needs a build with ALLOW_DIRECT_SUMMATION\n");
      return 1;
    }
#endif
#ifndef GPU_GRAVITY
  if(use_gpu)
    {
      fprintf(stderr, "ref_harness: gpu=%d needs a GPU_GRAVITY build (ref_harness_*_gpu)\n", use_gpu);
      return 1;
    }
#endif
  if(first < 0 || first > n)
    first = 0;
  if(count < 0 || first + count > n)
    count = n - first;
  if(stride < 1)
    stride = 1;

  /* ---- run parameters (what read_parameter_file + init would set) ---- */
  All.BoxSize                = arg_d(argc, argv, "box", 1.0);
  All.ErrTolTheta            = arg_d(argc, argv, "theta", 0.7);
  All.ErrTolForceAcc         = arg_d(argc, argv, "erracc", 0.0025);
  All.TypeOfOpeningCriterion = 1;
  All.ComovingIntegrationOn  = 0;
  All.G                      = 1.0;
  All.MultipleDomains        = (int)arg_d(argc, argv, "mdom", 8);
  All.TopNodeFactor          = arg_d(argc, argv, "tnf", 2.5);
  All.TopNodeAllocFactor     = 0.08;
  All.TreeAllocFactor        = 0.7;
  if(n < 1000)
    All.TreeAllocFactor = 10.0; /* init/init.c */
  All.SofteningComoving[0] = arg_d(argc, argv, "eps0", 0.01);
  All.SofteningComoving[1] = arg_d(argc, argv, "eps1", 0.01);
  All.SofteningMaxPhys[0]  = All.SofteningComoving[0];
  All.SofteningMaxPhys[1]  = All.SofteningComoving[1];
  All.MaxPart              = n;
  All.MaxPartSph           = 0;
  All.TotNumPart           = n;
  All.TotNumGas            = 0;
  All.Ti_Current           = 0;
  All.Time                 = 1.0;
  All.TimeBegin            = 0.0;
  All.TimeMax              = 1.0;
  All.ActivePartFracForNewDomainDecomp = 0.01;
  size_t need_mb = (size_t)(((double)n * 1400.0) / (1024.0 * 1024.0)) + 512;
  All.MaxMemSize = (int)need_mb;
  boxSize        = All.BoxSize;
  boxHalf        = 0.5 * All.BoxSize;

  /* the log files the reference writes to (io/logs.c:70-213) go to /dev/null */
  FdInfo = FdEnergy = FdTimings = FdDomain = FdBalance = FdMemory = FdTimebin = FdCPU = fopen("/dev/null", "w");

  mymalloc_init();
  timebins_init(&TimeBinsHydro, "Hydro", &All.MaxPartSph);
  timebins_init(&TimeBinsGravity, "Gravity", &All.MaxPart);
  NumPart = n;
  NumGas  = 0;
  allocate_memory();

  for(int i = 0; i < GRAVCOSTLEVELS; i++)
    All.LevelToTimeBin[i] = -1;

  for(int i = 0; i < n; i++)
    {
      memset(&P[i], 0, sizeof(struct particle_data));
      for(int k = 0; k < 3; k++)
        P[i].Pos[k] = pos[3 * i + k];
      P[i].Mass          = mass[i];
      P[i].Type          = 1;
      P[i].SofteningType = stype[i];
      P[i].ID            = (MyIDType)(i + 1);
      P[i].TimeBinGrav   = 0;
      P[i].TimeBinHydro  = 0;
      P[i].Ti_Current    = 0;
      P[i].OldAcc        = 0;
    }
  for(int i = 0; i < TIMEBINS; i++)
    TimeBinSynchronized[i] = 1;
  reconstruct_timebins();
  mark_active_timebins();

  set_softenings();
  force_short_range_init();
#ifdef PMGRID
  All.Asmth[0] = arg_d(argc, argv, "asmth", 1.25 / PMGRID);
  All.Rcut[0]  = arg_d(argc, argv, "rcut", RCUT * All.Asmth[0]);
#endif
#if !defined(PMGRID) && !defined(GRAVITY_NOT_PERIODIC)
  /* periodic pure-tree build: the reference's Ewald correction tables (forcetree_ewald.c:89-254),
   * read from / written to ewald_table_64_64_64.dat in the working directory */
  ewald_init();
  {
    const char *tabout = arg_s(argc, argv, "ewaldout", NULL);
    if(tabout)
      {
        FILE *ft = fopen(tabout, "wb");
        if(!ft)
          return 1;
        int64_t sz = (int64_t)(ENX + 1) * (ENY + 1) * (ENZ + 1);
        wr(ft, &sz, 8, 1);
        wr(ft, &Ewd_fac_intp, 8, 1);
        wr(ft, Ewd_fcorrx, sizeof(MyFloat), sz);
        wr(ft, Ewd_fcorry, sizeof(MyFloat), sz);
        wr(ft, Ewd_fcorrz, sizeof(MyFloat), sz);
        wr(ft, Ewd_potcorr, sizeof(MyFloat), sz);
        fclose(ft);
      }
  }
#endif

  double t0 = wall();
  domain_Decomposition();
  double t_domain = wall() - t0;

  int bin   = All.HighestActiveTimeBin;
  FILE *fo  = fopen(argv[2], "wb");
  if(!fo)
    return 1;
  wr(fo, "GGREFOUT", 1, 8);

  wsec(fo, "domain", 10 * 8);
  double dom[10] = {DomainCorner[0], DomainCorner[1], DomainCorner[2], DomainCenter[0], DomainCenter[1],
                    DomainCenter[2], DomainLen,       DomainInverseLen, DomainBigFac,   (double)NTopnodes};
  wr(fo, dom, 8, 10);

  wsec(fo, "order", lite ? 0 : (int64_t)n * 8);
  for(int i = 0; i < n && !lite; i++)
    {
      int64_t o = (int64_t)P[i].ID - 1;
      wr(fo, &o, 8, 1);
    }
  wsec(fo, "keys", lite ? 0 : (int64_t)n * 16);
  for(int i = 0; i < n && !lite; i++)
    {
      peano1D xb = domain_double_to_int(((P[i].Pos[0] - DomainCorner[0]) * DomainInverseLen) + 1.0);
      peano1D yb = domain_double_to_int(((P[i].Pos[1] - DomainCorner[1]) * DomainInverseLen) + 1.0);
      peano1D zb = domain_double_to_int(((P[i].Pos[2] - DomainCorner[2]) * DomainInverseLen) + 1.0);
      uint64_t kk[2];
      split_key(peano_hilbert_key(xb, yb, zb, BITS_PER_DIMENSION), &kk[0], &kk[1]);
      wr(fo, kk, 8, 2);
    }
  wsec(fo, "topnodes", (int64_t)NTopnodes * 48);
  for(int i = 0; i < NTopnodes; i++)
    {
      uint64_t k[4];
      split_key(TopNodes[i].StartKey, &k[0], &k[1]);
      split_key(TopNodes[i].Size, &k[2], &k[3]);
      wr(fo, k, 8, 4);
      int32_t dl[2] = {TopNodes[i].Daughter, TopNodes[i].Leaf};
      wr(fo, dl, 4, 2);
      wr(fo, TopNodes[i].MortonToPeanoSubnode, 1, 8);
    }

  double *acc  = malloc(sizeof(double) * 3 * n);
  double *pot  = malloc(sizeof(double) * n);
  int *ninter  = malloc(sizeof(int) * n);
  double *gacc = malloc(sizeof(double) * 3 * n);

  for(int pass = 0; pass < passes; pass++)
    {
      if(pass == 0 && displace != 0)
        P[0].Pos[0] = DomainCorner[0] + DomainLen * (1.0 + displace);
      if(active > 1)
        set_active_every(active);
      memset(acc, 0, sizeof(double) * 3 * n);
      memset(pot, 0, sizeof(double) * n);
      memset(ninter, 0, sizeof(int) * n);
      double t_build = 0, t_walk = 0, t_gt = 0;
#ifdef GPU_GRAVITY
      if(use_gpu)
        {
          for(int i = 0; i < n; i++)
            for(int k = 0; k < 3; k++)
              P[i].GravAccel[k] = 0;
          double tg0     = wall();
          int recoveries = gpu_gravity_tree(bin, use_gpu == 2 ? GPUGRAV_PREC_FP32 : GPUGRAV_PREC_FP64);
          t_gt           = wall() - tg0;
          for(int i = 0; i < n; i++)
            {
              for(int k = 0; k < 3; k++)
                gacc[3 * i + k] = acc[3 * i + k] = P[i].GravAccel[k];
#ifdef EVALPOTENTIAL
              pot[i] = P[i].Potential;
#endif
            }
          printf("gpu pass=%d recoveries=%d time=%.6f\n", pass, recoveries, t_gt);
        }
      else
#endif
#ifdef ALLOW_DIRECT_SUMMATION
          if(use_direct)
        {
          double td0 = wall();
          gravity_direct(bin);
          t_gt = wall() - td0;
          for(int i = 0; i < n; i++)
            {
              for(int k = 0; k < 3; k++)
                gacc[3 * i + k] = acc[3 * i + k] = P[i].GravAccel[k];
#ifdef EVALPOTENTIAL
              pot[i] = P[i].Potential;
#endif
            }
        }
      else
#endif
        {
      double tb0 = wall();
      construct_forcetree(0, 1, 0, bin);
      t_build = wall() - tb0;

      if(dump && pass == 0)
        dump_tree(fo);

      if(active <= 1)
        t_walk = walk_targets(first, count, stride, procs, acc, pot, ninter);

      if(run_gt)
        {
          double tg0 = wall();
          gravity_tree(bin);
          t_gt = wall() - tg0;
          for(int i = 0; i < n; i++)
            for(int k = 0; k < 3; k++)
              gacc[3 * i + k] = P[i].GravAccel[k];
        }
      else if(All.TypeOfOpeningCriterion == 1)
        All.ErrTolTheta = 0; /* what gravity_tree() does at its end (gravity/gravtree.c:654-655) */
        }

      /* the bounded CPU timing: the same walk again, reps times, after the last pass's */
      for(int r = 0; !use_gpu && !use_direct && pass == passes - 1 && r < reps; r++)
        {
          double tr     = walk_targets(first, count, stride, procs, acc, pot, ninter);
          long long nir = 0;
          int ntr       = 0;
          for(int i = first; i < first + count; i += stride)
            nir += ninter[i], ntr++;
          printf("rep=%d walk=%.6f targets=%d interactions=%lld procs=%d\n", r, tr, ntr, nir, procs);
          fflush(stdout);
        }

      char nm[16];
      const size_t na = lite ? 0 : (size_t)n;
      snprintf(nm, sizeof(nm), "acc%d", pass);
      wsec(fo, nm, (int64_t)na * 24);
      wr(fo, acc, 8, 3 * na);
      snprintf(nm, sizeof(nm), "pot%d", pass);
      wsec(fo, nm, (int64_t)na * 8);
      wr(fo, pot, 8, na);
      snprintf(nm, sizeof(nm), "ninter%d", pass);
      wsec(fo, nm, (int64_t)na * 4);
      wr(fo, ninter, 4, na);
      if(run_gt || use_gpu || use_direct)
        {
          snprintf(nm, sizeof(nm), "gacc%d", pass);
          wsec(fo, nm, (int64_t)n * 24);
          wr(fo, gacc, 8, 3 * (size_t)n);
        }

      if(!run_gt && !use_gpu && !use_direct)
        {
          /* store the walk results where gravity_tree() would have put them */
          for(int i = 0; i < n; i++)
            for(int k = 0; k < 3; k++)
              P[i].GravAccel[k] = acc[3 * i + k];
        }
      gravity_force_finalize(bin);
      if(!use_gpu && !use_direct)
        free_tree();

      snprintf(nm, sizeof(nm), "oldacc%d", pass);
      wsec(fo, nm, (int64_t)na * 4);
      for(int i = 0; i < (int)na; i++)
        {
          float oa = P[i].OldAcc;
          wr(fo, &oa, 4, 1);
        }

      long long nint = 0;
      int nt         = 0;
      for(int i = first; i < first + count; i += stride)
        nint += ninter[i], nt++;
      snprintf(nm, sizeof(nm), "time%d", pass);
      wsec(fo, nm, 6 * 8);
      double tv[6] = {t_domain, t_build, t_walk, t_gt, (double)nt, (double)nint};
      wr(fo, tv, 8, 6);
      printf("pass=%d N=%d domain=%.6f build=%.6f walk=%.6f (targets=%d, interactions=%lld) gravity_tree=%.6f\n", pass, n,
             t_domain, t_build, t_walk, nt, nint, t_gt);
    }

#ifdef HARNESS_PM
  if(use_pm)
    {
      /* the reference's long-range force on the same particles (gravity/pm/pm_periodic.c:172-248, 1572-1936) */
      const double asmth = All.Asmth[0], rcut = All.Rcut[0];
      pm_init_periodic(); /* sets Asmth/Rcut from ASMTH and PMGRID */
      for(int i = 0; i < n; i++)
        {
          for(int k = 0; k < 3; k++)
            P[i].GravPM[k] = 0;
#ifdef EVALPOTENTIAL
          P[i].PM_Potential = 0;
#endif
        }
      double tp0 = wall();
      pmforce_periodic(0, NULL);
      double tpm = wall() - tp0;
      wsec(fo, "gravpm", (int64_t)n * 24);
      for(int i = 0; i < n; i++)
        {
          double g[3] = {P[i].GravPM[0], P[i].GravPM[1], P[i].GravPM[2]};
          wr(fo, g, 8, 3);
        }
#ifdef EVALPOTENTIAL
      wsec(fo, "pmpot", (int64_t)n * 8);
      for(int i = 0; i < n; i++)
        {
          double v = P[i].PM_Potential;
          wr(fo, &v, 8, 1);
        }
#endif
      printf("pm asmth=%.17g pm_time=%.6f\n", All.Asmth[0], tpm);
      All.Asmth[0] = asmth;
      All.Rcut[0]  = rcut;
    }
#endif

  if(use_tstep)
    {
      /* the time-step criterion on the final accelerations (time_integration/timestep.c:284-353, 725-770) */
      All.ErrTolIntAccuracy = arg_d(argc, argv, "eta", 0.025);
      All.cf_atime = All.cf_a2inv = All.cf_hubble_a = 1.0;
      All.MaxSizeTimestep   = arg_d(argc, argv, "dtmax", 0.01);
      All.MinSizeTimestep   = arg_d(argc, argv, "dtmin", 0.0);
      All.DtDisplacement    = arg_d(argc, argv, "dtdisp", 1.0e30);
      All.TimeBegin         = 0.0;
      All.TimeMax           = 1.0;
      All.Timebase_interval = (All.TimeMax - All.TimeBegin) / TIMEBASE;
      All.Ti_Current        = 0;
      wsec(fo, "tistep", (int64_t)n * 8);
      int64_t *tis = malloc(sizeof(int64_t) * n);
      int32_t *tbs = malloc(sizeof(int32_t) * n);
      for(int i = 0; i < n; i++)
        {
          integertime ti = get_timestep_gravity(i);
          int bin        = 0;
          timebins_get_bin_and_do_validity_checks(ti, &bin, P[i].TimeBinGrav);
          tis[i] = (int64_t)ti;
          tbs[i] = bin;
        }
      wr(fo, tis, 8, n);
      wsec(fo, "tbin", (int64_t)n * 4);
      wr(fo, tbs, 4, n);
      free(tis);
      free(tbs);
      printf("tstep timebase=%lld\n", (long long)TIMEBASE);
    }

  /* particle order after the passes (a -3 recovery redoes the domain decomposition) */
  wsec(fo, "order_end", (int64_t)n * 8);
  for(int i = 0; i < n; i++)
    {
      int64_t o = (int64_t)P[i].ID - 1;
      wr(fo, &o, 8, 1);
    }
#ifdef GPU_GRAVITY
  gpu_gravity_free();
#endif
  wsec(fo, "end", 0);
  fclose(fo);
  return 0;
}
