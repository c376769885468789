/*
 * gpu_gravity.c -- the AREPO side of libarepo_gpugrav: the binding a maintainer adds to the
 * reference (under a GPU_GRAVITY switch) so that gravity() (src/gravity/accel.c:127-134) calls the
 * library instead of the pair construct_forcetree(0, ...) + gravity_tree(timebin).
 *
 * It is compiled here against the reference's own headers and linked into a harness build of the
 * reference (ref_harness_*_gpu), so the drop-in runs from C on AREPO's own data structures: P[],
 * All, the domain globals, TopNodes and TimeBinsGravity.  TEST INFRASTRUCTURE for the library.
 *
 *  - every particle goes into the tree; the walk covers TimeBinsGravity.ActiveParticleList (the
 *    TargetList of gravtree.c:494-520) through gpugrav_walk_targets, or every particle;
 *  - the caller's domain (DomainCorner/Len/BigFac) and TopNodes are handed over, so keys, top
 *    leaves and the node numbering are the reference's;
 *  - a particle outside the domain box (GPUGRAV_ERR_OUT_OF_BOX, force_treebuild_construct's -3)
 *    is answered as force_treebuild answers it (forcetree.c:187-208): a new domain decomposition and
 *    another try.  (A run with gas also frees and rebuilds the neighbour tree there, forcetree.c:201-206.)
 *  - packing buffers come from mymalloc and are freed in reverse order (AREPO's LIFO allocator);
 *    the library's own memory never does.
 */
#include <stdint.h>
#include <string.h>

#include "allvars.h"
#include "proto.h"
#include "../domain/domain.h"

#include "gpugrav.h"

static gpugrav_ctx *GpuGrav;

static void gpu_gravity_params(gpugrav_params *p, int precision)
{
  memset(p, 0, sizeof(*p));
  p->abi_version = GPUGRAV_ABI_VERSION;
#ifdef GRAVITY_NOT_PERIODIC
  p->periodic = 0;
#else
  p->periodic = 1;
#ifdef PMGRID
  p->asmth = All.Asmth[0];
  p->rcut  = All.Rcut[0];
#endif
#endif
  p->box_size   = All.BoxSize;
  p->rcut_cells = RCUT;
  p->nsofttypes = NSOFTTYPES + NSOFTTYPES_HYDRO;
  for(int i = 0; i <= NSOFTTYPES + NSOFTTYPES_HYDRO; i++)
    p->force_softening[i] = All.ForceSoftening[i]; /* last entry 0 (set_softenings) */
  p->type_of_opening_criterion = All.TypeOfOpeningCriterion;
  p->err_tol_theta             = All.ErrTolTheta; /* 0 after the first pass: relative criterion */
  p->err_tol_force_acc         = All.ErrTolForceAcc;
  p->top_node_factor           = All.TopNodeFactor;
  p->multiple_domains          = All.MultipleDomains;
  p->precision                 = precision;
#ifdef MULTIPLE_NODE_SOFTENING
  p->flags = GPUGRAV_FLAG_MULTIPLE_NODE_SOFTENING;
#endif
}

/* construct_forcetree(0, ...) + gravity_tree(timebin) on the GPU: P[i].GravAccel (without G) and,
 * with EVALPOTENTIAL, P[i].Potential of the active particles.  Returns the number of domain
 * decompositions redone for particles outside the domain box. */
int gpu_gravity_tree(int timebin, int precision)
{
  gpugrav_params prm;
  gpu_gravity_params(&prm, precision);
  int status = GpuGrav ? gpugrav_set_params(GpuGrav, &prm) : gpugrav_create(&GpuGrav, 0, &prm);
  if(status != GPUGRAV_OK)
    terminate_program("gpugrav: parameters: %s", gpugrav_status_string(status));

  int recoveries = 0;
  for(;;)
    {
      double *pos   = (double *)mymalloc("gg_pos", 3 * (size_t)NumPart * sizeof(double));
      double *mass  = (double *)mymalloc("gg_mass", (size_t)NumPart * sizeof(double));
      uint8_t *st   = (uint8_t *)mymalloc("gg_st", (size_t)NumPart);
      float *oldacc = (float *)mymalloc("gg_oldacc", (size_t)NumPart * sizeof(float));
      for(int i = 0; i < NumPart; i++)
        {
          for(int k = 0; k < 3; k++)
            pos[3 * i + k] = P[i].Pos[k];
          mass[i]   = P[i].Mass;
          st[i]     = P[i].SofteningType;
          oldacc[i] = P[i].OldAcc;
        }
      gpugrav_domain dom;
      for(int k = 0; k < 3; k++)
        {
          dom.corner[k] = DomainCorner[k];
          dom.center[k] = DomainCenter[k];
        }
      dom.len         = DomainLen;
      dom.inverse_len = DomainInverseLen;
      dom.big_fac     = DomainBigFac;
      gpugrav_topnode *top = (gpugrav_topnode *)mymalloc("gg_top", (size_t)NTopnodes * sizeof(gpugrav_topnode));
      for(int i = 0; i < NTopnodes; i++)
        {
          top[i].start_key_hi = (uint64_t)((unsigned __int128)TopNodes[i].StartKey >> 64);
          top[i].start_key_lo = (uint64_t)TopNodes[i].StartKey;
          top[i].size_hi      = (uint64_t)((unsigned __int128)TopNodes[i].Size >> 64);
          top[i].size_lo      = (uint64_t)TopNodes[i].Size;
          top[i].daughter     = TopNodes[i].Daughter;
          top[i].leaf         = TopNodes[i].Leaf;
          memcpy(top[i].morton_to_peano, TopNodes[i].MortonToPeanoSubnode, 8);
        }

      status = gpugrav_load(GpuGrav, NumPart, pos, mass, st, GPUGRAV_MEM_HOST, &dom);
      if(status == GPUGRAV_OK)
        status = gpugrav_build(GpuGrav, top, NTopnodes);
      if(status == GPUGRAV_ERR_OUT_OF_BOX)
        {
          myfree(top);
          myfree(oldacc);
          myfree(st);
          myfree(mass);
          myfree(pos);
          if(++recoveries > 3)
            terminate_program("gpugrav: particles stay outside the domain box");
          domain_free();
          domain_Decomposition(); /* as force_treebuild does on -3 */
          continue;
        }
      if(status != GPUGRAV_OK)
        terminate_program("gpugrav: %s: %s", gpugrav_status_string(status), gpugrav_last_error(GpuGrav));

      /* the targets: gravity_tree's TargetList */
      int nact = 0;
      int *targets = (int *)mymalloc("gg_targets", (size_t)NumPart * sizeof(int));
      for(int idx = 0; idx < TimeBinsGravity.NActiveParticles; idx++)
        if(TimeBinsGravity.ActiveParticleList[idx] >= 0)
          targets[nact++] = TimeBinsGravity.ActiveParticleList[idx];
      double *acc = (double *)mymalloc("gg_acc", 3 * (size_t)nact * sizeof(double) + 8);
      double *pot = (double *)mymalloc("gg_pot", (size_t)nact * sizeof(double) + 8);
      status = gpugrav_walk_targets(GpuGrav, nact, targets, oldacc, acc, pot, NULL, GPUGRAV_MEM_HOST);
      if(status != GPUGRAV_OK)
        terminate_program("gpugrav: %s: %s", gpugrav_status_string(status), gpugrav_last_error(GpuGrav));
      for(int j = 0; j < nact; j++)
        {
          const int i = targets[j];
          for(int k = 0; k < 3; k++)
            P[i].GravAccel[k] = acc[3 * j + k];
#ifdef EVALPOTENTIAL
          P[i].Potential = pot[j];
#endif
        }
      myfree(pot);
      myfree(acc);
      myfree(targets);
      myfree(top);
      myfree(oldacc);
      myfree(st);
      myfree(mass);
      myfree(pos);
      break;
    }
  if(All.TypeOfOpeningCriterion == 1)
    All.ErrTolTheta = 0; /* what gravity_tree does at its end (gravtree.c:654-655) */
  return recoveries;
}

void gpu_gravity_free(void)
{
  if(GpuGrav)
    gpugrav_destroy(GpuGrav);
  GpuGrav = NULL;
}
