/*
 * mpi_shim.c -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Single-rank implementations of the MPI calls the reference's gravity and
 * domain sources make, plus inert stand-ins for the GSL/FFTW entry points they
 * reference but never call on the short-range gravity path.  With one rank,
 * every collective copies the send buffer into the receive buffer, point to
 * point exchange with oneself is a copy, and reductions are identities.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "mpi.h"
#include "gsl/gsl_errno.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_rng.h"

static size_t type_size(MPI_Datatype t)
{
  switch(t)
    {
      case MPI_BYTE:
      case MPI_CHAR:
        return 1;
      case MPI_INT:
      case MPI_UNSIGNED:
      case MPI_FLOAT:
        return 4;
      case MPI_LONG:
      case MPI_UNSIGNED_LONG:
      case MPI_LONG_LONG:
      case MPI_LONG_LONG_INT:
      case MPI_UNSIGNED_LONG_LONG:
      case MPI_DOUBLE:
      case MPI_INT64_T:
      case MPI_UINT64_T:
      case MPI_2INT:
        return 8;
      case MPI_DOUBLE_INT:
        return 16;
      default:
        fprintf(stderr, "mpi_shim: unknown datatype %d\n", t);
        abort();
    }
}

static void copy_in(const void *s, void *r, size_t bytes)
{
  if(s == MPI_IN_PLACE || s == r || bytes == 0)
    return;
  memmove(r, s, bytes);
}

int MPI_Init(int *argc, char ***argv) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm comm, int code)
{
  fprintf(stderr, "MPI_Abort(%d)\n", code);
  exit(code ? code : 1);
}
double MPI_Wtime(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}
int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
  *rank = 0;
  return 0;
}
int MPI_Comm_size(MPI_Comm comm, int *size)
{
  *size = 1;
  return 0;
}
int MPI_Type_size(MPI_Datatype t, int *size)
{
  *size = (int)type_size(t);
  return 0;
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
  copy_in(s, r, (size_t)n * type_size(t));
  return 0;
}
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
  copy_in(s, r, (size_t)n * type_size(t));
  return 0;
}
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{
  copy_in(s, r, (size_t)sn * type_size(st));
  return 0;
}
int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt,
                  MPI_Comm c)
{
  copy_in((const char *)s + (size_t)sd[0] * type_size(st), (char *)r + (size_t)rd[0] * type_size(rt), (size_t)sc[0] * type_size(st));
  return 0;
}
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{
  copy_in(s, r, (size_t)sn * type_size(st));
  return 0;
}
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c)
{
  if(s == MPI_IN_PLACE)
    return 0;
  copy_in(s, (char *)r + (size_t)rd[0] * type_size(rt), (size_t)sn * type_size(st));
  return 0;
}
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{
  copy_in(s, r, (size_t)sn * type_size(st));
  return 0;
}
int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt, int root, MPI_Comm c)
{
  copy_in(s, (char *)r + (size_t)rd[0] * type_size(rt), (size_t)sn * type_size(st));
  return 0;
}
int MPI_Scatter(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{
  copy_in(s, r, (size_t)sn * type_size(st));
  return 0;
}
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) { return 0; }
int MPI_Barrier(MPI_Comm c) { return 0; }
int MPI_Sendrecv(const void *s, int sn, MPI_Datatype st, int dest, int stag, void *r, int rn, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm c, MPI_Status *status)
{
  copy_in(s, r, (size_t)sn * type_size(st));
  return 0;
}

static void no_p2p(const char *what)
{
  fprintf(stderr, "mpi_shim: %s is not available with a single rank\n", what);
  abort();
}
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
  no_p2p("MPI_Send");
  return 1;
}
int MPI_Ssend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
  no_p2p("MPI_Ssend");
  return 1;
}
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{
  no_p2p("MPI_Recv");
  return 1;
}
/* non-blocking messages to oneself (the only rank): a send is kept until the receive with the same
 * tag takes it (or the other way round); both are complete once matched */
#define SELF_MSGS 64
static struct
{
  const void *sbuf;
  void *rbuf;
  size_t bytes;
  int tag, has_send, has_recv;
} self_msg[SELF_MSGS];
static void self_match(int k)
{
  if(self_msg[k].has_send && self_msg[k].has_recv)
    {
      copy_in(self_msg[k].sbuf, self_msg[k].rbuf, self_msg[k].bytes);
      self_msg[k].has_send = self_msg[k].has_recv = 0;
    }
}
static int self_slot(int tag, int want_send)
{
  for(int k = 0; k < SELF_MSGS; k++)
    if(self_msg[k].tag == tag && (want_send ? (self_msg[k].has_recv && !self_msg[k].has_send)
                                            : (self_msg[k].has_send && !self_msg[k].has_recv)))
      return k;
  for(int k = 0; k < SELF_MSGS; k++)
    if(!self_msg[k].has_send && !self_msg[k].has_recv)
      return k;
  no_p2p("more than 64 pending messages to oneself");
  return -1;
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq)
{
  if(dest != 0)
    no_p2p("MPI_Isend to another rank");
  int k              = self_slot(tag, 1);
  self_msg[k].sbuf   = b;
  self_msg[k].tag    = tag;
  self_msg[k].bytes  = (size_t)n * type_size(t);
  self_msg[k].has_send = 1;
  self_match(k);
  return 0;
}
int MPI_Issend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq)
{
  no_p2p("MPI_Issend");
  return 1;
}
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq)
{
  if(src != 0)
    no_p2p("MPI_Irecv from another rank");
  int k              = self_slot(tag, 0);
  self_msg[k].rbuf   = b;
  self_msg[k].tag    = tag;
  self_msg[k].has_recv = 1;
  self_match(k);
  return 0;
}
int MPI_Wait(MPI_Request *rq, MPI_Status *st) { return 0; }
int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st) { return 0; }
int MPI_Test(MPI_Request *rq, int *flag, MPI_Status *st)
{
  *flag = 1;
  return 0;
}
int MPI_Testall(int n, MPI_Request *rq, int *flag, MPI_Status *st)
{
  *flag = 1;
  return 0;
}
int MPI_Iprobe(int src, int tag, MPI_Comm c, int *flag, MPI_Status *st)
{
  *flag = 0;
  return 0;
}
int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st)
{
  no_p2p("MPI_Probe");
  return 1;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n)
{
  *n = 0;
  return 0;
}
int MPI_Get_processor_name(char *name, int *len)
{
  strcpy(name, "localhost");
  *len = 9;
  return 0;
}
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out)
{
  *out = c;
  return 0;
}
int MPI_Comm_dup(MPI_Comm c, MPI_Comm *out)
{
  *out = c;
  return 0;
}
int MPI_Comm_free(MPI_Comm *c) { return 0; }
int MPI_Ibarrier(MPI_Comm c, MPI_Request *rq) { return 0; }

/* ---- GSL: only the random-number set-up is reachable (begrun1); it is unused with
 *      DO_NOT_RANDOMIZE_DOMAINCENTER, so a fixed-seed LCG stands in ---- */
struct gsl_rng_type_s
{
  int dummy;
};
struct gsl_rng_s
{
  unsigned long long state;
};
static const struct gsl_rng_type_s ranlxd1_type = {0};
const gsl_rng_type *gsl_rng_ranlxd1             = &ranlxd1_type;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t)
{
  gsl_rng *r = malloc(sizeof(gsl_rng));
  r->state   = 1;
  return r;
}
void gsl_rng_set(const gsl_rng *r, unsigned long seed) { ((gsl_rng *)r)->state = seed * 2862933555777941757ULL + 3037000493ULL; }
double gsl_rng_uniform(const gsl_rng *r)
{
  gsl_rng *q = (gsl_rng *)r;
  q->state   = q->state * 6364136223846793005ULL + 1442695040888963407ULL;
  return (double)(q->state >> 11) * (1.0 / 9007199254740992.0);
}
void gsl_rng_free(gsl_rng *r) { free(r); }
gsl_error_handler_t *gsl_set_error_handler(gsl_error_handler_t *h) { return 0; }
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n)
{
  fprintf(stderr, "mpi_shim: GSL integration is not available in the oracle build\n");
  abort();
}
void gsl_integration_workspace_free(gsl_integration_workspace *w) {}
int gsl_integration_qag(const gsl_function *f, double a, double b, double epsabs, double epsrel, size_t limit, int key,
                        gsl_integration_workspace *w, double *result, double *abserr)
{
  fprintf(stderr, "mpi_shim: GSL integration is not available in the oracle build\n");
  abort();
}
