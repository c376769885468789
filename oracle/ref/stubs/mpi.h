/* Single-rank MPI interface used to compile the reference's gravity sources
 * without an MPI installation.  Test infrastructure only: every collective
 * degenerates to a copy from the send to the receive buffer (one rank). */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H
#include <stddef.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Win;
typedef int MPI_Group;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef struct
{
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
  int count;
} MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_ANY_SOURCE -1
#define MPI_ANY_TAG -1
#define MPI_SUCCESS 0
#define MPI_REQUEST_NULL 0
#define MPI_UNDEFINED -32766
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_THREAD_SINGLE 0
enum
{
  MPI_BYTE = 1,
  MPI_CHAR,
  MPI_INT,
  MPI_UNSIGNED,
  MPI_LONG,
  MPI_UNSIGNED_LONG,
  MPI_LONG_LONG,
  MPI_LONG_LONG_INT,
  MPI_UNSIGNED_LONG_LONG,
  MPI_FLOAT,
  MPI_DOUBLE,
  MPI_DOUBLE_INT,
  MPI_2INT,
  MPI_INT64_T,
  MPI_UINT64_T
};
enum
{
  MPI_SUM = 1,
  MPI_MIN,
  MPI_MAX,
  MPI_LOR,
  MPI_LAND,
  MPI_BOR,
  MPI_BAND,
  MPI_MAXLOC,
  MPI_MINLOC
};
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Type_size(MPI_Datatype t, int *size);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt,
                  MPI_Comm c);
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c);
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Scatter(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Barrier(MPI_Comm c);
int MPI_Sendrecv(const void *s, int sn, MPI_Datatype st, int dest, int stag, void *r, int rn, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm c, MPI_Status *status);
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Ssend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Issend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Wait(MPI_Request *rq, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st);
int MPI_Test(MPI_Request *rq, int *flag, MPI_Status *st);
int MPI_Testall(int n, MPI_Request *rq, int *flag, MPI_Status *st);
int MPI_Iprobe(int src, int tag, MPI_Comm c, int *flag, MPI_Status *st);
int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n);
int MPI_Get_processor_name(char *name, int *len);
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out);
int MPI_Comm_dup(MPI_Comm c, MPI_Comm *out);
int MPI_Comm_free(MPI_Comm *c);
int MPI_Ibarrier(MPI_Comm c, MPI_Request *rq);
#endif
