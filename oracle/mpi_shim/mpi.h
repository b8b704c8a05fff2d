/* Single-rank stand-in for <mpi.h>, used only to compile the reference's own
 * pipeline sources (oracle/_ref) as a one-process program.  No MPI library is
 * installed on this machine.
 *
 * With one rank every collective is a copy from the send buffer to the
 * receive buffer (or nothing, for MPI_IN_PLACE), point-to-point receives can
 * never be satisfied, and MPI_Iprobe reports no message.  This mirrors what a
 * real MPI does at world size 1 for the call shapes used by the reference
 * (src/chunked_exchange.c, src/dsort.c, src/fastga_order.c,
 * src/pga-mpi-merge.c).
 *
 * Test infrastructure: nothing in the product links this file.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* the element size in bytes */
typedef int MPI_Op;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD     0
#define MPI_SUCCESS        0
#define MPI_ANY_SOURCE    (-1)
#define MPI_ANY_TAG       (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_IN_PLACE      ((void *) 1)

#define MPI_BYTE       1
#define MPI_CHAR       1
#define MPI_INT        4
#define MPI_LONG_LONG  8
#define MPI_INT64_T    8
#define MPI_DOUBLE     8

#define MPI_SUM  1
#define MPI_MAX  2
#define MPI_MIN  3
#define MPI_BOR  4

static inline int MPI_Init(int *argc, char ***argv) { (void) argc; (void) argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void) c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void) c; *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void) c; return 0; }

static inline double MPI_Wtime(void)
{ struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static inline int MPI_Abort(MPI_Comm c, int code)
{ (void) c;
  fprintf(stderr, "MPI_Abort(%d) in single-rank oracle build\n", code);
  exit(code);
}

static inline void oracle_mpi_copy(const void *s, void *r, long long n)
{ if (s != MPI_IN_PLACE && s != r && n > 0) memmove(r, s, (size_t) n); }

static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) root; (void) c; return 0; }

static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void) op; (void) c; oracle_mpi_copy(s, r, (long long) n * t); return 0; }

static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void) op; (void) root; (void) c; oracle_mpi_copy(s, r, (long long) n * t); return 0; }

static inline int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void) rn; (void) rt; (void) c; oracle_mpi_copy(s, r, (long long) sn * st); return 0; }

static inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st,
                                void *r, const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c)
{ (void) rc; (void) rt; (void) c;
  if (sc[0] > 0)
    memmove((char *) r + (long long) rd[0] * rt, (const char *) s + (long long) sd[0] * st,
            (size_t) sc[0] * st);
  return 0;
}

static inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void) rn; (void) rt; (void) c; oracle_mpi_copy(s, r, (long long) sn * st); return 0; }

static inline int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{ (void) rn; (void) rt; (void) root; (void) c; oracle_mpi_copy(s, r, (long long) sn * st); return 0; }

static inline int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd,
                              MPI_Datatype rt, int root, MPI_Comm c)
{ (void) rc; (void) root; (void) c;
  if (sn > 0) memmove((char *) r + (long long) rd[0] * rt, s, (size_t) sn * st);
  return 0;
}

static inline int MPI_Iprobe(int src, int tag, MPI_Comm c, int *flag, MPI_Status *st)
{ (void) src; (void) tag; (void) c; (void) st; *flag = 0; return 0; }

static inline int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st)
{ (void) src; (void) tag; (void) st; return MPI_Abort(c, 90); }

static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{ (void) b; (void) n; (void) t; (void) src; (void) tag; (void) st; return MPI_Abort(c, 91); }

static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) dst; (void) tag; return MPI_Abort(c, 92); }

static inline int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dst, int stag,
                               void *rb, int rn, MPI_Datatype rt, int src, int rtag,
                               MPI_Comm c, MPI_Status *status)
{ (void) dst; (void) stag; (void) rn; (void) rt; (void) src; (void) rtag; (void) status; (void) c;
  oracle_mpi_copy(sb, rb, (long long) sn * st); return 0;
}

#endif
