/*
 * Single-rank stand-in for the handful of MPI entry points that the
 * reference's 3D driver (3D/MPI/KHI) and its halo library (mpi/common_mpi.c)
 * touch.  It exists only so that the reference's own 3D stepping code can be
 * compiled from its sources and run as the CPU oracle on one process.
 *
 * Semantics at one rank:
 *   - MPI_Init / Finalize / Barrier / Bcast: no-ops returning MPI_SUCCESS.
 *   - MPI_Comm_size -> 1, MPI_Comm_rank -> 0.
 *   - MPI_Allreduce copies the send buffer (the max over one rank).
 *   - MPI_Sendrecv is never reached at one rank (mpi/common_mpi.c:221,280,339
 *     guard it with mpi_num{x,y,z} != 1); if it is, the harness aborts.
 *   - MPI_Wtime uses the monotonic clock.
 * This file is test infrastructure of the oracle, not part of the product.
 */
#ifndef QAS_ORACLE_MPI_STUB_H
#define QAS_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_DOUBLE 1
#define MPI_MAX 1

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code); }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void)op; (void)c; if (t == MPI_DOUBLE) memcpy(r, s, sizeof(double) * (size_t)n); return MPI_SUCCESS; }
static inline int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dst, int stag,
                               void *rb, int rn, MPI_Datatype rt, int src, int rtag,
                               MPI_Comm c, MPI_Status *s)
{
  (void)sb; (void)sn; (void)st; (void)dst; (void)stag; (void)rb; (void)rn; (void)rt;
  (void)src; (void)rtag; (void)c; (void)s;
  fprintf(stderr, "single-rank MPI stand-in: MPI_Sendrecv reached\n");
  abort();
}
static inline double MPI_Wtime(void)
{ struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec; }

#endif
