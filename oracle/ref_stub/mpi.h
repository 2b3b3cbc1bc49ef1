/* Single-rank stand-in for the few MPI calls made by the reference's CPU path
 * (setup_mlfma.cpp, solve.cpp, bicgs.cpp).  Test infrastructure only: it lets
 * the reference's unmodified sources compile and run as one process, so that
 * they can serve as the checker for the restated oracle and the CUDA path.
 *
 * With one rank every collective is a copy of the send buffer into the
 * receive buffer, and point-to-point calls are never reached (the pair
 * schedules are empty for one rank).  Datatypes are represented by their size
 * in bytes.
 */
#ifndef ISG_ORACLE_MPI_STUB_H
#define ISG_ORACLE_MPI_STUB_H

#include <string.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INTEGER ((MPI_Datatype)sizeof(int))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_DOUBLE_COMPLEX ((MPI_Datatype)(2 * sizeof(double)))
#define MPI_SUM 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }

static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)count * (size_t)t);
  return 0;
}

static inline int MPI_Allgather(const void *s, int scount, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)scount * (size_t)st);
  return 0;
}

static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int, MPI_Datatype, int, int, MPI_Comm,
                               MPI_Status *) {
  fprintf(stderr, "single-rank MPI stand-in: MPI_Sendrecv reached with one rank\n");
  abort();
  return 0;
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *out) {
  *out = 0;
  return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Gather(const void *s, int scount, MPI_Datatype st, void *r, int, MPI_Datatype, int, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)scount * (size_t)st);
  return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)count * (size_t)t);
  return 0;
}

static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#endif
