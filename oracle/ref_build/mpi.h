/* Single-rank MPI stand-in used only to compile the reference PFDD sources
 * into a CPU oracle (test infrastructure; nothing in the product links it).
 *
 * The reference calls a small MPI-1 subset (Init/Finalize/Abort, Comm_rank/size,
 * Barrier, Wtime, Bcast, Allreduce, Reduce and a few point-to-point calls that
 * are only reached when nprocs > 1, e.g. fft_fftw_slab.cpp:933 and the iproc
 * loops in dump.cpp).  With one rank every collective is a copy and every
 * point-to-point call is unreachable, so those abort loudly if ever hit.
 */
#ifndef PFDD_ORACLE_MPI_STUB_H
#define PFDD_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_LONG 8
#define MPI_LONG_LONG 9
#define MPI_DOUBLE 10
#define MPI_FLOAT 11

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t pfdd_stub_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_LONG_LONG: return sizeof(long long);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_FLOAT: return sizeof(float);
  }
  fprintf(stderr, "mpi stub: unknown datatype %d\n", t);
  abort();
}

static inline void pfdd_stub_unreachable(const char *what) {
  fprintf(stderr, "mpi stub: %s reached with a single rank\n", what);
  abort();
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code ? code : 1); }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline double MPI_Wtime() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)n * pfdd_stub_type_size(t));
  return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)n * pfdd_stub_type_size(t));
  return 0;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
  pfdd_stub_unreachable("MPI_Send"); return 0;
}
static inline int MPI_Rsend(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
  pfdd_stub_unreachable("MPI_Rsend"); return 0;
}
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  pfdd_stub_unreachable("MPI_Recv"); return 0;
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  pfdd_stub_unreachable("MPI_Irecv"); return 0;
}
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Get_count(const MPI_Status *, MPI_Datatype, int *c) { *c = 0; return 0; }

#endif
