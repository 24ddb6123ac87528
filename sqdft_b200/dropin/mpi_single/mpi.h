/* Single-process stand-in for the subset of MPI-3 that SQDFT uses.
 *
 * It lets the SQDFT sources compile and run as one rank where no MPI is
 * installed: the drop-in build (reference host code + the GPU SQ path) and
 * the oracle build of the reference use it.  With a real MPI, put its
 * include directory first instead.  With one rank every neighbour of the
 * distributed-graph topologies (initialize.cpp:335,458) is rank 0 itself, so a
 * neighbourhood all-to-all copies send block k into receive block k (MPI's
 * in-order matching of repeated edges).  That turns the halo exchanges of
 * sq.cpp:400-492 and poisson.cpp:740-800 into the periodic wrap-around of the
 * whole domain.  Reductions, gathers and broadcasts over one rank are copies.
 */
#ifndef SQB_ORACLE_MPI_STUB_H
#define SQB_ORACLE_MPI_STUB_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_CHAR 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_UNWEIGHTED ((int *)0)
#define MPI_IN_PLACE ((void *)1)

/* Degree of each distributed-graph communicator, indexed by handle - 16.
 * C++17 inline variables, so every translation unit shares one table. */
inline int sqb_stub_graph_degree[64];
inline int sqb_stub_graph_count = 0;

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE && n > 0) memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
static inline int MPI_Allgather(const void *s, int ns, MPI_Datatype ts, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE && ns > 0) memmove(r, s, (size_t)ns * (size_t)ts);
  return 0;
}
static inline int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *c) { *c = 1; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int nd, int *co) {
  for (int i = 0; i < nd; i++) co[i] = 0;
  return 0;
}
static inline int MPI_Cart_rank(MPI_Comm, const int *, int *r) { *r = 0; return 0; }
static inline int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst) { *src = 0; *dst = 0; return 0; }
static inline int MPI_Dist_graph_create_adjacent(MPI_Comm, int indegree, const int *, const int *, int,
                                                 const int *, const int *, MPI_Info, int, MPI_Comm *c) {
  int k = sqb_stub_graph_count++ % 64;
  sqb_stub_graph_degree[k] = indegree;
  *c = 16 + k;
  return 0;
}
static inline int MPI_Neighbor_alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r,
                                         const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c) {
  int deg = (c >= 16 && c < 16 + 64) ? sqb_stub_graph_degree[c - 16] : 0;
  for (int k = 0; k < deg; k++) {
    size_t bytes = (size_t)(sc[k] < rc[k] ? sc[k] : rc[k]) * (size_t)st;
    memmove((char *)r + (size_t)rd[k] * (size_t)rt, (const char *)s + (size_t)sd[k] * (size_t)st, bytes);
  }
  return 0;
}
static inline int MPI_Ineighbor_alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r,
                                          const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c,
                                          MPI_Request *req) {
  *req = 0;
  return MPI_Neighbor_alltoallv(s, sc, sd, st, r, rc, rd, rt, c);
}
#endif
