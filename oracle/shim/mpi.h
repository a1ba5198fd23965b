/*
 * Single-rank MPI shim for building the reference's hot-path sources as a CPU
 * oracle (test infrastructure only; never linked into the product).
 *
 * Every call behaves as MPI would with exactly one rank in MPI_COMM_WORLD:
 * reductions and gathers copy the send buffer to the receive buffer, the
 * Cartesian topology is 1x1 with rank 0 as its own (periodic) neighbour, and a
 * Sendrecv to self delivers the send buffer into the receive buffer.  Only the
 * symbols that the reference's Cell/Face/Riemann/TimeStep/GravMass/Sim/
 * MPIsetup sources use are provided.
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* value = element size in bytes */
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

static inline int MPI_Dims_create(int nnodes, int ndims, int *dims) {
  int d;
  (void)nnodes;
  for (d = 0; d < ndims; ++d)
    if (dims[d] == 0) dims[d] = 1;
  return 0;
}
static inline int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods,
                                  int reorder, MPI_Comm *cart) {
  (void)old; (void)ndims; (void)dims; (void)periods; (void)reorder;
  *cart = 0;
  return 0;
}
static inline int MPI_Cart_coords(MPI_Comm c, int rank, int maxdims, int *coords) {
  int d;
  (void)c; (void)rank;
  for (d = 0; d < maxdims; ++d) coords[d] = 0;
  return 0;
}
static inline int MPI_Cart_rank(MPI_Comm c, const int *coords, int *rank) {
  (void)c; (void)coords;
  *rank = 0;
  return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op,
                                MPI_Comm c) {
  (void)op; (void)c;
  memmove(r, s, (size_t)count * (size_t)t);
  return 0;
}
static inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int rc,
                                MPI_Datatype rt, MPI_Comm c) {
  (void)rc; (void)rt; (void)c;
  memmove(r, s, (size_t)sc * (size_t)st);
  return 0;
}
static inline int MPI_Sendrecv(const void *s, int sc, MPI_Datatype st, int dest, int stag,
                               void *r, int rc, MPI_Datatype rt, int src, int rtag, MPI_Comm c,
                               MPI_Status *status) {
  int n = sc < rc ? sc : rc;
  (void)dest; (void)stag; (void)rt; (void)src; (void)rtag; (void)c; (void)status;
  memmove(r, s, (size_t)n * (size_t)st);
  return 0;
}

#endif
