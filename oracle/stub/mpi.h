/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * header-only SparseLDL as a CPU test oracle. The reference headers name a
 * handful of MPI types and calls (node_owners.h, ordering_utils.h) that the
 * serial LDL path never executes; these definitions satisfy the compiler and
 * behave as a one-process communicator.
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_C_COMPLEX 4
#define MPI_C_DOUBLE_COMPLEX 5
#define MPI_DATATYPE_NULL 0
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int MPI_Comm_size(MPI_Comm, int* size) {
  *size = 1;
  return 0;
}
static inline int MPI_Comm_rank(MPI_Comm, int* rank) {
  *rank = 0;
  return 0;
}
static inline int MPI_Scatter(const void*, int, MPI_Datatype, void*, int,
                              MPI_Datatype, int, MPI_Comm) {
  return 0;
}
static inline int MPI_Scatterv(const void*, const int*, const int*,
                               MPI_Datatype, void*, int, MPI_Datatype, int,
                               MPI_Comm) {
  return 0;
}

#endif
