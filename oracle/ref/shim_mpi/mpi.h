/* A serial stand-in for the few MPI calls the reference ASCI headers use,
 * written for the oracle (test infrastructure only). It lets the reference's
 * constraint-partitioned contribution path
 * (include/macis/asci/determinant_search.hpp:143-391), which MACIS compiles
 * only with MPI, run in one process as any one rank of a job of `size`
 * ranks: a communicator is the integer (size << 16) | rank, and
 * MPI_Comm_rank / MPI_Comm_size decode it. That path and the constraint
 * split it calls (mask_constraints.hpp:486-605) use no collective. Every
 * data-moving call is implemented only for a communicator of size 1 and
 * aborts otherwise, so a rank of a larger job can never silently skip an
 * exchange. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* the element size in bytes */
typedef int MPI_Op;

#define MPI_COMM_WORLD ((1 << 16) | 0)
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_UINT64_T ((MPI_Datatype)8)
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

static inline int oracle_mpi_size(MPI_Comm c) {
  return (c >> 16) > 0 ? (c >> 16) : 1;
}
static inline void oracle_mpi_serial_only(MPI_Comm c, const char* what) {
  if(oracle_mpi_size(c) != 1) {
    fprintf(stderr, "oracle MPI shim: %s needs a real MPI job\n", what);
    abort();
  }
}
static inline int MPI_Comm_rank(MPI_Comm c, int* r) {
  *r = c & 0xFFFF;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm c, int* s) {
  *s = oracle_mpi_size(c);
  return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm c) {
  oracle_mpi_serial_only(c, "MPI_Barrier");
  return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm c) {
  oracle_mpi_serial_only(c, "MPI_Bcast");
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t,
                                MPI_Op, MPI_Comm c) {
  oracle_mpi_serial_only(c, "MPI_Allreduce");
  if(s != MPI_IN_PLACE) memcpy(r, s, (size_t)n * (size_t)t);
  return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r,
                                int, MPI_Datatype, MPI_Comm c) {
  oracle_mpi_serial_only(c, "MPI_Allgather");
  if(s != MPI_IN_PLACE) memcpy(r, s, (size_t)n * (size_t)t);
  return MPI_SUCCESS;
}
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r,
                                 const int*, const int* displs, MPI_Datatype rt,
                                 MPI_Comm c) {
  oracle_mpi_serial_only(c, "MPI_Allgatherv");
  if(s != MPI_IN_PLACE)
    memcpy((char*)r + (size_t)displs[0] * (size_t)rt, s, (size_t)n * (size_t)t);
  return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int n, MPI_Datatype t, MPI_Datatype* out) {
  *out = n * t;
  return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }
#endif
