/* TEST INFRASTRUCTURE ONLY — never part of the product path.
 *
 * A single-rank stand-in for <mpi.h>, so that the reference's own multi-level
 * glue (communication/internal_halo_manager.cpp, multiresolution/averager.cpp
 * and the topology they need) compiles into oracle/_ref without an MPI
 * installation. One rank owns every node: the rank queries answer 0 and 1,
 * the collectives copy the local contribution, derived datatypes are handles
 * without content. A point-to-point call never happens on one rank (every
 * partner is local); if one does, the process stops with a message instead of
 * computing something wrong. The declarations follow the MPI standard's C
 * binding for the calls the reference uses. */
#ifndef ALPACA_ORACLE_MPI_SHIM_H
#define ALPACA_ORACLE_MPI_SHIM_H

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_ORDER_C 0
#define MPI_TAG_UB 1
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_REQUEST_NULL 0
#define MPI_LOR 1
#define MPI_SUM 2
#define MPI_MAX 3
#define MPI_MIN 4
#define MPI_LAND 5

/* predefined datatypes carry their byte size; derived ones count up from 1024 */
#define MPI_CHAR 1
#define MPI_BYTE 1
#define MPI_INT8_T 1
#define MPI_CXX_BOOL 1
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_DOUBLE 8
#define MPI_LONG 8
#define MPI_LONG_LONG_INT 8
#define MPI_UNSIGNED_LONG_LONG 8

namespace alpaca_oracle_mpi {
inline std::size_t type_size(MPI_Datatype t) {
  if (t > 0 && t <= 8) return (std::size_t)t;
  std::fprintf(stderr, "single-rank MPI shim: a derived datatype reached a collective\n");
  std::abort();
}
[[noreturn]] inline void point_to_point(char const *what) {
  std::fprintf(stderr, "single-rank MPI shim: %s called, but one rank has no partner\n", what);
  std::abort();
}
inline int &next_type() {
  static int n = 1024;
  return n;
}
}  // namespace alpaca_oracle_mpi

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
inline int MPI_Comm_get_attr(MPI_Comm, int key, void *value, int *flag) {
  static int tag_ub = 1 << 30;
  *flag = key == MPI_TAG_UB;
  if (*flag) *static_cast<int **>(value) = &tag_ub;
  return MPI_SUCCESS;
}
inline int MPI_Allreduce(void const *send, void *recv, int count, MPI_Datatype t, MPI_Op,
                         MPI_Comm) {
  if (send != MPI_IN_PLACE)
    std::memcpy(recv, send, (std::size_t)count * alpaca_oracle_mpi::type_size(t));
  return MPI_SUCCESS;
}
inline int MPI_Allgather(void const *send, int count, MPI_Datatype t, void *recv, int, MPI_Datatype,
                         MPI_Comm) {
  if (send != MPI_IN_PLACE)
    std::memcpy(recv, send, (std::size_t)count * alpaca_oracle_mpi::type_size(t));
  return MPI_SUCCESS;
}
inline int MPI_Allgatherv(void const *send, int count, MPI_Datatype t, void *recv, int const *,
                          int const *displs, MPI_Datatype, MPI_Comm) {
  std::size_t const size = alpaca_oracle_mpi::type_size(t);
  if (send != MPI_IN_PLACE)
    std::memcpy(static_cast<char *>(recv) + (std::size_t)displs[0] * size, send,
                (std::size_t)count * size);
  return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Type_create_subarray(int, int const *, int const *, int const *, int, MPI_Datatype,
                                    MPI_Datatype *newtype) {
  *newtype = alpaca_oracle_mpi::next_type()++;
  return MPI_SUCCESS;
}
inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype *newtype) {
  *newtype = alpaca_oracle_mpi::next_type()++;
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *t) {
  *t = 0;
  return MPI_SUCCESS;
}
inline int MPI_Send(void const *, int, MPI_Datatype, int, int, MPI_Comm) {
  alpaca_oracle_mpi::point_to_point("MPI_Send");
}
inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  alpaca_oracle_mpi::point_to_point("MPI_Recv");
}
inline int MPI_Isend(void const *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  alpaca_oracle_mpi::point_to_point("MPI_Isend");
}
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  alpaca_oracle_mpi::point_to_point("MPI_Irecv");
}
inline int MPI_Waitall(int count, MPI_Request *, MPI_Status *) {
  if (count != 0) alpaca_oracle_mpi::point_to_point("MPI_Waitall");
  return MPI_SUCCESS;
}

#endif /* ALPACA_ORACLE_MPI_SHIM_H */
