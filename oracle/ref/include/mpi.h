// ORACLE — TEST INFRASTRUCTURE ONLY.
// Single-process stand-in for the MPI API surface that Free CFD's sources use,
// so that the unmodified reference sources compile and run as ONE rank
// (rank 0 of 1).  Collectives copy the send buffer to the receive buffer;
// point-to-point calls are never reached with one rank (every exchange loop
// in the reference skips its own rank) and do nothing.
#ifndef FCFD_REF_STUB_MPI_H
#define FCFD_REF_STUB_MPI_H

#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <sys/time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };

#define MPI_COMM_WORLD 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

// Datatypes are encoded as their size in bytes (derived types: see
// MPI_Type_create_struct, never used with one rank).
static inline size_t fcfd_mpi_size(MPI_Datatype t) { return t > 0 ? (size_t)t : 0; }

// An MPI error in the single-rank build is a harness error, not an exit.
struct FcfdRefAbort : std::runtime_error {
  int code;
  explicit FcfdRefAbort(int c) : std::runtime_error("reference called MPI_Abort"), code(c) {}
};

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { throw FcfdRefAbort(code); }
static inline double MPI_Wtime() {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r) std::memmove(r, s, (size_t)n * fcfd_mpi_size(t));
  return 0;
}
static inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r) std::memmove(r, s, (size_t)sn * fcfd_mpi_size(st));
  return 0;
}
static inline int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *, const int *displs,
                                 MPI_Datatype rt, MPI_Comm) {
  char *dst = (char *)r + (size_t)displs[0] * fcfd_mpi_size(rt);
  if (s != MPI_IN_PLACE && s != dst) std::memmove(dst, s, (size_t)sn * fcfd_mpi_size(st));
  return 0;
}
static inline int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r) std::memmove(r, s, (size_t)sn * fcfd_mpi_size(st));
  return 0;
}
// Point to point: unreachable with one rank.
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int, MPI_Datatype, int, int, MPI_Comm,
                               MPI_Status *) {
  return 0;
}
static inline int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *, MPI_Datatype *t) {
  *t = 0;
  return 0;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return 0; }

#endif
