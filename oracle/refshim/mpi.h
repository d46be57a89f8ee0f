// Single-rank MPI stand-in for the host-compiled reference solver (test
// infrastructure only).
//
// With one rank and kParallelSizeY == 1 the reference's halo exchange
// (MHDSolver::communicate, src/library/mhd_solver.inlrb:283-493) sends every
// message to itself, which is exactly its single-box shearing-periodic
// boundary.  Irecv records the receive buffer under its tag; the Isend with the
// same tag copies into it; Wait/Barrier do nothing; Allreduce copies.
#pragma once
#include <cstring>
#include <map>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };

#define MPI_COMM_WORLD 0
#define MPI_REAL 4
#define MPI_FLOAT 4
#define MPI_DOUBLE_PRECISION 8
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_SUCCESS 0

namespace nmhd_mpi_stub {
struct Pending { void *buf; int bytes; };
inline std::map<int, Pending> &pending() { static std::map<int, Pending> p; return p; }
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request *req) {
  nmhd_mpi_stub::Pending p = {buf, count * t};
  nmhd_mpi_stub::pending()[tag] = p;
  *req = tag;
  return 0;
}
static inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request *req) {
  nmhd_mpi_stub::Pending &p = nmhd_mpi_stub::pending()[tag];
  int n = count * t < p.bytes ? count * t : p.bytes;
  std::memcpy(p.buf, buf, n);
  nmhd_mpi_stub::pending().erase(tag);
  *req = tag;
  return 0;
}
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  std::memcpy(out, in, count * t);
  return 0;
}
