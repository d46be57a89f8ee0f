// MPI stand-in for the host-compiled reference solver (test infrastructure
// only).
//
// Ranks are processes started by the caller with NMHD_REF_RANK (this rank) and
// NMHD_REF_NRANKS (world size, default 1) in the environment.  Messages to the
// own rank stay in memory; messages to other ranks and the contributions to
// collectives go through files in the directory NMHD_REF_MAILBOX, each written
// under a temporary name and renamed into place, so a reader sees whole files
// only.  Sends are buffered (complete at once); a receive completes in
// MPI_Wait, which polls for the matching file.  Every wait gives up after
// NMHD_REF_MPI_TIMEOUT seconds (default 600) and aborts the process.
//
// With one rank the reference's halo exchange (MHDSolver::communicate,
// src/library/mhd_solver.inlrb:283-493) sends every message to itself, which is
// exactly its single-box shearing-periodic boundary; with P ranks along Y it is
// the reference's radial slab decomposition.
#pragma once
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; };

// datatype codes: low byte = size in bytes, bit 8 set for integers
#define MPI_COMM_WORLD 0
#define MPI_REAL 4
#define MPI_FLOAT 4
#define MPI_DOUBLE_PRECISION 8
#define MPI_DOUBLE 8
#define MPI_INT 0x104
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_SUCCESS 0

namespace nmhd_mpi_stub {

struct Recv { void *buf; int bytes; int source; int tag; };

struct State {
  int rank = 0, size = 1;
  std::string box;
  double timeout = 600.0;
  long collective = 0;
  std::map<int, Recv> recvs;                 // request id -> posted receive
  std::map<long long, std::vector<char>> self;  // tag -> message to self
  int next_req = 1;
  State() {
    if (const char *r = std::getenv("NMHD_REF_RANK")) rank = std::atoi(r);
    if (const char *n = std::getenv("NMHD_REF_NRANKS")) size = std::atoi(n);
    if (const char *b = std::getenv("NMHD_REF_MAILBOX")) box = b;
    if (const char *t = std::getenv("NMHD_REF_MPI_TIMEOUT")) timeout = std::atof(t);
    if (size < 1) size = 1;
    if (size > 1 && box.empty()) {
      std::fprintf(stderr, "mpi stub: NMHD_REF_MAILBOX must be set for %d ranks\n", size);
      std::abort();
    }
  }
};
inline State &st() { static State s; return s; }

inline int type_bytes(MPI_Datatype t) { return t & 0xff; }

inline void put_file(const std::string &name, const void *data, size_t bytes) {
  const std::string tmp = name + ".tmp";
  FILE *fp = std::fopen(tmp.c_str(), "wb");
  if (!fp || std::fwrite(data, 1, bytes, fp) != bytes || std::fclose(fp) != 0 ||
      std::rename(tmp.c_str(), name.c_str()) != 0) {
    std::fprintf(stderr, "mpi stub: cannot write %s\n", name.c_str());
    std::abort();
  }
}

// Waits (bounded) for `name`, reads `bytes` bytes of it; removes it if asked.
inline void take_file(const std::string &name, void *data, size_t bytes, bool remove) {
  const long polls = (long)(st().timeout * 2000.0);
  for (long i = 0;; ++i) {
    FILE *fp = std::fopen(name.c_str(), "rb");
    if (fp) {
      const size_t got = std::fread(data, 1, bytes, fp);
      std::fclose(fp);
      if (got != bytes) {
        std::fprintf(stderr, "mpi stub: short message %s\n", name.c_str());
        std::abort();
      }
      if (remove) std::remove(name.c_str());
      return;
    }
    if (i >= polls) {
      std::fprintf(stderr, "mpi stub: rank %d timed out waiting for %s\n", st().rank, name.c_str());
      std::abort();
    }
    usleep(500);
  }
}

inline std::string msg_name(int src, int dst, int tag) {
  char b[96];
  std::snprintf(b, sizeof b, "/m_%d_%d_%d", src, dst, tag);
  return st().box + b;
}

template <class T>
void reduce(T *acc, const T *v, int n, MPI_Op op) {
  for (int i = 0; i < n; ++i) {
    if (op == MPI_MIN) acc[i] = v[i] < acc[i] ? v[i] : acc[i];
    else if (op == MPI_MAX) acc[i] = v[i] > acc[i] ? v[i] : acc[i];
    else acc[i] = acc[i] + v[i];
  }
}

}  // namespace nmhd_mpi_stub

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = nmhd_mpi_stub::st().size; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = nmhd_mpi_stub::st().rank; return 0; }

static inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm,
                            MPI_Request *req) {
  nmhd_mpi_stub::State &s = nmhd_mpi_stub::st();
  const int id = s.next_req++;
  s.recvs[id] = nmhd_mpi_stub::Recv{buf, count * nmhd_mpi_stub::type_bytes(t), source, tag};
  *req = id;
  return 0;
}

static inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm,
                            MPI_Request *req) {
  nmhd_mpi_stub::State &s = nmhd_mpi_stub::st();
  const size_t bytes = (size_t)count * nmhd_mpi_stub::type_bytes(t);
  if (dest == s.rank) {
    const char *p = (const char *)buf;
    s.self[tag] = std::vector<char>(p, p + bytes);
  } else {
    nmhd_mpi_stub::put_file(nmhd_mpi_stub::msg_name(s.rank, dest, tag), buf, bytes);
  }
  *req = 0;  // buffered: complete
  return 0;
}

static inline int MPI_Wait(MPI_Request *req, MPI_Status *) {
  nmhd_mpi_stub::State &s = nmhd_mpi_stub::st();
  auto it = s.recvs.find(*req);
  if (it == s.recvs.end()) return 0;  // a send
  const nmhd_mpi_stub::Recv r = it->second;
  s.recvs.erase(it);
  if (r.source == s.rank) {
    auto m = s.self.find(r.tag);
    if (m == s.self.end() || (int)m->second.size() < r.bytes) {
      std::fprintf(stderr, "mpi stub: no message to self with tag %d\n", r.tag);
      std::abort();
    }
    std::memcpy(r.buf, m->second.data(), r.bytes);
    s.self.erase(m);
  } else {
    nmhd_mpi_stub::take_file(nmhd_mpi_stub::msg_name(r.source, s.rank, r.tag), r.buf, r.bytes, true);
  }
  return 0;
}

// Every rank writes its contribution to collective k; every rank reads all
// of them and reduces them in rank order, so all ranks get the same result.
static inline int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op op, MPI_Comm) {
  nmhd_mpi_stub::State &s = nmhd_mpi_stub::st();
  const size_t bytes = (size_t)count * nmhd_mpi_stub::type_bytes(t);
  if (s.size == 1) {
    std::memcpy(out, in, bytes);
    return 0;
  }
  const long k = s.collective++;
  char b[96];
  std::snprintf(b, sizeof b, "/c_%ld_%d", k, s.rank);
  nmhd_mpi_stub::put_file(s.box + b, in, bytes);
  std::vector<char> acc(bytes), v(bytes);
  for (int r = 0; r < s.size; ++r) {
    std::snprintf(b, sizeof b, "/c_%ld_%d", k, r);
    nmhd_mpi_stub::take_file(s.box + b, r == 0 ? acc.data() : v.data(), bytes, false);
    if (r == 0) continue;
    if (t == MPI_DOUBLE) nmhd_mpi_stub::reduce((double *)acc.data(), (const double *)v.data(), count, op);
    else if (t == MPI_FLOAT) nmhd_mpi_stub::reduce((float *)acc.data(), (const float *)v.data(), count, op);
    else nmhd_mpi_stub::reduce((int *)acc.data(), (const int *)v.data(), count, op);
  }
  std::memcpy(out, acc.data(), bytes);
  return 0;
}

static inline int MPI_Barrier(MPI_Comm c) {
  int one = 1, all = 0;
  return MPI_Allreduce(&one, &all, 1, MPI_INT, MPI_SUM, c);
}
