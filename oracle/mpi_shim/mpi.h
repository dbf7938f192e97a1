/*
 * Serial MPI stand-in for compiling the reference sbd headers at world size 1.
 *
 * TEST INFRASTRUCTURE ONLY: this header is used by the oracle recipe
 * (oracle/Makefile) to build the unmodified reference library
 * (include/sbd/sbd.h of walkup/sbd-ykt) into oracle/_ref/ as a CPU checker.
 * It is never linked into the product library.
 *
 * Semantics at one rank:
 *   - every communicator has size 1 and rank 0; MPI_Comm_split returns a comm;
 *   - MPI_Allreduce / MPI_Reduce copy send -> recv (a sum over one rank);
 *   - MPI_Bcast is a no-op;
 *   - point-to-point to self (MPI_Isend/Irecv/Send/Recv): a send copies its
 *     buffer into a per-tag queue; a receive takes the oldest message with
 *     that tag (or registers itself and is filled by the next matching send).
 *     The reference's ring slide (framework/mpi_utility.h:441-515) sends to
 *     itself at world size 1 and relies on this;
 *   - MPI_Waitall / MPI_Barrier are no-ops.
 */
#ifndef SBDX_ORACLE_MPI_SHIM_H
#define SBDX_ORACLE_MPI_SHIM_H

#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <deque>
#include <map>
#include <vector>

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

typedef int MPI_Comm;
typedef int MPI_Datatype; /* value = element size in bytes */
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 0
#define MPI_SUCCESS 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_C_BOOL 1
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_UNSIGNED_LONG 8
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_LONG 8
#define MPI_DOUBLE 8
#define MPI_CXX_FLOAT_COMPLEX 8
#define MPI_CXX_DOUBLE_COMPLEX 16
#define MPI_C_DOUBLE_COMPLEX 16

namespace sbdx_mpi_shim {
struct PendingRecv { void* buf; size_t bytes; };
inline std::map<int, std::deque<std::vector<char>>>& sends() {
  static std::map<int, std::deque<std::vector<char>>> q; return q;
}
inline std::map<int, std::deque<PendingRecv>>& recvs() {
  static std::map<int, std::deque<PendingRecv>> q; return q;
}
inline void post_send(const void* buf, size_t bytes, int tag) {
  auto& r = recvs()[tag];
  if (!r.empty()) {
    PendingRecv p = r.front(); r.pop_front();
    std::memcpy(p.buf, buf, bytes < p.bytes ? bytes : p.bytes);
    return;
  }
  std::vector<char> m(bytes);
  if (bytes) std::memcpy(m.data(), buf, bytes);
  sends()[tag].push_back(std::move(m));
}
inline void post_recv(void* buf, size_t bytes, int tag) {
  auto& s = sends()[tag];
  if (!s.empty()) {
    std::vector<char> m = std::move(s.front()); s.pop_front();
    std::memcpy(buf, m.data(), m.size() < bytes ? m.size() : bytes);
    return;
  }
  recvs()[tag].push_back(PendingRecv{buf, bytes});
}
}  // namespace sbdx_mpi_shim

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Init_thread(int*, char***, int req, int* prov) { if (prov) *prov = req; return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm* out) { *out = 0; return 0; }
inline int MPI_Comm_free(MPI_Comm*) { return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::fprintf(stderr, "MPI_Abort(%d)\n", code); std::exit(code); }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r && n > 0) std::memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Allreduce_c(const void* s, void* r, long long n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r && n > 0) std::memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r && n > 0) std::memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* q) {
  sbdx_mpi_shim::post_send(b, (size_t)n * (size_t)t, tag); if (q) *q = 0; return 0;
}
inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* q) {
  sbdx_mpi_shim::post_recv(b, (size_t)n * (size_t)t, tag); if (q) *q = 0; return 0;
}
inline int MPI_Isend_c(const void* b, long long n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* q) {
  sbdx_mpi_shim::post_send(b, (size_t)n * (size_t)t, tag); if (q) *q = 0; return 0;
}
inline int MPI_Irecv_c(void* b, long long n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* q) {
  sbdx_mpi_shim::post_recv(b, (size_t)n * (size_t)t, tag); if (q) *q = 0; return 0;
}
inline int MPI_Send(const void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm) {
  sbdx_mpi_shim::post_send(b, (size_t)n * (size_t)t, tag); return 0;
}
inline int MPI_Recv(void* b, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Status*) {
  sbdx_mpi_shim::post_recv(b, (size_t)n * (size_t)t, tag); return 0;
}
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }

#endif
