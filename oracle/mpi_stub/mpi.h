/*
 * Single-rank stand-in for <mpi.h>.
 *
 * Test infrastructure only: it lets the reference sbd headers compile and run
 * at MPI world size 1 in a container that has no MPI installation.  Every
 * communicator has exactly one rank (rank 0).  Collectives copy send buffers to
 * receive buffers; point-to-point messages a rank sends to itself go through a
 * tag-keyed mailbox, which is what the reference's ring shift (Mpi2dSlide,
 * include/sbd/framework/mpi_utility.h:437-502) does at world size 1.
 */
#ifndef SBD_ORACLE_MPI_STUB_H
#define SBD_ORACLE_MPI_STUB_H

#include <cstddef>
#include <cstring>
#include <map>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_THREAD_FUNNELED 1
#define MPI_SUCCESS 0
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

/* Datatype handles encode the element size in bytes. */
#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_C_BOOL 1
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_UNSIGNED_LONG 8
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_CXX_FLOAT_COMPLEX 8
#define MPI_CXX_DOUBLE_COMPLEX 16

namespace sbd_mpi_stub {
struct Pending { void* buf; int bytes; int tag; };
inline std::map<int, std::vector<std::vector<char>>>& mailbox() {
  static std::map<int, std::vector<std::vector<char>>> m;
  return m;
}
inline int next_request() {
  static int r = 0;
  return ++r;
}
inline std::map<int, Pending>& requests() {
  static std::map<int, Pending> q;
  return q;
}
inline void deliver(int bytes, int tag, void* buf) {
  auto& box = mailbox()[tag];
  if (!box.empty()) {
    std::vector<char> msg = box.front();
    box.erase(box.begin());
    std::memcpy(buf, msg.data(), msg.size() < (size_t)bytes ? msg.size() : (size_t)bytes);
  }
}
}  // namespace sbd_mpi_stub

inline int MPI_Init_thread(int*, char***, int, int* provided) { *provided = MPI_THREAD_FUNNELED; return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm* out) { *out = 0; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r && n > 0) std::memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != r && n > 0) std::memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Send(const void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm) {
  const char* p = static_cast<const char*>(buf);
  sbd_mpi_stub::mailbox()[tag].emplace_back(p, p + (size_t)n * (size_t)t);
  return 0;
}
inline int MPI_Recv(void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Status*) {
  sbd_mpi_stub::deliver(n * t, tag, buf);
  return 0;
}
inline int MPI_Isend(const void* buf, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request* req) {
  MPI_Send(buf, n, t, dst, tag, c);
  *req = 0;
  return 0;
}
inline int MPI_Irecv(void* buf, int n, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Request* req) {
  int id = sbd_mpi_stub::next_request();
  sbd_mpi_stub::requests()[id] = sbd_mpi_stub::Pending{buf, n * t, tag};
  *req = id;
  return 0;
}
inline int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status*) {
  for (int i = 0; i < n; i++) {
    auto it = sbd_mpi_stub::requests().find(reqs[i]);
    if (it != sbd_mpi_stub::requests().end()) {
      sbd_mpi_stub::deliver(it->second.bytes, it->second.tag, it->second.buf);
      sbd_mpi_stub::requests().erase(it);
    }
  }
  return 0;
}

#endif
