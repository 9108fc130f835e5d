// Single-rank MPI stand-in: TEST INFRASTRUCTURE ONLY.
//
// This header lets the reference's header-only TPB solver (sbd-pub, include/sbd/...) be
// compiled unchanged on a host without an MPI installation, so that its own CPU path can
// serve as the checker for this repository's GPU path.  Every communicator has exactly one
// rank: collectives copy send buffers to receive buffers, broadcasts do nothing, and
// point-to-point messages to self are buffered in a mailbox and matched by (comm, tag).
// It implements only the MPI-3 subset that the reference names (MPI_VERSION is 3 so the
// large-count `_c` calls are compiled out, mpi_utility.h:505,519,538,597,677).
// Nothing in the product library includes or links this file.
#ifndef SBD_ORACLE_MPI_SHIM_H
#define SBD_ORACLE_MPI_SHIM_H

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <vector>
#include <complex>

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef long MPI_Aint;
typedef int MPI_Request;
struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  size_t shim_bytes;
};

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_REQUEST_NULL (-1)
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

// operations (values only need to be distinct; a single rank never combines data)
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4

// predefined datatypes: the handle indexes the size table below
#define MPI_CHAR 1
#define MPI_BYTE 2
#define MPI_INT 3
#define MPI_UNSIGNED 4
#define MPI_UNSIGNED_CHAR 5
#define MPI_UNSIGNED_SHORT 6
#define MPI_UNSIGNED_LONG 7
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_FLOAT 9
#define MPI_DOUBLE 10
#define MPI_CXX_FLOAT_COMPLEX 11
#define MPI_CXX_DOUBLE_COMPLEX 12
#define MPI_C_BOOL 13
#define MPI_INT32_T 14
#define MPI_UINT32_T 15
#define MPI_UINT64_T 16
#define MPI_INT64_T 17
#define MPI_LONG 18
#define MPI_LONG_LONG 19
#define MPI_SHORT 20

namespace mpi_shim {

inline std::vector<size_t> &type_sizes() {
  static std::vector<size_t> sizes = {
      0,
      sizeof(char),
      1,
      sizeof(int),
      sizeof(unsigned),
      sizeof(unsigned char),
      sizeof(unsigned short),
      sizeof(unsigned long),
      sizeof(unsigned long long),
      sizeof(float),
      sizeof(double),
      sizeof(std::complex<float>),
      sizeof(std::complex<double>),
      sizeof(bool),
      sizeof(int32_t),
      sizeof(uint32_t),
      sizeof(uint64_t),
      sizeof(int64_t),
      sizeof(long),
      sizeof(long long),
      sizeof(short),
  };
  return sizes;
}

inline size_t bytes(long long count, MPI_Datatype t) {
  auto &s = type_sizes();
  if (t <= 0 || static_cast<size_t>(t) >= s.size()) {
    std::fprintf(stderr, "mpi_shim: unknown datatype %d\n", t);
    std::abort();
  }
  return static_cast<size_t>(count) * s[t];
}

struct Message {
  MPI_Comm comm;
  int tag;
  std::vector<char> data;
};

struct PendingRecv {
  bool active = false;
  bool done = false;
  void *buf = nullptr;
  size_t cap = 0;
  MPI_Comm comm = 0;
  int tag = 0;
  size_t got = 0;
};

inline std::deque<Message> &mailbox() {
  static std::deque<Message> m;
  return m;
}

inline std::vector<PendingRecv> &recvs() {
  static std::vector<PendingRecv> r;
  return r;
}

inline int &next_comm() {
  static int c = 16;
  return c;
}

inline bool try_match(PendingRecv &r) {
  auto &mb = mailbox();
  for (auto it = mb.begin(); it != mb.end(); ++it) {
    if (it->comm == r.comm && (r.tag == MPI_ANY_TAG || it->tag == r.tag)) {
      if (it->data.size() > r.cap) {
        std::fprintf(stderr, "mpi_shim: message truncated (%zu > %zu)\n", it->data.size(), r.cap);
        std::abort();
      }
      if (!it->data.empty()) std::memcpy(r.buf, it->data.data(), it->data.size());
      r.got = it->data.size();
      r.done = true;
      mb.erase(it);
      return true;
    }
  }
  return false;
}

inline void post_send(const void *buf, size_t nbytes, int tag, MPI_Comm comm) {
  Message m;
  m.comm = comm;
  m.tag = tag;
  m.data.resize(nbytes);
  if (nbytes) std::memcpy(m.data.data(), buf, nbytes);
  mailbox().push_back(std::move(m));
}

inline void copy_unless_in_place(const void *sendbuf, void *recvbuf, size_t nbytes) {
  if (sendbuf == MPI_IN_PLACE || sendbuf == recvbuf || nbytes == 0) return;
  std::memmove(recvbuf, sendbuf, nbytes);
}

}  // namespace mpi_shim

inline int MPI_Init_thread(int *, char ***, int required, int *provided) {
  if (provided) *provided = required;
  return MPI_SUCCESS;
}
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) {
  std::fprintf(stderr, "MPI_Abort(%d)\n", code);
  std::exit(code == 0 ? 1 : code);
}
inline int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
inline int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *out) {
  *out = mpi_shim::next_comm()++;
  return MPI_SUCCESS;
}
inline int MPI_Comm_free(MPI_Comm *c) {
  *c = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

inline int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op,
                         MPI_Comm) {
  mpi_shim::copy_unless_in_place(sendbuf, recvbuf, mpi_shim::bytes(count, t));
  return MPI_SUCCESS;
}
inline int MPI_Exscan(const void *, void *recvbuf, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  // rank 0's result is undefined in MPI; the reference overwrites it or ignores it.
  std::memset(recvbuf, 0, mpi_shim::bytes(count, t));
  return MPI_SUCCESS;
}
inline int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int,
                         MPI_Datatype, MPI_Comm) {
  mpi_shim::copy_unless_in_place(sendbuf, recvbuf, mpi_shim::bytes(scount, st));
  return MPI_SUCCESS;
}
inline int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf,
                          const int *, const int *displs, MPI_Datatype rt, MPI_Comm) {
  char *dst = static_cast<char *>(recvbuf) + mpi_shim::bytes(displs[0], rt);
  mpi_shim::copy_unless_in_place(sendbuf, dst, mpi_shim::bytes(scount, st));
  return MPI_SUCCESS;
}
inline int MPI_Gather(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int,
                      MPI_Datatype, int, MPI_Comm) {
  mpi_shim::copy_unless_in_place(sendbuf, recvbuf, mpi_shim::bytes(scount, st));
  return MPI_SUCCESS;
}
inline int MPI_Gatherv(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf,
                       const int *, const int *displs, MPI_Datatype rt, int, MPI_Comm) {
  char *dst = static_cast<char *>(recvbuf) + mpi_shim::bytes(displs[0], rt);
  mpi_shim::copy_unless_in_place(sendbuf, dst, mpi_shim::bytes(scount, st));
  return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype st, void *recvbuf, int,
                        MPI_Datatype, MPI_Comm) {
  mpi_shim::copy_unless_in_place(sendbuf, recvbuf, mpi_shim::bytes(scount, st));
  return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void *sendbuf, const int *scounts, const int *sdispls,
                         MPI_Datatype st, void *recvbuf, const int *, const int *rdispls,
                         MPI_Datatype rt, MPI_Comm) {
  const char *src = static_cast<const char *>(sendbuf) + mpi_shim::bytes(sdispls[0], st);
  char *dst = static_cast<char *>(recvbuf) + mpi_shim::bytes(rdispls[0], rt);
  mpi_shim::copy_unless_in_place(src, dst, mpi_shim::bytes(scounts[0], st));
  return MPI_SUCCESS;
}

inline int MPI_Send(const void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm comm) {
  mpi_shim::post_send(buf, mpi_shim::bytes(count, t), tag, comm);
  return MPI_SUCCESS;
}
inline int MPI_Recv(void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm comm,
                    MPI_Status *status) {
  mpi_shim::PendingRecv r;
  r.active = true;
  r.buf = buf;
  r.cap = mpi_shim::bytes(count, t);
  r.comm = comm;
  r.tag = tag;
  if (!mpi_shim::try_match(r)) {
    std::fprintf(stderr, "mpi_shim: blocking receive with no matching send to self\n");
    std::abort();
  }
  if (status) {
    status->MPI_SOURCE = 0;
    status->MPI_TAG = tag;
    status->MPI_ERROR = 0;
    status->shim_bytes = r.got;
  }
  return MPI_SUCCESS;
}
inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm comm,
                     MPI_Request *req) {
  mpi_shim::post_send(buf, mpi_shim::bytes(count, t), tag, comm);
  *req = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}
inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm comm,
                     MPI_Request *req) {
  auto &rs = mpi_shim::recvs();
  mpi_shim::PendingRecv r;
  r.active = true;
  r.buf = buf;
  r.cap = mpi_shim::bytes(count, t);
  r.comm = comm;
  r.tag = tag;
  mpi_shim::try_match(r);
  rs.push_back(r);
  *req = static_cast<int>(rs.size()) - 1;
  return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request *req, MPI_Status *status) {
  if (*req == MPI_REQUEST_NULL) return MPI_SUCCESS;
  auto &r = mpi_shim::recvs()[*req];
  if (!r.done && !mpi_shim::try_match(r)) {
    std::fprintf(stderr, "mpi_shim: wait on a receive with no matching send to self\n");
    std::abort();
  }
  if (status) {
    status->MPI_SOURCE = 0;
    status->MPI_TAG = r.tag;
    status->MPI_ERROR = 0;
    status->shim_bytes = r.got;
  }
  r.active = false;
  *req = MPI_REQUEST_NULL;
  // drop fully-consumed receive records so the table does not grow without bound
  auto &rs = mpi_shim::recvs();
  while (!rs.empty() && !rs.back().active) rs.pop_back();
  return MPI_SUCCESS;
}
inline int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *statuses) {
  for (int i = 0; i < n; ++i) MPI_Wait(&reqs[i], statuses ? &statuses[i] : MPI_STATUS_IGNORE);
  return MPI_SUCCESS;
}

inline int MPI_Get_address(const void *p, MPI_Aint *a) {
  *a = reinterpret_cast<MPI_Aint>(p);
  return MPI_SUCCESS;
}
inline int MPI_Type_create_struct(int n, const int *blocklens, const MPI_Aint *disps,
                                  const MPI_Datatype *types, MPI_Datatype *out) {
  size_t extent = 0;
  for (int i = 0; i < n; ++i) {
    size_t end = static_cast<size_t>(disps[i]) + mpi_shim::bytes(blocklens[i], types[i]);
    if (end > extent) extent = end;
  }
  extent = (extent + 7) & ~static_cast<size_t>(7);
  auto &s = mpi_shim::type_sizes();
  s.push_back(extent);
  *out = static_cast<int>(s.size()) - 1;
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *t) {
  *t = 0;
  return MPI_SUCCESS;
}

#endif  // SBD_ORACLE_MPI_SHIM_H
