/* Test infrastructure: a single-process stand-in for the MPI calls that the
 * reference's vlp4d_mpi OpenMP sources make, so that they compile and run as
 * one rank without an MPI library.
 *
 * Semantics for one process (rank 0 of a world of size 1):
 *  - reductions (MPI_Reduce, MPI_Allreduce) copy the send buffer into the
 *    receive buffer (the sum over one rank);
 *  - point-to-point messages can only go to the process itself: MPI_Irecv
 *    posts a receive, MPI_Isend delivers into the oldest posted receive with a
 *    matching tag (non-overtaking order, as MPI guarantees between one pair of
 *    ranks), MPI_Waitall fills in the statuses;
 *  - MPI_Init, MPI_Init_thread, MPI_Barrier, MPI_Finalize do nothing.
 * Written from the MPI standard's description of these calls; it is not an
 * MPI implementation and supports nothing beyond the calls listed here. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_bytes;
} MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_SUM 1
/* Datatype handles carry their size in bytes. */
#define MPI_BYTE 1
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_DOUBLE 8

namespace oracle_mpi {
struct Posted {
  void *buf;
  int bytes;
  int tag;
  int request;
  bool done;
  int status_bytes;
};
inline Posted *posted() {
  static Posted p[4096];
  return p;
}
inline int &nposted() {
  static int n = 0;
  return n;
}
inline int &next_request() {
  static int r = 1;
  return r;
}
}  // namespace oracle_mpi

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Init_thread(int *, char ***, int required, int *provided) {
  *provided = required;
  return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
  if (send != recv) memmove(recv, send, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  if (send != recv) memmove(recv, send, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}
static inline int MPI_Irecv(void *buf, int count, MPI_Datatype type, int, int tag, MPI_Comm, MPI_Request *req) {
  using namespace oracle_mpi;
  if (nposted() >= 4096) abort();
  Posted &p = posted()[nposted()++];
  p.buf = buf;
  p.bytes = count * type;
  p.tag = tag;
  p.request = next_request()++;
  p.done = false;
  p.status_bytes = 0;
  *req = p.request;
  return MPI_SUCCESS;
}
static inline int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm,
                            MPI_Request *req) {
  using namespace oracle_mpi;
  if (dest != 0) abort();
  const int bytes = count * type;
  for (int i = 0; i < nposted(); ++i) {
    Posted &p = posted()[i];
    if (!p.done && (p.tag == tag || p.tag == MPI_ANY_TAG)) {
      if (bytes > p.bytes) abort();
      memcpy(p.buf, buf, (size_t)bytes);
      p.done = true;
      p.status_bytes = bytes;
      *req = 0; /* a send to oneself completes at once */
      return MPI_SUCCESS;
    }
  }
  abort(); /* no receive posted: would deadlock under real MPI too */
}
static inline int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *stats) {
  using namespace oracle_mpi;
  for (int k = 0; k < count; ++k) {
    if (stats) {
      stats[k].MPI_SOURCE = 0;
      stats[k].MPI_ERROR = MPI_SUCCESS;
      stats[k].MPI_TAG = 0;
      stats[k].count_bytes = 0;
    }
    if (reqs[k] == 0) continue;
    for (int i = 0; i < nposted(); ++i) {
      Posted &p = posted()[i];
      if (p.request == reqs[k]) {
        if (!p.done) abort(); /* a receive nothing will ever match */
        if (stats) {
          stats[k].MPI_TAG = p.tag;
          stats[k].count_bytes = p.status_bytes;
        }
      }
    }
  }
  /* Drop the completed receives. */
  int w = 0;
  for (int i = 0; i < nposted(); ++i)
    if (!posted()[i].done) posted()[w++] = posted()[i];
  nposted() = w;
  return MPI_SUCCESS;
}

#endif
