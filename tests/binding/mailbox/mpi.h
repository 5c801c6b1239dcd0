/*
 * Two-party stand-in for <mpi.h>: a master (world rank 0) and one worker (world rank 1) that
 * run as two threads of one process, for the test of the GPU sub-lattice binding.
 *
 * Test infrastructure, not product code.  MPI_COMM_WORLD joins the two parties; the workers'
 * communicator (MAILBOX_WORKER_COMM) holds the worker alone.  A thread says which party it is
 * with mailbox::set_rank.  Collectives on the world move bytes through two FIFO channels:
 * down (from the root to the other party: broadcast, scatter) and up (to the root: gather);
 * a receive waits for its bytes with a time limit and throws std::runtime_error when they do
 * not come.  Barriers return at once: every transfer is ordered by its channel.  Packing is a
 * plain byte copy.  Reductions over both parties are not provided (the code under test makes
 * none).
 */
#ifndef MAILBOX_MPI_H
#define MAILBOX_MPI_H

#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <stdexcept>
#include <string>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Op;
typedef int MPI_Group;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; int count; } MPI_Status;

#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MAILBOX_WORKER_COMM ((MPI_Comm)2)
#define MPI_GROUP_NULL ((MPI_Group)0)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)5)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_LONG ((MPI_Datatype)9)
#define MPI_UNSIGNED ((MPI_Datatype)10)
#define MPI_UNSIGNED_LONG ((MPI_Datatype)11)
#define MPI_BYTE ((MPI_Datatype)12)
#define MPI_PACKED ((MPI_Datatype)13)
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_MAX_PROCESSOR_NAME 64

namespace mailbox {

struct State {
  std::mutex m;
  std::condition_variable cv;
  std::deque<char> down, up;
  std::string aborted;  // set when a party has failed: every later wait throws at once
  double wait_s = 60.0;
};

inline State& state() {
  static State s;
  return s;
}

inline thread_local int world_rank = 0;

inline void set_rank(int r) { world_rank = r; }

inline void reset() {
  State& s = state();
  std::lock_guard<std::mutex> g(s.m);
  s.down.clear();
  s.up.clear();
  s.aborted.clear();
}

inline void abort_all(const std::string& why) {
  State& s = state();
  {
    std::lock_guard<std::mutex> g(s.m);
    s.aborted = why.empty() ? "failed" : why;
  }
  s.cv.notify_all();
}

inline size_t pending() {
  State& s = state();
  std::lock_guard<std::mutex> g(s.m);
  return s.down.size() + s.up.size();
}

inline void push(std::deque<char>& q, const void* p, size_t n) {
  State& s = state();
  {
    std::lock_guard<std::mutex> g(s.m);
    const char* c = static_cast<const char*>(p);
    q.insert(q.end(), c, c + n);
  }
  s.cv.notify_all();
}

inline void pop(std::deque<char>& q, void* p, size_t n, const char* what) {
  State& s = state();
  std::unique_lock<std::mutex> g(s.m);
  const auto limit = std::chrono::steady_clock::now() + std::chrono::duration<double>(s.wait_s);
  while (q.size() < n) {
    if (!s.aborted.empty()) throw std::runtime_error(std::string("mailbox: ") + what + ": the other party failed");
    if (s.cv.wait_until(g, limit) == std::cv_status::timeout && q.size() < n)
      throw std::runtime_error(std::string("mailbox: ") + what + " waited too long for its data (rank " +
                               std::to_string(world_rank) + ")");
  }
  char* c = static_cast<char*>(p);
  for (size_t i = 0; i < n; ++i) c[i] = q[i];
  q.erase(q.begin(), q.begin() + n);
}

inline int type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_PACKED: return 1;
    case MPI_INT: case MPI_FLOAT: case MPI_UNSIGNED: return 4;
    case MPI_DOUBLE: case MPI_LONG: case MPI_UNSIGNED_LONG: return 8;
    default: return t > 16 ? t - 16 : 1;  /* derived types carry their extent: 16 + bytes */
  }
}

inline bool shared(MPI_Comm c) { return c == MPI_COMM_WORLD; }
inline int rank_in(MPI_Comm c) { return shared(c) ? world_rank : 0; }

}  // namespace mailbox

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Initialized(int* f) { *f = 1; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); return MPI_SUCCESS; }
static inline double MPI_Wtime() {
  struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { *r = mailbox::rank_in(c); return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { *s = mailbox::shared(c) ? 2 : 1; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm*) { return MPI_SUCCESS; }
static inline int MPI_Comm_group(MPI_Comm c, MPI_Group* g) { *g = c; return MPI_SUCCESS; }
static inline int MPI_Comm_create(MPI_Comm, MPI_Group g, MPI_Comm* n) { *n = g; return MPI_SUCCESS; }
static inline int MPI_Group_size(MPI_Group g, int* s) { return MPI_Comm_size(g, s); }
static inline int MPI_Group_rank(MPI_Group g, int* r) { return MPI_Comm_rank(g, r); }
static inline int MPI_Group_incl(MPI_Group, int, const int*, MPI_Group* n) { *n = MAILBOX_WORKER_COMM; return MPI_SUCCESS; }
static inline int MPI_Group_excl(MPI_Group, int, const int*, MPI_Group* n) { *n = MAILBOX_WORKER_COMM; return MPI_SUCCESS; }
static inline int MPI_Group_free(MPI_Group*) { return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Get_address(const void* p, MPI_Aint* a) { *a = (MPI_Aint)p; return MPI_SUCCESS; }
static inline int MPI_Address(void* p, MPI_Aint* a) { *a = (MPI_Aint)p; return MPI_SUCCESS; }

/* The workers' Cartesian grid: one worker, no neighbours. */
static inline int MPI_Dims_create(int, int ndims, int* dims) {
  for (int i = 0; i < ndims; ++i) if (dims[i] == 0) dims[i] = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Cart_create(MPI_Comm c, int, const int*, const int*, int, MPI_Comm* n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords) {
  for (int i = 0; i < maxdims; ++i) coords[i] = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Cart_rank(MPI_Comm, const int*, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Cart_shift(MPI_Comm, int, int, int* src, int* dst) {
  *src = MPI_PROC_NULL; *dst = MPI_PROC_NULL; return MPI_SUCCESS;
}

/* Point to point: between the parties through the channels, MPI_PROC_NULL ignored. */
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int dst, int, MPI_Comm c) {
  if (dst == MPI_PROC_NULL || !mailbox::shared(c)) return MPI_SUCCESS;
  mailbox::push(mailbox::world_rank == 0 ? mailbox::state().down : mailbox::state().up, b, (size_t)n * mailbox::type_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status* s) {
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  if (src == MPI_PROC_NULL || !mailbox::shared(c)) return MPI_SUCCESS;
  mailbox::pop(mailbox::world_rank == 0 ? mailbox::state().up : mailbox::state().down, b,
               (size_t)n * mailbox::type_size(t), "MPI_Recv");
  if (s) s->count = n;
  return MPI_SUCCESS;
}
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request* r) {
  *r = 0; return MPI_Send(b, n, t, dst, tag, c);
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int src, int, MPI_Comm c, MPI_Request* r) {
  *r = 0;
  if (src != MPI_PROC_NULL && mailbox::shared(c)) throw std::runtime_error("mailbox: MPI_Irecv between the parties");
  return MPI_SUCCESS;
}
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int dst, int, void*, int, MPI_Datatype,
                               int src, int tag, MPI_Comm c, MPI_Status* s) {
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  if ((dst != MPI_PROC_NULL || src != MPI_PROC_NULL) && mailbox::shared(c))
    throw std::runtime_error("mailbox: MPI_Sendrecv between the parties");
  return MPI_SUCCESS;
}
static inline int MPI_Sendrecv_replace(void* b, int n, MPI_Datatype t, int dst, int st, int src, int rt, MPI_Comm c,
                                       MPI_Status* s) {
  return MPI_Sendrecv(b, n, t, dst, st, b, n, t, src, rt, c, s);
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status* s) {
  if (src != MPI_PROC_NULL && mailbox::shared(c)) throw std::runtime_error("mailbox: MPI_Probe between the parties");
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  return MPI_SUCCESS;
}
static inline int MPI_Get_count(const MPI_Status* s, MPI_Datatype, int* c) { *c = s ? s->count : 0; return MPI_SUCCESS; }

/* Collectives.  On the workers' communicator (one rank) they are local copies. */
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  if (!mailbox::shared(c)) return MPI_SUCCESS;
  const size_t bytes = (size_t)n * mailbox::type_size(t);
  if (mailbox::world_rank == root) mailbox::push(mailbox::state().down, b, bytes);
  else mailbox::pop(mailbox::state().down, b, bytes, "MPI_Bcast");
  return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* sb, int sn, MPI_Datatype st, void* rb, int rn, MPI_Datatype rt, int root,
                             MPI_Comm c) {
  const size_t sbytes = (size_t)sn * mailbox::type_size(st);
  if (!mailbox::shared(c)) { if (sb != rb) memcpy(rb, sb, sbytes); return MPI_SUCCESS; }
  if (mailbox::world_rank != root) { mailbox::push(mailbox::state().up, sb, sbytes); return MPI_SUCCESS; }
  const size_t slot = (size_t)rn * mailbox::type_size(rt);
  memcpy((char*)rb + (size_t)root * slot, sb, sbytes);
  mailbox::pop(mailbox::state().up, (char*)rb + (size_t)(1 - root) * slot, slot, "MPI_Gather");
  return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void* sb, int sn, MPI_Datatype st, void* rb, const int* rcounts, const int* displs,
                              MPI_Datatype rt, int root, MPI_Comm c) {
  const size_t sbytes = (size_t)sn * mailbox::type_size(st);
  const size_t rsz = (size_t)mailbox::type_size(rt);
  if (!mailbox::shared(c)) { memcpy((char*)rb + (size_t)displs[0] * rsz, sb, sbytes); return MPI_SUCCESS; }
  if (mailbox::world_rank != root) { mailbox::push(mailbox::state().up, sb, sbytes); return MPI_SUCCESS; }
  memcpy((char*)rb + (size_t)displs[root] * rsz, sb, sbytes);
  const int other = 1 - root;
  mailbox::pop(mailbox::state().up, (char*)rb + (size_t)displs[other] * rsz, (size_t)rcounts[other] * rsz, "MPI_Gatherv");
  return MPI_SUCCESS;
}
static inline int MPI_Scatter(const void* sb, int sn, MPI_Datatype st, void* rb, int rn, MPI_Datatype rt, int root,
                              MPI_Comm c) {
  const size_t rbytes = (size_t)rn * mailbox::type_size(rt);
  if (!mailbox::shared(c)) { if (sb != rb) memcpy(rb, sb, rbytes); return MPI_SUCCESS; }
  if (mailbox::world_rank != root) { mailbox::pop(mailbox::state().down, rb, rbytes, "MPI_Scatter"); return MPI_SUCCESS; }
  const size_t slot = (size_t)sn * mailbox::type_size(st);
  memcpy(rb, (const char*)sb + (size_t)root * slot, rbytes);
  mailbox::push(mailbox::state().down, (const char*)sb + (size_t)(1 - root) * slot, slot);
  return MPI_SUCCESS;
}
static inline int MPI_Scatterv(const void* sb, const int* counts, const int* displs, MPI_Datatype st, void* rb, int rn,
                               MPI_Datatype rt, int root, MPI_Comm c) {
  const size_t ssz = (size_t)mailbox::type_size(st), rbytes = (size_t)rn * mailbox::type_size(rt);
  if (!mailbox::shared(c)) { memcpy(rb, (const char*)sb + (size_t)displs[0] * ssz, rbytes); return MPI_SUCCESS; }
  if (mailbox::world_rank != root) { mailbox::pop(mailbox::state().down, rb, rbytes, "MPI_Scatterv"); return MPI_SUCCESS; }
  memcpy(rb, (const char*)sb + (size_t)displs[root] * ssz, rbytes);
  const int other = 1 - root;
  mailbox::push(mailbox::state().down, (const char*)sb + (size_t)displs[other] * ssz, (size_t)counts[other] * ssz);
  return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm c) {
  if (mailbox::shared(c)) throw std::runtime_error("mailbox: MPI_Reduce over both parties");
  if (sb != rb) memcpy(rb, sb, (size_t)n * mailbox::type_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op, MPI_Comm c) {
  if (mailbox::shared(c)) throw std::runtime_error("mailbox: MPI_Allreduce over both parties");
  if (sb != rb) memcpy(rb, sb, (size_t)n * mailbox::type_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* sb, int sn, MPI_Datatype st, void* rb, int, MPI_Datatype, MPI_Comm c) {
  if (mailbox::shared(c)) throw std::runtime_error("mailbox: MPI_Allgather over both parties");
  if (sb != rb) memcpy(rb, sb, (size_t)sn * mailbox::type_size(st));
  return MPI_SUCCESS;
}

/* Packing: a byte-copy format private to this process. */
static inline int MPI_Pack_size(int n, MPI_Datatype t, MPI_Comm, int* size) { *size = n * mailbox::type_size(t); return MPI_SUCCESS; }
static inline int MPI_Pack(const void* in, int n, MPI_Datatype t, void* out, int outsize, int* pos, MPI_Comm) {
  int b = n * mailbox::type_size(t);
  if (*pos + b > outsize) return 1;
  memcpy((char*)out + *pos, in, (size_t)b); *pos += b; return MPI_SUCCESS;
}
static inline int MPI_Unpack(const void* in, int insize, int* pos, void* out, int n, MPI_Datatype t, MPI_Comm) {
  int b = n * mailbox::type_size(t);
  if (*pos + b > insize) return 1;
  memcpy(out, (const char*)in + *pos, (size_t)b); *pos += b; return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype* nt) {
  *nt = 16 + n * mailbox::type_size(old); return MPI_SUCCESS;
}
/* A struct type's extent: its last block's end, rounded up to its widest member (as MPI
 * implementations pad struct extents for alignment). */
static inline int MPI_Type_create_struct(int cnt, const int* bl, const MPI_Aint* disp, const MPI_Datatype* ts,
                                         MPI_Datatype* nt) {
  long end = 0, align = 1;
  for (int i = 0; i < cnt; ++i) {
    const long sz = mailbox::type_size(ts[i]);
    const long e = (long)(disp[i] - disp[0]) + (long)bl[i] * sz;
    if (e > end) end = e;
    if (sz <= 8 && sz > align) align = sz;
  }
  end = (end + align - 1) / align * align;
  *nt = (MPI_Datatype)(16 + end);
  return MPI_SUCCESS;
}
static inline int MPI_Type_struct(int cnt, int* bl, MPI_Aint* disp, MPI_Datatype* ts, MPI_Datatype* nt) {
  return MPI_Type_create_struct(cnt, bl, disp, ts, nt);
}
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }

#endif
