/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * own hot-path sources into the CPU oracle library (oracle/_ref).
 *
 * Test infrastructure, not product code.  Every communicator has exactly
 * one rank (rank 0, size 1); point-to-point traffic only ever targets
 * MPI_PROC_NULL (Cart_shift returns it, because a 1x1x1 Cartesian grid
 * has no neighbours); collectives degenerate to a local copy.  This is the
 * compute path of `mpirun -np 2` with one worker and mpiDimList=[1,1,1].
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <string.h>
#include <time.h>
#include <stdlib.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Op;
typedef int MPI_Group;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; int count; } MPI_Status;

#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_COMM_WORLD ((MPI_Comm)1)
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

static inline int oracle_mpi_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_PACKED: return 1;
    case MPI_INT: case MPI_FLOAT: case MPI_UNSIGNED: return 4;
    case MPI_DOUBLE: case MPI_LONG: case MPI_UNSIGNED_LONG: return 8;
    default: return t > 16 ? t - 16 : 1;  /* contiguous types: see Type_contiguous */
  }
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Initialized(int* f) { *f = 1; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); return MPI_SUCCESS; }
static inline double MPI_Wtime() {
  struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm*) { return MPI_SUCCESS; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group, MPI_Comm* n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Group_size(MPI_Group, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Group_rank(MPI_Group, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Group_incl(MPI_Group g, int, const int*, MPI_Group* n) { *n = g; return MPI_SUCCESS; }
static inline int MPI_Group_excl(MPI_Group g, int, const int*, MPI_Group* n) { *n = g; return MPI_SUCCESS; }
static inline int MPI_Group_free(MPI_Group*) { return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Get_address(const void* p, MPI_Aint* a) { *a = (MPI_Aint)p; return MPI_SUCCESS; }
static inline int MPI_Address(void* p, MPI_Aint* a) { *a = (MPI_Aint)p; return MPI_SUCCESS; }

/* Cartesian topology with every dimension of extent 1 and no neighbours. */
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

/* Point-to-point: the only partner a single rank ever has is MPI_PROC_NULL. */
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int src, int tag, MPI_Comm, MPI_Status* s) {
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  return MPI_SUCCESS;
}
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype,
                               int src, int tag, MPI_Comm, MPI_Status* s) {
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  return MPI_SUCCESS;
}
static inline int MPI_Sendrecv_replace(void*, int, MPI_Datatype, int, int, int src, int tag, MPI_Comm, MPI_Status* s) {
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  return MPI_SUCCESS;
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline int MPI_Probe(int src, int tag, MPI_Comm, MPI_Status* s) {
  if (s) { s->MPI_SOURCE = src; s->MPI_TAG = tag; s->MPI_ERROR = 0; s->count = 0; }
  return MPI_SUCCESS;
}
static inline int MPI_Get_count(const MPI_Status* s, MPI_Datatype, int* c) { *c = s ? s->count : 0; return MPI_SUCCESS; }

/* Collectives on one rank: a copy from send to receive buffer. */
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Reduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (sb != rb) memcpy(rb, sb, (size_t)n * oracle_mpi_type_size(t)); return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (sb != rb) memcpy(rb, sb, (size_t)n * oracle_mpi_type_size(t)); return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* sb, int sn, MPI_Datatype st, void* rb, int, MPI_Datatype, int, MPI_Comm) {
  if (sb != rb) memcpy(rb, sb, (size_t)sn * oracle_mpi_type_size(st)); return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void* sb, int sn, MPI_Datatype st, void* rb, const int*, const int* displs, MPI_Datatype rt, int, MPI_Comm) {
  memcpy((char*)rb + (size_t)displs[0] * oracle_mpi_type_size(rt), sb, (size_t)sn * oracle_mpi_type_size(st)); return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* sb, int sn, MPI_Datatype st, void* rb, int, MPI_Datatype, MPI_Comm) {
  if (sb != rb) memcpy(rb, sb, (size_t)sn * oracle_mpi_type_size(st)); return MPI_SUCCESS;
}
static inline int MPI_Scatter(const void* sb, int, MPI_Datatype, void* rb, int rn, MPI_Datatype rt, int, MPI_Comm) {
  if (sb != rb) memcpy(rb, sb, (size_t)rn * oracle_mpi_type_size(rt)); return MPI_SUCCESS;
}
static inline int MPI_Scatterv(const void* sb, const int*, const int* displs, MPI_Datatype st, void* rb, int rn, MPI_Datatype rt, int, MPI_Comm) {
  memcpy(rb, (const char*)sb + (size_t)displs[0] * oracle_mpi_type_size(st), (size_t)rn * oracle_mpi_type_size(rt)); return MPI_SUCCESS;
}

/* Packing: a byte-copy format private to this process. */
static inline int MPI_Pack_size(int n, MPI_Datatype t, MPI_Comm, int* size) { *size = n * oracle_mpi_type_size(t); return MPI_SUCCESS; }
static inline int MPI_Pack(const void* in, int n, MPI_Datatype t, void* out, int outsize, int* pos, MPI_Comm) {
  int b = n * oracle_mpi_type_size(t);
  if (*pos + b > outsize) return 1;
  memcpy((char*)out + *pos, in, (size_t)b); *pos += b; return MPI_SUCCESS;
}
static inline int MPI_Unpack(const void* in, int insize, int* pos, void* out, int n, MPI_Datatype t, MPI_Comm) {
  int b = n * oracle_mpi_type_size(t);
  if (*pos + b > insize) return 1;
  memcpy(out, (const char*)in + *pos, (size_t)b); *pos += b; return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype* nt) {
  *nt = 16 + n * oracle_mpi_type_size(old); return MPI_SUCCESS;
}
static inline int MPI_Type_create_struct(int, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Datatype* nt) { *nt = MPI_BYTE; return MPI_SUCCESS; }
static inline int MPI_Type_struct(int, int*, MPI_Aint*, MPI_Datatype*, MPI_Datatype* nt) { *nt = MPI_BYTE; return MPI_SUCCESS; }
static inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype*) { return MPI_SUCCESS; }

#endif
