/*
 * Single-rank MPI shim — test infrastructure for the oracle only (see mpi.h).
 *
 * Semantics at one rank:
 *   - Bcast/Barrier: no-ops; Reduce/Allreduce: copy send -> recv.
 *   - Gather/Gatherv: copy unless MPI_IN_PLACE (then the data is already there).
 *   - Isend to self is queued; the next Irecv takes it.  A message longer than
 *     the receive count is truncated to it.  Real MPI would raise
 *     MPI_ERR_TRUNCATE there; at one rank the only self-messages are the z halo
 *     slabs (MDcode/Parallel.c:427-460) which carry the rank's own, unchanged
 *     coordinates, so dropping the tail changes no value.
 *   - Derived struct types record their extent (offset of the last member +
 *     its size, rounded up to 8 bytes, i.e. sizeof of the C struct).
 */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAX_DERIVED 16
static long derived_extent[MAX_DERIVED];
static int n_derived = 0;

static long type_size(MPI_Datatype t) {
  if (t == MPI_INT) return 4;
  if (t == MPI_DOUBLE) return 8;
  if (t == MPI_UNSIGNED_LONG_LONG) return 8;
  if (t >= 100 && t < 100 + n_derived) return derived_extent[t - 100];
  fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
  abort();
}

/* one pending self-message and a small request table */
typedef struct { int used; int is_recv; long bytes; } req_slot;
#define MAX_REQ 64
static req_slot reqs[MAX_REQ];
static void *pend_msg = NULL;
static long pend_bytes = -1;

static int new_req(int is_recv, long bytes) {
  for (int i = 0; i < MAX_REQ; i++)
    if (!reqs[i].used) {
      reqs[i].used = 1;
      reqs[i].is_recv = is_recv;
      reqs[i].bytes = bytes;
      return i;
    }
  fprintf(stderr, "mpi shim: request table full\n");
  abort();
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c;
  return MPI_SUCCESS;
}
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
  (void)op; (void)root; (void)c;
  if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)n * type_size(t));
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  return MPI_Reduce(s, r, n, t, op, 0, c);
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *q) {
  (void)dest; (void)tag; (void)c;
  long bytes = (long)n * type_size(t);
  free(pend_msg);
  pend_msg = malloc(bytes > 0 ? (size_t)bytes : 1);
  if (bytes > 0) memcpy(pend_msg, b, (size_t)bytes);
  pend_bytes = bytes;
  *q = new_req(0, bytes);
  return MPI_SUCCESS;
}
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *q) {
  (void)src; (void)tag; (void)c;
  long cap = (long)n * type_size(t);
  if (pend_bytes < 0) {
    fprintf(stderr, "mpi shim: receive with no matching self-send\n");
    abort();
  }
  long got = pend_bytes < cap ? pend_bytes : cap;
  if (got > 0) memcpy(b, pend_msg, (size_t)got);
  pend_bytes = -1;
  *q = new_req(1, got);
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *q, MPI_Status *st) {
  req_slot *r = &reqs[*q];
  if (st) {
    st->count_bytes = (int)r->bytes;
    st->MPI_SOURCE = 0;
    st->MPI_TAG = 0;
    st->MPI_ERROR = 0;
  }
  r->used = 0;
  return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n) {
  *n = (int)(st->count_bytes / type_size(t));
  return MPI_SUCCESS;
}
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rn; (void)rt; (void)root; (void)c;
  if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)sn * type_size(st));
  return MPI_SUCCESS;
}
int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rn, const int *d,
                MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rn; (void)rt; (void)root; (void)c;
  if (s != MPI_IN_PLACE && s != r)
    memmove((char *)r + (long)d[0] * type_size(rt), s, (size_t)sn * type_size(st));
  return MPI_SUCCESS;
}
/* blocking point-to-point: the analysis program only sends to ranks >= 1
 * (Analysis/main.c:135-150), which do not exist at one rank */
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)dest; (void)tag; (void)c;
  fprintf(stderr, "mpi shim: MPI_Send has no peer at one rank\n");
  abort();
}
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st) {
  (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; (void)st;
  fprintf(stderr, "mpi shim: MPI_Recv has no peer at one rank\n");
  abort();
}
int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *off, const MPI_Datatype *types,
                           MPI_Datatype *out) {
  long ext = 0;
  for (int i = 0; i < n; i++) {
    long end = off[i] + (long)bl[i] * type_size(types[i]);
    if (end > ext) ext = end;
  }
  ext = (ext + 7) / 8 * 8;
  if (n_derived >= MAX_DERIVED) abort();
  derived_extent[n_derived] = ext;
  *out = 100 + n_derived++;
  return MPI_SUCCESS;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
