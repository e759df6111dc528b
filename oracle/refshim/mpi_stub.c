/* mpi_stub.c -- single-rank implementation of oracle/refshim/mpi.h (test infrastructure).
 * Point-to-point messages can only go to rank 0 itself: a send and a receive with the
 * same tag are matched (in either posting order) and the data is copied. */
#include "mpi.h"
#include <stdio.h>
#include <string.h>
#include <time.h>

#define MAXPEND 64
typedef struct { const void *sbuf; void *rbuf; size_t bytes; int tag; int used; } pend_t;
static pend_t g_send[MAXPEND], g_recv[MAXPEND];

static size_t type_size(MPI_Datatype t) { return t == MPI_FLOAT ? 4 : t == MPI_INT ? sizeof(int) : t == MPI_DOUBLE ? 8 : 1; }
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return MPI_SUCCESS; }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c) { (void)buf; (void)count; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
double MPI_Wtime(void) { struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return ts.tv_sec + 1e-9 * ts.tv_nsec; }

static int post(pend_t *mine, pend_t *other, const void *sb, void *rb, size_t bytes, int tag, int peer) {
  int i;
  if (peer != 0) { fprintf(stderr, "refshim: message to rank %d in a single-rank run\n", peer); return MPI_ERR_OTHER; }
  for (i = 0; i < MAXPEND; i++)
    if (other[i].used && other[i].tag == tag) {
      void *dst = rb ? rb : other[i].rbuf;
      const void *src = sb ? sb : other[i].sbuf;
      memcpy(dst, src, bytes < other[i].bytes ? bytes : other[i].bytes);
      other[i].used = 0;
      return MPI_SUCCESS;
    }
  for (i = 0; i < MAXPEND; i++)
    if (!mine[i].used) {
      mine[i].sbuf = sb; mine[i].rbuf = rb; mine[i].bytes = bytes; mine[i].tag = tag; mine[i].used = 1;
      return MPI_SUCCESS;
    }
  return MPI_ERR_OTHER;
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c, MPI_Request *r) {
  (void)c; if (r) *r = 0; return post(g_send, g_recv, b, NULL, (size_t)n * type_size(t), g, d); }
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Request *r) {
  (void)c; if (r) *r = 0; return post(g_recv, g_send, NULL, b, (size_t)n * type_size(t), g, s); }
int MPI_Wait(MPI_Request *r, MPI_Status *s) { (void)r; (void)s; return MPI_SUCCESS; }
int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int dest, int stag, void *rb, int rc, MPI_Datatype rt, int src, int rtag, MPI_Comm c, MPI_Status *s) {
  (void)dest; (void)stag; (void)rt; (void)src; (void)rtag; (void)c; (void)s; (void)rc;
  memcpy(rb, sb, (size_t)sc * type_size(st)); return MPI_SUCCESS; }
int MPI_Scatter(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rc; (void)rt; (void)root; (void)c; if (sb != rb) memcpy(rb, sb, (size_t)sc * type_size(st)); return MPI_SUCCESS; }
int MPI_Gather(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rc; (void)rt; (void)root; (void)c; if (sb != rb) memcpy(rb, sb, (size_t)sc * type_size(st)); return MPI_SUCCESS; }
