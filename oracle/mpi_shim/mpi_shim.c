/*
 * Single-rank MPI shim (see mpi.h).  Test infrastructure for the CPU oracle
 * build of the TIOGA reference; not part of the product library.
 *
 * Point-to-point: a send whose tag matches an already posted receive is
 * copied straight into it; otherwise the payload is copied into a pending
 * list that a later receive with the same tag drains in FIFO order.  This is
 * exactly the message order a real MPI gives one rank talking to itself.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct pending_send {
  int tag;
  size_t nbytes;
  void *data;
  struct pending_send *next;
} pending_send;

typedef struct posted_recv {
  int tag;
  size_t nbytes;
  void *buf;
  int *done;
  struct posted_recv *next;
} posted_recv;

static pending_send *g_sends = NULL;   /* FIFO of unmatched sends */
static posted_recv *g_recvs = NULL;    /* FIFO of unmatched receives */

/* request table: a request is an index; done[] tracks completion */
#define SHIM_MAX_REQ (1 << 16)
static int g_done[SHIM_MAX_REQ];
static int g_next_req = 1;

static int new_request(void) {
  int r = g_next_req++;
  if (g_next_req >= SHIM_MAX_REQ) g_next_req = 1;
  g_done[r] = 0;
  return r;
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
MPI_Comm MPI_Comm_f2c(MPI_Fint comm) { (void)comm; return MPI_COMM_WORLD; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm comm, int code) {
  (void)comm;
  fprintf(stderr, "#mpi_shim: MPI_Abort(%d) called by the reference\n", code);
  fflush(stderr);
  abort();
  return code;
}

double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void copy_if_distinct(const void *src, void *dst, size_t n) {
  if (src != dst && n > 0) memmove(dst, src, n);
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
  (void)op; (void)comm;
  copy_if_distinct(sendbuf, recvbuf, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count,
               MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm) {
  (void)op; (void)root; (void)comm;
  copy_if_distinct(sendbuf, recvbuf, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype,
                  void *recvbuf, int rcount, MPI_Datatype rtype, MPI_Comm comm) {
  (void)rcount; (void)rtype; (void)comm;
  copy_if_distinct(sendbuf, recvbuf, (size_t)scount * (size_t)stype);
  return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype,
                   void *recvbuf, const int *rcounts, const int *displs,
                   MPI_Datatype rtype, MPI_Comm comm) {
  (void)rcounts; (void)comm;
  copy_if_distinct(sendbuf, (char *)recvbuf + (size_t)displs[0] * (size_t)rtype,
                   (size_t)scount * (size_t)stype);
  return MPI_SUCCESS;
}

int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype stype,
                 void *recvbuf, int rcount, MPI_Datatype rtype, MPI_Comm comm) {
  (void)rcount; (void)rtype; (void)comm;
  copy_if_distinct(sendbuf, recvbuf, (size_t)scount * (size_t)stype);
  return MPI_SUCCESS;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest,
              int tag, MPI_Comm comm, MPI_Request *req) {
  (void)dest; (void)comm;
  size_t nbytes = (size_t)count * (size_t)type;
  int r = new_request();
  *req = r;
  /* match the oldest posted receive with this tag */
  posted_recv *prev = NULL, *p = g_recvs;
  while (p && p->tag != tag) { prev = p; p = p->next; }
  if (p) {
    if (nbytes > p->nbytes) {
      fprintf(stderr, "#mpi_shim: message truncated (%zu > %zu)\n", nbytes, p->nbytes);
      abort();
    }
    copy_if_distinct(buf, p->buf, nbytes);
    *(p->done) = 1;
    if (prev) prev->next = p->next; else g_recvs = p->next;
    free(p);
  } else {
    pending_send *s = (pending_send *)malloc(sizeof(pending_send));
    s->tag = tag;
    s->nbytes = nbytes;
    s->data = malloc(nbytes ? nbytes : 1);
    copy_if_distinct(buf, s->data, nbytes);
    s->next = NULL;
    if (!g_sends) g_sends = s;
    else { pending_send *t = g_sends; while (t->next) t = t->next; t->next = s; }
  }
  g_done[r] = 1; /* the payload is copied: the send buffer is free */
  return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req) {
  (void)source; (void)comm;
  size_t nbytes = (size_t)count * (size_t)type;
  int r = new_request();
  *req = r;
  pending_send *prev = NULL, *s = g_sends;
  while (s && s->tag != tag) { prev = s; s = s->next; }
  if (s) {
    if (s->nbytes > nbytes) {
      fprintf(stderr, "#mpi_shim: message truncated (%zu > %zu)\n", s->nbytes, nbytes);
      abort();
    }
    copy_if_distinct(s->data, buf, s->nbytes);
    g_done[r] = 1;
    if (prev) prev->next = s->next; else g_sends = s->next;
    free(s->data);
    free(s);
  } else {
    posted_recv *p = (posted_recv *)malloc(sizeof(posted_recv));
    p->tag = tag;
    p->nbytes = nbytes;
    p->buf = buf;
    p->done = &g_done[r];
    p->next = NULL;
    if (!g_recvs) g_recvs = p;
    else { posted_recv *t = g_recvs; while (t->next) t = t->next; t->next = p; }
  }
  return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *stats) {
  for (int i = 0; i < count; i++) {
    if (!g_done[reqs[i]]) {
      fprintf(stderr, "#mpi_shim: Waitall on an unmatched request (one rank "
                      "cannot complete it)\n");
      abort();
    }
    if (stats) {
      stats[i].MPI_SOURCE = 0;
      stats[i].MPI_TAG = 0;
      stats[i].MPI_ERROR = 0;
      stats[i].count_bytes = 0;
    }
  }
  return MPI_SUCCESS;
}
