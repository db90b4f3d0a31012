/*
 * Single-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE ONLY.
 *
 * Semantics kept from the MPI standard for a one-process world:
 *  - a Cartesian communicator has coordinates 0 in every dimension; a shift
 *    along a periodic dimension names this rank, along a non-periodic one
 *    it names MPI_PROC_NULL;
 *  - a subarray datatype describes a C-ordered box inside a bigger C-ordered
 *    array of a basic type; Sendrecv to/from this rank packs the send box and
 *    unpacks it into the receive box (through a bounce buffer, because the
 *    reference sends and receives on the same array);
 *  - Isend/Irecv to this rank are matched by tag at MPI_Waitall;
 *  - a blocking Send to this rank is buffered until the Recv with its tag.
 */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXTYPES 4096
#define MAXDIMS 4

typedef struct {
  int base;                 /* basic type handle */
  int ndims;
  int sizes[MAXDIMS], subsizes[MAXDIMS], starts[MAXDIMS];
} subarray_t;

static subarray_t g_types[MAXTYPES];
static int g_ntypes = 0;
static int g_cart_ndims = 0;
static int g_cart_periods[MAXDIMS];

static size_t basic_size(int t)
{
  switch (t) {
  case 1: return sizeof(double);
  case 2: return sizeof(int);
  case 3: return 1;
  case 4: return 1;
  default: fprintf(stderr, "fakempi: bad basic type %d\n", t); abort();
  }
}

static int is_basic(int t) { return t >= 1 && t <= 4; }

static subarray_t *derived(int t)
{
  if (t < 16 || t >= 16 + g_ntypes) { fprintf(stderr, "fakempi: bad type %d\n", t); abort(); }
  return &g_types[t - 16];
}

/* bytes of payload carried by `count` items of type t */
static size_t payload_bytes(int t, int count)
{
  if (is_basic(t)) return basic_size(t) * (size_t)count;
  subarray_t *s = derived(t);
  size_t n = basic_size(s->base);
  for (int d = 0; d < s->ndims; d++) n *= (size_t)s->subsizes[d];
  return n * (size_t)count;
}

/* walk the subarray box in C order; dir=0 packs buf->flat, dir=1 unpacks flat->buf */
static void walk(int t, char *buf, char *flat, int dir)
{
  if (is_basic(t)) { fprintf(stderr, "fakempi: walk on basic type\n"); abort(); }
  subarray_t *s = derived(t);
  size_t es = basic_size(s->base);
  int nd = s->ndims;
  size_t stride[MAXDIMS];
  stride[nd - 1] = es;
  for (int d = nd - 2; d >= 0; d--) stride[d] = stride[d + 1] * (size_t)s->sizes[d + 1];
  int idx[MAXDIMS] = {0};
  size_t row = (size_t)s->subsizes[nd - 1] * es;
  for (;;) {
    size_t off = 0;
    for (int d = 0; d < nd - 1; d++) off += (size_t)(s->starts[d] + idx[d]) * stride[d];
    off += (size_t)s->starts[nd - 1] * es;
    if (dir == 0) memcpy(flat, buf + off, row); else memcpy(buf + off, flat, row);
    flat += row;
    int d = nd - 2;
    while (d >= 0) {
      if (++idx[d] < s->subsizes[d]) break;
      idx[d] = 0;
      d--;
    }
    if (d < 0) break;
  }
}

static void copy_typed(const void *sbuf, int scount, int stype, void *rbuf, int rcount, int rtype)
{
  size_t sb = payload_bytes(stype, scount), rb = payload_bytes(rtype, rcount);
  if (sb != rb) { fprintf(stderr, "fakempi: size mismatch %zu vs %zu (types %d %d)\n", sb, rb, stype, rtype); abort(); }
  char *tmp = (char *)malloc(sb ? sb : 1);
  if (is_basic(stype)) memcpy(tmp, sbuf, sb);
  else for (int c = 0; c < scount; c++) walk(stype, (char *)sbuf, tmp, 0);
  if (is_basic(rtype)) memcpy(rbuf, tmp, rb);
  else for (int c = 0; c < rcount; c++) walk(rtype, (char *)rbuf, tmp, 1);
  free(tmp);
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

int MPI_Dims_create(int nnodes, int ndims, int dims[])
{
  if (nnodes != 1) { fprintf(stderr, "fakempi: one rank only\n"); abort(); }
  for (int d = 0; d < ndims; d++) if (dims[d] == 0) dims[d] = 1;
  return 0;
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *cart)
{
  (void)old; (void)reorder;
  for (int d = 0; d < ndims; d++) {
    if (dims[d] != 1) { fprintf(stderr, "fakempi: grid dim %d = %d, one rank only\n", d, dims[d]); abort(); }
    g_cart_periods[d] = periods[d];
  }
  g_cart_ndims = ndims;
  *cart = 1;
  return 0;
}

int MPI_Cart_coords(MPI_Comm c, int rank, int maxdims, int coords[])
{
  (void)c; (void)rank;
  for (int d = 0; d < maxdims; d++) coords[d] = 0;
  return 0;
}

int MPI_Cart_rank(MPI_Comm c, const int coords[], int *rank)
{
  (void)c;
  for (int d = 0; d < g_cart_ndims; d++)
    if (coords[d] != 0 && !g_cart_periods[d]) { *rank = MPI_PROC_NULL; return 0; }
  *rank = 0;
  return 0;
}

int MPI_Cart_shift(MPI_Comm c, int direction, int disp, int *src, int *dst)
{
  (void)c;
  if (disp == 0 || g_cart_periods[direction]) { *src = 0; *dst = 0; }
  else { *src = MPI_PROC_NULL; *dst = MPI_PROC_NULL; }
  return 0;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order, MPI_Datatype old,
                             MPI_Datatype *newtype)
{
  if (order != MPI_ORDER_C || ndims > MAXDIMS || !is_basic(old) || g_ntypes >= MAXTYPES) {
    fprintf(stderr, "fakempi: unsupported subarray\n"); abort();
  }
  subarray_t *s = &g_types[g_ntypes];
  s->base = old; s->ndims = ndims;
  for (int d = 0; d < ndims; d++) {
    s->sizes[d] = sizes[d]; s->subsizes[d] = subsizes[d]; s->starts[d] = starts[d];
    if (starts[d] < 0 || starts[d] + subsizes[d] > sizes[d]) {
      fprintf(stderr, "fakempi: subarray out of range (dim %d)\n", d); abort();
    }
  }
  *newtype = 16 + g_ntypes++;
  return 0;
}

int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }

int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int source, int rtag,
                 MPI_Comm c, MPI_Status *st)
{
  (void)stag; (void)rtag; (void)c; (void)st;
  if (dest == MPI_PROC_NULL && source == MPI_PROC_NULL) return 0;
  if (dest != 0 || source != 0) { fprintf(stderr, "fakempi: one-sided self Sendrecv\n"); abort(); }
  copy_typed(sbuf, scount, stype, rbuf, rcount, rtype);
  return 0;
}

int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
  (void)op; (void)c;
  if (sbuf != MPI_IN_PLACE) memcpy(rbuf, sbuf, payload_bytes(t, count));
  return 0;
}

/* blocking self messages of basic types (the tracer hand-over,
   tracers.c:266-289): a send to this rank is buffered, as an eager MPI
   implementation would, and the receive with the same tag takes it */
#define MAXMSG 1024
typedef struct { int tag; size_t bytes; void *data; } msg_t;
static msg_t g_msg[MAXMSG];
static int g_nmsg = 0;

int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
  (void)c;
  if (dest == MPI_PROC_NULL) return 0;
  if (dest != 0 || !is_basic(t) || g_nmsg >= MAXMSG) { fprintf(stderr, "fakempi: unsupported MPI_Send\n"); abort(); }
  size_t b = payload_bytes(t, count);
  void *d = malloc(b ? b : 1);
  if (!d) abort();
  memcpy(d, buf, b);
  g_msg[g_nmsg].tag = tag;
  g_msg[g_nmsg].bytes = b;
  g_msg[g_nmsg].data = d;
  g_nmsg++;
  return 0;
}
int MPI_Recv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c, MPI_Status *st)
{
  (void)c; (void)st;
  if (source == MPI_PROC_NULL) return 0;
  if (source != 0 || !is_basic(t)) { fprintf(stderr, "fakempi: unsupported MPI_Recv\n"); abort(); }
  for (int k = 0; k < g_nmsg; k++)
    if (g_msg[k].tag == tag) {
      size_t b = payload_bytes(t, count);
      if (b != g_msg[k].bytes) { fprintf(stderr, "fakempi: MPI_Recv size mismatch\n"); abort(); }
      memcpy(buf, g_msg[k].data, b);
      free(g_msg[k].data);
      g_msg[k] = g_msg[--g_nmsg];
      return 0;
    }
  fprintf(stderr, "fakempi: MPI_Recv with no matching send (tag %d)\n", tag); abort();
}

/* nonblocking self messages: queue them and match sends to receives by tag */
#define MAXREQ 65536
typedef struct { int is_send; const void *sbuf; void *rbuf; int count, type, tag; } pending_t;
static pending_t g_pend[MAXREQ];
static int g_npend = 0;

int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *req)
{
  (void)c;
  if (dest == MPI_PROC_NULL) { *req = -1; return 0; }
  if (g_npend >= MAXREQ) abort();
  g_pend[g_npend] = (pending_t){1, buf, NULL, count, t, tag};
  *req = g_npend++;
  return 0;
}
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c, MPI_Request *req)
{
  (void)c;
  if (source == MPI_PROC_NULL) { *req = -1; return 0; }
  if (g_npend >= MAXREQ) abort();
  g_pend[g_npend] = (pending_t){0, NULL, buf, count, t, tag};
  *req = g_npend++;
  return 0;
}
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status sts[])
{
  (void)sts;
  /* the sends' data are packed first (MPI semantics: a send buffer is read
     as it stood when the send was posted and was not modified since) */
  for (int r = 0; r < count; r++) {
    if (reqs[r] < 0 || g_pend[reqs[r]].is_send) continue;
    pending_t *rv = &g_pend[reqs[r]];
    int found = 0;
    for (int s = 0; s < count; s++) {
      if (reqs[s] < 0) continue;
      pending_t *sd = &g_pend[reqs[s]];
      if (sd->is_send && sd->tag == rv->tag && sd->count >= 0) {
        copy_typed(sd->sbuf, sd->count, sd->type, rv->rbuf, rv->count, rv->type);
        sd->count = -1;
        found = 1;
        break;
      }
    }
    if (!found) { fprintf(stderr, "fakempi: unmatched Irecv tag %d\n", rv->tag); abort(); }
  }
  g_npend = 0;
  return 0;
}
