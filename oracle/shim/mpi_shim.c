/*
 * Single-rank MPI stand-in for building the reference solver as the CPU oracle.
 * Test infrastructure only: nothing in the product links this file.
 *
 * Datatypes are flattened at creation time into a list of contiguous byte
 * segments relative to the start of one element; a message of `count`
 * elements is then the segment list repeated at multiples of the extent.
 * With a single rank every point-to-point message is a self message, so
 * Sendrecv packs the send layout into a scratch buffer and unpacks it with
 * the receive layout.  Collectives degenerate to copies (the reduction of a
 * single contribution is that contribution).
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
  size_t off, len;
} seg_t;

typedef struct {
  size_t size;   /* bytes of payload per element */
  size_t extent; /* bytes spanned by one element */
  int nseg;
  seg_t *seg;
} dtype_t;

#define MAX_TYPES 256
static dtype_t g_types[MAX_TYPES];
static int g_ntypes = 0;

static void shim_fail(const char *what) {
  fprintf(stderr, "mpi shim: %s\n", what);
  exit(2);
}

static void ensure_basic(void) {
  if (g_ntypes) return;
  static seg_t s_double = {0, sizeof(double)}, s_float = {0, sizeof(float)}, s_int = {0, sizeof(int)},
               s_ld = {0, sizeof(long double)}, s_char = {0, 1};
  g_types[0] = (dtype_t){0, 0, 0, NULL};
  g_types[MPI_DOUBLE] = (dtype_t){sizeof(double), sizeof(double), 1, &s_double};
  g_types[MPI_FLOAT] = (dtype_t){sizeof(float), sizeof(float), 1, &s_float};
  g_types[MPI_INT] = (dtype_t){sizeof(int), sizeof(int), 1, &s_int};
  g_types[MPI_LONG_DOUBLE] = (dtype_t){sizeof(long double), sizeof(long double), 1, &s_ld};
  g_types[MPI_CHAR] = (dtype_t){1, 1, 1, &s_char};
  g_ntypes = 6;
}

static const dtype_t *get_type(MPI_Datatype t) {
  ensure_basic();
  if (t <= 0 || t >= g_ntypes) shim_fail("unknown datatype handle");
  return &g_types[t];
}

/* append a segment, merging with the previous one when contiguous */
static void push_seg(seg_t **v, int *n, int *cap, size_t off, size_t len) {
  if (*n > 0) {
    seg_t *last = &(*v)[*n - 1];
    if (last->off + last->len == off) {
      last->len += len;
      return;
    }
  }
  if (*n == *cap) {
    *cap = *cap ? 2 * *cap : 16;
    *v = (seg_t *)realloc(*v, sizeof(seg_t) * (size_t)*cap);
    if (!*v) shim_fail("out of memory");
  }
  (*v)[(*n)++] = (seg_t){off, len};
}

static MPI_Datatype new_type(size_t size, size_t extent, seg_t *seg, int nseg) {
  ensure_basic();
  if (g_ntypes >= MAX_TYPES) shim_fail("too many datatypes");
  g_types[g_ntypes] = (dtype_t){size, extent, nseg, seg};
  return g_ntypes++;
}

int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype, MPI_Datatype *newtype) {
  const dtype_t *o = get_type(oldtype);
  seg_t *v = NULL;
  int n = 0, cap = 0;
  for (int c = 0; c < count; c++)
    for (int b = 0; b < blocklength; b++) {
      size_t base = ((size_t)c * (size_t)stride + (size_t)b) * o->extent;
      for (int s = 0; s < o->nseg; s++) push_seg(&v, &n, &cap, base + o->seg[s].off, o->seg[s].len);
    }
  size_t extent = count > 0 ? ((size_t)(count - 1) * (size_t)stride + (size_t)blocklength) * o->extent : 0;
  *newtype = new_type((size_t)count * (size_t)blocklength * o->size, extent, v, n);
  return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype) {
  return MPI_Type_vector(count, 1, 1, oldtype, newtype);
}

int MPI_Type_commit(MPI_Datatype *type) {
  (void)get_type(*type);
  return MPI_SUCCESS;
}

static void pack(const char *buf, int count, const dtype_t *t, char *out) {
  for (int i = 0; i < count; i++)
    for (int s = 0; s < t->nseg; s++) {
      memcpy(out, buf + (size_t)i * t->extent + t->seg[s].off, t->seg[s].len);
      out += t->seg[s].len;
    }
}

static void unpack(const char *in, char *buf, int count, const dtype_t *t) {
  for (int i = 0; i < count; i++)
    for (int s = 0; s < t->nseg; s++) {
      memcpy(buf + (size_t)i * t->extent + t->seg[s].off, in, t->seg[s].len);
      in += t->seg[s].len;
    }
}

static void typed_copy(const void *src, int scount, MPI_Datatype stype, void *dst, int rcount, MPI_Datatype rtype) {
  const dtype_t *s = get_type(stype), *r = get_type(rtype);
  size_t bytes = (size_t)scount * s->size;
  if (bytes != (size_t)rcount * r->size) shim_fail("send/recv size mismatch");
  if (bytes == 0) return;
  char *tmp = (char *)malloc(bytes);
  if (!tmp) shim_fail("out of memory");
  pack((const char *)src, scount, s, tmp);
  unpack(tmp, (char *)dst, rcount, r);
  free(tmp);
}

int MPI_Init(int *argc, char ***argv) {
  (void)argc;
  (void)argv;
  ensure_basic();
  return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  (void)comm;
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int *size) {
  (void)comm;
  *size = 1;
  return MPI_SUCCESS;
}
double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
double MPI_Wtick(void) { return 1e-9; }
int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  return MPI_SUCCESS;
}
int MPI_Op_create(MPI_User_function *fn, int commute, MPI_Op *op) {
  (void)fn;
  (void)commute;
  static int next = 2;
  *op = next++;
  return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag, void *recvbuf,
                 int recvcount, MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm, MPI_Status *status) {
  (void)sendtag;
  (void)recvtag;
  (void)comm;
  if (dest != 0 || source != 0) shim_fail("Sendrecv with a rank other than 0");
  typed_copy(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
  if (status) *status = (MPI_Status){0, 0, 0};
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op, MPI_Comm comm) {
  (void)op;
  (void)comm;
  if (sendbuf != recvbuf) typed_copy(sendbuf, count, datatype, recvbuf, count, datatype);
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op, int root,
               MPI_Comm comm) {
  (void)root;
  return MPI_Allreduce(sendbuf, recvbuf, count, datatype, op, comm);
}

int MPI_Bcast(void *buffer, int count, MPI_Datatype datatype, int root, MPI_Comm comm) {
  (void)buffer;
  (void)count;
  (void)datatype;
  (void)root;
  (void)comm;
  return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm) {
  (void)comm;
  if (sendbuf != recvbuf) typed_copy(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype);
  return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, const int *recvcounts,
                   const int *displs, MPI_Datatype recvtype, MPI_Comm comm) {
  (void)comm;
  const dtype_t *r = get_type(recvtype);
  char *dst = (char *)recvbuf + (size_t)displs[0] * r->extent;
  if (sendbuf != dst) typed_copy(sendbuf, sendcount, sendtype, dst, recvcounts[0], recvtype);
  return MPI_SUCCESS;
}

int MPI_Dims_create(int nnodes, int ndims, int *dims) {
  (void)nnodes;
  for (int i = 0; i < ndims; i++)
    if (dims[i] == 0) dims[i] = 1;
  return MPI_SUCCESS;
}
int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder, MPI_Comm *cart) {
  (void)old;
  (void)ndims;
  (void)dims;
  (void)periods;
  (void)reorder;
  *cart = 0;
  return MPI_SUCCESS;
}
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords) {
  (void)comm;
  (void)rank;
  for (int i = 0; i < maxdims; i++) coords[i] = 0;
  return MPI_SUCCESS;
}
int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank) {
  (void)comm;
  (void)coords;
  *rank = 0;
  return MPI_SUCCESS;
}
