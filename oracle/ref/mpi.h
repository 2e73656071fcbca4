/*
 * mpi.h -- single-rank MPI stand-in used ONLY to compile the reference's own
 * hot-path sources (lattice_util.cpp, solvers.cpp, blas_qkxTM.cpp, util.cpp,
 * blas.cpp, contractions.cpp, read_conf_lime.cpp, write_conf_lime.cpp) into the
 * test oracle under oracle/_ref/.  Test infrastructure.
 *
 * With one rank and P = (1,1,1,1) the reference never exchanges halos
 * (every communicate* call is guarded by lL < L), so point-to-point calls are
 * no-ops and reductions / gathers copy the send buffer to the receive buffer.
 */
#ifndef QKX_REF_MPI_STUB_H
#define QKX_REF_MPI_STUB_H

#include <string.h>
#include <time.h>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Request;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_FLOAT 4
#define MPI_CHAR 1
#define MPI_BYTE 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

static inline size_t qkx_stub_elem_bytes(MPI_Datatype t) { return t > 0 ? (size_t)t : 1; }

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Abort(MPI_Comm, int) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) memmove(r, s, n * qkx_stub_elem_bytes(t));
  return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != r) memmove(r, s, n * qkx_stub_elem_bytes(t));
  return 0;
}
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int,
                             MPI_Comm) {
  if (s != r) memmove(r, s, n * qkx_stub_elem_bytes(t));
  return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype,
                               int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Type_vector(int, int, int, MPI_Datatype, MPI_Datatype* o) { *o = 0; return 0; }
static inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype* o) { *o = 0; return 0; }
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Type_free(MPI_Datatype*) { return 0; }
static inline int MPI_Comm_group(MPI_Comm, MPI_Group* g) { *g = 0; return 0; }
static inline int MPI_Group_incl(MPI_Group, int, const int*, MPI_Group* g) { *g = 0; return 0; }
static inline int MPI_Group_rank(MPI_Group, int* r) { *r = 0; return 0; }
static inline int MPI_Group_size(MPI_Group, int* n) { *n = 1; return 0; }
static inline int MPI_Comm_create(MPI_Comm, MPI_Group, MPI_Comm* c) { *c = 0; return 0; }

/* MPI-IO for one rank (lib/read_conf_lime.cpp, lib/write_conf_lime.cpp): the subarray a rank
 * owns is the whole array, so a view is a byte offset and an element size, and a collective
 * read or write is one contiguous stdio transfer at that offset. */
#include <stdio.h>
typedef long long MPI_Offset;
typedef int MPI_Info;
typedef struct qkx_stub_file {
  FILE* fp;
  MPI_Offset disp;
  size_t esize;
} * MPI_File;
#define MPI_INFO_NULL 0
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_ORDER_C 56

static inline int MPI_Type_create_subarray(int nd, const int* sizes, const int* sub, const int* starts, int,
                                           MPI_Datatype old, MPI_Datatype* out) {
  for (int i = 0; i < nd; i++)
    if (sub[i] != sizes[i] || starts[i] != 0) return 1; /* one rank owns everything */
  *out = old;
  return 0;
}
static inline int MPI_File_open(MPI_Comm, const char* name, int amode, MPI_Info, MPI_File* fh) {
  FILE* fp = fopen(name, amode == MPI_MODE_RDONLY ? "rb" : "r+b");
  if (!fp) return 1;
  *fh = new qkx_stub_file{fp, 0, 1};
  return 0;
}
static inline int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype, const char*,
                                    MPI_Info) {
  fh->disp = disp;
  fh->esize = qkx_stub_elem_bytes(etype);
  return 0;
}
static inline int MPI_File_read_all(MPI_File fh, void* buf, int count, MPI_Datatype t, MPI_Status*) {
  const size_t n = (size_t)count * qkx_stub_elem_bytes(t);
  if (fseeko(fh->fp, (off_t)fh->disp, SEEK_SET) != 0) return 1;
  return fread(buf, 1, n, fh->fp) == n ? MPI_SUCCESS : 1;
}
static inline int MPI_File_write_all(MPI_File fh, const void* buf, int count, MPI_Datatype t, MPI_Status*) {
  const size_t n = (size_t)count * qkx_stub_elem_bytes(t);
  if (fseeko(fh->fp, (off_t)fh->disp, SEEK_SET) != 0) return 1;
  return fwrite(buf, 1, n, fh->fp) == n ? MPI_SUCCESS : 1;
}
static inline int MPI_File_close(MPI_File* fh) {
  const int rc = fclose((*fh)->fp);
  delete *fh;
  *fh = 0;
  return rc == 0 ? MPI_SUCCESS : 1;
}

#endif
