#define _POSIX_C_SOURCE 200809L
/*
 * Single-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE ONLY.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "mpi.h"

struct svof_mpi_type_s svof_mpi_double_s = {sizeof(double), 1, 0, {0}, {0}, {0}};
struct svof_mpi_type_s svof_mpi_int_s = {sizeof(int), 1, 0, {0}, {0}, {0}};
struct svof_mpi_type_s svof_mpi_byte_s = {1, 1, 0, {0}, {0}, {0}};

struct svof_mpi_file_s {
  FILE *fp;
  long disp;
  MPI_Datatype filetype;
};

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; fprintf(stderr, "MPI_Abort(%d)\n", code); exit(1); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1.e-9 * (double)ts.tv_nsec;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm) {
  (void)buf; (void)count; (void)type; (void)root; (void)comm;
  return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
  (void)op; (void)comm;
  if (MPI_IN_PLACE != sendbuf) memcpy(recvbuf, sendbuf, (size_t)count * type->size);
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm) {
  (void)op; (void)root; (void)comm;
  if (MPI_IN_PLACE != sendbuf) memcpy(recvbuf, sendbuf, (size_t)count * type->size);
  return MPI_SUCCESS;
}

/* the only peer of rank 0 is rank 0 itself (periodic y) or MPI_PROC_NULL */
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status) {
  (void)sendtag; (void)recvtag; (void)comm; (void)status; (void)recvtype; (void)recvcount;
  if (MPI_PROC_NULL == dest || MPI_PROC_NULL == source) return MPI_SUCCESS;
  memmove(recvbuf, sendbuf, (size_t)sendcount * sendtype->size);
  return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype) {
  MPI_Datatype t = calloc(1, sizeof(*t));
  t->size = (size_t)count * oldtype->size;
  t->builtin = 0;
  *newtype = t;
  return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[],
                             int order, MPI_Datatype oldtype, MPI_Datatype *newtype) {
  (void)order;
  MPI_Datatype t = calloc(1, sizeof(*t));
  t->builtin = 0;
  t->ndims = ndims;
  size_t n = 1;
  for (int d = 0; d < ndims && d < 8; d++) {
    t->sizes[d] = sizes[d];
    t->subsizes[d] = subsizes[d];
    t->starts[d] = starts[d];
    n *= (size_t)subsizes[d];
  }
  t->size = n * oldtype->size;
  *newtype = t;
  return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *type) { (void)type; return MPI_SUCCESS; }

int MPI_Type_free(MPI_Datatype *type) {
  if (*type && !(*type)->builtin) free(*type);
  *type = MPI_DATATYPE_NULL;
  return MPI_SUCCESS;
}

int MPI_Error_string(int code, char *string, int *len) {
  *len = snprintf(string, MPI_MAX_ERROR_STRING, "MPI error %d", code);
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh) {
  (void)comm; (void)info;
  const char *mode = (amode & MPI_MODE_RDWR) ? "r+b" : "rb";
  FILE *fp = fopen(filename, mode);
  if (NULL == fp && (amode & MPI_MODE_CREATE)) fp = fopen(filename, "w+b");
  if (NULL == fp) return MPI_ERR_OTHER;
  *fh = calloc(1, sizeof(**fh));
  (*fh)->fp = fp;
  return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh) {
  if (*fh) {
    fclose((*fh)->fp);
    free(*fh);
  }
  *fh = NULL;
  return MPI_SUCCESS;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *datarep, MPI_Info info) {
  (void)etype; (void)datarep; (void)info;
  fh->disp = (long)disp;
  fh->filetype = filetype;
  return MPI_SUCCESS;
}

/* one rank owns the whole array: the subarray view must equal the full array */
static int check_full_view(MPI_File fh) {
  const MPI_Datatype t = fh->filetype;
  if (NULL == t) return 0;
  for (int d = 0; d < t->ndims; d++) {
    if (t->sizes[d] != t->subsizes[d] || 0 != t->starts[d]) {
      fprintf(stderr, "single-rank MPI-IO: partial subarray views are not supported\n");
      return 1;
    }
  }
  return 0;
}

int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype type, MPI_Status *status) {
  (void)status;
  if (check_full_view(fh)) return MPI_ERR_OTHER;
  if (0 != fseek(fh->fp, fh->disp, SEEK_SET)) return MPI_ERR_OTHER;
  const size_t n = fread(buf, type->size, (size_t)count, fh->fp);
  return n == (size_t)count ? MPI_SUCCESS : MPI_ERR_OTHER;
}

int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Status *status) {
  (void)status;
  if (check_full_view(fh)) return MPI_ERR_OTHER;
  if (0 != fseek(fh->fp, fh->disp, SEEK_SET)) return MPI_ERR_OTHER;
  const size_t n = fwrite(buf, type->size, (size_t)count, fh->fp);
  return n == (size_t)count ? MPI_SUCCESS : MPI_ERR_OTHER;
}
