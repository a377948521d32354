/*
 * Single-rank stand-in for <mpi.h>.  TEST INFRASTRUCTURE ONLY: it exists so
 * that the reference's own src/*.c compile into the oracle library on a
 * machine without MPI.  Every routine implements the one-process meaning of
 * the MPI call as the reference uses it (halo.c, decide_dt.c, config.c,
 * fileio.c, memory.c, timer.c): collectives copy, point-to-point to self is a
 * memcpy, MPI-IO with a full-array subarray view is a plain file read/write.
 */
#ifndef SVOF_SHIM_MPI_H
#define SVOF_SHIM_MPI_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct svof_mpi_type_s *MPI_Datatype;
typedef struct svof_mpi_file_s *MPI_File;
typedef struct { int source, tag, error; } MPI_Status;

struct svof_mpi_type_s {
  size_t size;     /* bytes covered by one element of this type */
  int builtin;     /* 1 for the predefined types (never freed) */
  int ndims;       /* subarray types only */
  int sizes[8], subsizes[8], starts[8];
};

extern struct svof_mpi_type_s svof_mpi_double_s, svof_mpi_int_s, svof_mpi_byte_s;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_DOUBLE (&svof_mpi_double_s)
#define MPI_INT (&svof_mpi_int_s)
#define MPI_BYTE (&svof_mpi_byte_s)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_PROC_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_ERROR_STRING 256
#define MPI_INFO_NULL 0
#define MPI_ORDER_C 0
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR 8
#define MPI_MODE_CREATE 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[],
                             int order, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);
int MPI_Error_string(int code, char *string, int *len);
int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *datarep, MPI_Info info);
int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype type, MPI_Status *status);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Status *status);

#endif
