/*
 * Single-rank stand-in for the subset of MPI that SimpleTCSolver's C sources
 * call (test infrastructure for the oracle build only; never linked into the
 * GPU library).
 *
 * One process is the whole world: communicators have one member, reductions
 * with MPI_IN_PLACE are no-ops, MPI_Sendrecv to oneself is a typed memcpy and
 * MPI-IO reads/writes the whole file through stdio at the view's displacement.
 * Call sites this covers (reference paths):
 *   src/halo.c:45-76,110-139       MPI_Type_vector / MPI_Type_contiguous + MPI_Sendrecv
 *   src/fileio.c:84-99,406-505     subarray file views, MPI_File_read_all/write_all
 *   src/decide_dt.c:77             MPI_Allreduce(MPI_IN_PLACE, MIN)
 *   src/logging/*.c                MPI_Reduce(MPI_IN_PLACE at root)
 *   src/config.c, array.c, timer.c, memory.c, main.c
 */
#if !defined(TCREF_SHIM_MPI_H)
#define TCREF_SHIM_MPI_H

#include <stddef.h>
#include <stdint.h>

/* a datatype is a pointer to a description of its memory footprint */
typedef struct shim_mpi_type_t_ shim_mpi_type_t;
typedef const shim_mpi_type_t * MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct shim_mpi_file_t_ * MPI_File;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

/* a description: "count" blocks of "blocklen" elements of "base",
 * consecutive blocks "stride" base-extents apart; a basic type has base NULL */
struct shim_mpi_type_t_ {
  size_t extent;              /* bytes of one basic element (basic types only) */
  int count;
  int blocklen;
  long stride;
  const shim_mpi_type_t * base;
};

extern const shim_mpi_type_t shim_mpi_byte_, shim_mpi_int_, shim_mpi_double_;
#define MPI_BYTE   (&shim_mpi_byte_)
#define MPI_INT    (&shim_mpi_int_)
#define MPI_DOUBLE (&shim_mpi_double_)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0)

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL  0
#define MPI_PROC_NULL  (-1)
#define MPI_INFO_NULL  0
#define MPI_SUCCESS    0
#define MPI_MAX_ERROR_STRING 256
#define MPI_ORDER_C    56
#define MPI_MODE_RDONLY 2
#define MPI_MODE_RDWR   8
#define MPI_MODE_CREATE 1
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

int MPI_Init(int * argc, char *** argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Barrier(MPI_Comm comm);
int MPI_Comm_rank(MPI_Comm comm, int * rank);
int MPI_Comm_size(MPI_Comm comm, int * size);
double MPI_Wtime(void);
int MPI_Error_string(int code, char * string, int * length);

int MPI_Bcast(void * buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void * sendbuf, void * recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void * sendbuf, void * recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Sendrecv(
    const void * sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
    void * recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
    MPI_Comm comm, MPI_Status * status);

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype * newtype);
int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype, MPI_Datatype * newtype);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[], int order, MPI_Datatype oldtype, MPI_Datatype * newtype);
int MPI_Type_commit(MPI_Datatype * type);
int MPI_Type_free(MPI_Datatype * type);

int MPI_File_open(MPI_Comm comm, const char * filename, int amode, MPI_Info info, MPI_File * fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype, const char * datarep, MPI_Info info);
int MPI_File_read_all(MPI_File fh, void * buf, int count, MPI_Datatype type, MPI_Status * status);
int MPI_File_write_all(MPI_File fh, const void * buf, int count, MPI_Datatype type, MPI_Status * status);
int MPI_File_close(MPI_File * fh);

#endif // TCREF_SHIM_MPI_H
