/*
 * Single-rank implementation of oracle/shim/mpi.h (oracle build only).
 * The world has one rank, so every collective is local and every
 * point-to-point message goes to oneself.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "mpi.h"

const shim_mpi_type_t shim_mpi_byte_   = {1, 1, 1, 1, NULL};
const shim_mpi_type_t shim_mpi_int_    = {sizeof(int), 1, 1, 1, NULL};
const shim_mpi_type_t shim_mpi_double_ = {sizeof(double), 1, 1, 1, NULL};

struct shim_mpi_file_t_ {
  FILE * fp;
  MPI_Offset disp;
};

static size_t type_extent(MPI_Datatype t){
  if(NULL == t->base){
    return t->extent;
  }
  return (size_t)((t->count - 1) * t->stride + t->blocklen) * type_extent(t->base);
}

static size_t type_size(MPI_Datatype t){
  if(NULL == t->base){
    return t->extent;
  }
  return (size_t)t->count * (size_t)t->blocklen * type_size(t->base);
}

/* visit every basic element of one instance of "t" placed at byte offset "off"
 * and copy it between the packed stream and the typed buffer */
static void walk(MPI_Datatype t, size_t off, char * typed, char * packed, size_t * pos, int unpack){
  if(NULL == t->base){
    if(unpack){
      memcpy(typed + off, packed + *pos, t->extent);
    }else{
      memcpy(packed + *pos, typed + off, t->extent);
    }
    *pos += t->extent;
    return;
  }
  const size_t bext = type_extent(t->base);
  for(int b = 0; b < t->count; b++){
    for(int e = 0; e < t->blocklen; e++){
      walk(t->base, off + ((size_t)b * (size_t)t->stride + (size_t)e) * bext, typed, packed, pos, unpack);
    }
  }
}

int MPI_Init(int * argc, char *** argv){ (void)argc; (void)argv; return 0; }
int MPI_Finalize(void){ return 0; }
int MPI_Abort(MPI_Comm comm, int code){ (void)comm; exit(code == 0 ? 1 : code); }
int MPI_Barrier(MPI_Comm comm){ (void)comm; return 0; }
int MPI_Comm_rank(MPI_Comm comm, int * rank){ (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int * size){ (void)comm; *size = 1; return 0; }

double MPI_Wtime(void){
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1.e-9 * (double)ts.tv_nsec;
}

int MPI_Error_string(int code, char * string, int * length){
  *length = snprintf(string, MPI_MAX_ERROR_STRING, "shim MPI error %d", code);
  return 0;
}

int MPI_Bcast(void * buf, int count, MPI_Datatype type, int root, MPI_Comm comm){
  (void)buf; (void)count; (void)type; (void)root; (void)comm;
  return 0;
}

static void copy_reduce(const void * sendbuf, void * recvbuf, int count, MPI_Datatype type){
  if(MPI_IN_PLACE == sendbuf){
    return;
  }
  memcpy(recvbuf, sendbuf, (size_t)count * type_size(type));
}

int MPI_Allreduce(const void * sendbuf, void * recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm){
  (void)op; (void)comm;
  copy_reduce(sendbuf, recvbuf, count, type);
  return 0;
}

int MPI_Reduce(const void * sendbuf, void * recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm){
  (void)op; (void)root; (void)comm;
  copy_reduce(sendbuf, recvbuf, count, type);
  return 0;
}

int MPI_Sendrecv(
    const void * sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
    void * recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
    MPI_Comm comm, MPI_Status * status){
  (void)dest; (void)sendtag; (void)source; (void)recvtag; (void)comm; (void)status;
  const size_t nbytes = (size_t)sendcount * type_size(sendtype);
  if(nbytes != (size_t)recvcount * type_size(recvtype)){
    fprintf(stderr, "shim MPI_Sendrecv: message size mismatch\n");
    exit(1);
  }
  char * packed = malloc(nbytes > 0 ? nbytes : 1);
  size_t pos = 0;
  for(int n = 0; n < sendcount; n++){
    walk(sendtype, (size_t)n * type_extent(sendtype), (char *)sendbuf, packed, &pos, 0);
  }
  pos = 0;
  for(int n = 0; n < recvcount; n++){
    walk(recvtype, (size_t)n * type_extent(recvtype), (char *)recvbuf, packed, &pos, 1);
  }
  free(packed);
  return 0;
}

static MPI_Datatype new_type(int count, int blocklen, long stride, MPI_Datatype base){
  shim_mpi_type_t * t = calloc(1, sizeof(shim_mpi_type_t));
  t->count = count;
  t->blocklen = blocklen;
  t->stride = stride;
  t->base = base;
  return t;
}

int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype * newtype){
  *newtype = new_type(count, 1, 1, oldtype);
  return 0;
}

int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype, MPI_Datatype * newtype){
  *newtype = new_type(count, blocklength, stride, oldtype);
  return 0;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[], int order, MPI_Datatype oldtype, MPI_Datatype * newtype){
  (void)order;
  /* one rank owns the whole array, so the view must be the full array */
  long n = 1;
  for(int d = 0; d < ndims; d++){
    if(sizes[d] != subsizes[d] || 0 != starts[d]){
      fprintf(stderr, "shim MPI_Type_create_subarray: only whole-array views are supported\n");
      exit(1);
    }
    n *= sizes[d];
  }
  *newtype = new_type((int)n, 1, 1, oldtype);
  return 0;
}

int MPI_Type_commit(MPI_Datatype * type){ (void)type; return 0; }

int MPI_Type_free(MPI_Datatype * type){
  if(NULL != *type && NULL != (*type)->base){
    free((void *)*type);
  }
  *type = MPI_DATATYPE_NULL;
  return 0;
}

int MPI_File_open(MPI_Comm comm, const char * filename, int amode, MPI_Info info, MPI_File * fh){
  (void)comm; (void)info;
  const char * mode = (amode & MPI_MODE_RDONLY) ? "rb" : "r+b";
  FILE * fp = fopen(filename, mode);
  if(NULL == fp && (amode & MPI_MODE_CREATE)){
    fp = fopen(filename, "w+b");
  }
  if(NULL == fp){
    return 1;
  }
  *fh = calloc(1, sizeof(struct shim_mpi_file_t_));
  (*fh)->fp = fp;
  return 0;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype, const char * datarep, MPI_Info info){
  (void)etype; (void)filetype; (void)datarep; (void)info;
  fh->disp = disp;
  return 0;
}

int MPI_File_read_all(MPI_File fh, void * buf, int count, MPI_Datatype type, MPI_Status * status){
  (void)status;
  const size_t nbytes = (size_t)count * type_size(type);
  if(0 != fseek(fh->fp, (long)fh->disp, SEEK_SET)) return 1;
  if(nbytes != fread(buf, 1, nbytes, fh->fp)){
    fprintf(stderr, "shim MPI_File_read_all: short read\n");
    return 1;
  }
  return 0;
}

int MPI_File_write_all(MPI_File fh, const void * buf, int count, MPI_Datatype type, MPI_Status * status){
  (void)status;
  const size_t nbytes = (size_t)count * type_size(type);
  if(0 != fseek(fh->fp, (long)fh->disp, SEEK_SET)) return 1;
  if(nbytes != fwrite(buf, 1, nbytes, fh->fp)){
    fprintf(stderr, "shim MPI_File_write_all: short write\n");
    return 1;
  }
  return 0;
}

int MPI_File_close(MPI_File * fh){
  if(NULL != *fh){
    fclose((*fh)->fp);
    free(*fh);
    *fh = NULL;
  }
  return 0;
}
