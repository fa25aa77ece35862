/*
 * Single-rank implementation of oracle/shim/sdecomp.h (oracle build only).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "sdecomp.h"

struct sdecomp_info_t_ {
  size_t ndims;
};

struct sdecomp_transpose_plan_t_ {
  size_t glsizes[3];
  size_t size_elem;
  sdecomp_pencil_t bef;
  sdecomp_pencil_t aft;
};

/* memory order of each pencil: order[0] is the fastest-varying direction */
static void pencil_order(const sdecomp_pencil_t pencil, int order[3]){
  switch(pencil){
    case SDECOMP_X1PENCIL:
    case SDECOMP_X2PENCIL:
      order[0] = 0; order[1] = 1; order[2] = 2; break;
    case SDECOMP_Y1PENCIL:
    case SDECOMP_Y2PENCIL:
      order[0] = 1; order[1] = 2; order[2] = 0; break;
    default:
      order[0] = 2; order[1] = 0; order[2] = 1; break;
  }
}

static int info_construct(const MPI_Comm comm_default, const size_t ndims, const size_t * dims, const bool * periods, sdecomp_info_t ** info){
  (void)comm_default; (void)periods;
  for(size_t d = 0; d < ndims; d++){
    if(1 != dims[d]){
      fprintf(stderr, "sdecomp shim: only a single process is supported\n");
      return 1;
    }
  }
  *info = calloc(1, sizeof(sdecomp_info_t));
  (*info)->ndims = ndims;
  return 0;
}

static int info_destruct(sdecomp_info_t * info){
  free(info);
  return 0;
}

static int get_comm_cart(const sdecomp_info_t * info, MPI_Comm * comm_cart){
  (void)info;
  *comm_cart = MPI_COMM_WORLD;
  return 0;
}

static int get_comm_rank(const sdecomp_info_t * info, int * rank){
  (void)info;
  *rank = 0;
  return 0;
}

static int get_neighbours(const sdecomp_info_t * info, const sdecomp_pencil_t pencil, const sdecomp_dir_t dir, int neighbours[2]){
  (void)info; (void)pencil; (void)dir;
  neighbours[0] = 0;
  neighbours[1] = 0;
  return 0;
}

static int get_pencil_mysize(const sdecomp_info_t * info, const sdecomp_pencil_t pencil, const sdecomp_dir_t dir, const size_t glsize, size_t * mysize){
  (void)info; (void)pencil; (void)dir;
  *mysize = glsize;
  return 0;
}

static int get_pencil_offset(const sdecomp_info_t * info, const sdecomp_pencil_t pencil, const sdecomp_dir_t dir, const size_t glsize, size_t * offset){
  (void)info; (void)pencil; (void)dir; (void)glsize;
  *offset = 0;
  return 0;
}

static int transpose_construct(const sdecomp_info_t * info, const sdecomp_pencil_t bef, const sdecomp_pencil_t aft, const size_t * gl_sizes, const size_t size_elem, sdecomp_transpose_plan_t ** plan){
  (void)info;
  *plan = calloc(1, sizeof(sdecomp_transpose_plan_t));
  for(int d = 0; d < 3; d++){
    (*plan)->glsizes[d] = gl_sizes[d];
  }
  (*plan)->size_elem = size_elem;
  (*plan)->bef = bef;
  (*plan)->aft = aft;
  return 0;
}

static int transpose_execute(sdecomp_transpose_plan_t * plan, const void * sendbuf, void * recvbuf){
  int ob[3], oa[3];
  pencil_order(plan->bef, ob);
  pencil_order(plan->aft, oa);
  const size_t * n = plan->glsizes;
  const size_t es = plan->size_elem;
  /* strides of each physical direction in both layouts */
  size_t sb[3], sa[3];
  sb[ob[0]] = 1; sb[ob[1]] = n[ob[0]]; sb[ob[2]] = n[ob[0]] * n[ob[1]];
  sa[oa[0]] = 1; sa[oa[1]] = n[oa[0]]; sa[oa[2]] = n[oa[0]] * n[oa[1]];
  const char * src = sendbuf;
  char * dst = recvbuf;
  for(size_t z = 0; z < n[2]; z++){
    for(size_t y = 0; y < n[1]; y++){
      for(size_t x = 0; x < n[0]; x++){
        const size_t ib = x * sb[0] + y * sb[1] + z * sb[2];
        const size_t ia = x * sa[0] + y * sa[1] + z * sa[2];
        memcpy(dst + es * ia, src + es * ib, es);
      }
    }
  }
  return 0;
}

static int transpose_destruct(sdecomp_transpose_plan_t * plan){
  free(plan);
  return 0;
}

const sdecomp_t sdecomp = {
  .construct = info_construct,
  .destruct = info_destruct,
  .get_comm_cart = get_comm_cart,
  .get_comm_rank = get_comm_rank,
  .get_neighbours = get_neighbours,
  .get_pencil_mysize = get_pencil_mysize,
  .get_pencil_offset = get_pencil_offset,
  .transpose = {
    .construct = transpose_construct,
    .execute = transpose_execute,
    .destruct = transpose_destruct,
  },
};
