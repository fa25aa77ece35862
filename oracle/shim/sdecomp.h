/*
 * Single-rank stand-in for the SimpleDecomp API surface that SimpleTCSolver
 * calls (oracle build only). SimpleDecomp's sources are not vendored with the
 * reference (empty submodule, reference .gitmodules:1-4), so this restates the
 * behaviour its call sites rely on for a 1x1x1 process grid:
 *   - every pencil holds the whole global array (mysize == glsize, offset 0);
 *   - neighbours in y and z are the rank itself (periodic);
 *   - a transpose is a local permutation between the pencils' memory orders.
 * Memory orders (fastest index first), as the consumers index them:
 *   X1, X2: (x, y, z)   src/fluid/compute_potential.c:467-484
 *   Y1, Y2: (y, z, x)   src/fluid/predict/linear_system.c:61-67
 *   Z1, Z2: (z, x, y)   src/fluid/predict/linear_system.c:94-100
 */
#if !defined(TCREF_SHIM_SDECOMP_H)
#define TCREF_SHIM_SDECOMP_H

#include <stddef.h>
#include <stdbool.h>
#include <mpi.h>

typedef enum {
  SDECOMP_X1PENCIL = 0,
  SDECOMP_Y1PENCIL = 1,
  SDECOMP_Z1PENCIL = 2,
  SDECOMP_X2PENCIL = 3,
  SDECOMP_Y2PENCIL = 4,
  SDECOMP_Z2PENCIL = 5,
} sdecomp_pencil_t;

typedef enum {
  SDECOMP_XDIR = 0,
  SDECOMP_YDIR = 1,
  SDECOMP_ZDIR = 2,
} sdecomp_dir_t;

typedef struct sdecomp_info_t_ sdecomp_info_t;
typedef struct sdecomp_transpose_plan_t_ sdecomp_transpose_plan_t;

typedef struct {
  int (* const construct)(
      const sdecomp_info_t * info,
      const sdecomp_pencil_t pencil_bef,
      const sdecomp_pencil_t pencil_aft,
      const size_t * gl_sizes,
      const size_t size_elem,
      sdecomp_transpose_plan_t ** plan
  );
  int (* const execute)(
      sdecomp_transpose_plan_t * plan,
      const void * sendbuf,
      void * recvbuf
  );
  int (* const destruct)(
      sdecomp_transpose_plan_t * plan
  );
} sdecomp_transpose_t;

typedef struct {
  int (* const construct)(
      const MPI_Comm comm_default,
      const size_t ndims,
      const size_t * dims,
      const bool * periods,
      sdecomp_info_t ** info
  );
  int (* const destruct)(
      sdecomp_info_t * info
  );
  int (* const get_comm_cart)(
      const sdecomp_info_t * info,
      MPI_Comm * comm_cart
  );
  int (* const get_comm_rank)(
      const sdecomp_info_t * info,
      int * rank
  );
  int (* const get_neighbours)(
      const sdecomp_info_t * info,
      const sdecomp_pencil_t pencil,
      const sdecomp_dir_t dir,
      int neighbours[2]
  );
  int (* const get_pencil_mysize)(
      const sdecomp_info_t * info,
      const sdecomp_pencil_t pencil,
      const sdecomp_dir_t dir,
      const size_t glsize,
      size_t * mysize
  );
  int (* const get_pencil_offset)(
      const sdecomp_info_t * info,
      const sdecomp_pencil_t pencil,
      const sdecomp_dir_t dir,
      const size_t glsize,
      size_t * offset
  );
  const sdecomp_transpose_t transpose;
} sdecomp_t;

extern const sdecomp_t sdecomp;

#endif // TCREF_SHIM_SDECOMP_H
