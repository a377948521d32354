/*
 * Single-rank stand-in for SimpleDecomp's "sdecomp.h".  TEST INFRASTRUCTURE
 * ONLY.  SimpleDecomp (github.com/NaokiHori/SimpleDecomp, branch
 * "submodule"; commit not recorded in the mounted tree) is an un-vendored
 * submodule of the reference.  Only the call sites the reference makes are
 * provided (src/domain.c:195-206, src/halo.c:24-29, src/linear_system.c:46-61,
 * src/fluid/compute_potential/{dct,dft}.c), with one-process meaning:
 *   - every pencil holds the whole global array (mysize = glsize, offset 0);
 *   - the periodic y neighbours of rank 0 are rank 0 itself, the x
 *     neighbours are MPI_PROC_NULL;
 *   - an x1 pencil is stored x-fastest ([j][i]), a y1 pencil y-fastest
 *     ([i][j]); the x1<->y1 transpose is the local 2D transpose.
 */
#ifndef SVOF_SHIM_SDECOMP_H
#define SVOF_SHIM_SDECOMP_H

#include <stdbool.h>
#include <stddef.h>
#include <mpi.h>

typedef enum {
  SDECOMP_XDIR = 0,
  SDECOMP_YDIR = 1,
  SDECOMP_ZDIR = 2
} sdecomp_dir_t;

typedef enum {
  SDECOMP_X1PENCIL = 0,
  SDECOMP_Y1PENCIL = 1,
  SDECOMP_Z1PENCIL = 2,
  SDECOMP_X2PENCIL = 3,
  SDECOMP_Y2PENCIL = 4,
  SDECOMP_Z2PENCIL = 5
} sdecomp_pencil_t;

typedef struct sdecomp_info_t_ sdecomp_info_t;
typedef struct sdecomp_transpose_plan_t_ sdecomp_transpose_plan_t;

typedef struct {
  int (*const construct)(const sdecomp_info_t *info, const sdecomp_pencil_t pencil_before,
                         const sdecomp_pencil_t pencil_after, const size_t *gsizes,
                         const size_t size_elem, sdecomp_transpose_plan_t **plan);
  int (*const execute)(sdecomp_transpose_plan_t *plan, const void *sendbuf, void *recvbuf);
  int (*const destruct)(sdecomp_transpose_plan_t *plan);
} sdecomp_transpose_t;

typedef struct {
  int (*const construct)(const MPI_Comm comm_default, const size_t ndims, const size_t *dims,
                         const bool *periods, sdecomp_info_t **info);
  int (*const destruct)(sdecomp_info_t *info);
  int (*const get_comm_cart)(const sdecomp_info_t *info, MPI_Comm *comm_cart);
  int (*const get_comm_rank)(const sdecomp_info_t *info, int *rank);
  int (*const get_neighbours)(const sdecomp_info_t *info, const sdecomp_pencil_t pencil,
                              const sdecomp_dir_t dir, int neighbours[2]);
  int (*const get_pencil_mysize)(const sdecomp_info_t *info, const sdecomp_pencil_t pencil,
                                 const sdecomp_dir_t dir, const size_t glsize, size_t *mysize);
  int (*const get_pencil_offset)(const sdecomp_info_t *info, const sdecomp_pencil_t pencil,
                                 const sdecomp_dir_t dir, const size_t glsize, size_t *offset);
  sdecomp_transpose_t transpose;
} sdecomp_t;

extern const sdecomp_t sdecomp;

#endif
