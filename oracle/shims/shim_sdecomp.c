/*
 * Single-rank SimpleDecomp stand-in (see sdecomp.h).  TEST INFRASTRUCTURE ONLY.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "sdecomp.h"

struct sdecomp_info_t_ {
  size_t ndims;
  bool periods[3];
};

struct sdecomp_transpose_plan_t_ {
  size_t nx, ny;      /* global sizes in x and y */
  size_t elem;        /* bytes per element */
  int x1_to_y1;       /* direction */
};

static int construct(const MPI_Comm comm_default, const size_t ndims, const size_t *dims,
                     const bool *periods, sdecomp_info_t **info) {
  (void)comm_default; (void)dims;
  if (2 != ndims) {
    fprintf(stderr, "single-rank sdecomp: only 2D domains are supported\n");
    return 1;
  }
  *info = calloc(1, sizeof(sdecomp_info_t));
  (*info)->ndims = ndims;
  for (size_t d = 0; d < ndims; d++) (*info)->periods[d] = periods[d];
  return 0;
}

static int destruct(sdecomp_info_t *info) { free(info); return 0; }

static int get_comm_cart(const sdecomp_info_t *info, MPI_Comm *comm_cart) {
  (void)info;
  *comm_cart = MPI_COMM_WORLD;
  return 0;
}

static int get_comm_rank(const sdecomp_info_t *info, int *rank) { (void)info; *rank = 0; return 0; }

static int get_neighbours(const sdecomp_info_t *info, const sdecomp_pencil_t pencil,
                          const sdecomp_dir_t dir, int neighbours[2]) {
  (void)pencil;
  const int self = info->periods[dir] ? 0 : MPI_PROC_NULL;
  neighbours[0] = self;
  neighbours[1] = self;
  return 0;
}

static int get_pencil_mysize(const sdecomp_info_t *info, const sdecomp_pencil_t pencil,
                             const sdecomp_dir_t dir, const size_t glsize, size_t *mysize) {
  (void)info; (void)pencil; (void)dir;
  *mysize = glsize;
  return 0;
}

static int get_pencil_offset(const sdecomp_info_t *info, const sdecomp_pencil_t pencil,
                             const sdecomp_dir_t dir, const size_t glsize, size_t *offset) {
  (void)info; (void)pencil; (void)dir; (void)glsize;
  *offset = 0;
  return 0;
}

static int tr_construct(const sdecomp_info_t *info, const sdecomp_pencil_t pencil_before,
                        const sdecomp_pencil_t pencil_after, const size_t *gsizes,
                        const size_t size_elem, sdecomp_transpose_plan_t **plan) {
  (void)info;
  int fwd;
  if (SDECOMP_X1PENCIL == pencil_before && SDECOMP_Y1PENCIL == pencil_after) {
    fwd = 1;
  } else if (SDECOMP_Y1PENCIL == pencil_before && SDECOMP_X1PENCIL == pencil_after) {
    fwd = 0;
  } else {
    fprintf(stderr, "single-rank sdecomp: unsupported transpose %d -> %d\n", pencil_before, pencil_after);
    return 1;
  }
  *plan = calloc(1, sizeof(sdecomp_transpose_plan_t));
  (*plan)->nx = gsizes[0];
  (*plan)->ny = gsizes[1];
  (*plan)->elem = size_elem;
  (*plan)->x1_to_y1 = fwd;
  return 0;
}

/* x1 pencil: element (i, j) at j * nx + i; y1 pencil: element (i, j) at i * ny + j */
static int tr_execute(sdecomp_transpose_plan_t *plan, const void *sendbuf, void *recvbuf) {
  const size_t nx = plan->nx, ny = plan->ny, e = plan->elem;
  const char *s = sendbuf;
  char *r = recvbuf;
  for (size_t j = 0; j < ny; j++) {
    for (size_t i = 0; i < nx; i++) {
      const size_t x1 = j * nx + i, y1 = i * ny + j;
      if (plan->x1_to_y1) {
        memcpy(r + e * y1, s + e * x1, e);
      } else {
        memcpy(r + e * x1, s + e * y1, e);
      }
    }
  }
  return 0;
}

static int tr_destruct(sdecomp_transpose_plan_t *plan) { free(plan); return 0; }

const sdecomp_t sdecomp = {
  .construct = construct,
  .destruct = destruct,
  .get_comm_cart = get_comm_cart,
  .get_comm_rank = get_comm_rank,
  .get_neighbours = get_neighbours,
  .get_pencil_mysize = get_pencil_mysize,
  .get_pencil_offset = get_pencil_offset,
  .transpose = {
    .construct = tr_construct,
    .execute = tr_execute,
    .destruct = tr_destruct,
  },
};
