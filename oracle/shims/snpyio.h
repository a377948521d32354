/*
 * Stand-in for SimpleNpyIO's "snpyio.h" (github.com/NaokiHori/SimpleNpyIO,
 * branch "submodule"; commit not recorded in the mounted tree).  TEST
 * INFRASTRUCTURE ONLY.  Reads and writes NPY v1.0/v2.0 headers with the
 * signatures the reference calls at src/fileio.c:193 and src/fileio.c:250.
 * The dtype string keeps its quotes ("'<f8'"), as the reference compares it
 * against NPY_DOUBLE = "'<f8'" (src/fileio.c:21).
 */
#ifndef SVOF_SHIM_SNPYIO_H
#define SVOF_SHIM_SNPYIO_H

#include <stdbool.h>
#include <stddef.h>
#include <stdio.h>

int snpyio_r_header(size_t *ndim, size_t **shape, char **dtype, bool *is_fortran_order,
                    FILE *fp, size_t *header_size);
int snpyio_w_header(const size_t ndim, const size_t *shape, const char dtype[],
                    const bool is_fortran_order, FILE *fp, size_t *header_size);

#endif
