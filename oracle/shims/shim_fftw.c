#define _POSIX_C_SOURCE 200809L
/*
 * FFTW3 stand-in (see fftw3.h).  TEST INFRASTRUCTURE ONLY.
 * Supports rank-1 batched transforms with unit stride, as the reference uses.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"
#include "../svof_fft.h"

enum { K_R2R_DCT2, K_R2R_DCT3, K_R2C, K_C2R };

struct svof_fftw_plan_s {
  int kind;
  int howmany;
  int idist, odist;
  double *in, *out;
  svof_fft_plan_t *plan;
};

static fftw_plan make(int kind, int rank, const int *n, int howmany, void *in, int istride,
                      int idist, void *out, int ostride, int odist) {
  if (1 != rank || 1 != istride || 1 != ostride) {
    fprintf(stderr, "fftw shim: only rank-1 unit-stride transforms are supported\n");
    return NULL;
  }
  fftw_plan p = calloc(1, sizeof(*p));
  p->kind = kind;
  p->howmany = howmany;
  p->idist = idist;
  p->odist = odist;
  p->in = in;
  p->out = out;
  p->plan = svof_fft_plan_create((size_t)n[0]);
  return p;
}

fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany,
                             double *in, const int *inembed, int istride, int idist,
                             double *out, const int *onembed, int ostride, int odist,
                             const fftw_r2r_kind *kind, unsigned flags) {
  (void)inembed; (void)onembed; (void)flags;
  int k;
  if (FFTW_REDFT10 == kind[0]) {
    k = K_R2R_DCT2;
  } else if (FFTW_REDFT01 == kind[0]) {
    k = K_R2R_DCT3;
  } else {
    fprintf(stderr, "fftw shim: unsupported r2r kind %d\n", (int)kind[0]);
    return NULL;
  }
  return make(k, rank, n, howmany, in, istride, idist, out, ostride, odist);
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)inembed; (void)onembed; (void)flags;
  return make(K_R2C, rank, n, howmany, in, istride, idist, (double *)out, ostride, odist);
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)inembed; (void)onembed; (void)flags;
  return make(K_C2R, rank, n, howmany, (double *)in, istride, idist, out, ostride, odist);
}

void fftw_execute(const fftw_plan p) {
  for (int m = 0; m < p->howmany; m++) {
    switch (p->kind) {
      case K_R2R_DCT2:
        svof_dct2(p->plan, p->in + (size_t)m * p->idist, p->out + (size_t)m * p->odist);
        break;
      case K_R2R_DCT3:
        svof_dct3(p->plan, p->in + (size_t)m * p->idist, p->out + (size_t)m * p->odist);
        break;
      case K_R2C:
        svof_fft_r2c(p->plan, p->in + (size_t)m * p->idist, p->out + 2 * (size_t)m * p->odist);
        break;
      case K_C2R:
        svof_fft_c2r(p->plan, p->in + 2 * (size_t)m * p->idist, p->out + (size_t)m * p->odist);
        break;
    }
  }
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  svof_fft_plan_destroy(p->plan);
  free(p);
}

void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (0 != posix_memalign(&p, 64, n ? n : 1)) return NULL;
  return p;
}

void fftw_free(void *p) { free(p); }
