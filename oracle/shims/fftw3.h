/*
 * Stand-in for <fftw3.h>.  TEST INFRASTRUCTURE ONLY.  FFTW3 is a system
 * library of the reference (CI installs Ubuntu's libfftw3-dev, version not
 * pinned: .github/workflows/ci.yml:29) and is absent here.  This header
 * provides exactly the calls of src/fluid/compute_potential/dct.c:197-231 and
 * src/fluid/compute_potential/dft.c:226-261 with FFTW's documented
 * unnormalised definitions, computed by oracle/svof_fft.c.  As in FFTW, when
 * <complex.h> is included first, fftw_complex is the native C99 complex type
 * (the reference's tdm.c does arithmetic on it).
 */
#ifndef SVOF_SHIM_FFTW3_H
#define SVOF_SHIM_FFTW3_H

#include <complex.h>
#include <stddef.h>

typedef double _Complex fftw_complex;
typedef struct svof_fftw_plan_s *fftw_plan;

typedef enum {
  FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
  FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
  FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_r2r(int rank, const int *n, int howmany,
                             double *in, const int *inembed, int istride, int idist,
                             double *out, const int *onembed, int ostride, int odist,
                             const fftw_r2r_kind *kind, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#endif
