/*
 * svof_fft.h -- CPU fast Fourier / cosine transforms used by the oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This file belongs to the oracle (the CPU checker
 * of the CUDA path); the product library never links it.
 *
 * The reference (SimpleVOFSolver) calls FFTW3 for four one-dimensional real
 * transforms (src/fluid/compute_potential/dct.c:209-220 and
 * src/fluid/compute_potential/dft.c:239-250).  FFTW is absent from this
 * machine, so the oracle implements FFTW's documented, unnormalised
 * definitions itself:
 *
 *   REDFT10 (DCT-II)  Y_k = 2 sum_{n=0}^{N-1} x_n cos(pi k (2n+1) / (2N))
 *   REDFT01 (DCT-III) y_n = X_0 + 2 sum_{k=1}^{N-1} X_k cos(pi k (2n+1) / (2N))
 *   r2c               X_k = sum_n x_n exp(-2 pi i k n / N),  k = 0 .. N/2
 *   c2r               x_n = sum_{k=0}^{N-1} X_k exp(+2 pi i k n / N), X
 *                     Hermitian; Im X_0 and Im X_{N/2} are ignored
 *
 * Power-of-two lengths use an iterative radix-2 decimation-in-time complex
 * FFT with twiddles from libm cos/sin; the DCTs use Makhoul's N-point
 * reordering.  The CUDA kernels perform the same butterflies in the same
 * order with the same twiddle tables (uploaded from the host), so the two
 * agree to the last bit when the CUDA code is compiled without FMA
 * contraction.  Other lengths fall back to direct O(N^2) sums.
 */
#ifndef SVOF_FFT_H
#define SVOF_FFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  size_t n;
  int pow2;
  /* forward (exp(-i...)) and backward (exp(+i...)) twiddles, interleaved
   * (re, im), n/2 entries each: w_m = exp(-+ 2 pi i m / n) */
  double *twf;
  double *twb;
  /* DCT post/pre twiddles, interleaved (cos, sin) of pi k / (2n), n entries */
  double *cs;
  /* bit-reversal permutation (power-of-two lengths only) */
  size_t *rev;
  /* scratch, 2n doubles */
  double *work;
} svof_fft_plan_t;

svof_fft_plan_t *svof_fft_plan_create(size_t n);
void svof_fft_plan_destroy(svof_fft_plan_t *plan);

/* in-place complex transform of n interleaved (re, im) pairs;
 * sign = -1 forward, +1 backward (unnormalised) */
void svof_fft_c2c(const svof_fft_plan_t *plan, double *z, int sign);
/* real -> half-complex: out holds n/2+1 interleaved pairs */
void svof_fft_r2c(const svof_fft_plan_t *plan, const double *in, double *out);
/* half-complex -> real (unnormalised) */
void svof_fft_c2r(const svof_fft_plan_t *plan, const double *in, double *out);
/* FFTW_REDFT10 */
void svof_dct2(const svof_fft_plan_t *plan, const double *in, double *out);
/* FFTW_REDFT01 */
void svof_dct3(const svof_fft_plan_t *plan, const double *in, double *out);

/* twiddle tables exactly as the plan builds them (for device upload) */
void svof_fft_twiddles(size_t n, int sign, double *tw /* n/2 pairs */);
void svof_dct_twiddles(size_t n, double *cs /* n pairs */);

#ifdef __cplusplus
}
#endif

#endif
