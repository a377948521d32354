/*
 * svof_fft.c -- see svof_fft.h.  TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Transform definitions follow FFTW3's documented kinds as called by the
 * reference at src/fluid/compute_potential/dct.c:209-220 (REDFT10, REDFT01)
 * and src/fluid/compute_potential/dft.c:239-250 (r2c, c2r).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "svof_fft.h"

static const double SVOF_PI = 3.14159265358979323846;

static int is_pow2(size_t n) { return n >= 1 && 0 == (n & (n - 1)); }

void svof_fft_twiddles(size_t n, int sign, double *tw) {
  for (size_t m = 0; m < n / 2; m++) {
    const double ang = 2.0 * SVOF_PI * (double)m / (double)n;
    tw[2 * m + 0] = cos(ang);
    tw[2 * m + 1] = sign < 0 ? -sin(ang) : sin(ang);
  }
}

void svof_dct_twiddles(size_t n, double *cs) {
  for (size_t k = 0; k < n; k++) {
    const double ang = SVOF_PI * (double)k / (2.0 * (double)n);
    cs[2 * k + 0] = cos(ang);
    cs[2 * k + 1] = sin(ang);
  }
}

svof_fft_plan_t *svof_fft_plan_create(size_t n) {
  if (n < 1) return NULL;
  svof_fft_plan_t *p = calloc(1, sizeof(*p));
  p->n = n;
  p->pow2 = is_pow2(n);
  p->twf = calloc(n / 2 + 1, 2 * sizeof(double));
  p->twb = calloc(n / 2 + 1, 2 * sizeof(double));
  p->cs = calloc(n, 2 * sizeof(double));
  p->work = calloc(2 * n + 2, sizeof(double));
  svof_fft_twiddles(n, -1, p->twf);
  svof_fft_twiddles(n, +1, p->twb);
  svof_dct_twiddles(n, p->cs);
  if (p->pow2) {
    p->rev = calloc(n, sizeof(size_t));
    size_t bits = 0;
    while (((size_t)1 << bits) < n) bits++;
    for (size_t i = 0; i < n; i++) {
      size_t r = 0;
      for (size_t b = 0; b < bits; b++) {
        if (i & ((size_t)1 << b)) r |= (size_t)1 << (bits - 1 - b);
      }
      p->rev[i] = r;
    }
  }
  return p;
}

void svof_fft_plan_destroy(svof_fft_plan_t *p) {
  if (!p) return;
  free(p->twf);
  free(p->twb);
  free(p->cs);
  free(p->rev);
  free(p->work);
  free(p);
}

/* radix-2 DIT; butterfly: t = w * z[b]; z[a] = z[a] + t; z[b] = z[a] - t */
static void c2c_pow2(const svof_fft_plan_t *p, double *z, int sign) {
  const size_t n = p->n;
  const double *tw = sign < 0 ? p->twf : p->twb;
  for (size_t i = 0; i < n; i++) {
    const size_t j = p->rev[i];
    if (j > i) {
      const double r = z[2 * i], im = z[2 * i + 1];
      z[2 * i] = z[2 * j];
      z[2 * i + 1] = z[2 * j + 1];
      z[2 * j] = r;
      z[2 * j + 1] = im;
    }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const size_t half = len >> 1;
    const size_t step = n / len;
    for (size_t s = 0; s < n; s += len) {
      for (size_t k = 0; k < half; k++) {
        const double wr = tw[2 * (k * step) + 0];
        const double wi = tw[2 * (k * step) + 1];
        const size_t a = s + k, b = a + half;
        const double xr = z[2 * b], xi = z[2 * b + 1];
        const double tr = wr * xr - wi * xi;
        const double ti = wr * xi + wi * xr;
        const double ur = z[2 * a], ui = z[2 * a + 1];
        z[2 * a] = ur + tr;
        z[2 * a + 1] = ui + ti;
        z[2 * b] = ur - tr;
        z[2 * b + 1] = ui - ti;
      }
    }
  }
}

/* direct O(n^2) DFT for other lengths */
static void c2c_naive(const svof_fft_plan_t *p, double *z, int sign) {
  const size_t n = p->n;
  double *w = p->work;
  for (size_t k = 0; k < n; k++) {
    double sr = 0.0, si = 0.0;
    for (size_t m = 0; m < n; m++) {
      const size_t idx = (k * m) % n;
      const double ang = 2.0 * SVOF_PI * (double)idx / (double)n;
      const double c = cos(ang), s = sign < 0 ? -sin(ang) : sin(ang);
      sr += c * z[2 * m] - s * z[2 * m + 1];
      si += c * z[2 * m + 1] + s * z[2 * m];
    }
    w[2 * k] = sr;
    w[2 * k + 1] = si;
  }
  memcpy(z, w, 2 * n * sizeof(double));
}

void svof_fft_c2c(const svof_fft_plan_t *p, double *z, int sign) {
  if (p->pow2) {
    c2c_pow2(p, z, sign);
  } else {
    c2c_naive(p, z, sign);
  }
}

void svof_fft_r2c(const svof_fft_plan_t *p, const double *in, double *out) {
  const size_t n = p->n;
  double *z = malloc(2 * n * sizeof(double));
  for (size_t i = 0; i < n; i++) {
    z[2 * i] = in[i];
    z[2 * i + 1] = 0.0;
  }
  svof_fft_c2c(p, z, -1);
  memcpy(out, z, 2 * (n / 2 + 1) * sizeof(double));
  free(z);
}

void svof_fft_c2r(const svof_fft_plan_t *p, const double *in, double *out) {
  const size_t n = p->n;
  double *z = malloc(2 * n * sizeof(double));
  z[0] = in[0];
  z[1] = 0.0;
  for (size_t k = 1; k < n; k++) {
    if (2 * k < n) {
      z[2 * k] = in[2 * k];
      z[2 * k + 1] = in[2 * k + 1];
    } else if (2 * k == n) {
      z[2 * k] = in[2 * k];
      z[2 * k + 1] = 0.0;
    } else {
      const size_t m = n - k;
      z[2 * k] = in[2 * m];
      z[2 * k + 1] = -in[2 * m + 1];
    }
  }
  svof_fft_c2c(p, z, +1);
  for (size_t i = 0; i < n; i++) out[i] = z[2 * i];
  free(z);
}

/* REDFT10 via Makhoul: v_i = x_{2i}, v_{n-1-i} = x_{2i+1};
 * Y_k = 2 (cos(pi k/2n) Re V_k + sin(pi k/2n) Im V_k) */
void svof_dct2(const svof_fft_plan_t *p, const double *in, double *out) {
  const size_t n = p->n;
  if (!p->pow2 || n < 2) {
    for (size_t k = 0; k < n; k++) {
      double s = 0.0;
      for (size_t m = 0; m < n; m++) {
        s += in[m] * cos(SVOF_PI * (double)(k * (2 * m + 1)) / (2.0 * (double)n));
      }
      out[k] = 2.0 * s;
    }
    return;
  }
  double *z = malloc(2 * n * sizeof(double));
  for (size_t i = 0; i < n / 2; i++) {
    z[2 * i] = in[2 * i];
    z[2 * i + 1] = 0.0;
    z[2 * (n - 1 - i)] = in[2 * i + 1];
    z[2 * (n - 1 - i) + 1] = 0.0;
  }
  svof_fft_c2c(p, z, -1);
  for (size_t k = 0; k < n; k++) {
    const double c = p->cs[2 * k], s = p->cs[2 * k + 1];
    out[k] = 2.0 * (c * z[2 * k] + s * z[2 * k + 1]);
  }
  free(z);
}

/* REDFT01 via the inverse reordering: Z_k = exp(i pi k/2n) (X_k - i X_{n-k}),
 * X_n = 0; z = backward FFT(Z); y_{2i} = Re z_i, y_{2i+1} = Re z_{n-1-i} */
void svof_dct3(const svof_fft_plan_t *p, const double *in, double *out) {
  const size_t n = p->n;
  if (!p->pow2 || n < 2) {
    for (size_t m = 0; m < n; m++) {
      double s = 0.0;
      for (size_t k = 1; k < n; k++) {
        s += in[k] * cos(SVOF_PI * (double)(k * (2 * m + 1)) / (2.0 * (double)n));
      }
      out[m] = in[0] + 2.0 * s;
    }
    return;
  }
  double *z = malloc(2 * n * sizeof(double));
  for (size_t k = 0; k < n; k++) {
    const double a = in[k];
    const double b = 0 == k ? 0.0 : in[n - k];
    const double c = p->cs[2 * k], s = p->cs[2 * k + 1];
    z[2 * k] = c * a + s * b;
    z[2 * k + 1] = s * a - c * b;
  }
  svof_fft_c2c(p, z, +1);
  for (size_t i = 0; i < n / 2; i++) {
    out[2 * i] = z[2 * i];
    out[2 * i + 1] = z[2 * (n - 1 - i)];
  }
  free(z);
}
