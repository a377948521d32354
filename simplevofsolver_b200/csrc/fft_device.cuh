// fft_device.cuh -- radix-2 decimation-in-time butterflies shared by the 2D
// and 3D Poisson kernels.  The stages are the oracle's (oracle/svof_fft.c):
// data in bit-reversed order, twiddle w_m = exp(-+ 2 pi i m / n) from a host
// table, t = w * x_b, (x_a, x_b) <- (x_a + t, x_a - t).  With FMA contraction
// disabled the results agree with the oracle bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace svof_fft_dev {

__device__ __forceinline__ int bitrev(int q, int log2n) { return (int)(__brev((unsigned)q) >> (32 - log2n)); }

// butterfly stages of `lines` independent transforms of length n = 2^log2n
// stored back to back as interleaved complex values, already in bit-reversed
// order; all threads of the block take part and the call ends synchronised
__device__ __forceinline__ void fft_stages(double *z, int log2n, int lines, const double *__restrict__ tw) {
  const int n = 1 << log2n;
  const int nb = lines * (n >> 1);
  for (int s = 1; s <= log2n; s++) {
    const int half = 1 << (s - 1);
    const int len = half << 1;
    const int step = n >> s;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int line = b / (n >> 1);
      const int bb = b - line * (n >> 1);
      const int grp = bb >> (s - 1);
      const int k = bb & (half - 1);
      double *zz = z + 2 * line * n;
      const int ia = grp * len + k, ib = ia + half;
      const double wr = tw[2 * (k * step) + 0];
      const double wi = tw[2 * (k * step) + 1];
      const double xr = zz[2 * ib], xi = zz[2 * ib + 1];
      const double tr = wr * xr - wi * xi;
      const double ti = wr * xi + wi * xr;
      const double ur = zz[2 * ia], ui = zz[2 * ia + 1];
      zz[2 * ia] = ur + tr;
      zz[2 * ia + 1] = ui + ti;
      zz[2 * ib] = ur - tr;
      zz[2 * ib + 1] = ui - ti;
    }
    __syncthreads();
  }
}


// ---------------------------------------------------------------------------
// Register-blocked passes over COLS independent lines of N = 2^L2N points
// (N a compile-time constant): the same radix-2 butterflies (pairs, twiddles,
// association and stage order) run in passes of up to three stages.  In a
// pass a thread takes (line, group) pairs, lines fastest across the lanes,
// loads the 2^NS points of its group, runs their butterflies in registers and
// stores them.  The first pass reads its points (in bit-reversed order)
// through a caller's `first` and the last one hands its results to `last`;
// the passes between go through shared memory, re / im separately, point p
// of line c at c LD + p + p / 8 with LD = N + N / 8 + 1 odd, so the lanes of
// a half warp, on distinct lines, fall on distinct banks.

template <class R>
struct Cplx;
template <>
struct Cplx<double> {
  using T = double2;
  static __device__ __forceinline__ T make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Cplx<float> {
  using T = float2;
  static __device__ __forceinline__ T make(float a, float b) { return make_float2(a, b); }
};

__device__ __forceinline__ int fpad(int p) { return p + (p >> 3); }

// the shared-memory pitch of a line of 2^l2n points
__host__ __device__ constexpr int fft_ld(int l2n) { return (1 << l2n) + ((1 << l2n) >> 3) + 1; }

// twiddle loads: read-only path, kept in L1 ahead of the streaming data
__device__ __forceinline__ double2 tw_ld(const double2 *p) {
  double2 v;
  asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ float2 tw_ld(const float2 *p) {
  float2 v;
  asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
}

// the butterflies of stages S0 .. S0 + NS - 1 of group gi, in registers
template <class R, int L2N, int S0, int NS>
__device__ __forceinline__ void butterflies(int gi, R *xr, R *xi, const R *__restrict__ tw) {
  using C2 = typename Cplx<R>::T;
  constexpr int G = 1 << NS, H = 1 << (S0 - 1);
#pragma unroll
  for (int t = 0; t < NS; t++) {
    const int st_ = S0 + t, dist = 1 << t;
#pragma unroll
    for (int m = 0; m < G; m++) {
      if (m & dist) continue;
      // twiddle of the pair (base + m H, base + (m + dist) H) at stage st_
      const int kk = (gi & (H - 1)) + (m & (dist - 1)) * H;
      const C2 w = tw_ld(reinterpret_cast<const C2 *>(tw) + (kk << (L2N - st_)));
      const R br = xr[m + dist], bi = xi[m + dist];
      const R tr = w.x * br - w.y * bi;
      const R ti = w.x * bi + w.y * br;
      const R ur = xr[m], ui = xi[m];
      xr[m] = ur + tr;
      xi[m] = ui + ti;
      xr[m + dist] = ur - tr;
      xi[m + dist] = ui - ti;
    }
  }
}

// stages S0 .. S0 + NS - 1 of the block's COLS lines: ld(c, base, G, H, re,
// im) fetches the G points base + m H (m < G) of line c into re[m], im[m],
// st(c, base, G, H, re, im) stores them (G and H as integral constants)
template <class R, int L2N, int COLS, int S0, int NS, int THREADS, class LdF, class StF>
__device__ __forceinline__ void fft_pass(const R *__restrict__ tw, LdF ld, StF st) {
  constexpr int G = 1 << NS, H = 1 << (S0 - 1), NG = (1 << L2N) >> NS, PAIRS = COLS * NG;
  using GC = std::integral_constant<int, G>;
  using HC = std::integral_constant<int, H>;
#pragma unroll
  for (int p0 = 0; p0 < PAIRS; p0 += THREADS) {
    const int pr = p0 + (int)threadIdx.x;
    if (0 == PAIRS % THREADS || pr < PAIRS) {
      const int c = pr % COLS, gi = pr / COLS;
      const int base = (gi & (H - 1)) + ((gi >> (S0 - 1)) << (S0 - 1 + NS));
      R xr[G], xi[G];
      ld(c, base, GC(), HC(), xr, xi);
      butterflies<R, L2N, S0, NS>(gi, xr, xi, tw);
      st(c, base, GC(), HC(), xr, xi);
    }
  }
}

// all passes: the first reads through `first`, the last writes through `last`
template <class R, int L2N, int COLS, int S0 = 1, int THREADS = 256, class FirstF, class LastF>
__device__ __forceinline__ void fft_lines(R *__restrict__ re, R *__restrict__ im, const R *__restrict__ tw,
                                          FirstF first, LastF last) {
  constexpr int LD = fft_ld(L2N);
  constexpr int NS = (L2N - S0 + 1) < 3 ? (L2N - S0 + 1) : 3;
  constexpr bool IS_FIRST = (1 == S0), IS_LAST = (S0 + NS > L2N);
  auto lds = [&](int c, int base, auto gc, auto hc, R *xr, R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int m = 0; m < G; m++) {
      xr[m] = re[c * LD + fpad(base + m * H)];
      xi[m] = im[c * LD + fpad(base + m * H)];
    }
  };
  auto sts = [&](int c, int base, auto gc, auto hc, const R *xr, const R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int m = 0; m < G; m++) {
      re[c * LD + fpad(base + m * H)] = xr[m];
      im[c * LD + fpad(base + m * H)] = xi[m];
    }
  };
  if constexpr (IS_FIRST && IS_LAST) {
    fft_pass<R, L2N, COLS, S0, NS, THREADS>(tw, first, last);
  } else if constexpr (IS_FIRST) {
    fft_pass<R, L2N, COLS, S0, NS, THREADS>(tw, first, sts);
  } else if constexpr (IS_LAST) {
    fft_pass<R, L2N, COLS, S0, NS, THREADS>(tw, lds, last);
  } else {
    fft_pass<R, L2N, COLS, S0, NS, THREADS>(tw, lds, sts);
  }
  if constexpr (!IS_LAST) {
    __syncthreads();
    fft_lines<R, L2N, COLS, S0 + NS, THREADS>(re, im, tw, first, last);
  }
}

}  // namespace svof_fft_dev
