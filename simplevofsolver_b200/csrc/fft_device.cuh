// fft_device.cuh -- radix-2 decimation-in-time butterflies shared by the 2D
// and 3D Poisson kernels.  The stages are the oracle's (oracle/svof_fft.c):
// data in bit-reversed order, twiddle w_m = exp(-+ 2 pi i m / n) from a host
// table, t = w * x_b, (x_a, x_b) <- (x_a + t, x_a - t).  With FMA contraction
// disabled the results agree with the oracle bit for bit.
#pragma once

#include <cuda_runtime.h>

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

}  // namespace svof_fft_dev
