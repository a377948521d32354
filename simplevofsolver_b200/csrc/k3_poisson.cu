// k3_poisson.cu -- pressure Poisson solve of the FP64 3D path.
//
// Right-hand side (divergence / (gamma dt ny nz)), r2c along y, complex DFT
// along z, complex Neumann Thomas along x for every (ky, kz), inverse DFT
// along z, c2r along y (src/fluid/compute_potential/dft.c:406-468 in 2D,
// with the second periodic direction of the restatement
// oracle/svof_oracle3d.c).  The spectral array is S[kz][ky][i], complex,
// x fastest: every transform reads and writes runs of consecutive i, and the
// x line solve reads each line contiguously.  No transpose pass exists.
//
//   k3_pois_fwd_y  a block owns COLS consecutive i of one plane k
//   k3_pois_z      a block owns COLS consecutive i of one ky, both signs
//   k3_pois_x      a block owns 32 lines (ky, kz), walked in 32-cell chunks:
//                  forward recurrence (values back into S, v into scratch),
//                  then back substitution in reverse chunk order
//   k3_pois_inv_y  a block owns COLS consecutive i of one plane k; writes psi
//                  with its halo images and Neumann walls
#include <type_traits>

#include "fft_device.cuh"
#include "svof3d_internal.cuh"

namespace svof3 {

using svof_fft_dev::bitrev;

// One warp per line.  Lines are stored re / im separately in shared memory
// with a row stride of n + 1 doubles, so that the column-wise loads and stores
// (consecutive threads on consecutive lines) and the butterflies (consecutive
// lanes on consecutive positions) are free of bank conflicts.  The butterflies
// are those of fft_stages (same pairs, same twiddles, same association).
__device__ __forceinline__ void warp_fft_line(double *__restrict__ re, double *__restrict__ im, int log2n,
                                              const double *__restrict__ tw) {
  const int lane = threadIdx.x & 31;
  const int nb = 1 << (log2n - 1);
  for (int st = 1; st <= log2n; st++) {
    const int half = 1 << (st - 1);
    const int sh = log2n - st;
    for (int b = lane; b < nb; b += 32) {
      const int grp = b >> (st - 1);
      const int kk = b & (half - 1);
      const int ia = (grp << st) + kk, ib = ia + half;
      const double2 w = __ldg(reinterpret_cast<const double2 *>(tw) + (kk << sh));
      const double xr = re[ib], xi = im[ib];
      const double tr = w.x * xr - w.y * xi;
      const double ti = w.x * xi + w.y * xr;
      const double ur = re[ia], ui = im[ia];
      re[ia] = ur + tr;
      im[ia] = ui + ti;
      re[ib] = ur - tr;
      im[ib] = ui - ti;
    }
    __syncwarp();
  }
}

template <int COLS>
__global__ void __launch_bounds__(32 * COLS) k3_pois_fwd_y(const double *__restrict__ ux,
                                                          const double *__restrict__ uy,
                                                          const double *__restrict__ uz, double *__restrict__ spec,
                                                          const double *__restrict__ tw,
                                                          const double *__restrict__ dtp, double gam, int log2n,
                                                          Grid3 g) {
  extern __shared__ double sm[];
  const int n = 1 << log2n, ld = n + 1, nx = g.nx, nky = n / 2 + 1;
  double *re = sm, *im = sm + COLS * ld;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  const double dt = ldg(dtp);
  const double prefactor = 1. / (gam * dt) / (1. * g.ny * g.nz);
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int q = w / COLS, col = w % COLS;
    const int m = bitrev(q, log2n);
    double v = 0.;
    if (col < nc) {
      const int i = i0 + col, j = m + 1;
      const double dx = ldg(g.dxf + i - 1);
      v = prefactor * (+(ldg(ux + ix_ux(g, i + 1, j, k)) - ldg(ux + ix_ux(g, i, j, k))) / dx +
                       (ldg(uy + ix_cc(g, i, j + 1, k)) - ldg(uy + ix_cc(g, i, j, k))) / g.dy +
                       (ldg(uz + ix_cc(g, i, j, k + 1)) - ldg(uz + ix_cc(g, i, j, k))) / g.dz);
    }
    re[col * ld + q] = v;
    im[col * ld + q] = 0.;
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line(re + col * ld, im + col * ld, log2n, tw);
  }
  __syncthreads();
  for (int w = threadIdx.x; w < nky * COLS; w += 32 * COLS) {
    const int ky = w / COLS, col = w % COLS;
    if (col < nc) {
      reinterpret_cast<double2 *>(spec)[((size_t)(k - 1) * nky + ky) * nx + (i0 - 1 + col)] =
          make_double2(re[col * ld + ky], im[col * ld + ky]);
    }
  }
}

// complex DFT along z, in place, for COLS consecutive i of one ky; the sign is
// the twiddle table's
template <int COLS>
__global__ void __launch_bounds__(32 * COLS) k3_pois_z(double *__restrict__ spec, const double *__restrict__ tw,
                                                      int log2n, Grid3 g) {
  extern __shared__ double sm[];
  const int n = 1 << log2n, ld = n + 1, nx = g.nx, nky = g.ny / 2 + 1;
  double *re = sm, *im = sm + COLS * ld;
  const int i0 = blockIdx.x * COLS;
  const int ky = blockIdx.y;
  const int nc = min(COLS, nx - i0);
  double2 *sp = reinterpret_cast<double2 *>(spec);
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int q = w / COLS, col = w % COLS;
    const int m = bitrev(q, log2n);
    double2 v = make_double2(0., 0.);
    if (col < nc) v = sp[((size_t)m * nky + ky) * nx + (i0 + col)];
    re[col * ld + q] = v.x;
    im[col * ld + q] = v.y;
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line(re + col * ld, im + col * ld, log2n, tw);
  }
  __syncthreads();
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int kz = w / COLS, col = w % COLS;
    if (col < nc) sp[((size_t)kz * nky + ky) * nx + (i0 + col)] = make_double2(re[col * ld + kz], im[col * ld + kz]);
  }
}

// complex Neumann Thomas along x per line (ky, kz): tdm_c = -pl - pu + lambda,
// lambda = evy[ky] + evz[kz], first / last diagonal + pl[0] / + pu[nx-1], then
// gtsv component-wise (src/tdm.c:17-50; dft.c:364-395 in 2D).  Warp 0 runs
// the recurrences with one line per lane; the other warps move the tiles.
constexpr int XL = kXsLines, XC = kXsChunk;

__global__ void __launch_bounds__(256) k3_pois_x(double *__restrict__ spec, double *__restrict__ scratch,
                                                 const double *__restrict__ pl, const double *__restrict__ pu,
                                                 const double *__restrict__ evy, const double *__restrict__ evz,
                                                 Grid3 g) {
  __shared__ double sre[XL][XC + 1], sim[XL][XC + 1], sv[XL][XC + 1];
  __shared__ double spl[XC], spu[XC];
  const int nx = g.nx, nky = g.ny / 2 + 1;
  const long nlines = (long)nky * g.nz;
  const long l0 = (long)blockIdx.x * XL;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int nchunks = (nx + XC - 1) / XC;
  const bool sweeper = (0 == ty) && (l0 + tx < nlines);
  double lam = 0.;
  if (sweeper) {
    const long l = l0 + tx;
    lam = evy[l % nky] + evz[l / nky];
  }
  double vprev = 0., qr = 0., qi = 0.;
  // ---------------------------------------------------------- forward
  for (int c = 0; c < nchunks; c++) {
    const int p0 = c * XC;
    if (tid < XC) {
      spl[tid] = (p0 + tid < nx) ? pl[p0 + tid] : 0.;
      spu[tid] = (p0 + tid < nx) ? pu[p0 + tid] : 0.;
    }
    for (int m = 0; m < XL / 8; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l < nlines && p < nx) {
        const double2 v = *reinterpret_cast<const double2 *>(spec + 2 * ((size_t)l * nx + p));
        sre[ll][tx] = v.x;
        sim[ll][tx] = v.y;
      }
    }
    __syncthreads();
    if (sweeper) {
      const int smax = min(XC, nx - p0);
      for (int s = 0; s < smax; s++) {
        const int i = p0 + s;
        const double l = spl[s], u = spu[s];
        double c = -l - u + lam;
        if (0 == i) c += l;
        if (nx - 1 == i) c += u;
        double xr = sre[tx][s], xi = sim[tx][s];
        if (0 == i) {
          vprev = u / c;
          qr = xr / c;
          qi = xi / c;
        } else if (i < nx - 1) {
          const double val = 1. / (c - l * vprev);
          vprev = val * (u);
          qr = val * (xr - l * qr);
          qi = val * (xi - l * qi);
        } else {
          const double val = c - l * vprev;
          if (fabs(val) > kDblEpsilon) {
            qr = 1. / val * (xr - l * qr);
            qi = 1. / val * (xi - l * qi);
          } else {
            qr = 0.;
            qi = 0.;
          }
        }
        sre[tx][s] = qr;
        sim[tx][s] = qi;
        sv[tx][s] = vprev;
      }
    }
    __syncthreads();
    for (int m = 0; m < XL / 8; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l < nlines && p < nx) {
        *reinterpret_cast<double2 *>(spec + 2 * ((size_t)l * nx + p)) = make_double2(sre[ll][tx], sim[ll][tx]);
        scratch[(size_t)l * nx + p] = sv[ll][tx];
      }
    }
    __syncthreads();
  }
  // ---------------------------------------------------------- backward
  double nr = 0., ni = 0.;
  for (int c = nchunks - 1; c >= 0; c--) {
    const int p0 = c * XC;
    for (int m = 0; m < XL / 8; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l < nlines && p < nx) {
        const double2 v = *reinterpret_cast<const double2 *>(spec + 2 * ((size_t)l * nx + p));
        sre[ll][tx] = v.x;
        sim[ll][tx] = v.y;
        sv[ll][tx] = scratch[(size_t)l * nx + p];
      }
    }
    __syncthreads();
    if (sweeper) {
      const int smax = min(XC, nx - p0);
      for (int s = smax - 1; s >= 0; s--) {
        const int i = p0 + s;
        if (nx - 1 == i) {
          nr = sre[tx][s];
          ni = sim[tx][s];
        } else {
          const double v = sv[tx][s];
          nr = sre[tx][s] - v * nr;
          ni = sim[tx][s] - v * ni;
          sre[tx][s] = nr;
          sim[tx][s] = ni;
        }
      }
    }
    __syncthreads();
    for (int m = 0; m < XL / 8; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l < nlines && p < nx) {
        *reinterpret_cast<double2 *>(spec + 2 * ((size_t)l * nx + p)) = make_double2(sre[ll][tx], sim[ll][tx]);
      }
    }
    __syncthreads();
  }
}

// c2r along y (Hermitian extension as FFTW's c2r reads it: Im of X_0 and
// X_{ny/2} ignored), psi of COLS consecutive i of plane k with the halo images;
// the Neumann walls take the new neighbour value and hand their old value to
// the halo images
template <int COLS>
__global__ void __launch_bounds__(32 * COLS) k3_pois_inv_y(const double *__restrict__ spec,
                                                          double *__restrict__ psi,
                                                          const double *__restrict__ tw, int log2n, Grid3 g) {
  extern __shared__ double sm[];
  const int n = 1 << log2n, ld = n + 1, nx = g.nx, ny = g.ny, nz = g.nz, nky = n / 2 + 1;
  double *re = sm, *im = sm + COLS * ld;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  const double2 *sp = reinterpret_cast<const double2 *>(spec);
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int q = w / COLS, col = w % COLS;
    const int m = bitrev(q, log2n);
    double r = 0., x = 0.;
    if (col < nc) {
      const size_t base = ((size_t)(k - 1) * nky) * nx + (i0 - 1 + col);
      if (0 == m) {
        r = __ldg(&sp[base].x);
      } else if (2 * m < n) {
        const double2 v = __ldg(&sp[base + (size_t)m * nx]);
        r = v.x;
        x = v.y;
      } else if (2 * m == n) {
        r = __ldg(&sp[base + (size_t)m * nx].x);
      } else {
        const double2 v = __ldg(&sp[base + (size_t)(n - m) * nx]);
        r = v.x;
        x = -v.y;
      }
    }
    re[col * ld + q] = r;
    im[col * ld + q] = x;
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line(re + col * ld, im + col * ld, log2n, tw);
  }
  __syncthreads();
  for (int w = threadIdx.x; w < n * COLS; w += 32 * COLS) {
    const int r = w / COLS, col = w % COLS;
    if (col >= nc) continue;
    const int i = i0 + col, j = r + 1;
    const double y = re[col * ld + r];
    for_images(j, k, ny, nz, true, [&](int jj, int kk) { psi[ix_cc(g, i, jj, kk)] = y; });
  }
  // Neumann walls of the interior rows of this plane
  const bool has_left = (1 == i0), has_right = (i0 + nc - 1 == nx);
  for (int w = threadIdx.x; w < 2 * n; w += 32 * COLS) {
    const int side = w / n, j = 1 + (w - side * n);
    if ((0 == side && !has_left) || (1 == side && !has_right)) continue;
    const int iw = side ? nx + 1 : 0;
    const int col = side ? nc - 1 : 0;
    const double nv = re[col * ld + (j - 1)];
    const double old = psi[ix_cc(g, iw, j, k)];
    psi[ix_cc(g, iw, j, k)] = nv;
    for_images(j, k, ny, nz, false, [&](int jj, int kk) { psi[ix_cc(g, iw, jj, kk)] = old; });
  }
}

// ---- host-side launchers (the templates stay in this translation unit)
namespace {
template <class F>
cudaError_t by_cols(int cols, F f) {
  switch (cols) {
    case 16: return f(std::integral_constant<int, 16>());
    case 8: return f(std::integral_constant<int, 8>());
    case 4: return f(std::integral_constant<int, 4>());
    default: return cudaErrorInvalidValue;
  }
}
size_t fft_smem(int n, int cols) { return sizeof(double) * 2 * (size_t)(n + 1) * cols; }
}  // namespace

cudaError_t pois_prepare(int ny, int cols_y, int nz, int cols_z) {
  cudaError_t e = by_cols(cols_y, [&](auto c) {
    constexpr int C = decltype(c)::value;
    cudaError_t r = cudaFuncSetAttribute(k3_pois_fwd_y<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fft_smem(ny, C));
    if (cudaSuccess != r) return r;
    return cudaFuncSetAttribute(k3_pois_inv_y<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fft_smem(ny, C));
  });
  if (cudaSuccess != e) return e;
  return by_cols(cols_z, [&](auto c) {
    constexpr int C = decltype(c)::value;
    return cudaFuncSetAttribute(k3_pois_z<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fft_smem(nz, C));
  });
}

cudaError_t pois_fwd_y(int cols, cudaStream_t st, const double *ux, const double *uy, const double *uz, double *spec,
                       const double *tw, const double *dtp, double gam, int log2n, Grid3 g) {
  return by_cols(cols, [&](auto c) {
    constexpr int C = decltype(c)::value;
    dim3 gr((g.nx + C - 1) / C, g.nz);
    k3_pois_fwd_y<C><<<gr, 32 * C, fft_smem(g.ny, C), st>>>(ux, uy, uz, spec, tw, dtp, gam, log2n, g);
    return cudaGetLastError();
  });
}

cudaError_t pois_z(int cols, cudaStream_t st, double *spec, const double *tw, int log2n, Grid3 g) {
  return by_cols(cols, [&](auto c) {
    constexpr int C = decltype(c)::value;
    dim3 gr((g.nx + C - 1) / C, g.ny / 2 + 1);
    k3_pois_z<C><<<gr, 32 * C, fft_smem(g.nz, C), st>>>(spec, tw, log2n, g);
    return cudaGetLastError();
  });
}

cudaError_t pois_inv_y(int cols, cudaStream_t st, const double *spec, double *psi, const double *tw, int log2n,
                       Grid3 g) {
  return by_cols(cols, [&](auto c) {
    constexpr int C = decltype(c)::value;
    dim3 gr((g.nx + C - 1) / C, g.nz);
    k3_pois_inv_y<C><<<gr, 32 * C, fft_smem(g.ny, C), st>>>(spec, psi, tw, log2n, g);
    return cudaGetLastError();
  });
}

}  // namespace svof3
