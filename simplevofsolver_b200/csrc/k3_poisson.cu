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
//   k3_pois_fwd_y  a block owns `cols` consecutive i of one plane k
//   k3_pois_z      a block owns `cols` consecutive i of one ky, both signs
//   k3_pois_x      a block owns 32 lines (ky, kz), walked in 32-cell chunks:
//                  forward recurrence (values back into S, v into scratch),
//                  then back substitution in reverse chunk order
//   k3_pois_inv_y  a block owns `cols` consecutive i of one plane k; writes psi
//                  with its halo images and Neumann walls
#include "fft_device.cuh"
#include "svof3d_internal.cuh"

namespace svof3 {

using svof_fft_dev::bitrev;
using svof_fft_dev::fft_stages;

__global__ void k3_pois_fwd_y(const double *__restrict__ ux, const double *__restrict__ uy,
                              const double *__restrict__ uz, double *__restrict__ spec,
                              const double *__restrict__ tw, const double *__restrict__ dtp, double gam,
                              int log2n, int cols, Grid3 g) {
  extern __shared__ double z[];  // [cols][ny] complex
  const int n = g.ny, nx = g.nx, nky = n / 2 + 1;
  const int i0 = 1 + blockIdx.x * cols;
  const int k = 1 + blockIdx.y;
  const int nc = min(cols, nx - i0 + 1);
  const double dt = *dtp;
  const double prefactor = 1. / (gam * dt) / (1. * g.ny * g.nz);
  for (int w = threadIdx.x; w < cols * n; w += blockDim.x) {
    const int q = w / cols, col = w - q * cols;
    const int m = bitrev(q, log2n);
    double v = 0.;
    if (col < nc) {
      const int i = i0 + col, j = m + 1;
      const double dx = g.dxf[i - 1];
      v = prefactor * (+(ux[ix_ux(g, i + 1, j, k)] - ux[ix_ux(g, i, j, k)]) / dx +
                       (uy[ix_cc(g, i, j + 1, k)] - uy[ix_cc(g, i, j, k)]) / g.dy +
                       (uz[ix_cc(g, i, j, k + 1)] - uz[ix_cc(g, i, j, k)]) / g.dz);
    }
    z[2 * (col * n + q)] = v;
    z[2 * (col * n + q) + 1] = 0.;
  }
  __syncthreads();
  fft_stages(z, log2n, cols, tw);
  for (int w = threadIdx.x; w < nc * nky; w += blockDim.x) {
    const int ky = w / nc, col = w - ky * nc;
    const size_t o = 2 * (((size_t)(k - 1) * nky + ky) * nx + (i0 - 1 + col));
    spec[o] = z[2 * (col * n + ky)];
    spec[o + 1] = z[2 * (col * n + ky) + 1];
  }
}

// complex DFT along z, in place, for `cols` consecutive i of one ky; the sign
// is the twiddle table's
__global__ void k3_pois_z(double *__restrict__ spec, const double *__restrict__ tw, int log2n, int cols, Grid3 g) {
  extern __shared__ double z[];  // [cols][nz] complex
  const int n = g.nz, nx = g.nx, nky = g.ny / 2 + 1;
  const int i0 = blockIdx.x * cols;
  const int ky = blockIdx.y;
  const int nc = min(cols, nx - i0);
  for (int w = threadIdx.x; w < cols * n; w += blockDim.x) {
    const int q = w / cols, col = w - q * cols;
    const int m = bitrev(q, log2n);
    double re = 0., im = 0.;
    if (col < nc) {
      const size_t o = 2 * (((size_t)m * nky + ky) * nx + (i0 + col));
      re = spec[o];
      im = spec[o + 1];
    }
    z[2 * (col * n + q)] = re;
    z[2 * (col * n + q) + 1] = im;
  }
  __syncthreads();
  fft_stages(z, log2n, cols, tw);
  for (int w = threadIdx.x; w < nc * n; w += blockDim.x) {
    const int kz = w / nc, col = w - kz * nc;
    const size_t o = 2 * (((size_t)kz * nky + ky) * nx + (i0 + col));
    spec[o] = z[2 * (col * n + kz)];
    spec[o + 1] = z[2 * (col * n + kz) + 1];
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
// X_{ny/2} ignored), psi of `cols` consecutive i of plane k with the halo
// images; the Neumann walls take the new neighbour value and hand their old
// value to the halo images
__global__ void k3_pois_inv_y(const double *__restrict__ spec, double *__restrict__ psi,
                              const double *__restrict__ tw, int log2n, int cols, Grid3 g) {
  extern __shared__ double z[];  // [cols][ny] complex
  const int n = g.ny, nx = g.nx, ny = g.ny, nz = g.nz, nky = n / 2 + 1;
  const int i0 = 1 + blockIdx.x * cols;
  const int k = 1 + blockIdx.y;
  const int nc = min(cols, nx - i0 + 1);
  for (int w = threadIdx.x; w < cols * n; w += blockDim.x) {
    const int q = w / cols, col = w - q * cols;
    const int m = bitrev(q, log2n);
    double re = 0., im = 0.;
    if (col < nc) {
      const size_t base = ((size_t)(k - 1) * nky) * nx + (i0 - 1 + col);
      if (0 == m) {
        re = spec[2 * base];
      } else if (2 * m < n) {
        const size_t o = 2 * (base + (size_t)m * nx);
        re = spec[o];
        im = spec[o + 1];
      } else if (2 * m == n) {
        re = spec[2 * (base + (size_t)m * nx)];
      } else {
        const size_t o = 2 * (base + (size_t)(n - m) * nx);
        re = spec[o];
        im = -spec[o + 1];
      }
    }
    z[2 * (col * n + q)] = re;
    z[2 * (col * n + q) + 1] = im;
  }
  __syncthreads();
  fft_stages(z, log2n, cols, tw);
  for (int w = threadIdx.x; w < nc * n; w += blockDim.x) {
    const int r = w / nc, col = w - r * nc;
    const int i = i0 + col, j = r + 1;
    const double y = z[2 * (col * n + r)];
    int js[4], ks[4];
    const int nimg = halo_images(j, k, ny, nz, js, ks);
    for (int q = 0; q < nimg; q++) psi[ix_cc(g, i, js[q], ks[q])] = y;
  }
  // Neumann walls of the interior rows of this plane
  const bool has_left = (1 == i0), has_right = (i0 + nc - 1 == nx);
  for (int w = threadIdx.x; w < 2 * n; w += blockDim.x) {
    const int side = w / n, j = 1 + (w - side * n);
    if ((0 == side && !has_left) || (1 == side && !has_right)) continue;
    const int iw = side ? nx + 1 : 0;
    const int col = side ? nc - 1 : 0;
    const double nv = z[2 * (col * n + (j - 1))];
    const double old = psi[ix_cc(g, iw, j, k)];
    int js[4], ks[4];
    const int nimg = halo_images(j, k, ny, nz, js, ks);
    psi[ix_cc(g, iw, j, k)] = nv;
    for (int q = 1; q < nimg; q++) psi[ix_cc(g, iw, js[q], ks[q])] = old;
  }
}

}  // namespace svof3
