// k3_poisson.cu -- pressure Poisson solve of the 3D path.
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
//
// Templates on R, the type of the spectrum, the twiddles and the transform
// arithmetic: R = double is the FP64 path (the restatement's butterflies bit
// for bit); R = float is the mixed path.  The x line solve is FP64 in both.
// The mixed path solves twice (defect correction): the second pass
// transforms the FP64 residual b - A psi of the first solution (RESID) and
// adds its solution to psi (ACCUM); its singular (ky, kz) = (0, 0) line has
// its gauge pinned (last unknown zero) so that the FP32 round-off of the
// compatibility condition cannot blow the additive constant up.
#include <type_traits>

#include "fft_device.cuh"
#include "svof3d_internal.cuh"

namespace svof3 {

using svof_fft_dev::bitrev;

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

// One warp per line.  Lines are stored re / im separately in shared memory,
// position p at padded index pad(p) = p + p / 8 and lines ld = n + n / 8 + 1
// apart, which keeps the column-wise loads and stores (consecutive threads on
// consecutive lines) and the register passes below free of bank conflicts.
// The transform is the oracle's radix-2 decimation in time (same butterfly
// pairs, same twiddles, same association), executed in passes of up to three
// stages: a lane loads the 2^ns points a pass combines, runs their butterflies
// in registers and stores them back, so shared memory is touched once per
// pass instead of once per stage.
__device__ __forceinline__ int fpad(int p) { return p + (p >> 3); }
__host__ __device__ __forceinline__ int fft_ld(int n) { return n + (n >> 3) + 1; }

template <class R, int NS>
__device__ __forceinline__ void fft_pass(R *__restrict__ re, R *__restrict__ im, int log2n, int s0,
                                         const R *__restrict__ tw) {
  using C2 = typename Cplx<R>::T;
  constexpr int G = 1 << NS;
  const int lane = threadIdx.x & 31;
  const int h = 1 << (s0 - 1);
  const int ngroups = (1 << log2n) >> NS;
  for (int gi = lane; gi < ngroups; gi += 32) {
    const int base = (gi & (h - 1)) + ((gi >> (s0 - 1)) << (s0 - 1 + NS));
    R xr[G], xi[G];
#pragma unroll
    for (int m = 0; m < G; m++) {
      const int q = fpad(base + m * h);
      xr[m] = re[q];
      xi[m] = im[q];
    }
#pragma unroll
    for (int t = 0; t < NS; t++) {
      const int st = s0 + t, dist = 1 << t;
#pragma unroll
      for (int m = 0; m < G; m++) {
        if (m & dist) continue;
        const int pa = base + m * h;
        const int kk = pa & ((h << t) - 1);
        const C2 w = __ldg(reinterpret_cast<const C2 *>(tw) + (kk << (log2n - st)));
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
#pragma unroll
    for (int m = 0; m < G; m++) {
      const int q = fpad(base + m * h);
      re[q] = xr[m];
      im[q] = xi[m];
    }
  }
  __syncwarp();
}

template <class R>
__device__ __forceinline__ void warp_fft_line(R *__restrict__ re, R *__restrict__ im, int log2n,
                                              const R *__restrict__ tw) {
  int s0 = 1;
  while (s0 <= log2n) {
    const int ns = min(3, log2n - s0 + 1);
    if (3 == ns) fft_pass<R, 3>(re, im, log2n, s0, tw);
    else if (2 == ns) fft_pass<R, 2>(re, im, log2n, s0, tw);
    else fft_pass<R, 1>(re, im, log2n, s0, tw);
    s0 += ns;
  }
}

// right-hand side (or, RESID, the residual b - A psi) at (i, j, k); FP64
template <bool RESID>
__device__ __forceinline__ double pois_rhs(const double *__restrict__ ux, const double *__restrict__ uy,
                                           const double *__restrict__ uz, const double *__restrict__ psi,
                                           const double *__restrict__ pl, const double *__restrict__ pu,
                                           const Grid3 &g, int i, int j, int k, double prefactor, double gdt) {
  const double dx = ldg(g.dxf + i - 1);
  const double div = +(ldg(ux + ix_ux(g, i + 1, j, k)) - ldg(ux + ix_ux(g, i, j, k))) / dx +
                     (ldg(uy + ix_cc(g, i, j + 1, k)) - ldg(uy + ix_cc(g, i, j, k))) / g.dy +
                     (ldg(uz + ix_cc(g, i, j, k + 1)) - ldg(uz + ix_cc(g, i, j, k))) / g.dz;
  if (!RESID) return prefactor * div;
  const double c = ldg(psi + ix_cc(g, i, j, k));
  const double l = ldg(pl + i - 1), u = ldg(pu + i - 1);
  const double ap = l * ldg(psi + ix_cc(g, i - 1, j, k)) + (-l - u) * c + u * ldg(psi + ix_cc(g, i + 1, j, k)) +
                    (ldg(psi + ix_cc(g, i, j - 1, k)) - 2. * c + ldg(psi + ix_cc(g, i, j + 1, k))) / (g.dy * g.dy) +
                    (ldg(psi + ix_cc(g, i, j, k - 1)) - 2. * c + ldg(psi + ix_cc(g, i, j, k + 1))) / (g.dz * g.dz);
  return (div / gdt - ap) / (1. * g.ny * g.nz);
}

template <int COLS, class R, bool RESID>
__global__ void __launch_bounds__(32 * COLS) k3_pois_fwd_y(const double *__restrict__ ux,
                                                          const double *__restrict__ uy,
                                                          const double *__restrict__ uz,
                                                          const double *__restrict__ psi,
                                                          const double *__restrict__ pl,
                                                          const double *__restrict__ pu, R *__restrict__ spec,
                                                          const R *__restrict__ tw, const double *__restrict__ dtp,
                                                          double gam, int log2n, Grid3 g) {
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  const int n = 1 << log2n, ld = fft_ld(n), nx = g.nx, nky = n / 2 + 1;
  R *im = re + COLS * ld;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  const double dt = ldg(dtp);
  const double prefactor = 1. / (gam * dt) / (1. * g.ny * g.nz);
  const double gdt = gam * dt;
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int q = w / COLS, col = w % COLS;
    const int m = bitrev(q, log2n);
    double v = 0.;
    if (col < nc) v = pois_rhs<RESID>(ux, uy, uz, psi, pl, pu, g, i0 + col, m + 1, k, prefactor, gdt);
    re[col * ld + fpad(q)] = R(v);
    im[col * ld + fpad(q)] = R(0.);
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line<R>(re + col * ld, im + col * ld, log2n, tw);
  }
  __syncthreads();
  using C2 = typename Cplx<R>::T;
  for (int w = threadIdx.x; w < nky * COLS; w += 32 * COLS) {
    const int ky = w / COLS, col = w % COLS;
    if (col < nc) {
      reinterpret_cast<C2 *>(spec)[((size_t)(k - 1) * nky + ky) * nx + (i0 - 1 + col)] =
          Cplx<R>::make(re[col * ld + fpad(ky)], im[col * ld + fpad(ky)]);
    }
  }
}

// complex DFT along z, in place, for COLS consecutive i of one ky; the sign is
// the twiddle table's
template <int COLS, class R>
__global__ void __launch_bounds__(32 * COLS) k3_pois_z(R *__restrict__ spec, const R *__restrict__ tw, int log2n,
                                                      Grid3 g) {
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  const int n = 1 << log2n, ld = fft_ld(n), nx = g.nx, nky = g.ny / 2 + 1;
  R *im = re + COLS * ld;
  const int i0 = blockIdx.x * COLS;
  const int ky = blockIdx.y;
  const int nc = min(COLS, nx - i0);
  using C2 = typename Cplx<R>::T;
  C2 *sp = reinterpret_cast<C2 *>(spec);
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int q = w / COLS, col = w % COLS;
    const int m = bitrev(q, log2n);
    C2 v = Cplx<R>::make(R(0.), R(0.));
    if (col < nc) v = sp[((size_t)m * nky + ky) * nx + (i0 + col)];
    re[col * ld + fpad(q)] = v.x;
    im[col * ld + fpad(q)] = v.y;
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line<R>(re + col * ld, im + col * ld, log2n, tw);
  }
  __syncthreads();
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int kz = w / COLS, col = w % COLS;
    if (col < nc)
      sp[((size_t)kz * nky + ky) * nx + (i0 + col)] = Cplx<R>::make(re[col * ld + fpad(kz)], im[col * ld + fpad(kz)]);
  }
}

// complex Neumann Thomas along x per line (ky, kz): tdm_c = -pl - pu + lambda,
// lambda = evy[ky] + evz[kz], first / last diagonal + pl[0] / + pu[nx-1], then
// gtsv component-wise (src/tdm.c:17-50; dft.c:364-395 in 2D).  Warp 0 runs
// the recurrences with one line per lane; the other warps move the tiles.
// FP64 arithmetic; the spectrum and the scratch of v are R.
constexpr int XL = kXsLines, XC = kXsChunk;

template <class R>
__global__ void __launch_bounds__(256) k3_pois_x(R *__restrict__ spec, R *__restrict__ scratch,
                                                 const double *__restrict__ pl, const double *__restrict__ pu,
                                                 const double *__restrict__ evy, const double *__restrict__ evz,
                                                 int pin_gauge, Grid3 g) {
  __shared__ double sre[XL][XC + 1], sim[XL][XC + 1], sv[XL][XC + 1];
  __shared__ double spl[XC], spu[XC];
  using C2 = typename Cplx<R>::T;
  C2 *sp = reinterpret_cast<C2 *>(spec);
  const int nx = g.nx, nky = g.ny / 2 + 1;
  const long nlines = (long)nky * g.nz;
  const long l0 = (long)blockIdx.x * XL;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int nchunks = (nx + XC - 1) / XC;
  const bool sweeper = (0 == ty) && (l0 + tx < nlines);
  double lam = 0.;
  bool pinned = false;
  if (sweeper) {
    const long l = l0 + tx;
    lam = ldg(evy + l % nky) + ldg(evz + l / nky);
    pinned = pin_gauge && (0 == l);
  }
  double vprev = 0., qr = 0., qi = 0.;
  // ---------------------------------------------------------- forward
  for (int c = 0; c < nchunks; c++) {
    const int p0 = c * XC;
    if (tid < XC) {
      spl[tid] = (p0 + tid < nx) ? ldg(pl + p0 + tid) : 0.;
      spu[tid] = (p0 + tid < nx) ? ldg(pu + p0 + tid) : 0.;
    }
    for (int m = 0; m < XL / 8; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l < nlines && p < nx) {
        const C2 v = sp[(size_t)l * nx + p];
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
        const double xr = sre[tx][s], xi = sim[tx][s];
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
          if (fabs(val) > kDblEpsilon && !pinned) {
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
        sp[(size_t)l * nx + p] = Cplx<R>::make(R(sre[ll][tx]), R(sim[ll][tx]));
        scratch[(size_t)l * nx + p] = R(sv[ll][tx]);
      }
    }
    __syncthreads();
  }
  // ---------------------------------------------------------- backward
  // (FP64 arithmetic; in the mixed path the forward values come back rounded
  // to FP32, an error the defect-correction pass removes)
  double nr = 0., ni = 0.;
  for (int c = nchunks - 1; c >= 0; c--) {
    const int p0 = c * XC;
    for (int m = 0; m < XL / 8; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l < nlines && p < nx) {
        const C2 v = sp[(size_t)l * nx + p];
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
      if (l < nlines && p < nx) sp[(size_t)l * nx + p] = Cplx<R>::make(R(sre[ll][tx]), R(sim[ll][tx]));
    }
    __syncthreads();
  }
}

// c2r along y (Hermitian extension as FFTW's c2r reads it: Im of X_0 and
// X_{ny/2} ignored), psi of COLS consecutive i of plane k (ACCUM: psi +=) with
// the halo images; the Neumann walls take the new neighbour value and hand
// their old value to the halo images
template <int COLS, class R, bool ACCUM>
__global__ void __launch_bounds__(32 * COLS) k3_pois_inv_y(const R *__restrict__ spec, double *__restrict__ psi,
                                                          const R *__restrict__ tw, int log2n, Grid3 g) {
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  const int n = 1 << log2n, ld = fft_ld(n), nx = g.nx, ny = g.ny, nz = g.nz, nky = n / 2 + 1;
  R *im = re + COLS * ld;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  using C2 = typename Cplx<R>::T;
  const C2 *sp = reinterpret_cast<const C2 *>(spec);
  for (int w = threadIdx.x; w < COLS * n; w += 32 * COLS) {
    const int q = w / COLS, col = w % COLS;
    const int m = bitrev(q, log2n);
    R r = R(0.), x = R(0.);
    if (col < nc) {
      const size_t base = ((size_t)(k - 1) * nky) * nx + (i0 - 1 + col);
      if (0 == m) {
        r = __ldg(&sp[base].x);
      } else if (2 * m < n) {
        const C2 v = __ldg(&sp[base + (size_t)m * nx]);
        r = v.x;
        x = v.y;
      } else if (2 * m == n) {
        r = __ldg(&sp[base + (size_t)m * nx].x);
      } else {
        const C2 v = __ldg(&sp[base + (size_t)(n - m) * nx]);
        r = v.x;
        x = -v.y;
      }
    }
    re[col * ld + fpad(q)] = r;
    im[col * ld + fpad(q)] = x;
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line<R>(re + col * ld, im + col * ld, log2n, tw);
  }
  __syncthreads();
  for (int w = threadIdx.x; w < n * COLS; w += 32 * COLS) {
    const int r = w / COLS, col = w % COLS;
    if (col >= nc) continue;
    const int i = i0 + col, j = r + 1;
    double y = (double)re[col * ld + fpad(r)];
    if (ACCUM) y += psi[ix_cc(g, i, j, k)];
    for_images(j, k, ny, nz, true, [&](int jj, int kk) { psi[ix_cc(g, i, jj, kk)] = y; });
  }
  // (ACCUM: the walls below read the accumulated neighbour values)
  if (ACCUM) __syncthreads();
  // Neumann walls of the interior rows of this plane
  const bool has_left = (1 == i0), has_right = (i0 + nc - 1 == nx);
  for (int w = threadIdx.x; w < 2 * n; w += 32 * COLS) {
    const int side = w / n, j = 1 + (w - side * n);
    if ((0 == side && !has_left) || (1 == side && !has_right)) continue;
    const int iw = side ? nx + 1 : 0;
    const int col = side ? nc - 1 : 0;
    const double nv = ACCUM ? psi[ix_cc(g, i0 + col, j, k)] : (double)re[col * ld + fpad(j - 1)];
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
template <class R>
size_t fft_smem(int n, int cols) {
  return sizeof(R) * 2 * (size_t)fft_ld(n) * cols;
}
}  // namespace

template <class R>
cudaError_t pois_prepare(int ny, int cols_y, int nz, int cols_z) {
  cudaError_t e = by_cols(cols_y, [&](auto c) {
    constexpr int C = decltype(c)::value;
    const int sy = (int)fft_smem<R>(ny, C);
    const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t r;
    if (cudaSuccess != (r = cudaFuncSetAttribute(k3_pois_fwd_y<C, R, false>, at, sy))) return r;
    if (cudaSuccess != (r = cudaFuncSetAttribute(k3_pois_fwd_y<C, R, true>, at, sy))) return r;
    if (cudaSuccess != (r = cudaFuncSetAttribute(k3_pois_inv_y<C, R, false>, at, sy))) return r;
    return cudaFuncSetAttribute(k3_pois_inv_y<C, R, true>, at, sy);
  });
  if (cudaSuccess != e) return e;
  return by_cols(cols_z, [&](auto c) {
    constexpr int C = decltype(c)::value;
    return cudaFuncSetAttribute(k3_pois_z<C, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fft_smem<R>(nz, C));
  });
}

template <class R>
cudaError_t pois_fwd_y(int cols, bool resid, cudaStream_t st, const double *ux, const double *uy, const double *uz,
                       const double *psi, const double *pl, const double *pu, R *spec, const R *tw,
                       const double *dtp, double gam, int log2n, Grid3 g) {
  return by_cols(cols, [&](auto c) {
    constexpr int C = decltype(c)::value;
    dim3 gr((g.nx + C - 1) / C, g.nz);
    const size_t sm = fft_smem<R>(g.ny, C);
    if (resid) {
      k3_pois_fwd_y<C, R, true><<<gr, 32 * C, sm, st>>>(ux, uy, uz, psi, pl, pu, spec, tw, dtp, gam, log2n, g);
    } else {
      k3_pois_fwd_y<C, R, false><<<gr, 32 * C, sm, st>>>(ux, uy, uz, psi, pl, pu, spec, tw, dtp, gam, log2n, g);
    }
    return cudaGetLastError();
  });
}

template <class R>
cudaError_t pois_z(int cols, cudaStream_t st, R *spec, const R *tw, int log2n, Grid3 g) {
  return by_cols(cols, [&](auto c) {
    constexpr int C = decltype(c)::value;
    dim3 gr((g.nx + C - 1) / C, g.ny / 2 + 1);
    k3_pois_z<C, R><<<gr, 32 * C, fft_smem<R>(g.nz, C), st>>>(spec, tw, log2n, g);
    return cudaGetLastError();
  });
}

template <class R>
cudaError_t pois_x(cudaStream_t st, R *spec, R *scratch, const double *pl, const double *pu, const double *evy,
                   const double *evz, int pin_gauge, Grid3 g) {
  const long nlines = (long)(g.ny / 2 + 1) * g.nz;
  k3_pois_x<R><<<(unsigned)((nlines + XL - 1) / XL), 256, 0, st>>>(spec, scratch, pl, pu, evy, evz, pin_gauge, g);
  return cudaGetLastError();
}

template <class R>
cudaError_t pois_inv_y(int cols, bool accum, cudaStream_t st, const R *spec, double *psi, const R *tw, int log2n,
                       Grid3 g) {
  return by_cols(cols, [&](auto c) {
    constexpr int C = decltype(c)::value;
    dim3 gr((g.nx + C - 1) / C, g.nz);
    const size_t sm = fft_smem<R>(g.ny, C);
    if (accum) {
      k3_pois_inv_y<C, R, true><<<gr, 32 * C, sm, st>>>(spec, psi, tw, log2n, g);
    } else {
      k3_pois_inv_y<C, R, false><<<gr, 32 * C, sm, st>>>(spec, psi, tw, log2n, g);
    }
    return cudaGetLastError();
  });
}

#define SVOF3_POISSON_INST(R)                                                                                    \
  template cudaError_t pois_prepare<R>(int, int, int, int);                                                      \
  template cudaError_t pois_fwd_y<R>(int, bool, cudaStream_t, const double *, const double *, const double *,   \
                                     const double *, const double *, const double *, R *, const R *,            \
                                     const double *, double, int, Grid3);                                       \
  template cudaError_t pois_z<R>(int, cudaStream_t, R *, const R *, int, Grid3);                                 \
  template cudaError_t pois_x<R>(cudaStream_t, R *, R *, const double *, const double *, const double *,        \
                                 const double *, int, Grid3);                                                    \
  template cudaError_t pois_inv_y<R>(int, bool, cudaStream_t, const R *, double *, const R *, int, Grid3);
SVOF3_POISSON_INST(double)
SVOF3_POISSON_INST(float)
#undef SVOF3_POISSON_INST

}  // namespace svof3
