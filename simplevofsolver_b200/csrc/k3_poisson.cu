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

// One warp per line, the line length N = 2^L2N a compile-time constant.
// Lines are stored re / im separately in shared memory, position p at padded
// index pad(p) = p + p / 8 and lines LD = N + N / 8 + 1 apart, which keeps the
// column-wise loads and stores (consecutive threads on consecutive lines) and
// the register passes below free of bank conflicts.  The transform is the
// oracle's radix-2 decimation in time (same butterfly pairs, same twiddles,
// same association), executed in passes of up to three stages: a lane loads
// the 2^NS points a pass combines, runs their butterflies in registers and
// stores them back, so shared memory is touched once per pass instead of once
// per stage.
__device__ __forceinline__ int fpad(int p) { return p + (p >> 3); }

// Shape of a block of one transform direction: COLS lines of N points, one
// warp each.  COLS is the widest of 16 / 8 / 4 whose shared memory stays
// within 80 KB (the rows the y transforms read are COLS x 8 bytes wide and,
// with the reference's x pitch of nx + 2, not sector aligned: wider rows waste
// less of each sector), MINB the resident blocks per SM the launch bounds ask
// for (shared memory permitting, and no fewer than 64 registers a thread).
constexpr int line_cols(int col_bytes) {
  return (16 * col_bytes <= 81920) ? 16 : ((8 * col_bytes <= 81920) ? 8 : 4);
}
constexpr int line_minb(int smem, int threads) {
  return (232448 / (smem + 1024) < 1024 / threads) ? ((232448 / (smem + 1024)) < 1 ? 1 : 232448 / (smem + 1024))
                                                    : ((1024 / threads) < 1 ? 1 : 1024 / threads);
}
template <class R, int L2N>
struct Line {
  static constexpr int N = 1 << L2N;
  static constexpr int LD = N + (N >> 3) + 1;
  static constexpr int COL_BYTES = 2 * (int)sizeof(R) * LD;
  static constexpr int COLS = line_cols(COL_BYTES);
  static constexpr int THREADS = 32 * COLS;
  static constexpr int SMEM = COLS * COL_BYTES;
  static constexpr int MINB = line_minb(SMEM, THREADS);
  static constexpr int ITER = (N + 31) / 32;  // points per thread in the load / store loops
};

template <class R, int L2N, int S0, int NS>
__device__ __forceinline__ void fft_pass(R *__restrict__ re, R *__restrict__ im, const R *__restrict__ tw) {
  using C2 = typename Cplx<R>::T;
  constexpr int G = 1 << NS, H = 1 << (S0 - 1), NG = (1 << L2N) >> NS;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int g0 = 0; g0 < NG; g0 += 32) {
    const int gi = g0 + lane;
    if (NG >= 32 || gi < NG) {
      const int base = (gi & (H - 1)) + ((gi >> (S0 - 1)) << (S0 - 1 + NS));
      R xr[G], xi[G];
#pragma unroll
      for (int m = 0; m < G; m++) {
        const int q = fpad(base + m * H);
        xr[m] = re[q];
        xi[m] = im[q];
      }
#pragma unroll
      for (int t = 0; t < NS; t++) {
        const int st = S0 + t, dist = 1 << t;
#pragma unroll
        for (int m = 0; m < G; m++) {
          if (m & dist) continue;
          // twiddle index of the pair (base + m H, base + (m + dist) H) at stage st
          const int kk = (gi & (H - 1)) + (m & (dist - 1)) * H;
          const C2 w = __ldg(reinterpret_cast<const C2 *>(tw) + (kk << (L2N - st)));
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
        const int q = fpad(base + m * H);
        re[q] = xr[m];
        im[q] = xi[m];
      }
    }
  }
  __syncwarp();
}

template <class R, int L2N, int S0 = 1>
__device__ __forceinline__ void warp_fft_line(R *__restrict__ re, R *__restrict__ im, const R *__restrict__ tw) {
  if constexpr (S0 <= L2N) {
    constexpr int NS = (L2N - S0 + 1) < 3 ? (L2N - S0 + 1) : 3;
    fft_pass<R, L2N, S0, NS>(re, im, tw);
    warp_fft_line<R, L2N, S0 + NS>(re, im, tw);
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

// forward transform along y of COLS consecutive i of plane k: the right-hand
// side (RESID: the residual) of each point, in bit-reversed order, then the
// warp transforms, then the ky = 0 .. N/2 half of the spectrum
template <int L2N, class R, bool RESID>
__global__ void __launch_bounds__(Line<R, L2N>::THREADS, Line<R, L2N>::MINB)
    k3_pois_fwd_y(const double *__restrict__ ux, const double *__restrict__ uy, const double *__restrict__ uz,
                  const double *__restrict__ psi, const double *__restrict__ pl, const double *__restrict__ pu,
                  R *__restrict__ spec, const R *__restrict__ tw, const double *__restrict__ dtp, double gam,
                  Grid3 g) {
  using L = Line<R, L2N>;
  constexpr int N = L::N, LD = L::LD, COLS = L::COLS, NKY = N / 2 + 1;
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  R *im = re + COLS * LD;
  const int nx = g.nx;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  const double dt = ldg(dtp);
  const double prefactor = 1. / (gam * dt) / (1. * g.ny * g.nz);
  const double gdt = gam * dt;
#pragma unroll 4
  for (int it = 0; it < L::ITER; it++) {
    const int w = threadIdx.x + it * L::THREADS;
    if (N >= 32 || w < COLS * N) {
      const int q = w / COLS, col = w % COLS;
      const int m = bitrev(q, L2N);
      double v = 0.;
      if (col < nc) v = pois_rhs<RESID>(ux, uy, uz, psi, pl, pu, g, i0 + col, m + 1, k, prefactor, gdt);
      re[col * LD + fpad(q)] = R(v);
      im[col * LD + fpad(q)] = R(0.);
    }
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line<R, L2N>(re + col * LD, im + col * LD, tw);
  }
  __syncthreads();
  using C2 = typename Cplx<R>::T;
  C2 *out = reinterpret_cast<C2 *>(spec) + (size_t)(k - 1) * NKY * nx + (i0 - 1);
#pragma unroll 4
  for (int it = 0; it < (NKY * COLS + L::THREADS - 1) / L::THREADS; it++) {
    const int w = threadIdx.x + it * L::THREADS;
    const int ky = w / COLS, col = w % COLS;
    if (ky < NKY && col < nc) out[(size_t)ky * nx + col] = Cplx<R>::make(re[col * LD + fpad(ky)], im[col * LD + fpad(ky)]);
  }
}

// complex DFT along z, in place, for COLS consecutive i of one ky; the sign is
// the twiddle table's
template <int L2N, class R>
__global__ void __launch_bounds__(Line<R, L2N>::THREADS, Line<R, L2N>::MINB)
    k3_pois_z(R *__restrict__ spec, const R *__restrict__ tw, Grid3 g) {
  using L = Line<R, L2N>;
  constexpr int N = L::N, LD = L::LD, COLS = L::COLS;
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  R *im = re + COLS * LD;
  const int nx = g.nx, nky = g.ny / 2 + 1;
  const int i0 = blockIdx.x * COLS;
  const int ky = blockIdx.y;
  const int nc = min(COLS, nx - i0);
  using C2 = typename Cplx<R>::T;
  C2 *sp = reinterpret_cast<C2 *>(spec) + (size_t)ky * nx + i0;
  const size_t rs = (size_t)nky * nx;  // stride of kz
#pragma unroll 4
  for (int it = 0; it < L::ITER; it++) {
    const int w = threadIdx.x + it * L::THREADS;
    if (N >= 32 || w < COLS * N) {
      const int q = w / COLS, col = w % COLS;
      const int m = bitrev(q, L2N);
      C2 v = Cplx<R>::make(R(0.), R(0.));
      if (col < nc) v = sp[m * rs + col];
      re[col * LD + fpad(q)] = v.x;
      im[col * LD + fpad(q)] = v.y;
    }
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line<R, L2N>(re + col * LD, im + col * LD, tw);
  }
  __syncthreads();
#pragma unroll 4
  for (int it = 0; it < L::ITER; it++) {
    const int w = threadIdx.x + it * L::THREADS;
    if (N >= 32 || w < COLS * N) {
      const int kz = w / COLS, col = w % COLS;
      if (col < nc) sp[kz * rs + col] = Cplx<R>::make(re[col * LD + fpad(kz)], im[col * LD + fpad(kz)]);
    }
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
template <int L2N, class R, bool ACCUM>
__global__ void __launch_bounds__(Line<R, L2N>::THREADS, Line<R, L2N>::MINB)
    k3_pois_inv_y(const R *__restrict__ spec, double *__restrict__ psi, const R *__restrict__ tw, Grid3 g) {
  using L = Line<R, L2N>;
  constexpr int N = L::N, LD = L::LD, COLS = L::COLS, NKY = N / 2 + 1;
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  R *im = re + COLS * LD;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  using C2 = typename Cplx<R>::T;
  const C2 *sp = reinterpret_cast<const C2 *>(spec) + (size_t)(k - 1) * NKY * nx + (i0 - 1);
#pragma unroll 4
  for (int it = 0; it < L::ITER; it++) {
    const int w = threadIdx.x + it * L::THREADS;
    if (N >= 32 || w < COLS * N) {
      const int q = w / COLS, col = w % COLS;
      const int m = bitrev(q, L2N);
      R r = R(0.), x = R(0.);
      if (col < nc) {
        // X_m for m <= N/2, conj(X_{N-m}) above; Im of X_0 and X_{N/2} ignored
        const int row = (2 * m <= N) ? m : N - m;
        const C2 v = __ldg(&sp[(size_t)row * nx + col]);
        r = v.x;
        x = (0 == m || 2 * m == N) ? R(0.) : ((2 * m < N) ? v.y : -v.y);
      }
      re[col * LD + fpad(q)] = r;
      im[col * LD + fpad(q)] = x;
    }
  }
  __syncthreads();
  {
    const int col = threadIdx.x >> 5;
    warp_fft_line<R, L2N>(re + col * LD, im + col * LD, tw);
  }
  __syncthreads();
#pragma unroll 4
  for (int it = 0; it < L::ITER; it++) {
    const int w = threadIdx.x + it * L::THREADS;
    if (N >= 32 || w < COLS * N) {
      const int r = w / COLS, col = w % COLS;
      if (col < nc) {
        const int i = i0 + col, j = r + 1;
        double y = (double)re[col * LD + fpad(r)];
        if (ACCUM) y += psi[ix_cc(g, i, j, k)];
        for_images(j, k, ny, nz, true, [&](int jj, int kk) { psi[ix_cc(g, i, jj, kk)] = y; });
      }
    }
  }
  // (ACCUM: the walls below read the accumulated neighbour values)
  if (ACCUM) __syncthreads();
  // Neumann walls of the interior rows of this plane
  const bool has_left = (1 == i0), has_right = (i0 + nc - 1 == nx);
  if (!has_left && !has_right) return;
  for (int w = threadIdx.x; w < 2 * N; w += L::THREADS) {
    const int side = w / N, j = 1 + (w - side * N);
    if ((0 == side && !has_left) || (1 == side && !has_right)) continue;
    const int iw = side ? nx + 1 : 0;
    const int col = side ? nc - 1 : 0;
    const double nv = ACCUM ? psi[ix_cc(g, i0 + col, j, k)] : (double)re[col * LD + fpad(j - 1)];
    const double old = psi[ix_cc(g, iw, j, k)];
    psi[ix_cc(g, iw, j, k)] = nv;
    for_images(j, k, ny, nz, false, [&](int jj, int kk) { psi[ix_cc(g, iw, jj, kk)] = old; });
  }
}

// ---- host-side launchers (the templates stay in this translation unit)
namespace {
constexpr int kMinL2N = 1, kMaxL2N = 11;
template <class F>
cudaError_t by_l2n(int l2n, F f) {
  switch (l2n) {
    case 1: return f(std::integral_constant<int, 1>());
    case 2: return f(std::integral_constant<int, 2>());
    case 3: return f(std::integral_constant<int, 3>());
    case 4: return f(std::integral_constant<int, 4>());
    case 5: return f(std::integral_constant<int, 5>());
    case 6: return f(std::integral_constant<int, 6>());
    case 7: return f(std::integral_constant<int, 7>());
    case 8: return f(std::integral_constant<int, 8>());
    case 9: return f(std::integral_constant<int, 9>());
    case 10: return f(std::integral_constant<int, 10>());
    case 11: return f(std::integral_constant<int, 11>());
    default: return cudaErrorInvalidValue;
  }
}
template <class K>
cudaError_t line_attrs(K kernel, int smem) {
  cudaError_t r = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (cudaSuccess != r) return r;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}
}  // namespace

template <class R>
cudaError_t pois_prepare(int log2ny, int log2nz) {
  if (log2ny < kMinL2N || log2ny > kMaxL2N || log2nz < kMinL2N || log2nz > kMaxL2N) return cudaErrorInvalidValue;
  cudaError_t e = by_l2n(log2ny, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    constexpr int sm = Line<R, L2>::SMEM;
    cudaError_t r;
    if (cudaSuccess != (r = line_attrs(k3_pois_fwd_y<L2, R, false>, sm))) return r;
    if (cudaSuccess != (r = line_attrs(k3_pois_fwd_y<L2, R, true>, sm))) return r;
    if (cudaSuccess != (r = line_attrs(k3_pois_inv_y<L2, R, false>, sm))) return r;
    return line_attrs(k3_pois_inv_y<L2, R, true>, sm);
  });
  if (cudaSuccess != e) return e;
  return by_l2n(log2nz, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    return line_attrs(k3_pois_z<L2, R>, Line<R, L2>::SMEM);
  });
}

template <class R>
cudaError_t pois_fwd_y(bool resid, cudaStream_t st, const double *ux, const double *uy, const double *uz,
                       const double *psi, const double *pl, const double *pu, R *spec, const R *tw,
                       const double *dtp, double gam, int log2n, Grid3 g) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.nz);
    if (resid) {
      k3_pois_fwd_y<L2, R, true><<<gr, L::THREADS, L::SMEM, st>>>(ux, uy, uz, psi, pl, pu, spec, tw, dtp, gam, g);
    } else {
      k3_pois_fwd_y<L2, R, false><<<gr, L::THREADS, L::SMEM, st>>>(ux, uy, uz, psi, pl, pu, spec, tw, dtp, gam, g);
    }
    return cudaGetLastError();
  });
}

template <class R>
cudaError_t pois_z(cudaStream_t st, R *spec, const R *tw, int log2n, Grid3 g) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.ny / 2 + 1);
    k3_pois_z<L2, R><<<gr, L::THREADS, L::SMEM, st>>>(spec, tw, g);
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
cudaError_t pois_inv_y(bool accum, cudaStream_t st, const R *spec, double *psi, const R *tw, int log2n, Grid3 g) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.nz);
    if (accum) {
      k3_pois_inv_y<L2, R, true><<<gr, L::THREADS, L::SMEM, st>>>(spec, psi, tw, g);
    } else {
      k3_pois_inv_y<L2, R, false><<<gr, L::THREADS, L::SMEM, st>>>(spec, psi, tw, g);
    }
    return cudaGetLastError();
  });
}

#define SVOF3_POISSON_INST(R)                                                                                    \
  template cudaError_t pois_prepare<R>(int, int);                                                                \
  template cudaError_t pois_fwd_y<R>(bool, cudaStream_t, const double *, const double *, const double *,   \
                                     const double *, const double *, const double *, R *, const R *,            \
                                     const double *, double, int, Grid3);                                       \
  template cudaError_t pois_z<R>(cudaStream_t, R *, const R *, int, Grid3);                                      \
  template cudaError_t pois_x<R>(cudaStream_t, R *, R *, const double *, const double *, const double *,        \
                                 const double *, int, Grid3);                                                    \
  template cudaError_t pois_inv_y<R>(bool, cudaStream_t, const R *, double *, const R *, int, Grid3);
SVOF3_POISSON_INST(double)
SVOF3_POISSON_INST(float)
#undef SVOF3_POISSON_INST

}  // namespace svof3
