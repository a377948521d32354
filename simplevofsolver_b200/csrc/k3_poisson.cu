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
//   k3_pois_b      the right-hand side of every cell, compact
//   k3_pois_fwd_y  a block owns COLS consecutive i of one plane k
//   k3_pois_z      a block owns COLS consecutive i of one ky, both signs
//                  (in place)
//   k3_pois_x      a block owns 64 or 128 lines (ky, kz), one per thread,
//                  walked in 16-cell chunks: forward recurrence (values back
//                  into S, v into scratch), then back substitution in reverse
//                  chunk order
//   k3_pois_inv_y  a block owns COLS consecutive i of one plane k; writes psi
//                  with its halo images and Neumann walls
//
//   k3_pois_resid  the FP64 residual b - L psi of a solve (the defect of an
//                  FP32 pass), into a compact array
//
// Templates on R, the type of the spectrum, the twiddles and the transform
// arithmetic; the x line solve computes in FP64.  The FP64 and the mixed path
// instantiate R = double (the restatement's butterflies bit for bit); the
// defect-corrected form (SVOF3_MIXED_DC) instantiates R = float: an FP32
// pass, the FP64 residual of its psi, a second FP32 pass on the residual,
// accumulated into psi.
#include <cuda_pipeline.h>

#include <type_traits>

#include "fft_device.cuh"
#include "svof3d_internal.cuh"
#include "smem_limit.cuh"

namespace svof3 {

using svof_fft_dev::bitrev;
using svof_fft_dev::Cplx;
using svof_fft_dev::fft_lines;
using svof_fft_dev::fpad;


// The transforms (the register-blocked passes of fft_device.cuh).  A block
// owns COLS lines of N = 2^L2N points: consecutive i of one plane k for y, of
// one ky for z.  The first pass reads its points from global memory and the
// last one writes its results there, so a warp's global accesses are runs of
// consecutive i.

constexpr int kLineThreads = 256;
// COLS: the widest of 16 / 8 / 4 lines whose shared memory stays within 80 KB
// (the rows the y transforms read are COLS x 8 bytes wide and, with the
// reference's x pitch of nx + 2, not sector aligned: wider rows waste less of
// each sector).  MINB: resident blocks per SM, shared memory permitting, at
// most 4 (64 registers a thread).
constexpr int line_cols(int col_bytes) {
  return (16 * col_bytes <= 81920) ? 16 : ((8 * col_bytes <= 81920) ? 8 : 4);
}
constexpr int line_minb(int smem) {
  return (232448 / (smem + 1024) < 1) ? 1 : ((232448 / (smem + 1024) > 4) ? 4 : 232448 / (smem + 1024));
}
template <class R, int L2N>
struct Line {
  static constexpr int N = 1 << L2N;
  static constexpr int LD = svof_fft_dev::fft_ld(L2N);
  static constexpr int COL_BYTES = 2 * (int)sizeof(R) * LD;
  static constexpr int COLS = line_cols(COL_BYTES);
  static constexpr int SMEM = COLS * COL_BYTES;
  static constexpr int MINB = line_minb(SMEM);
};



// the right-hand side b = div u / (gamma dt ny nz) of every interior cell,
// FP64, into a compact array (x fastest, nx ny per plane), with the
// reference's association: one thread per (i, j) walking kBPlanes planes, uz
// at k + 1 carried to the next plane, every load of the thread's planes
// issued before its first division
constexpr int kBPlanes = 4;
__global__ void __launch_bounds__(256, 4) k3_pois_b(const double *__restrict__ ux, const double *__restrict__ uy,
                                                    const double *__restrict__ uz, double *__restrict__ b,
                                                    const double *__restrict__ dtp, double gam, Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 1 + blockIdx.z * kBPlanes;
  if (i > nx || j > ny || k0 > nz) return;
  const double dt = ldg(dtp);
  const double prefactor = 1. / (gam * dt) / (1. * g.ny * g.nz);
  const double dx = ldg(g.dxf + i - 1);
  double *bo = b + (i - 1) + (size_t)nx * (j - 1);
  const size_t bplane = (size_t)nx * ny;
  double uzk = ldg(uz + ix_cc(g, i, j, k0));  // uz at the current plane
  constexpr int B = kBPlanes;
  double x0[B], x1[B], y0[B], y1[B], zp[B];
#pragma unroll
  for (int h = 0; h < B; h++) {
    const int k = min(k0 + h, nz);
    x0[h] = ldg(ux + ix_ux(g, i, j, k));
    x1[h] = ldg(ux + ix_ux(g, i + 1, j, k));
    y0[h] = ldg(uy + ix_cc(g, i, j, k));
    y1[h] = ldg(uy + ix_cc(g, i, j + 1, k));
    zp[h] = ldg(uz + ix_cc(g, i, j, k + 1));
  }
#pragma unroll
  for (int h = 0; h < B; h++) {
    const int k = k0 + h;
    if (k > nz) break;
    const double div = +(x1[h] - x0[h]) / dx + (y1[h] - y0[h]) / g.dy + (zp[h] - uzk) / g.dz;
    uzk = zp[h];
    bo[bplane * (k - 1)] = prefactor * div;
  }
}

// the residual r = b - L psi / (ny nz) of every interior cell, FP64, into a
// compact array like b: L the operator the spectral solve inverts (x:
// pl (psi(i-1) - psi) + pu (psi(i+1) - psi), the wall cells holding their
// neighbour's value (Neumann); y, z: the periodic second differences over
// the halo images); 1 / (ny nz) undoes the unnormalised transforms' scale
// that b carries.  One thread per (i, j), kBPlanes planes.
__global__ void __launch_bounds__(256, 4) k3_pois_resid(const double *__restrict__ b, const double *__restrict__ psi,
                                                        double *__restrict__ r, const double *__restrict__ pl,
                                                        const double *__restrict__ pu, Grid3 g) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 1 + blockIdx.z * kBPlanes;
  if (i > nx || j > ny || k0 > nz) return;
  const double l = ldg(pl + i - 1), u = ldg(pu + i - 1);
  const double ry = 1. / (g.dy * g.dy), rz = 1. / (g.dz * g.dz);
  const double scale = 1. / ((double)ny * (double)nz);
  const size_t o = (i - 1) + (size_t)nx * (j - 1), bplane = (size_t)nx * ny;
  for (int k = k0; k < min(k0 + kBPlanes, nz + 1); k++) {
    const double pc = ldg(psi + ix_cc(g, i, j, k));
    const double lx = l * (ldg(psi + ix_cc(g, i - 1, j, k)) - pc) + u * (ldg(psi + ix_cc(g, i + 1, j, k)) - pc);
    const double lyy = ry * (ldg(psi + ix_cc(g, i, j - 1, k)) - 2. * pc + ldg(psi + ix_cc(g, i, j + 1, k)));
    const double lzz = rz * (ldg(psi + ix_cc(g, i, j, k - 1)) - 2. * pc + ldg(psi + ix_cc(g, i, j, k + 1)));
    const size_t q = o + bplane * (k - 1);
    r[q] = ldg(b + q) - scale * (lx + lyy + lzz);
  }
}

// forward transform along y of COLS consecutive i of plane k: the first pass
// reads the right-hand side b (k3_pois_b), the last one writes the
// ky = 0 .. N/2 half of the spectrum
template <int L2N, class R>
__global__ void __launch_bounds__(kLineThreads, Line<R, L2N>::MINB)
    k3_pois_fwd_y(const double *__restrict__ b, R *__restrict__ spec, const R *__restrict__ tw, Grid3 g) {
  using L = Line<R, L2N>;
  using C2 = typename Cplx<R>::T;
  constexpr int N = L::N, COLS = L::COLS, NKY = N / 2 + 1;
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  R *im = re + COLS * L::LD;
  const int nx = g.nx;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  const double *bp = b + (size_t)nx * N * (k - 1) + (i0 - 1);
  C2 *out = reinterpret_cast<C2 *>(spec) + (size_t)(k - 1) * NKY * nx + (i0 - 1);
  auto first = [&](int c, int base, auto gc, auto hc, R *xr, R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int m = 0; m < G; m++) {
      xr[m] = R(c < nc ? ldg(bp + (size_t)nx * bitrev(base + m * H, L2N) + c) : 0.);
      xi[m] = R(0.);
    }
  };
  auto last = [&](int c, int base, auto gc, auto hc, const R *xr, const R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
    if (c >= nc) return;
#pragma unroll
    for (int m = 0; m < G; m++) {
      const int p = base + m * H;
      if (p <= N / 2) out[(size_t)p * nx + c] = Cplx<R>::make(xr[m], xi[m]);
    }
  };
  fft_lines<R, L2N, COLS>(re, im, tw, first, last);
}

// complex DFT along z, in place, for COLS consecutive i of one ky; the sign is
// the twiddle table's (every read of the first pass precedes every write of
// the last, the passes being separated by block barriers; a single-pass
// length has one group per line)
template <int L2N, class R>
__global__ void __launch_bounds__(kLineThreads, Line<R, L2N>::MINB)
    k3_pois_z(R *__restrict__ spec, const R *__restrict__ tw, Grid3 g) {
  using L = Line<R, L2N>;
  using C2 = typename Cplx<R>::T;
  constexpr int COLS = L::COLS;
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  R *im = re + COLS * L::LD;
  const int nx = g.nx, nky = g.ny / 2 + 1;
  const int i0 = blockIdx.x * COLS;
  const int ky = blockIdx.y;
  const int nc = min(COLS, nx - i0);
  C2 *sp = reinterpret_cast<C2 *>(spec) + (size_t)ky * nx + i0;
  const size_t rs = (size_t)nky * nx;  // stride of kz
  auto first = [&](int c, int base, auto gc, auto hc, R *xr, R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int m = 0; m < G; m++) {
      C2 v = Cplx<R>::make(R(0.), R(0.));
      if (c < nc) v = sp[bitrev(base + m * H, L2N) * rs + c];
      xr[m] = v.x;
      xi[m] = v.y;
    }
  };
  auto last = [&](int c, int base, auto gc, auto hc, const R *xr, const R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
    if (c >= nc) return;
#pragma unroll
    for (int m = 0; m < G; m++) sp[(base + m * H) * rs + c] = Cplx<R>::make(xr[m], xi[m]);
  };
  fft_lines<R, L2N, COLS>(re, im, tw, first, last);
}

// complex Neumann Thomas along x per line (ky, kz): tdm_c = -pl - pu + lambda,
// lambda = evy[ky] + evz[kz], first / last diagonal + pl[0] / + pu[nx-1], then
// gtsv component-wise (src/tdm.c:17-50; dft.c:364-395 in 2D).  Every thread
// sweeps one line of the block's LPB, the recurrence carried in registers in
// FP64 across chunks of XC points that the block stages in shared memory by
// cp.async (a warp's copies are runs of XC consecutive points of two lines):
// forward (values back into S, v into scratch), then back substitution in
// reverse chunk order.  The spectrum and the scratch of v are R.
// gauge0 (the FP32 passes of the defect-corrected solve): the line of the
// mode ky = kz = 0, whose Neumann system is singular, takes the gauge
// psi_hat(last) = 0 instead of the quotient by its round-off-sized last
// pivot (the FP64 path's choice, the reference's, whose solution then
// carries a large constant that FP32 storage of the line cannot resolve);
// psi changes by a constant only.
constexpr int XC = 16;
template <class R, int LPB>
struct XShape {
  using C2 = typename Cplx<R>::T;
  static constexpr size_t SQ = sizeof(C2) * LPB * (XC + 1);
  static constexpr size_t SMEM = SQ + sizeof(R) * LPB * (XC + 1) + 2 * sizeof(double) * XC;
};

template <class R, int LPB>
__global__ void __launch_bounds__(LPB) k3_pois_x(R *__restrict__ spec, R *__restrict__ scratch,
                                                 const double *__restrict__ pl, const double *__restrict__ pu,
                                                 const double *__restrict__ evy, const double *__restrict__ evz,
                                                 Grid3 g, int gauge0, unsigned long long *__restrict__ small_pivots) {
  using C2 = typename Cplx<R>::T;
  using S = XShape<R, LPB>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C2(*sq)[XC + 1] = reinterpret_cast<C2(*)[XC + 1]>(smraw);
  R(*sv)[XC + 1] = reinterpret_cast<R(*)[XC + 1]>(smraw + S::SQ);
  double *spl = reinterpret_cast<double *>(smraw + S::SQ + sizeof(R) * LPB * (XC + 1));
  double *spu = spl + XC;
  C2 *sp = reinterpret_cast<C2 *>(spec);
  const int nx = g.nx, nky = g.ny / 2 + 1;
  const long nlines = (long)nky * g.nz;
  const long l0 = (long)blockIdx.x * LPB;
  const int t = threadIdx.x;
  const bool live = l0 + t < nlines;
  const int nchunks = (nx + XC - 1) / XC;
  double lam = 0.;
  if (live) {
    const long l = l0 + t;
    lam = ldg(evy + l % nky) + ldg(evz + l / nky);
  }
  // chunk copies: element e = t + LPB r is point e % XC of line e / XC
  auto copy_in = [&](int p0, bool with_v) {
    const int pw = min(XC, nx - p0);
#pragma unroll 4
    for (int r = 0; r < XC; r++) {
      const int e = t + LPB * r, ll = e / XC, q = e % XC;
      const long l = l0 + ll;
      if (l < nlines && q < pw) {
        const size_t o = (size_t)l * nx + p0 + q;
        __pipeline_memcpy_async(&sq[ll][q], &sp[o], sizeof(C2));
        if (with_v) __pipeline_memcpy_async(&sv[ll][q], &scratch[o], sizeof(R));
      }
    }
    __pipeline_commit();
  };
  auto copy_out = [&](int p0, bool with_v) {
    const int pw = min(XC, nx - p0);
#pragma unroll 4
    for (int r = 0; r < XC; r++) {
      const int e = t + LPB * r, ll = e / XC, q = e % XC;
      const long l = l0 + ll;
      if (l < nlines && q < pw) {
        const size_t o = (size_t)l * nx + p0 + q;
        sp[o] = sq[ll][q];
        if (with_v) scratch[o] = sv[ll][q];
      }
    }
  };
  double vprev = 0., qr = 0., qi = 0.;
  bool small = false;  // a pivot of this line at most DBL_EPSILON in magnitude
  // ---------------------------------------------------------- forward
  for (int c = 0; c < nchunks; c++) {
    const int p0 = c * XC;
    if (t < XC) {
      spl[t] = (p0 + t < nx) ? ldg(pl + p0 + t) : 0.;
      spu[t] = (p0 + t < nx) ? ldg(pu + p0 + t) : 0.;
    }
    copy_in(p0, false);
    __pipeline_wait_prior(0);
    __syncthreads();
    if (live) {
      const int smax = min(XC, nx - p0);
      for (int s = 0; s < smax; s++) {
        const int i = p0 + s;
        const double l = spl[s], u = spu[s];
        double c = -l - u + lam;
        if (0 == i) c += l;
        if (nx - 1 == i) c += u;
        const C2 x = sq[t][s];
        const double xr = x.x, xi = x.y;
        if (0 == i) {
          small |= !(fabs(c) > kDblEpsilon);
          vprev = u / c;
          qr = xr / c;
          qi = xi / c;
        } else if (i < nx - 1) {
          const double piv = c - l * vprev;
          small |= !(fabs(piv) > kDblEpsilon);
          const double val = 1. / piv;
          vprev = val * (u);
          qr = val * (xr - l * qr);
          qi = val * (xi - l * qi);
        } else {
          const double val = c - l * vprev;
          small |= !(fabs(val) > kDblEpsilon);
          if (fabs(val) > kDblEpsilon && !(gauge0 && 0 == l0 + t)) {
            qr = 1. / val * (xr - l * qr);
            qi = 1. / val * (xi - l * qi);
          } else {
            qr = 0.;
            qi = 0.;
          }
        }
        sq[t][s] = Cplx<R>::make(R(qr), R(qi));
        sv[t][s] = R(vprev);
      }
    }
    __syncthreads();
    copy_out(p0, true);
    __syncthreads();
  }
  // ---------------------------------------------------------- backward
  // (FP64 arithmetic; in the mixed path the forward values come back rounded
  // to FP32, an error the defect-correction pass removes)
  double nr = 0., ni = 0.;
  for (int c = nchunks - 1; c >= 0; c--) {
    const int p0 = c * XC;
    copy_in(p0, true);
    __pipeline_wait_prior(0);
    __syncthreads();
    if (live) {
      const int smax = min(XC, nx - p0);
      for (int s = smax - 1; s >= 0; s--) {
        const int i = p0 + s;
        const C2 x = sq[t][s];
        if (nx - 1 == i) {
          nr = x.x;
          ni = x.y;
        } else {
          const double v = sv[t][s];
          nr = x.x - v * nr;
          ni = x.y - v * ni;
          sq[t][s] = Cplx<R>::make(R(nr), R(ni));
        }
      }
    }
    __syncthreads();
    copy_out(p0, false);
    __syncthreads();
  }
  // the ky = kz = 0 line is singular by construction (its last pivot is
  // round-off sized) and is not counted
  const unsigned bad = __ballot_sync(0xffffffffu, live && small && 0 != l0 + t);
  if (small_pivots && bad && 0 == (t & 31)) atomicAdd(small_pivots, (unsigned long long)__popc(bad));
}

// c2r along y (Hermitian extension as FFTW's c2r reads it: Im of X_0 and
// X_{ny/2} ignored), psi of COLS consecutive i of plane k with the halo
// images; the Neumann walls take the new neighbour value and hand
// their old value to the halo images
// ACC (the correction pass of the defect-corrected form): psi += the result,
// the walls take their neighbour's new total and their halo images keep what
// the first pass gave them
template <int L2N, class R, bool ACC>
__global__ void __launch_bounds__(kLineThreads, Line<R, L2N>::MINB)
    k3_pois_inv_y(const R *__restrict__ spec, double *__restrict__ psi, const R *__restrict__ tw, Grid3 g) {
  using L = Line<R, L2N>;
  using C2 = typename Cplx<R>::T;
  constexpr int N = L::N, COLS = L::COLS, NKY = N / 2 + 1;
  extern __shared__ unsigned char smraw[];
  R *re = reinterpret_cast<R *>(smraw);
  R *im = re + COLS * L::LD;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i0 = 1 + blockIdx.x * COLS;
  const int k = 1 + blockIdx.y;
  const int nc = min(COLS, nx - i0 + 1);
  const C2 *sp = reinterpret_cast<const C2 *>(spec) + (size_t)(k - 1) * NKY * nx + (i0 - 1);
  auto first = [&](int c, int base, auto gc, auto hc, R *xr, R *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const int m = bitrev(base + q * H, L2N);
      R r = R(0.), x = R(0.);
      if (c < nc) {
        // X_m for m <= N/2, conj(X_{N-m}) above; Im of X_0 and X_{N/2} ignored
        const int row = (2 * m <= N) ? m : N - m;
        const C2 v = __ldg(&sp[(size_t)row * nx + c]);
        r = v.x;
        x = (0 == m || 2 * m == N) ? R(0.) : ((2 * m < N) ? v.y : -v.y);
      }
      xr[q] = r;
      xi[q] = x;
    }
  };
  // psi of rows j = p + 1 with their halo images
  auto last = [&](int c, int base, auto gc, auto hc, const R *xr, const R *) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
    if (c >= nc) return;
    const int i = i0 + c;
    double y[G];
#pragma unroll
    for (int q = 0; q < G; q++) y[q] = (double)xr[q];
#pragma unroll
    for (int q = 0; q < G; q++) {
      const double v = y[q];
      for_images(base + q * H + 1, k, ny, nz, true, [&](int jj, int kk) {
        if (ACC) psi[ix_cc(g, i, jj, kk)] += v;
        else psi[ix_cc(g, i, jj, kk)] = v;
      });
    }
  };
  fft_lines<R, L2N, COLS>(re, im, tw, first, last);
  // Neumann walls of the interior rows of this plane (the blocks at either end
  // of x): the wall cell takes its neighbour's new value, read back after the
  // barrier, and hands its old value to its halo images
  const bool has_left = (1 == i0), has_right = (i0 + nc - 1 == nx);
  if (!has_left && !has_right) return;
  __syncthreads();
  for (int w = threadIdx.x; w < 2 * N; w += kLineThreads) {
    const int side = w / N, j = 1 + (w - side * N);
    if ((0 == side && !has_left) || (1 == side && !has_right)) continue;
    const int iw = side ? nx + 1 : 0;
    const double nv = psi[ix_cc(g, side ? nx : 1, j, k)];
    if (ACC) {
      psi[ix_cc(g, iw, j, k)] = nv;
      continue;
    }
    const double old = psi[ix_cc(g, iw, j, k)];
    psi[ix_cc(g, iw, j, k)] = nv;
    for_images(j, k, ny, nz, false, [&](int jj, int kk) { psi[ix_cc(g, iw, jj, kk)] = old; });
  }
}

// ---------------------------------------------------------------------------
// Packed y transforms (the mixed path's single FP64 pass; not the FP64
// path's, whose transforms follow the restatement's rounding): two adjacent
// columns i, i + 1 travel as the real and imaginary parts of one complex
// line, so each transform carries two real lines instead of one real line
// with a zero imaginary part, and a block covers 2 COLS columns.
// Forward: Z = FFT(b_i + i b_{i+1}), then X_p = (Z_p + conj Z_{N-p}) / 2 and
// Y_p = (Z_p - conj Z_{N-p}) / 2i for p <= N/2 (a pass through shared memory
// after the last stage).  Inverse: Z_m = X_m + i Y_m from the two half
// spectra (conjugates above N/2, Im of X_0, X_{N/2} and Y_0, Y_{N/2} dropped
// as the c2r transform drops them), then Re -> psi_i, Im -> psi_{i+1}.
template <int L2N>
__global__ void __launch_bounds__(kLineThreads, Line<double, L2N>::MINB)
    k3_pois_fwd_y_pk(const double *__restrict__ b, double *__restrict__ spec, const double *__restrict__ tw,
                     Grid3 g) {
  using L = Line<double, L2N>;
  using C2 = typename Cplx<double>::T;
  constexpr int N = L::N, COLS = L::COLS, NKY = N / 2 + 1, LD = L::LD;
  extern __shared__ unsigned char smraw[];
  double *re = reinterpret_cast<double *>(smraw);
  double *im = re + COLS * LD;
  const int nx = g.nx;
  const int i0 = 1 + blockIdx.x * 2 * COLS;  // columns i0 .. i0 + 2 COLS - 1
  const int k = 1 + blockIdx.y;
  const int ncol = min(2 * COLS, nx - i0 + 1);
  const double *bp = b + (size_t)nx * N * (k - 1) + (i0 - 1);
  C2 *out = reinterpret_cast<C2 *>(spec) + (size_t)(k - 1) * NKY * nx + (i0 - 1);
  auto first = [&](int c, int base, auto gc, auto hc, double *xr, double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int m = 0; m < G; m++) {
      const size_t row = (size_t)nx * bitrev(base + m * H, L2N);
      xr[m] = (2 * c < ncol) ? ldg(bp + row + 2 * c) : 0.;
      xi[m] = (2 * c + 1 < ncol) ? ldg(bp + row + 2 * c + 1) : 0.;
    }
  };
  auto last = [&](int c, int base, auto gc, auto hc, const double *xr, const double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int m = 0; m < G; m++) {
      re[c * LD + svof_fft_dev::fpad(base + m * H)] = xr[m];
      im[c * LD + svof_fft_dev::fpad(base + m * H)] = xi[m];
    }
  };
  svof_fft_dev::fft_lines<double, L2N, COLS>(re, im, tw, first, last);
  __syncthreads();
  // split: (p, column pair c) with c fastest, two adjacent outputs per thread
  for (int w = threadIdx.x; w < NKY * COLS; w += kLineThreads) {
    const int c = w % COLS, p = w / COLS;
    if (2 * c >= ncol) continue;
    const int q = (N - p) & (N - 1);
    const double a = re[c * LD + svof_fft_dev::fpad(p)], bb = im[c * LD + svof_fft_dev::fpad(p)];
    const double cr = re[c * LD + svof_fft_dev::fpad(q)], d = im[c * LD + svof_fft_dev::fpad(q)];
    out[(size_t)p * nx + 2 * c] = Cplx<double>::make(0.5 * (a + cr), 0.5 * (bb - d));
    if (2 * c + 1 < ncol) out[(size_t)p * nx + 2 * c + 1] = Cplx<double>::make(0.5 * (bb + d), -0.5 * (a - cr));
  }
}

template <int L2N>
__global__ void __launch_bounds__(kLineThreads, Line<double, L2N>::MINB)
    k3_pois_inv_y_pk(const double *__restrict__ spec, double *__restrict__ psi, const double *__restrict__ tw,
                     Grid3 g) {
  using L = Line<double, L2N>;
  using C2 = typename Cplx<double>::T;
  constexpr int N = L::N, COLS = L::COLS, NKY = N / 2 + 1;
  extern __shared__ unsigned char smraw[];
  double *re = reinterpret_cast<double *>(smraw);
  double *im = re + COLS * L::LD;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i0 = 1 + blockIdx.x * 2 * COLS;
  const int k = 1 + blockIdx.y;
  const int ncol = min(2 * COLS, nx - i0 + 1);
  const C2 *sp = reinterpret_cast<const C2 *>(spec) + (size_t)(k - 1) * NKY * nx + (i0 - 1);
  auto first = [&](int c, int base, auto gc, auto hc, double *xr, double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const int m = bitrev(base + q * H, L2N);
      const int row = (2 * m <= N) ? m : N - m;
      const bool edge = (0 == m || 2 * m == N);
      const double sgn = (2 * m < N) ? 1. : -1.;
      C2 x = Cplx<double>::make(0., 0.), y = Cplx<double>::make(0., 0.);
      if (2 * c < ncol) x = __ldg(&sp[(size_t)row * nx + 2 * c]);
      if (2 * c + 1 < ncol) y = __ldg(&sp[(size_t)row * nx + 2 * c + 1]);
      const double xi_ = edge ? 0. : sgn * x.y, yi_ = edge ? 0. : sgn * y.y;
      xr[q] = x.x - yi_;  // Re (X + i Y)
      xi[q] = xi_ + y.x;  // Im (X + i Y)
    }
  };
  auto last = [&](int c, int base, auto gc, auto hc, const double *xr, const double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const double ve = xr[q], vo = xi[q];
      for_images(base + q * H + 1, k, ny, nz, true, [&](int jj, int kk) {
        if (2 * c < ncol) psi[ix_cc(g, i0 + 2 * c, jj, kk)] = ve;
        if (2 * c + 1 < ncol) psi[ix_cc(g, i0 + 2 * c + 1, jj, kk)] = vo;
      });
    }
  };
  svof_fft_dev::fft_lines<double, L2N, COLS>(re, im, tw, first, last);
  // Neumann walls, as k3_pois_inv_y
  const bool has_left = (1 == i0), has_right = (i0 + ncol - 1 == nx);
  if (!has_left && !has_right) return;
  __syncthreads();
  for (int w = threadIdx.x; w < 2 * N; w += kLineThreads) {
    const int side = w / N, j = 1 + (w - side * N);
    if ((0 == side && !has_left) || (1 == side && !has_right)) continue;
    const int iw = side ? nx + 1 : 0;
    const double nv = psi[ix_cc(g, side ? nx : 1, j, k)];
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
  cudaError_t r = raise_smem_limit(kernel, (size_t)smem);
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
    if (cudaSuccess != (r = line_attrs(k3_pois_fwd_y<L2, R>, sm))) return r;
    if (cudaSuccess != (r = line_attrs(k3_pois_inv_y<L2, R, true>, sm))) return r;
    if constexpr (std::is_same<R, double>::value) {
      if (cudaSuccess != (r = line_attrs(k3_pois_fwd_y_pk<L2>, sm))) return r;
      if (cudaSuccess != (r = line_attrs(k3_pois_inv_y_pk<L2>, sm))) return r;
    }
    return line_attrs(k3_pois_inv_y<L2, R, false>, sm);
  });
  if (cudaSuccess != e) return e;
  e = by_l2n(log2nz, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    return line_attrs(k3_pois_z<L2, R>, Line<R, L2>::SMEM);
  });
  if (cudaSuccess != e) return e;
  if (cudaSuccess != (e = line_attrs(k3_pois_x<R, 64>, (int)XShape<R, 64>::SMEM))) return e;
  return line_attrs(k3_pois_x<R, 128>, (int)XShape<R, 128>::SMEM);
}

template <class R>
cudaError_t pois_fwd_y(cudaStream_t st, const double *ux, const double *uy, const double *uz, double *b, R *spec,
                       const R *tw, const double *dtp, double gam, int log2n, Grid3 g) {
  const dim3 bb(32, 8), bg((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kBPlanes - 1) / kBPlanes);
  k3_pois_b<<<bg, bb, 0, st>>>(ux, uy, uz, b, dtp, gam, g);
  cudaError_t e = cudaGetLastError();
  if (cudaSuccess != e) return e;
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.nz);
    k3_pois_fwd_y<L2, R><<<gr, kLineThreads, L::SMEM, st>>>(b, spec, tw, g);
    return cudaGetLastError();
  });
}

template <class R>
cudaError_t pois_z(cudaStream_t st, R *spec, const R *tw, int log2n, Grid3 g) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.ny / 2 + 1);
    k3_pois_z<L2, R><<<gr, kLineThreads, L::SMEM, st>>>(spec, tw, g);
    return cudaGetLastError();
  });
}

// lines per block of the x solve: 128, or 64 when 128 would leave SMs idle
inline bool pois_x_narrow(long nlines) { return nlines < 148L * 4 * 128; }

template <class R>
cudaError_t pois_x(cudaStream_t st, R *spec, R *scratch, const double *pl, const double *pu, const double *evy,
                   const double *evz, Grid3 g, bool gauge0, unsigned long long *small_pivots) {
  const long nlines = (long)(g.ny / 2 + 1) * g.nz;
  const int gz = gauge0 ? 1 : 0;
  if (pois_x_narrow(nlines)) {
    k3_pois_x<R, 64><<<(unsigned)((nlines + 63) / 64), 64, XShape<R, 64>::SMEM, st>>>(spec, scratch, pl, pu, evy,
                                                                                      evz, g, gz, small_pivots);
  } else {
    k3_pois_x<R, 128><<<(unsigned)((nlines + 127) / 128), 128, XShape<R, 128>::SMEM, st>>>(spec, scratch, pl, pu,
                                                                                          evy, evz, g, gz,
                                                                                          small_pivots);
  }
  return cudaGetLastError();
}

template <class R>
cudaError_t pois_inv_y(cudaStream_t st, const R *spec, double *psi, const R *tw, int log2n, Grid3 g, bool acc) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.nz);
    if (acc) k3_pois_inv_y<L2, R, true><<<gr, kLineThreads, L::SMEM, st>>>(spec, psi, tw, g);
    else k3_pois_inv_y<L2, R, false><<<gr, kLineThreads, L::SMEM, st>>>(spec, psi, tw, g);
    return cudaGetLastError();
  });
}

template <class R>
cudaError_t pois_fwd_y_array(cudaStream_t st, const double *b, R *spec, const R *tw, int log2n, Grid3 g) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<R, L2>;
    dim3 gr((g.nx + L::COLS - 1) / L::COLS, g.nz);
    k3_pois_fwd_y<L2, R><<<gr, kLineThreads, L::SMEM, st>>>(b, spec, tw, g);
    return cudaGetLastError();
  });
}

cudaError_t pois_fwd_y_packed(cudaStream_t st, const double *ux, const double *uy, const double *uz, double *b,
                              double *spec, const double *tw, const double *dtp, double gam, int log2n, Grid3 g) {
  const dim3 bb(32, 8), bg((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kBPlanes - 1) / kBPlanes);
  k3_pois_b<<<bg, bb, 0, st>>>(ux, uy, uz, b, dtp, gam, g);
  cudaError_t e = cudaGetLastError();
  if (cudaSuccess != e) return e;
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<double, L2>;
    dim3 gr((g.nx + 2 * L::COLS - 1) / (2 * L::COLS), g.nz);
    k3_pois_fwd_y_pk<L2><<<gr, kLineThreads, L::SMEM, st>>>(b, spec, tw, g);
    return cudaGetLastError();
  });
}

cudaError_t pois_inv_y_packed(cudaStream_t st, const double *spec, double *psi, const double *tw, int log2n,
                              Grid3 g) {
  return by_l2n(log2n, [&](auto c) {
    constexpr int L2 = decltype(c)::value;
    using L = Line<double, L2>;
    dim3 gr((g.nx + 2 * L::COLS - 1) / (2 * L::COLS), g.nz);
    k3_pois_inv_y_pk<L2><<<gr, kLineThreads, L::SMEM, st>>>(spec, psi, tw, g);
    return cudaGetLastError();
  });
}

cudaError_t pois_resid(cudaStream_t st, const double *b, const double *psi, double *r, const double *pl,
                       const double *pu, Grid3 g) {
  const dim3 bb(32, 8), bg((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kBPlanes - 1) / kBPlanes);
  k3_pois_resid<<<bg, bb, 0, st>>>(b, psi, r, pl, pu, g);
  return cudaGetLastError();
}

#define SVOF3_POISSON_INST(R)                                                                                    \
  template cudaError_t pois_prepare<R>(int, int);                                                                \
  template cudaError_t pois_fwd_y<R>(cudaStream_t, const double *, const double *, const double *, double *, R *, \
                                     const R *, const double *, double, int, Grid3);                            \
  template cudaError_t pois_z<R>(cudaStream_t, R *, const R *, int, Grid3);                                      \
  template cudaError_t pois_x<R>(cudaStream_t, R *, R *, const double *, const double *, const double *,        \
                                 const double *, Grid3, bool, unsigned long long *);                             \
  template cudaError_t pois_inv_y<R>(cudaStream_t, const R *, double *, const R *, int, Grid3, bool);          \
  template cudaError_t pois_fwd_y_array<R>(cudaStream_t, const double *, R *, const R *, int, Grid3);
SVOF3_POISSON_INST(double)
SVOF3_POISSON_INST(float)
#undef SVOF3_POISSON_INST

}  // namespace svof3
