// k_poisson.cu -- pressure Poisson solve of the FP64 2D path.
//
// Uniform x grid (src/fluid/compute_potential/dct.c:373-421):
//   k_dct_fwd     divergence right-hand side of one row, FFTW_REDFT10 along x
//   k_dct_ysolve  periodic tri-diagonal system along y for every x wavenumber
//                 (Sherman-Morrison, src/tdm.c:78-99), one wavenumber per thread
//   k_dct_inv     FFTW_REDFT01 along x, psi row with halo and Neumann walls
// Stretched x grid (src/fluid/compute_potential/dft.c:406-468):
//   k_dft_fwd     right-hand side of a tile of columns, r2c along y
//   k_dft_xsolve  complex Neumann tri-diagonal system along x for every y
//                 wavenumber (src/tdm.c:17-50, component-wise)
//   k_dft_inv     c2r along y, psi columns with halo and walls
//
// The reference transposes between x- and y-pencils around every transform;
// on one device the spectral array is instead laid out so that each line
// solve reads it coalesced: DCT path [j][kx] (threads over kx walk j), DFT
// path [i][ky] (threads over ky walk i).  No transpose pass exists.
//
// The transforms are the radix-2 decimation-in-time FFT of the oracle
// (oracle/svof_fft.c) with the same butterflies and the same twiddle tables,
// so with FMA contraction disabled they agree with it bit for bit.  Lengths
// must be powers of two (the DCT path's row transforms: 4 .. 4096 points).
#include <type_traits>

#include "fft_device.cuh"
#include "smem_limit.cuh"
#include "svof_internal.cuh"

namespace svof {

using svof_fft_dev::bitrev;
using svof_fft_dev::fft_stages;

// assign_input, dct.c:285-315 / dft.c:315-345
__device__ __forceinline__ double poisson_rhs(const double *__restrict__ ux, const double *__restrict__ uy,
                                              const Grid2 &g, int i, int j, double prefactor) {
  const int nx = g.nx;
  const double dx = g.dxf[i - 1];
  const double ux_xm = ux[ix_ux(nx, i, j)];
  const double ux_xp = ux[ix_ux(nx, i + 1, j)];
  const double uy_ym = uy[ix_cc(nx, i, j)];
  const double uy_yp = uy[ix_cc(nx, i, j + 1)];
  return prefactor * (+(ux_xp - ux_xm) / dx + (uy_yp - uy_ym) / g.dy);
}

// the right-hand side of the forward solve (assign_input): the divergence of
// the predicted velocity times the substep's prefactor
struct DivRhs {
  const double *ux, *uy;
  Grid2 g;
  double prefactor;
  __device__ __forceinline__ double operator()(int i, int j) const { return poisson_rhs(ux, uy, g, i, j, prefactor); }
};

// a right-hand side given as an array [j-1][i-1] divided by the cell widths
// dxf (the adjoint's solve with the grid-metric weights of the x grid)
struct ArrayRhs {
  const double *r;
  const double *dxf;
  int nx;
  __device__ __forceinline__ double operator()(int i, int j) const {
    return r[(size_t)(j - 1) * nx + (i - 1)] / dxf[i - 1];
  }
};

// ---------------------------------------------------------------- DCT path
// A block owns DctShape<L2N>::ROWS consecutive rows j (N = nx = 2^L2N points
// each; THREADS threads, pairs of (row, butterfly group) across the lanes)
// and runs their transforms as the register-blocked passes of fft_device.cuh:
// the same butterflies, twiddles and stage order as the oracle, three stages
// per pass between shared-memory round trips.  Dynamic shared memory: re / im
// (ROWS fft_ld(L2N) each), the rows' input (ROWS N) and, for the inverse, the
// rows' output (ROWS N).
// ROWS: one row up to 256 points (those grids have few rows: one block per
// row keeps the SMs busy), then 2048 / N; THREADS: the first pass's pairs,
// 32 .. 256
template <int L2N>
struct DctShape {
  static constexpr int N = 1 << L2N;
  static constexpr int ROWS = (L2N <= 8 || (2048 >> L2N) < 1) ? 1 : (2048 >> L2N);
  static constexpr int PAIRS = ROWS * (N >> (L2N < 3 ? L2N : 3));
  static constexpr int THREADS = PAIRS < 32 ? 32 : (PAIRS > 256 ? 256 : (PAIRS + 31) / 32 * 32);
  static constexpr int LD = svof_fft_dev::fft_ld(L2N);
  static constexpr size_t SMEM_FWD = sizeof(double) * ROWS * (2 * (size_t)LD + N);
  static constexpr size_t SMEM_INV = sizeof(double) * ROWS * (2 * (size_t)LD + 2 * N);
};

// rows j0 .. j0 + ROWS - 1 of the right-hand side, FFTW_REDFT10 along x into
// spec (Makhoul: v_m = x_{2m}, v_{n-1-m} = x_{2m+1}, an FFT of v, then
// 2 Re(w_k V_k) with the pre/post twiddles cs)
template <int L2N, class Rhs>
__device__ __forceinline__ void dct_fwd_rows(const Rhs &rhs, double *__restrict__ spec,
                                             const double *__restrict__ tw, const double *__restrict__ cs, int ny) {
  using S = DctShape<L2N>;
  constexpr int N = S::N, ROWS = S::ROWS, LD = S::LD;
  extern __shared__ double dsm[];
  double *re = dsm, *im = re + ROWS * LD, *rr = im + ROWS * LD;  // rr [ROWS][N]
  const int j0 = 1 + blockIdx.x * ROWS;
  const int nr = min(ROWS, ny - j0 + 1);
  // the rows' right-hand sides, read in order (coalesced)
  for (int w = threadIdx.x; w < ROWS * N; w += S::THREADS) {
    const int c = w >> L2N, i = w & (N - 1);
    rr[w] = (c < nr) ? rhs(i + 1, j0 + c) : 0.;
  }
  __syncthreads();
  // point p of the bit-reversed FFT input holds v_m, m = bitrev(p)
  auto first = [&](int c, int base, auto gc, auto hc, double *xr, double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const int m = bitrev(base + q * H, L2N);
      const int src = (m < N / 2) ? 2 * m : 2 * (N - 1 - m) + 1;
      xr[q] = rr[c * N + src];
      xi[q] = 0.;
    }
  };
  auto last = [&](int c, int base, auto gc, auto hc, const double *xr, const double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
    if (c >= nr) return;
    double *out = spec + (size_t)(j0 + c - 1) * N;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const int k = base + q * H;
      const double2 w = __ldg(reinterpret_cast<const double2 *>(cs) + k);
      out[k] = 2.0 * (w.x * xr[q] + w.y * xi[q]);
    }
  };
  svof_fft_dev::fft_lines<double, L2N, ROWS, 1, S::THREADS>(re, im, tw, first, last);
}

template <int L2N>
__global__ void __launch_bounds__(DctShape<L2N>::THREADS) k_dct_fwd(const double *__restrict__ ux, const double *__restrict__ uy,
                                                        double *__restrict__ spec, const double *__restrict__ tw,
                                                        const double *__restrict__ cs, const double *__restrict__ dtp,
                                                        double gam, Grid2 g) {
  pdl_enter();
  const double dt = *dtp;
  const double prefactor = 1. / (gam * dt) / (2. * (1 << L2N));
  dct_fwd_rows<L2N>(DivRhs{ux, uy, g, prefactor}, spec, tw, cs, g.ny);
}

template <int L2N>
__global__ void __launch_bounds__(DctShape<L2N>::THREADS) k_dct_fwd_rhs(const double *__restrict__ r, double *__restrict__ spec,
                                                            const double *__restrict__ tw,
                                                            const double *__restrict__ cs, Grid2 g) {
  dct_fwd_rows<L2N>(ArrayRhs{r, g.dxf, g.nx}, spec, tw, cs, g.ny);
}

// periodic tri-diagonal solve along y per wavenumber k (src/tdm.c:78-99 with
// gtsv :17-50).  The k-dependent, time-independent quantities the reference
// recomputes on every call are tables: vt[j][k] (gtsv's v), rvt[j][k]
// (gtsv's val = 1 / (c - l v[j-1]), j = 1 .. n-3), lastf[k] (1 / val of the
// last row, 0 where the reference zeroes that row), q1t[j][k] and den[k]
// (Sherman-Morrison).  A block owns kt consecutive wavenumbers; all its
// threads stage the lines and their tables in shared memory ([j][t],
// coalesced), then one thread per line runs the recurrences on shared memory
// only, and all threads apply the Sherman-Morrison correction on the way out.
__global__ void k_dct_ysolve(double *__restrict__ spec, const double *__restrict__ vt,
                             const double *__restrict__ rvt, const double *__restrict__ q1t,
                             const double *__restrict__ ck, const double *__restrict__ lastf,
                             const double *__restrict__ den, double lap, int nx, int ny, int kt) {
  pdl_enter();
  extern __shared__ double sm[];
  double *sq = sm;                       // [ny][kt] line data
  double *sv = sm + (size_t)ny * kt;     // [ny][kt] v
  double *sr = sm + 2 * (size_t)ny * kt; // [ny][kt] val
  __shared__ double sl[64];
  const int k0 = blockIdx.x * kt;
  const int n = ny;
  const int nk = min(kt, nx - k0);
  for (int w = threadIdx.x; w < n * kt; w += blockDim.x) {
    const int j = w / kt, t = w - j * kt;
    const size_t g = (size_t)j * nx + k0 + t;
    const bool ok = t < nk;
    sq[w] = ok ? spec[g] : 0.;
    sv[w] = ok ? vt[g] : 0.;
    sr[w] = ok ? rvt[g] : 0.;
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < nk) {
    const int k = k0 + t;
    const double l = lap, u = lap, c = ck[k];
    const double lf = lastf[k];
    const double d = den[k];
    double *q = sq + t;
    const double *v = sv + t, *r = sr + t;
#define Q(jj) q[(size_t)(jj) * kt]
#define V(jj) v[(size_t)(jj) * kt]
#define RV(jj) r[(size_t)(jj) * kt]
    // gtsv of size n-1 on rows 0 .. n-2.  The interior rows go in batches of
    // YB: the batch's loads first, then the dependent chain on registers,
    // then its stores (the same expressions in the same order as one row at
    // a time, which the remainder rows use).
    constexpr int YB = 8;
    double qprev = Q(0) / c;
    Q(0) = qprev;
    int i = 1;
    for (; i + YB <= n - 2; i += YB) {
      double xv[YB], rv[YB];
#pragma unroll
      for (int k = 0; k < YB; k++) {
        xv[k] = Q(i + k);
        rv[k] = RV(i + k);
      }
#pragma unroll
      for (int k = 0; k < YB; k++) {
        qprev = rv[k] * (xv[k] - l * qprev);
        xv[k] = qprev;
      }
#pragma unroll
      for (int k = 0; k < YB; k++) Q(i + k) = xv[k];
    }
    for (; i < n - 2; i++) {
      qprev = RV(i) * (Q(i) - l * qprev);
      Q(i) = qprev;
    }
    Q(n - 2) = (0. != lf) ? lf * (Q(n - 2) - l * qprev) : 0.;
    double qn = Q(n - 2);
    i = n - 3;
    for (; i - YB + 1 >= 0; i -= YB) {
      double xv[YB], vv[YB];
#pragma unroll
      for (int k = 0; k < YB; k++) {
        xv[k] = Q(i - k);
        vv[k] = V(i - k);
      }
#pragma unroll
      for (int k = 0; k < YB; k++) {
        qn = xv[k] - vv[k] * qn;
        xv[k] = qn;
      }
#pragma unroll
      for (int k = 0; k < YB; k++) Q(i - k) = xv[k];
    }
    for (; i >= 0; i--) {
      qn = Q(i) - V(i) * qn;
      Q(i) = qn;
    }
    // Sherman-Morrison correction
    const double num = Q(n - 1) - u * qn - l * Q(n - 2);
    const double qlast = fabs(d) < kDblEpsilon ? 0. : num / d;
    Q(n - 1) = qlast;
    sl[t] = qlast;
#undef Q
#undef V
#undef RV
  }
  __syncthreads();
  for (int w = threadIdx.x; w < n * kt; w += blockDim.x) {
    const int j = w / kt, tt = w - j * kt;
    if (tt < nk) {
      const size_t g = (size_t)j * nx + k0 + tt;
      spec[g] = (j < n - 1) ? sq[w] + sl[tt] * q1t[g] : sq[w];
    }
  }
}

// rows j0 .. j0 + ROWS - 1: REDFT01 then extract_output +
// fluid_update_boundaries_psi (the pre-twiddle pairs spectrum k and n - k;
// FFT point p is output position 2p below n/2, 2(n-1-p)+1 above)
template <int L2N>
__global__ void __launch_bounds__(DctShape<L2N>::THREADS) k_dct_inv(const double *__restrict__ spec, double *__restrict__ psi,
                                                        const double *__restrict__ tw, const double *__restrict__ cs,
                                                        Grid2 g) {
  pdl_enter();
  using S = DctShape<L2N>;
  constexpr int N = S::N, ROWS = S::ROWS, LD = S::LD;
  extern __shared__ double dsm[];
  double *re = dsm, *im = re + ROWS * LD, *in = im + ROWS * LD, *ro = in + ROWS * N;  // in, ro [ROWS][N]
  __shared__ double wold[4];  // old wall values of rows 1 and ny (left, right)
  const int nx = g.nx, ny = g.ny;
  const int j0 = 1 + blockIdx.x * ROWS;
  const int nr = min(ROWS, ny - j0 + 1);
  // old wall values of the rows that feed the halo, read before any write
  if (threadIdx.x < 4) {
    const int row = (threadIdx.x < 2) ? 1 : ny, side = threadIdx.x & 1;
    if (row >= j0 && row < j0 + nr) wold[threadIdx.x] = psi[ix_cc(nx, side ? nx + 1 : 0, row)];
  }
  // the spectrum rows, read in order (coalesced)
  for (int w = threadIdx.x; w < ROWS * N; w += S::THREADS) {
    const int c = w >> L2N;
    in[w] = (c < nr) ? spec[(size_t)(j0 - 1) * N + w] : 0.;
  }
  __syncthreads();
  auto first = [&](int c, int base, auto gc, auto hc, double *xr, double *xi) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const int m = bitrev(base + q * H, L2N);
      const double a = in[c * N + m];
      const double b = (0 == m) ? 0. : in[c * N + N - m];
      const double2 w = __ldg(reinterpret_cast<const double2 *>(cs) + m);
      xr[q] = w.x * a + w.y * b;
      xi[q] = w.y * a - w.x * b;
    }
  };
  auto last = [&](int c, int base, auto gc, auto hc, const double *xr, const double *) {
    constexpr int G = decltype(gc)::value, H = decltype(hc)::value;
#pragma unroll
    for (int q = 0; q < G; q++) {
      const int p = base + q * H;
      const int o = (p < N / 2) ? 2 * p : 2 * (N - 1 - p) + 1;
      ro[c * N + o] = xr[q];
    }
  };
  svof_fft_dev::fft_lines<double, L2N, ROWS, 1, S::THREADS>(re, im, tw, first, last);
  __syncthreads();
  // psi rows with their halo images, written in order (coalesced)
  for (int w = threadIdx.x; w < nr * N; w += S::THREADS) {
    const int c = w >> L2N, i = (w & (N - 1)) + 1, j = j0 + c;
    const double y = ro[w];
    psi[ix_cc(nx, i, j)] = y;
    if (ny == j) psi[ix_cc(nx, i, 0)] = y;
    if (1 == j) psi[ix_cc(nx, i, ny + 1)] = y;
  }
  // Neumann walls, psi.c:7-20 (the wall takes its neighbour), and the halo
  // rows' wall cells, which take the walls' old values
  for (int c = threadIdx.x; c < nr; c += S::THREADS) {
    const int j = j0 + c;
    psi[ix_cc(nx, 0, j)] = ro[c * N];
    psi[ix_cc(nx, nx + 1, j)] = ro[c * N + N - 1];
    if (ny == j) {
      psi[ix_cc(nx, 0, 0)] = wold[2];
      psi[ix_cc(nx, nx + 1, 0)] = wold[3];
    }
    if (1 == j) {
      psi[ix_cc(nx, 0, ny + 1)] = wold[0];
      psi[ix_cc(nx, nx + 1, ny + 1)] = wold[1];
    }
  }
}

// ---- launch plans of the DCT row transforms, by length
namespace {
template <class F>
auto by_log2n(int l2n, F f) {
  switch (l2n) {
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
    default: return f(std::integral_constant<int, 12>());
  }
}
}  // namespace

bool dct_length_ok(int log2n) { return log2n >= kDctMinL2N && log2n <= kDctMaxL2N; }
int dct_rows(int log2n) {
  return by_log2n(log2n, [](auto c) { return DctShape<decltype(c)::value>::ROWS; });
}
int dct_threads(int log2n) {
  return by_log2n(log2n, [](auto c) { return DctShape<decltype(c)::value>::THREADS; });
}
size_t dct_smem(int log2n, bool inverse) {
  return by_log2n(log2n, [&](auto c) {
    using S = DctShape<decltype(c)::value>;
    return inverse ? S::SMEM_INV : S::SMEM_FWD;
  });
}
DctFwdKernel dct_fwd_kernel(int log2n) {
  return by_log2n(log2n, [](auto c) { return (DctFwdKernel)&k_dct_fwd<decltype(c)::value>; });
}
DctFwdRhsKernel dct_fwd_rhs_kernel(int log2n) {
  return by_log2n(log2n, [](auto c) { return (DctFwdRhsKernel)&k_dct_fwd_rhs<decltype(c)::value>; });
}
DctInvKernel dct_inv_kernel(int log2n) {
  return by_log2n(log2n, [](auto c) { return (DctInvKernel)&k_dct_inv<decltype(c)::value>; });
}
cudaError_t dct_prepare(int log2n) {
  if (!dct_length_ok(log2n)) return cudaErrorInvalidValue;
  cudaError_t e = raise_smem_limit(dct_fwd_kernel(log2n), dct_smem(log2n, false));
  if (cudaSuccess == e) e = raise_smem_limit(dct_fwd_rhs_kernel(log2n), dct_smem(log2n, false));
  if (cudaSuccess == e) e = raise_smem_limit(dct_inv_kernel(log2n), dct_smem(log2n, true));
  return e;
}

// ---------------------------------------------------------------- DFT path
// columns i0 .. i0+cols-1 of the right-hand side, r2c along y into spec; the
// block's dynamic shared memory holds cols * 2 ny doubles
template <class Rhs>
__device__ __forceinline__ void dft_fwd_cols(const Rhs &rhs, double *__restrict__ spec, const double *__restrict__ tw,
                                             int log2n, int cols, int nx, int n, int i0) {
  extern __shared__ double z[];
  const int nky = n / 2 + 1;
  const int nc = min(cols, nx - i0 + 1);
  for (int w = threadIdx.x; w < cols * n; w += blockDim.x) {
    const int q = w / cols, col = w % cols;
    const int m = bitrev(q, log2n);
    double v = 0.;
    if (col < nc) v = rhs(i0 + col, m + 1);
    z[2 * (col * n + q)] = v;
    z[2 * (col * n + q) + 1] = 0.;
  }
  __syncthreads();
  fft_stages(z, log2n, cols, tw);
  for (int w = threadIdx.x; w < nc * nky; w += blockDim.x) {
    const int col = w / nky, k = w % nky;
    const size_t o = 2 * ((size_t)(i0 - 1 + col) * nky + k);
    spec[o] = z[2 * (col * n + k)];
    spec[o + 1] = z[2 * (col * n + k) + 1];
  }
}

// a block owns `cols` consecutive columns i0 .. i0+cols-1 and all ny rows;
// dynamic shared memory cols * 2 ny doubles
__global__ void k_dft_fwd(const double *__restrict__ ux, const double *__restrict__ uy,
                          double *__restrict__ spec, const double *__restrict__ tw,
                          const double *__restrict__ dtp, double gam, int log2n, int cols, Grid2 g) {
  pdl_enter();
  const int n = g.ny;
  const double dt = *dtp;
  const double prefactor = 1. / (gam * dt) / (1. * n);
  dft_fwd_cols(DivRhs{ux, uy, g, prefactor}, spec, tw, log2n, cols, g.nx, n, 1 + blockIdx.x * cols);
}

__global__ void k_dft_fwd_rhs(const double *__restrict__ r, double *__restrict__ spec, const double *__restrict__ tw,
                              int log2n, int cols, Grid2 g) {
  dft_fwd_cols(ArrayRhs{r, g.dxf, g.nx}, spec, tw, log2n, cols, g.nx, g.ny, 1 + blockIdx.x * cols);
}

// complex Neumann Thomas along x per ky (dft.c:364-395); spec layout [i][ky],
// vt[i][ky] and rvt[i][ky] hold the reference's v and val for each ky.  A
// block owns kt consecutive ky lines: all threads stage them and their tables
// in shared memory, one thread per line runs the recurrences there.
__global__ void k_dft_xsolve(double *__restrict__ spec, const double *__restrict__ vt,
                             const double *__restrict__ rvt, const double *__restrict__ pl,
                             const double *__restrict__ pu, const double *__restrict__ evals, int nx,
                             int nky, int kt) {
  pdl_enter();
  extern __shared__ double sm[];
  double *sre = sm;                        // [nx][kt]
  double *sim = sm + (size_t)nx * kt;      // [nx][kt]
  double *sv = sm + 2 * (size_t)nx * kt;   // [nx][kt]
  double *sr = sm + 3 * (size_t)nx * kt;   // [nx][kt]
  const int k0 = blockIdx.x * kt;
  const int nk = min(kt, nky - k0);
  const int n = nx;
  for (int w = threadIdx.x; w < n * kt; w += blockDim.x) {
    const int i = w / kt, t = w - i * kt;
    const size_t g = (size_t)i * nky + k0 + t;
    const bool ok = t < nk;
    sre[w] = ok ? spec[2 * g] : 0.;
    sim[w] = ok ? spec[2 * g + 1] : 0.;
    sv[w] = ok ? vt[g] : 0.;
    sr[w] = ok ? rvt[g] : 0.;
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < nk) {
    const double ev = evals[k0 + t];
#define QR(ii) sre[(size_t)(ii) * kt + t]
#define QI(ii) sim[(size_t)(ii) * kt + t]
#define V(ii) sv[(size_t)(ii) * kt + t]
#define RV(ii) sr[(size_t)(ii) * kt + t]
    // tdm_c with the Neumann boundary rows
    double c0 = -pl[0] - pu[0] + ev;
    c0 += pl[0];
    double pr = QR(0) / c0, pi = QI(0) / c0;
    QR(0) = pr;
    QI(0) = pi;
#pragma unroll 4
    for (int i = 1; i < n - 1; i++) {
      const double l = pl[i];
      const double val = RV(i);  // 1 / (c_i - l_i v_{i-1})
      pr = val * (QR(i) - l * pr);
      pi = val * (QI(i) - l * pi);
      QR(i) = pr;
      QI(i) = pi;
    }
    {
      const double l = pl[n - 1];
      double c = -l - pu[n - 1] + ev;
      c += pu[n - 1];
      const double val = c - l * V(n - 2);
      if (fabs(val) > kDblEpsilon) {
        QR(n - 1) = 1. / val * (QR(n - 1) - l * pr);
        QI(n - 1) = 1. / val * (QI(n - 1) - l * pi);
      } else {
        QR(n - 1) = 0.;
        QI(n - 1) = 0.;
      }
    }
    double nr = QR(n - 1), ni = QI(n - 1);
#pragma unroll 4
    for (int i = n - 2; i >= 0; i--) {
      const double v = V(i);
      nr = QR(i) - v * nr;
      ni = QI(i) - v * ni;
      QR(i) = nr;
      QI(i) = ni;
    }
#undef QR
#undef QI
#undef V
#undef RV
  }
  __syncthreads();
  for (int w = threadIdx.x; w < n * kt; w += blockDim.x) {
    const int i = w / kt, tt = w - i * kt;
    if (tt < nk) {
      const size_t g = (size_t)i * nky + k0 + tt;
      spec[2 * g] = sre[w];
      spec[2 * g + 1] = sim[w];
    }
  }
}

// c2r along y for a tile of columns, extract_output and the psi boundaries
__global__ void k_dft_inv(const double *__restrict__ spec, double *__restrict__ psi,
                          const double *__restrict__ tw, int log2n, int cols, Grid2 g) {
  pdl_enter();
  extern __shared__ double z[];
  const int n = g.ny, nx = g.nx, ny = g.ny;
  const int nky = n / 2 + 1;
  const int i0 = 1 + blockIdx.x * cols;
  const int nc = min(cols, nx - i0 + 1);
  const bool has_left = (1 == i0), has_right = (i0 + nc - 1 == nx);
  // old wall values feeding the halo rows (read before any write)
  double wl1 = 0., wln = 0., wr1 = 0., wrn = 0.;
  if (0 == threadIdx.x) {
    if (has_left) {
      wl1 = psi[ix_cc(nx, 0, 1)];
      wln = psi[ix_cc(nx, 0, ny)];
    }
    if (has_right) {
      wr1 = psi[ix_cc(nx, nx + 1, 1)];
      wrn = psi[ix_cc(nx, nx + 1, ny)];
    }
  }
  // Hermitian extension as FFTW's c2r reads it: Im of X_0 and X_{n/2} ignored
  for (int w = threadIdx.x; w < cols * n; w += blockDim.x) {
    const int q = w / cols, col = w % cols;
    const int m = bitrev(q, log2n);
    double re = 0., im = 0.;
    if (col < nc) {
      const size_t base = 2 * ((size_t)(i0 - 1 + col) * nky);
      if (0 == m) {
        re = spec[base];
      } else if (2 * m < n) {
        re = spec[base + 2 * m];
        im = spec[base + 2 * m + 1];
      } else if (2 * m == n) {
        re = spec[base + 2 * m];
      } else {
        re = spec[base + 2 * (n - m)];
        im = -spec[base + 2 * (n - m) + 1];
      }
    }
    z[2 * (col * n + q)] = re;
    z[2 * (col * n + q) + 1] = im;
  }
  __syncthreads();
  fft_stages(z, log2n, cols, tw);
  for (int w = threadIdx.x; w < nc * n; w += blockDim.x) {
    const int r = w / nc, col = w % nc;
    const int i = i0 + col, j = r + 1;
    const double y = z[2 * (col * n + r)];
    psi[ix_cc(nx, i, j)] = y;
    if (ny == j) psi[ix_cc(nx, i, 0)] = y;
    if (1 == j) psi[ix_cc(nx, i, ny + 1)] = y;
  }
  __syncthreads();
  if (0 == threadIdx.x) {
    if (has_left) {
      psi[ix_cc(nx, 0, 0)] = wln;
      psi[ix_cc(nx, 0, ny + 1)] = wl1;
    }
    if (has_right) {
      psi[ix_cc(nx, nx + 1, 0)] = wrn;
      psi[ix_cc(nx, nx + 1, ny + 1)] = wr1;
    }
  }
  // Neumann walls, psi.c:7-20
  for (int j = 1 + threadIdx.x; j <= ny; j += blockDim.x) {
    if (has_left) psi[ix_cc(nx, 0, j)] = z[2 * (0 * n + (j - 1))];
    if (has_right) psi[ix_cc(nx, nx + 1, j)] = z[2 * ((nc - 1) * n + (j - 1))];
  }
}

}  // namespace svof
