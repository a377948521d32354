// k3_adjoint.cu -- kernels of the 3D step's adjoint (FP64 path): the
// transposes, in reverse, of the step functions of the restatement
// oracle/svof_oracle3d.c (the reference's 2D step carried to a second,
// periodic direction z), as the 2D adjoint (k_adjoint.cu) does for the 2D
// step:
//
//   k3_adj_project    fluid_update_pressure and fluid_correct_velocity
//   k3_adj_div        the divergence right-hand side of the Poisson solve
//                     (its solve: the forward's own transforms and line
//                     solves on psi_bar / dxf, host side)
//   k3_adj_xsolve     the implicit-x Thomas solves of ux, uy, uz (from the
//                     forward's LU table) and the RK split of delta_bar
//   k3_adj_rhs        the momentum right-hand sides (advection x, y, z,
//                     diffusion, pressure, surface force)
//   k3_adj_interface  the THINC/QQ fluxes and the RK update of vof, the CSF
//                     force, the intercept (implicit function theorem) and
//                     the cell normal's normalisation
//   k3_adj_cgrad      per corner: the corner normals' adjoint from the eight
//                     cells around it (mean normal, curvature) through the
//                     normalisation's transpose
//   k3_adj_cvof       per cell: the corner gradients' transpose back to vof
//
// Adjoint fields are compact: ux faces i = 2..nx (ix_srcx), cells i = 1..nx
// (ix_src); y and z are periodic, so an index 0 or n + 1 wraps (a halo row
// or plane holds a copy of an interior one, and every primal function reads
// the copy with the same arithmetic as the original).  Wall values are
// constants and carry no adjoint.  The primal fields are read in their
// storage layouts, halos included.  Branches follow the primal state
// (upwind side, interfacial test, eps clamps).  Every kernel gathers (each
// thread owns its outputs): no atomics, results independent of scheduling.
// Spacings enter as reciprocals (AGrid3): no divisions but the normalisations'.
// The temperature is not differentiated (the adjoint needs add_buoyancy = 0).
#include <cuda_pipeline.h>

#include "adjoint3d_internal.cuh"

namespace svof3 {

namespace {

__constant__ double a3_gauss_p[2] = {-0.2886751345948129, +0.2886751345948129};
__constant__ double a3_gauss_w[2] = {+0.5, +0.5};
constexpr double kBeta3 = 1.;
constexpr double kVofMin3 = 1.e-8;
constexpr double kInvEps = 4503599627370496.;  // 1 / DBL_EPSILON = 2^52

__device__ __forceinline__ int wrap(int j, int n) { return j < 1 ? j + n : (j > n ? j - n : j); }
__device__ __forceinline__ bool interfacial3(double v) { return !(v < kVofMin3 || 1. - kVofMin3 < v); }

// H and H' of the THINC indicator 1 / (1 + exp(-2 beta z))
__device__ __forceinline__ void thinc_hh3(double z, double &h, double &hp) {
  h = 1. / (1. + exp(-2. * kBeta3 * z));
  hp = 2. * kBeta3 * h * (1. - h);
}

// transpose of the derivative of g / max(|g|, eps) (a symmetric Jacobian)
__device__ __forceinline__ void unit_adj3(double gx, double gy, double gz, double bx, double by, double bz,
                                          double &ox, double &oy, double &oz) {
  const double norm = sqrt(gx * gx + gy * gy + gz * gz);
  if (norm > kDblEpsilon) {
    const double rn = 1. / norm;
    const double nx_ = gx * rn, ny_ = gy * rn, nz_ = gz * rn;
    const double pr = nx_ * bx + ny_ * by + nz_ * bz;
    ox = (bx - nx_ * pr) * rn;
    oy = (by - ny_ * pr) * rn;
    oz = (bz - nz_ * pr) * rn;
  } else {
    ox = bx * kInvEps;
    oy = by * kInvEps;
    oz = bz * kInvEps;
  }
}

// the unnormalised corner gradient of compute_gradient at corner (ic, jc, kc)
// (storage rows jc - 1, jc and planes kc - 1, kc)
__device__ __forceinline__ void corner_grad3(const double *__restrict__ vof, const AGrid3 &ag, int ic, int jc,
                                             int kc, double &gx, double &gy, double &gz) {
  const Grid3 &g = ag.g;
  double a[2][4];
  for (int q = 0; q < 2; q++) {
    const long o = ix_vof(g, ic - 1, jc - 1, kc - 1 + q);
    const long r = g.nx + 2;
    a[q][0] = vof[o];
    a[q][1] = vof[o + 1];
    a[q][2] = vof[o + r];
    a[q][3] = vof[o + r + 1];
  }
  gx = ag.rxc[ic - 1] * ((-a[0][0] + a[0][1] - a[0][2] + a[0][3]) + (-a[1][0] + a[1][1] - a[1][2] + a[1][3]));
  gy = ag.rdy * ((-a[0][0] - a[0][1] + a[0][2] + a[0][3]) + (-a[1][0] - a[1][1] + a[1][2] + a[1][3]));
  gz = ag.rdz * ((+a[1][0] + a[1][1] + a[1][2] + a[1][3]) - (+a[0][0] + a[0][1] + a[0][2] + a[0][3]));
}

__device__ __forceinline__ bool cell3(const Grid3 &g, int &i, int &j, int &k) {
  i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  k = 1 + blockIdx.z;
  return i <= g.nx && j <= g.ny && k <= g.nz;
}

// offsets of the periodic neighbours of row j / plane k in a compact array of
// rows of w values (a row step s = w, a plane step p = w ny)
struct Wrap3 {
  long jp, jm, kp, km;
  __device__ __forceinline__ Wrap3(int j, int k, int ny, int nz, long w) {
    const long p = w * ny;
    jp = (j == ny) ? -(long)(ny - 1) * w : w;
    jm = (j == 1) ? (long)(ny - 1) * w : -w;
    kp = (k == nz) ? -(long)(nz - 1) * p : p;
    km = (k == 1) ? (long)(nz - 1) * p : -p;
  }
  __device__ __forceinline__ long at(int dj, int dk) const {
    return (dj == 0 ? 0L : (dj > 0 ? jp : jm)) + (dk == 0 ? 0L : (dk > 0 ? kp : km));
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// psi_bar += (d p' / d psi)^T p_bar' (mode & 1), (d u' / d psi)^T u_bar'
// (mode & 2); u_bar and p_bar pass through (u' = u* - ..., p' = p + ...).
// update_pressure: p'(i) = p(i) + psi(i) - pre / dxf_i (-dm + dp) with the
// Neumann walls (dm = 0 at i = 1, dp = 0 at i = nx); correct: u' = u* - gdt
// grad psi, y and z periodic.
__global__ void k3_adj_project(const double *__restrict__ aux, const double *__restrict__ auy,
                               const double *__restrict__ auz, const double *__restrict__ ap,
                               double *__restrict__ apsi, double gdt, double pre, int mode, AGrid3 ag) {
  int i, j, k;
  const Grid3 &g = ag.g;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx;
  const long oc = ix_src(g, i, j, k);
  double acc = 0.;
  if (mode & 1) {
    const double pb = ap[oc];
    const double ci = pre * ag.rxf[i - 1];
    double diag = 0.;
    if (i > 1) diag += ag.rxc[i - 1];
    if (i < nx) diag += ag.rxc[i];
    acc += pb + pb * ci * diag;
    if (i > 1) acc -= ap[oc - 1] * (pre * ag.rxf[i - 2]) * ag.rxc[i - 1];
    if (i < nx) acc -= ap[oc + 1] * (pre * ag.rxf[i]) * ag.rxc[i];
  }
  if (mode & 2) {
    const Wrap3 w(j, k, g.ny, g.nz, nx);
    const long of = ix_srcx(g, i, j, k);
    if (i >= 2) acc -= gdt * ag.rxc[i - 1] * aux[of];
    if (i + 1 <= nx) acc += gdt * ag.rxc[i] * aux[of + 1];
    acc -= gdt * ag.rdy * auy[oc];
    acc += gdt * ag.rdy * auy[oc + w.jp];
    acc -= gdt * ag.rdz * auz[oc];
    acc += gdt * ag.rdz * auz[oc + w.kp];
  }
  apsi[oc] += acc;
}

// b = psi_bar / dxf into the compact right-hand-side layout of the forward
// transforms (x fastest, nx ny per plane: the same as ix_src)
__global__ void k3_adj_scale(const double *__restrict__ apsi, double *__restrict__ b, AGrid3 ag) {
  int i, j, k;
  if (!cell3(ag.g, i, j, k)) return;
  const long o = ix_src(ag.g, i, j, k);
  b[o] = apsi[o] * ag.rxf[i - 1];
}

// the transpose of the divergence right-hand side b = pre (dux/dxf + duy/dy +
// duz/dz) applied to the adjoint solve's output s (psi layout): b_bar =
// dxf s; also clears psi_bar (the forward overwrites psi)
__global__ void k3_adj_div(double *__restrict__ aux, double *__restrict__ auy, double *__restrict__ auz,
                           const double *__restrict__ s, double *__restrict__ apsi, double pre_p, AGrid3 ag) {
  int i, j, k;
  const Grid3 &g = ag.g;
  if (!cell3(g, i, j, k)) return;
  const long oc = ix_src(g, i, j, k);
  const long q = ix_cc(g, i, j, k);  // psi layout: halos hold the periodic copies
  const double sc = s[q];
  if (i >= 2) aux[ix_srcx(g, i, j, k)] += pre_p * (s[q - 1] - sc);
  const double dxf = g.dxf[i - 1];
  auy[oc] += pre_p * (dxf * ag.rdy) * (s[q - (g.nx + 2)] - sc);
  auz[oc] += pre_p * (dxf * ag.rdz) * (s[q - (long)(g.nx + 2) * (g.ny + 2)] - sc);
  apsi[oc] = 0.;
}

// ---------------------------------------------------------------------------
// delta_bar = T^-T u_bar* for every x line of ux, uy, uz, T = L U the
// forward's factorisation (k3_tdm_coef: per system s at coef + 3 s nx, L[i],
// R[i] = 1 / d_i (R[0] = d_0), V[i] = v_i; systems 0 ux, 1 uy and uz):
// U^T z = b (z_0 = b_0, z_i = b_i - v_{i-1} z_{i-1}), then L^T y = z
// (y_{n-1} = R_{n-1} z_{n-1}, y_i = R_i (z_i - l_{i+1} y_{i+1}), y_0 = (z_0 -
// l_1 y_1) / d_0).  Then the RK weights: src_a_bar = a dt delta_bar + pend,
// src_g_bar = g dt delta_bar, pend = b dt delta_bar.
// A block owns kAdjXLines consecutive lines (j, k) of one field (blockIdx.y),
// one per thread, the recurrences carried in registers; the lines (rows of
// the compact arrays, contiguous) pass through two shared tiles kAdjXChunk
// points at a time: cp.async brings chunk c + 1 (runs of consecutive points)
// while chunk c is swept.  The forward sweep parks z in z_f (FP64: src_g_bar
// itself when S is double, a scratch array otherwise), which the backward
// sweep reads.
template <class S>
__global__ void __launch_bounds__(kAdjXLines) k3_adj_xsolve(
    const double *__restrict__ aux, const double *__restrict__ auy, const double *__restrict__ auz,
    const double *__restrict__ coef, S *__restrict__ sa_x, S *__restrict__ sg_x, S *__restrict__ sa_y,
    S *__restrict__ sg_y, S *__restrict__ sa_z, S *__restrict__ sg_z, S *__restrict__ pend_x,
    S *__restrict__ pend_y, S *__restrict__ pend_z, double *__restrict__ z_x, double *__restrict__ z_y,
    double *__restrict__ z_z, double adt, double bdt, double gdt, Grid3 g) {
  extern __shared__ double smx[];
  constexpr int NL = kAdjXLines, XC = kAdjXChunk, LD = kAdjXChunk + 1, PER = NL * XC / kAdjXLines;
  const int nx = g.nx;
  const int f = blockIdx.y;  // 0 ux, 1 uy, 2 uz
  const int n = (0 == f) ? nx - 1 : nx;
  const double *src = (0 == f) ? aux : (1 == f ? auy : auz);
  S *sa = (0 == f) ? sa_x : (1 == f ? sa_y : sa_z);
  S *sg = (0 == f) ? sg_x : (1 == f ? sg_y : sg_z);
  S *pend = (0 == f) ? pend_x : (1 == f ? pend_y : pend_z);
  double *zp = (0 == f) ? z_x : (1 == f ? z_y : z_z);  // the forward sweep's values
  const int set = (0 == f) ? 0 : 1;
  double *sL = smx, *sR = smx + nx, *sV = smx + 2 * nx;
  double *tiles = smx + 3 * nx;  // [2][NL][LD]
  for (int w = threadIdx.x; w < 3 * nx; w += NL) smx[w] = coef[(size_t)3 * set * nx + w];
  const long nlines = (long)g.ny * g.nz;
  const long l0 = (long)blockIdx.x * NL;
  const int nr = (int)min((long)NL, nlines - l0);
  const int t = threadIdx.x;
  const size_t base = (size_t)l0 * n;  // row l at base + (l - l0) n
  const int nch = (n + XC - 1) / XC;
  // element m of a thread's share of a chunk: row w / XC, point w % XC
  auto fetch = [&](const double *from, int c, int buf) {
    const int c0 = c * XC, cw = min(XC, n - c0);
    double *tl = tiles + (size_t)buf * NL * LD;
#pragma unroll
    for (int m = 0; m < PER; m++) {
      const int w = t + NL * m, r = w / XC, q = w - r * XC;
      if (r < nr && q < cw) __pipeline_memcpy_async(tl + r * LD + q, from + base + (size_t)r * n + c0 + q, 8);
    }
    __pipeline_commit();
  };
  // forward sweep
  double z = 0.;
  fetch(src, 0, 0);
  __syncthreads();  // (the coefficients)
  for (int c = 0; c < nch; c++) {
    const int c0 = c * XC, cw = min(XC, n - c0), buf = c & 1;
    double *tl = tiles + (size_t)buf * NL * LD;
    if (c + 1 < nch) {
      fetch(src, c + 1, buf ^ 1);
      __pipeline_wait_prior(1);
    } else {
      __pipeline_wait_prior(0);
    }
    __syncthreads();
    if (t < nr) {
      for (int q = 0; q < cw; q++) {
        const int p = c0 + q;
        const double b = tl[t * LD + q];
        z = (0 == p) ? b : b - sV[p - 1] * z;
        tl[t * LD + q] = z;
      }
    }
    __syncthreads();
#pragma unroll
    for (int m = 0; m < PER; m++) {
      const int w = t + NL * m, r = w / XC, q = w - r * XC;
      if (r < nr && q < cw) zp[base + (size_t)r * n + c0 + q] = tl[r * LD + q];
    }
    __syncthreads();  // the tile is refilled two chunks on
  }
  // the forward sweep's stores are read back by this block's copies
  __threadfence_block();
  __syncthreads();
  // backward sweep, chunks in reverse
  double y = 0.;
  const double rd0 = 1. / sR[0];
  fetch(zp, nch - 1, 0);
  for (int it = 0; it < nch; it++) {
    const int c = nch - 1 - it, c0 = c * XC, cw = min(XC, n - c0), buf = it & 1;
    double *tl = tiles + (size_t)buf * NL * LD;
    if (c - 1 >= 0) {
      fetch(zp, c - 1, buf ^ 1);
      __pipeline_wait_prior(1);
    } else {
      __pipeline_wait_prior(0);
    }
    __syncthreads();
    if (t < nr) {
      for (int q = cw - 1; q >= 0; q--) {
        const int p = c0 + q;
        const double zz = tl[t * LD + q];
        if (p == n - 1) y = zz * sR[n - 1];
        else if (p > 0) y = sR[p] * (zz - sL[p + 1] * y);
        else y = (zz - sL[1] * y) * rd0;
        tl[t * LD + q] = y;
      }
    }
    __syncthreads();
    // the RK split: the pending terms' loads issued together, then the stores
    double pv[PER];
#pragma unroll
    for (int m = 0; m < PER; m++) {
      const int w = t + NL * m, r = w / XC, q = w - r * XC;
      pv[m] = (r < nr && q < cw) ? (double)pend[base + (size_t)r * n + c0 + q] : 0.;
    }
#pragma unroll
    for (int m = 0; m < PER; m++) {
      const int w = t + NL * m, r = w / XC, q = w - r * XC;
      if (r < nr && q < cw) {
        const size_t o = base + (size_t)r * n + c0 + q;
        const double d = tl[r * LD + q];
        sa[o] = S(adt * d + pv[m]);
        sg[o] = S(gdt * d);
        pend[o] = S(bdt * d);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// transposes of the momentum right-hand sides (rhs_all of the restatement):
// u_bar = u_bar* + (d src / d u)^T src_bar, p_bar += (d src_g / d p)^T
// src_g_bar, ifrc_bar = src_a_bar.  A self-advection term l a + c b + u e with
// l = h (a + b) / 2, u = -h (b + e) / 2, c = -l - u equals h (a^2 - e^2) / 2:
// derivatives h a, 0, -h e; a cross term h [ul (a - b) - uu (e - b)] has
// derivatives h ul, h (uu - ul), -h uu in (a, b, e) and h (a - b), -h (e - b)
// in its advecting velocities ul, uu.  One thread per cell (i, j, k) writes
// ux face i (i >= 2), uy, uz and p of the cell, the three forces, and with
// the vof buoyancy extension on, vof_bar and the coefficient's adjoint.
// Neighbours are addressed by offsets (di, dj, dk) from the cell: compact
// arrays with periodic wraps (Wrap3), primal storage arrays through their
// halos.
// (64 registers and a 76-byte spill: four blocks of 256 threads per SM; the
// kernel is bound by memory latency, so resident warps set its speed: 2 %
// faster than three blocks without spill.  A z-marching form with the
// k -+ 1 planes of seven arrays in a cp.async shared-memory ring, two blocks
// per SM, was 19 % slower)
template <class S>
__global__ void __launch_bounds__(256, 4) k3_adj_rhs(Adj3RhsArgs<S> a) {
  int i, j, k;
  const AGrid3 &ag = a.ag;
  const Grid3 &g = ag.g;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx;
  const double rdy = ag.rdy, rdz = ag.rdz, nu = a.m_dif;
  const Wrap3 wc(j, k, g.ny, g.nz, nx), wf(j, k, g.ny, g.nz, nx - 1);
  const long oc = ix_src(g, i, j, k);
  const long of = ix_srcx(g, i, j, k);  // (face i; a face i + di at of + di)
  const long pu = ix_ux(g, i, j, k), pc = ix_cc(g, i, j, k);
  const long uj = nx + 1, uk = (long)(nx + 1) * (g.ny + 2), cj = nx + 2, ck = (long)(nx + 2) * (g.ny + 2);
  auto UX = [&](int di, int dj, int dk) { return a.ux[pu + di + dj * uj + dk * uk]; };
  auto V = [&](int di, int dj, int dk) { return a.uy[pc + di + dj * cj + dk * ck]; };
  auto W = [&](int di, int dj, int dk) { return a.uz[pc + di + dj * cj + dk * ck]; };
  auto SAX = [&](int di, int dj, int dk) { return (i + di >= 2 && i + di <= nx) ? a.sa_x[of + di + wf.at(dj, dk)] : 0.; };
  auto SGX = [&](int di, int dj, int dk) { return (i + di >= 2 && i + di <= nx) ? a.sg_x[of + di + wf.at(dj, dk)] : 0.; };
  auto SAY = [&](int di, int dj, int dk) { return (i + di >= 1 && i + di <= nx) ? a.sa_y[oc + di + wc.at(dj, dk)] : 0.; };
  auto SGY = [&](int di, int dj, int dk) { return (i + di >= 1 && i + di <= nx) ? a.sg_y[oc + di + wc.at(dj, dk)] : 0.; };
  auto SAZ = [&](int di, int dj, int dk) { return (i + di >= 1 && i + di <= nx) ? a.sa_z[oc + di + wc.at(dj, dk)] : 0.; };
  auto SGZ = [&](int di, int dj, int dk) { return (i + di >= 1 && i + di <= nx) ? a.sg_z[oc + di + wc.at(dj, dk)] : 0.; };
  const double rxf_i = ag.rxf[i - 1];
  const double rxf_m = (i >= 2) ? ag.rxf[i - 2] : 0., rxf_p = (i < nx) ? ag.rxf[i] : 0.;
  const double rxc_i = ag.rxc[i - 1], rxc_p = ag.rxc[i];
  // ---- ux face (i, j, k), i = 2..nx
  if (i >= 2) {
    double acc = a.aux[of];
    const double uxc = UX(0, 0, 0);
    // advection x of ux: (0.25 / dxc_f) (ux(f-1)^2 - ux(f+1)^2) at faces f = i -+ 1
    if (i + 1 <= nx) acc += 2. * (0.25 * rxc_p) * uxc * SAX(1, 0, 0);
    if (i - 1 >= 2) acc -= 2. * (0.25 * ag.rxc[i - 2]) * uxc * SAX(-1, 0, 0);
    const double w_xm = 0.5 * g.dxf[i - 2] * rxc_i;
    const double w_xp = 0.5 * g.dxf[i - 1] * rxc_i;
    {  // advection y of ux at rows j, j -+ 1, V(row) = w_xm uy(i-1, row) + w_xp uy(i, row)
      const double vj = w_xm * V(-1, 0, 0) + w_xp * V(0, 0, 0);
      const double vj1 = w_xm * V(-1, 1, 0) + w_xp * V(0, 1, 0);
      acc += (0.5 * rdy) * (vj1 * SAX(0, 1, 0) + (vj1 - vj) * SAX(0, 0, 0) - vj * SAX(0, -1, 0));
    }
    {  // advection z of ux
      const double wk = w_xm * W(-1, 0, 0) + w_xp * W(0, 0, 0);
      const double wk1 = w_xm * W(-1, 0, 1) + w_xp * W(0, 0, 1);
      acc += (0.5 * rdz) * (wk1 * SAX(0, 0, 1) + (wk1 - wk) * SAX(0, 0, 0) - wk * SAX(0, 0, -1));
    }
    // diffusion y, z (src_a) and x (src_g)
    acc += nu * (a.ly0 * SAX(0, 1, 0) + a.ly1 * SAX(0, 0, 0) + a.ly2 * SAX(0, -1, 0));
    acc += nu * (a.lz0 * SAX(0, 0, 1) + a.lz1 * SAX(0, 0, 0) + a.lz2 * SAX(0, 0, -1));
    {
      double d = a.lap_ux[3 * (i - 2) + 1] * SGX(0, 0, 0);
      if (i - 1 >= 2) d += a.lap_ux[3 * (i - 3) + 2] * SGX(-1, 0, 0);
      if (i + 1 <= nx) d += a.lap_ux[3 * (i - 1) + 0] * SGX(1, 0, 0);
      acc += nu * d;
    }
    // advection x of uy and of uz: ux(i, j, k) is half of U_l of cell i and of
    // U_u of cell i - 1 at rows j, j + 1 (uy) and planes k, k + 1 (uz)
    for (int s = 0; s < 2; s++) {
      const double du = V(-1, s, 0) - V(0, s, 0);
      acc += 0.25 * du * (SAY(0, s, 0) * rxf_i + SAY(-1, s, 0) * rxf_m);
      const double dw = W(-1, 0, s) - W(0, 0, s);
      acc += 0.25 * dw * (SAZ(0, 0, s) * rxf_i + SAZ(-1, 0, s) * rxf_m);
    }
    a.aux[of] = acc;
    a.aifx[of] = S(SAX(0, 0, 0));
  }
  const double dxf = g.dxf[i - 1];
  // ---- uy cell (i, j, k)
  {
    double acc = a.auy[oc];
    const double uyc = V(0, 0, 0);
    acc += 2. * (0.25 * rdy) * uyc * (SAY(0, 1, 0) - SAY(0, -1, 0));
    {  // advection x of uy (U of cells i, i -+ 1)
      const double ul = 0.5 * UX(0, -1, 0) + 0.5 * UX(0, 0, 0);
      const double uu = 0.5 * UX(1, -1, 0) + 0.5 * UX(1, 0, 0);
      acc += (0.5 * rxf_i) * (uu - ul) * SAY(0, 0, 0);
      if (i + 1 <= nx) acc += (0.5 * rxf_p) * uu * SAY(1, 0, 0);
      if (i - 1 >= 1) acc -= (0.5 * rxf_m) * ul * SAY(-1, 0, 0);
    }
    {  // advection z of uy (W(plane) = 0.5 uz(i, j-1, plane) + 0.5 uz(i, j, plane))
      const double wz = 0.5 * W(0, -1, 0) + 0.5 * W(0, 0, 0);
      const double wz1 = 0.5 * W(0, -1, 1) + 0.5 * W(0, 0, 1);
      acc += (0.5 * rdz) * (wz1 * SAY(0, 0, 1) + (wz1 - wz) * SAY(0, 0, 0) - wz * SAY(0, 0, -1));
    }
    // advection y of ux (V of faces i, i + 1 holds uy(i, j, k))
    for (int s = 0; s < 2; s++) {
      const int ip = i + s;
      if (ip < 2 || ip > nx) continue;
      const double w = 0.5 * dxf * ag.rxc[ip - 1];
      const double du = UX(s, -1, 0) - UX(s, 0, 0);
      acc += w * (0.5 * rdy) * du * (SAX(s, 0, 0) + SAX(s, -1, 0));
    }
    // advection y of uz (V(plane) = 0.5 uy(i, j, plane-1) + 0.5 uy(i, j, plane)
    // of uz cells (i, j, k), (i, j, k+1) and U_u of (i, j-1, .))
    for (int s = 0; s < 2; s++) {
      const double dw = W(0, -1, s) - W(0, 0, s);
      acc += (0.25 * rdy) * dw * (SAZ(0, 0, s) + SAZ(0, -1, s));
    }
    acc += nu * (a.ly0 * SAY(0, 1, 0) + a.ly1 * SAY(0, 0, 0) + a.ly2 * SAY(0, -1, 0));
    acc += nu * (a.lz0 * SAY(0, 0, 1) + a.lz1 * SAY(0, 0, 0) + a.lz2 * SAY(0, 0, -1));
    {
      double d = a.lap_cc[3 * (i - 1) + 1] * SGY(0, 0, 0);
      if (i - 1 >= 1) d += a.lap_cc[3 * (i - 2) + 2] * SGY(-1, 0, 0);
      if (i + 1 <= nx) d += a.lap_cc[3 * i + 0] * SGY(1, 0, 0);
      acc += nu * d;
    }
    a.auy[oc] = acc;
    a.aify[oc] = S(SAY(0, 0, 0));
    // the vof buoyancy grav (0.5 vof(j-1) + 0.5 vof(j) - vof_ref) of the uy
    // faces j and j + 1
    if (0. != a.grav_vof) {
      const long v0 = ix_vof(g, i, j, k);
      const double face = 0.5 * a.vof_post[v0 - (nx + 2)] + 0.5 * a.vof_post[v0] - a.vof_ref;
      a.agrv[oc] += SAY(0, 0, 0) * face;
      a.avof[oc] += a.grav_vof * 0.5 * (SAY(0, 0, 0) + SAY(0, 1, 0));
    }
  }
  // ---- uz cell (i, j, k)
  {
    double acc = a.auz[oc];
    const double uzc = W(0, 0, 0);
    acc += 2. * (0.25 * rdz) * uzc * (SAZ(0, 0, 1) - SAZ(0, 0, -1));
    {  // advection x of uz
      const double ul = 0.5 * UX(0, 0, -1) + 0.5 * UX(0, 0, 0);
      const double uu = 0.5 * UX(1, 0, -1) + 0.5 * UX(1, 0, 0);
      acc += (0.5 * rxf_i) * (uu - ul) * SAZ(0, 0, 0);
      if (i + 1 <= nx) acc += (0.5 * rxf_p) * uu * SAZ(1, 0, 0);
      if (i - 1 >= 1) acc -= (0.5 * rxf_m) * ul * SAZ(-1, 0, 0);
    }
    {  // advection y of uz (V(row) = 0.5 uy(i, row, k-1) + 0.5 uy(i, row, k))
      const double vy = 0.5 * V(0, 0, -1) + 0.5 * V(0, 0, 0);
      const double vy1 = 0.5 * V(0, 1, -1) + 0.5 * V(0, 1, 0);
      acc += (0.5 * rdy) * (vy1 * SAZ(0, 1, 0) + (vy1 - vy) * SAZ(0, 0, 0) - vy * SAZ(0, -1, 0));
    }
    // advection z of ux (W of faces i, i + 1 holds uz(i, j, k))
    for (int s = 0; s < 2; s++) {
      const int ip = i + s;
      if (ip < 2 || ip > nx) continue;
      const double w = 0.5 * dxf * ag.rxc[ip - 1];
      const double du = UX(s, 0, -1) - UX(s, 0, 0);
      acc += w * (0.5 * rdz) * du * (SAX(s, 0, 0) + SAX(s, 0, -1));
    }
    // advection z of uy (W(row) = 0.5 uz(i, row-1, k) + 0.5 uz(i, row, k) of
    // uy cells (i, j, k), (i, j+1, k) and U_u of (., ., k-1))
    for (int s = 0; s < 2; s++) {
      const double dv = V(0, s, -1) - V(0, s, 0);
      acc += (0.25 * rdz) * dv * (SAY(0, s, 0) + SAY(0, s, -1));
    }
    acc += nu * (a.ly0 * SAZ(0, 1, 0) + a.ly1 * SAZ(0, 0, 0) + a.ly2 * SAZ(0, -1, 0));
    acc += nu * (a.lz0 * SAZ(0, 0, 1) + a.lz1 * SAZ(0, 0, 0) + a.lz2 * SAZ(0, 0, -1));
    {
      double d = a.lap_cc[3 * (i - 1) + 1] * SGZ(0, 0, 0);
      if (i - 1 >= 1) d += a.lap_cc[3 * (i - 2) + 2] * SGZ(-1, 0, 0);
      if (i + 1 <= nx) d += a.lap_cc[3 * i + 0] * SGZ(1, 0, 0);
      acc += nu * d;
    }
    a.auz[oc] = acc;
    a.aifz[oc] = S(SAZ(0, 0, 0));
  }
  // ---- pressure gradients of the three src_g
  double pb = (SGY(0, 1, 0) - SGY(0, 0, 0)) * rdy + (SGZ(0, 0, 1) - SGZ(0, 0, 0)) * rdz;
  if (i >= 2) pb -= SGX(0, 0, 0) * rxc_i;
  if (i + 1 <= nx) pb += SGX(1, 0, 0) * rxc_p;
  a.ap[oc] += pb;
}

// ---------------------------------------------------------------------------
// k3_adj_interface: one thread per cell c = (i, j, k).
//  mode & 1 (update_vof): src_bar = a dt vof_bar' + pend; the face fluxes'
//    adjoints f_bar = div^T src_bar; u_bar of the faces c owns (x face i,
//    y face j, z face k) += (indicator sum or upwind vof) f_bar; for the
//    faces where c is upwind, vof_bar(c) += vel f_bar (single phase) or the
//    normal's adjoint n_bar(c) += vel f_bar sum_g w_g H'(z_g) (x_g, 1);
//    pend = b dt vof_bar' for the previous substep.
//  mode & 2 (force): vof_bar, kappa_bar and the tension's adjoint of the six
//    CSF faces of c.
//  mode & 4 (normal): the intercept (implicit function theorem over the
//    2 x 2 x 2 Gauss points) and the cell normal's normalisation: n_bar ->
//    vof_bar(c) and the adjoint m_bar of the unnormalised mean normal.
// With mode & 1 but not & 4, n_bar goes to anrm; with & 4 but not & 1 it is
// read from there.
// (64 registers, no spill: four blocks of 256 threads per SM)
template <class S>
__global__ void __launch_bounds__(256, 4) k3_adj_interface(Adj3IfaceArgs<S> a) {
  int i, j, k;
  const AGrid3 &ag = a.ag;
  const Grid3 &g = ag.g;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double rdy = ag.rdy, rdz = ag.rdz;
  const Wrap3 wc(j, k, ny, nz, nx);
  const long oc = ix_src(g, i, j, k);
  const double vofc = a.vof[ix_vof(g, i, j, k)];
  const bool inter = interfacial3(vofc);
  double vacc = a.avof_in[oc];
  double nb[4] = {0., 0., 0., 0.};
  if (a.mode & 1) {
    auto SRC = [&](int di, int dj, int dk) {  // src_bar of a neighbour, 0 outside x
      if (i + di < 1 || i + di > nx) return 0.;
      const long q = oc + di + wc.at(dj, dk);
      return a.adt * a.avof_in[q] + a.pend_in[q];
    };
    const double sc = SRC(0, 0, 0);
    const double fx_i = (i >= 2) ? sc * ag.rxf[i - 1] - SRC(-1, 0, 0) * ag.rxf[i - 2] : 0.;
    const double fx_ip = (i + 1 <= nx) ? SRC(1, 0, 0) * ag.rxf[i] - sc * ag.rxf[i - 1] : 0.;
    const double fy_j = (sc - SRC(0, -1, 0)) * rdy, fy_jp = (SRC(0, 1, 0) - sc) * rdy;
    const double fz_k = (sc - SRC(0, 0, -1)) * rdz, fz_kp = (SRC(0, 0, 1) - sc) * rdz;
    a.pend_out[oc] = a.bdt * a.avof_in[oc];
    // the indicator sum of a face whose upwind cell (ii, jj, kk) is interfacial,
    // or its vof; axis 0 / 1 / 2 and the face coordinate xf
    auto phi_of = [&](int ii, int jj, int kk, int axis, double xf) {
      const double lvof = a.vof[ix_vof(g, ii, jj, kk)];
      if (!interfacial3(lvof)) return lvof;
      const double *n = a.normal + ix_nrm(g, ii, wrap(jj, ny), wrap(kk, nz));
      double phi = 0.;
      for (int q1 = 0; q1 < 2; q1++)
        for (int q0 = 0; q0 < 2; q0++) {
          const double pa = a3_gauss_p[q0], pb = a3_gauss_p[q1];
          const double x0 = (0 == axis) ? xf : pa, x1 = (1 == axis) ? xf : (0 == axis ? pa : pb);
          const double x2 = (2 == axis) ? xf : pb;
          double h, hp;
          thinc_hh3(n[0] * x0 + n[1] * x1 + n[2] * x2 + n[3], h, hp);
          phi += a3_gauss_w[q0] * a3_gauss_w[q1] * h;
        }
      return phi;
    };
    // the faces c owns
    if (i >= 2) {
      const double vel = a.ux[ix_ux(g, i, j, k)];
      const bool neg = vel < 0.;
      a.aux[ix_srcx(g, i, j, k)] += phi_of(neg ? i : i - 1, j, k, 0, neg ? -0.5 : +0.5) * fx_i;
    }
    {
      const double vel = a.uy[ix_cc(g, i, j, k)];
      const bool neg = vel < 0.;
      a.auy[oc] += phi_of(i, neg ? j : j - 1, k, 1, neg ? -0.5 : +0.5) * fy_j;
    }
    {
      const double vel = a.uz[ix_cc(g, i, j, k)];
      const bool neg = vel < 0.;
      a.auz[oc] += phi_of(i, j, neg ? k : k - 1, 2, neg ? -0.5 : +0.5) * fz_k;
    }
    // the faces where c is upwind
    const double *nc = a.normal + ix_nrm(g, i, j, k);
    auto upwind = [&](double vel, double fb, int axis, double xf) {
      if (!inter) {
        vacc += vel * fb;
        return;
      }
      for (int q1 = 0; q1 < 2; q1++)
        for (int q0 = 0; q0 < 2; q0++) {
          const double pa = a3_gauss_p[q0], pb = a3_gauss_p[q1];
          const double x0 = (0 == axis) ? xf : pa, x1 = (1 == axis) ? xf : (0 == axis ? pa : pb);
          const double x2 = (2 == axis) ? xf : pb;
          double h, hp;
          thinc_hh3(nc[0] * x0 + nc[1] * x1 + nc[2] * x2 + nc[3], h, hp);
          const double c = vel * fb * a3_gauss_w[q0] * a3_gauss_w[q1] * hp;
          nb[0] += c * x0;
          nb[1] += c * x1;
          nb[2] += c * x2;
          nb[3] += c;
        }
    };
    if (i >= 2) {
      const double vel = a.ux[ix_ux(g, i, j, k)];
      if (vel < 0.) upwind(vel, fx_i, 0, -0.5);
    }
    if (i + 1 <= nx) {
      const double vel = a.ux[ix_ux(g, i + 1, j, k)];
      if (!(vel < 0.)) upwind(vel, fx_ip, 0, +0.5);
    }
    {
      const double vel = a.uy[ix_cc(g, i, j, k)];
      if (vel < 0.) upwind(vel, fy_j, 1, -0.5);
    }
    {
      const double vel = a.uy[ix_cc(g, i, j + 1, k)];
      if (!(vel < 0.)) upwind(vel, fy_jp, 1, +0.5);
    }
    {
      const double vel = a.uz[ix_cc(g, i, j, k)];
      if (vel < 0.) upwind(vel, fz_k, 2, -0.5);
    }
    {
      const double vel = a.uz[ix_cc(g, i, j, k + 1)];
      if (!(vel < 0.)) upwind(vel, fz_kp, 2, +0.5);
    }
    if (!(a.mode & 4))
      for (int m = 0; m < 4; m++) a.anrm[4 * oc + m] = S(nb[m]);
  }
  if (a.mode & 2) {
    const double sig = a.tension;
    const double *curv = a.curv, *vof = a.vof;
    double kb = 0., sb = 0.;
    // x faces f = i (c on the right) and f = i + 1 (c on the left), 2..nx
    for (int s = 0; s < 2; s++) {
      const int f = i + s;
      if (f < 2 || f > nx) continue;
      const double ib = a.aifx[ix_srcx(g, f, j, k)];
      const double rx = ag.rxc[f - 1];
      const double grad = rx * (-vof[ix_vof(g, f - 1, j, k)] + vof[ix_vof(g, f, j, k)]);
      const double kap = 0.5 * (+curv[ix_cc(g, f - 1, j, k)] + curv[ix_cc(g, f, j, k)]);
      vacc += (0 == s ? 1. : -1.) * sig * kap * rx * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    // y faces j (c above) and j + 1 (c below)
    for (int s = 0; s < 2; s++) {
      const int r = j + s;  // storage row of the face's upper cell
      const double ib = a.aify[oc + wc.at(s, 0)];
      const double grad = rdy * (-vof[ix_vof(g, i, r - 1, k)] + vof[ix_vof(g, i, r, k)]);
      const double kap = 0.5 * (+curv[ix_cc(g, i, wrap(r - 1, ny), k)] + curv[ix_cc(g, i, wrap(r, ny), k)]);
      vacc += (0 == s ? 1. : -1.) * sig * kap * rdy * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    // z faces k (c above) and k + 1 (c below)
    for (int s = 0; s < 2; s++) {
      const int r = k + s;
      const double ib = a.aifz[oc + wc.at(0, s)];
      const double grad = rdz * (-vof[ix_vof(g, i, j, r - 1)] + vof[ix_vof(g, i, j, r)]);
      const double kap = 0.5 * (+curv[ix_cc(g, i, j, wrap(r - 1, nz))] + curv[ix_cc(g, i, j, wrap(r, nz))]);
      vacc += (0 == s ? 1. : -1.) * sig * kap * rdz * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    a.akap[oc] = S(kb);
    a.asig[oc] += sb;
  }
  if (a.mode & 4) {
    if (!(a.mode & 1))
      for (int m = 0; m < 4; m++) nb[m] = a.anrm[4 * oc + m];
    double mb[3] = {0., 0., 0.};
    if (inter) {
      const double *nc = a.normal + ix_nrm(g, i, j, k);
      double fd = 0., f[3] = {0., 0., 0.};
      for (int q2 = 0; q2 < 2; q2++)
        for (int q1 = 0; q1 < 2; q1++)
          for (int q0 = 0; q0 < 2; q0++) {
            const double w = a3_gauss_w[q0] * a3_gauss_w[q1] * a3_gauss_w[q2];
            const double x[3] = {a3_gauss_p[q0], a3_gauss_p[q1], a3_gauss_p[q2]};
            double h, hp;
            thinc_hh3(nc[0] * x[0] + nc[1] * x[1] + nc[2] * x[2] + nc[3], h, hp);
            fd += w * hp;
            for (int m = 0; m < 3; m++) f[m] += w * hp * x[m];
          }
      // d = d(vof, n): dd = (dvof - f . dn) / fd
      const double r = nb[3] / fd;
      vacc += r;
      for (int m = 0; m < 3; m++) nb[m] -= f[m] * r;
      // n = m / max(|m|, eps), m = (sum of the eight corner normals) / (dxf, dy, dz)
      double mv[3] = {0., 0., 0.};
      for (int q = 0; q < 8; q++) {
        const int ic = i + (q & 1), jc = j + ((q >> 1) & 1), kc = k + (q >> 2);
        double gx, gy, gz;
        corner_grad3(a.vof, ag, ic, jc, kc, gx, gy, gz);
        const double norm = sqrt(+gx * gx + gy * gy + gz * gz);
        const double ninv = 1. / fmax(norm, kDblEpsilon);
        mv[0] += gx * ninv;
        mv[1] += gy * ninv;
        mv[2] += gz * ninv;
      }
      mv[0] *= ag.rxf[i - 1];
      mv[1] *= rdy;
      mv[2] *= rdz;
      unit_adj3(mv[0], mv[1], mv[2], nb[0], nb[1], nb[2], mb[0], mb[1], mb[2]);
    }
    for (int m = 0; m < 3; m++) a.am[3 * oc + m] = S(mb[m]);
  }
  a.avof_out[oc] = vacc;
}

// ---------------------------------------------------------------------------
// k3_adj_cgrad: one thread per corner (ic, jc, kc), ic in [1, nx + 1], jc in
// [1, ny], kc in [1, nz] (the periodic corners once each): the corner normal's
// adjoint from the eight cells around it, cell (ic-1+dp, jc-1+dq, kc-1+dr):
// m_bar / (dxf, dy, dz) of the cell's mean normal and -+ kappa_bar / (4 dxf,
// 4 dy, 4 dz) of its curvature (+ for the cell's left / lower corner), then
// the normalisation's transpose (zero at a corner flatter than the gradient
// floor tau); gbar[3 corner] = the corner gradient's adjoint, corner =
// (ic - 1) + (nx + 1) ((jc - 1) + ny (kc - 1)).
template <class S>
__global__ void k3_adj_cgrad(const double *__restrict__ vof, const S *__restrict__ am, const S *__restrict__ akap,
                             S *__restrict__ gbar, AGrid3 ag) {
  const Grid3 &g = ag.g;
  const int ic = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int jc = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int kc = 1 + blockIdx.z;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (ic > nx + 1 || jc > ny || kc > nz) return;
  double b[3] = {0., 0., 0.};
  for (int dr = 0; dr < 2; dr++)
    for (int dq = 0; dq < 2; dq++)
      for (int dp = 0; dp < 2; dp++) {
        const int p = ic - 1 + dp;
        if (p < 1 || p > nx) continue;
        const long o = ix_src(g, p, wrap(jc - 1 + dq, ny), wrap(kc - 1 + dr, nz));
        const double kap = 0.25 * akap[o];
        const double rxp = ag.rxf[p - 1];
        b[0] += (am[3 * o + 0] + (dp ? kap : -kap)) * rxp;
        b[1] += (am[3 * o + 1] + (dq ? kap : -kap)) * ag.rdy;
        b[2] += (am[3 * o + 2] + (dr ? kap : -kap)) * ag.rdz;
      }
  double gx, gy, gz;
  corner_grad3(vof, ag, ic, jc, kc, gx, gy, gz);
  double o0, o1, o2;
  unit_adj3(gx, gy, gz, b[0], b[1], b[2], o0, o1, o2);
  if (ag.tau > 0.) {
    // |g| h < tau with h = min(dxc, dy, dz): a flat corner, no derivative
    const double rmax = fmax(ag.rxc[ic - 1], fmax(ag.rdy, ag.rdz));
    if (sqrt(gx * gx + gy * gy + gz * gz) < ag.tau * rmax) o0 = o1 = o2 = 0.;
  }
  const long q = (long)(ic - 1) + (long)(nx + 1) * ((long)(jc - 1) + (long)ny * (kc - 1));
  gbar[3 * q + 0] = S(o0);
  gbar[3 * q + 1] = S(o1);
  gbar[3 * q + 2] = S(o2);
}

// k3_adj_cvof: one thread per cell: vof_bar += the corner gradients'
// transposes of its eight corners (ic in {i, i+1}, jc, kc wrapped): the cell is
// the corner's (ic-1+dp, jc-1+dq, kc-1+dr) cell, with coefficients
// -+1 / dxc(ic), -+1 / dy, -+1 / dz (+ for dp, dq, dr = 1)
template <class S>
__global__ void k3_adj_cvof(const S *__restrict__ gbar, double *__restrict__ avof, AGrid3 ag) {
  int i, j, k;
  const Grid3 &g = ag.g;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  double sx = 0., sy = 0., sz = 0.;
  for (int sr = 0; sr < 2; sr++)
    for (int sq = 0; sq < 2; sq++)
      for (int sp = 0; sp < 2; sp++) {
        const int ic = i + sp, jc = wrap(j + sq, ny), kc = wrap(k + sr, nz);
        const long q = (long)(ic - 1) + (long)(nx + 1) * ((long)(jc - 1) + (long)ny * (kc - 1));
        // the cell's place in the corner's stencil: dp = 1 - sp, dq = 1 - sq, dr = 1 - sr
        const double gxv = (double)gbar[3 * q + 0] * ag.rxc[ic - 1];
        const double gyv = gbar[3 * q + 1], gzv = gbar[3 * q + 2];
        sx += sp ? -gxv : gxv;
        sy += sq ? -gyv : gyv;
        sz += sr ? -gzv : gzv;
      }
  avof[ix_src(g, i, j, k)] += sx + sy * ag.rdy + sz * ag.rdz;
}

// deterministic sum of n values (one block of 256 threads)
__global__ void k3_adj_sum(const double *__restrict__ x, long n, double *__restrict__ out) {
  __shared__ double part[256];
  double s = 0.;
  for (long q = threadIdx.x; q < n; q += blockDim.x) s += x[q];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (0 == threadIdx.x) *out = part[0];
}

__global__ void k3_adj_set(double *dst, double v) { *dst = v; }

// ---- launchers (the kernels' instantiations stay in this translation unit)
template <class S>
cudaError_t adj3_xsolve_launch(cudaStream_t st, long lines, size_t smem, const double *aux, const double *auy,
                               const double *auz, const double *coef, S *sa_x, S *sg_x, S *sa_y, S *sg_y, S *sa_z,
                               S *sg_z, S *pend_x, S *pend_y, S *pend_z, double *z_x, double *z_y, double *z_z,
                               double adt, double bdt, double gdt, Grid3 g) {
  k3_adj_xsolve<S><<<dim3((unsigned)((lines + kAdjXLines - 1) / kAdjXLines), 3), kAdjXLines, smem, st>>>(
      aux, auy, auz, coef, sa_x, sg_x, sa_y, sg_y, sa_z, sg_z, pend_x, pend_y, pend_z, z_x, z_y, z_z, adt, bdt, gdt,
      g);
  return cudaGetLastError();
}

template <class S>
cudaError_t adj3_xsolve_prepare(size_t smem) {
  return cudaFuncSetAttribute(k3_adj_xsolve<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <class S>
cudaError_t adj3_rhs_launch(cudaStream_t st, const Adj3RhsArgs<S> &a) {
  const Grid3 &g = a.ag.g;
  k3_adj_rhs<S><<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz), dim3(32, 8), 0, st>>>(a);
  return cudaGetLastError();
}

template <class S>
cudaError_t adj3_interface_launch(cudaStream_t st, const Adj3IfaceArgs<S> &a) {
  const Grid3 &g = a.ag.g;
  k3_adj_interface<S><<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz), dim3(32, 8), 0, st>>>(a);
  return cudaGetLastError();
}

template <class S>
cudaError_t adj3_corners_launch(cudaStream_t st, const double *vof, const S *am, const S *akap, S *gbar,
                                double *avof, AGrid3 ag) {
  const Grid3 &g = ag.g;
  k3_adj_cgrad<S><<<dim3((g.nx + 1 + 31) / 32, (g.ny + 7) / 8, g.nz), dim3(32, 8), 0, st>>>(vof, am, akap, gbar,
                                                                                            ag);
  cudaError_t e = cudaGetLastError();
  if (cudaSuccess != e) return e;
  k3_adj_cvof<S><<<dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz), dim3(32, 8), 0, st>>>(gbar, avof, ag);
  return cudaGetLastError();
}

// the two storage types of the adjoint's intermediates
#define SVOF3_ADJ_INST(S)                                                                                         \
  template cudaError_t adj3_xsolve_launch<S>(cudaStream_t, long, size_t, const double *, const double *,           \
                                             const double *, const double *, S *, S *, S *, S *, S *, S *, S *, S *, \
                                             S *, double *, double *, double *, double, double, double, Grid3);     \
  template cudaError_t adj3_xsolve_prepare<S>(size_t);                                                           \
  template cudaError_t adj3_rhs_launch<S>(cudaStream_t, const Adj3RhsArgs<S> &);                                 \
  template cudaError_t adj3_interface_launch<S>(cudaStream_t, const Adj3IfaceArgs<S> &);                         \
  template cudaError_t adj3_corners_launch<S>(cudaStream_t, const double *, const S *, const S *, S *, double *,  \
                                              AGrid3);
SVOF3_ADJ_INST(double)
SVOF3_ADJ_INST(float)
#undef SVOF3_ADJ_INST

}  // namespace svof3
