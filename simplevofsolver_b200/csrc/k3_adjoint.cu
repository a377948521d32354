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
// The temperature is not differentiated (the adjoint needs add_buoyancy = 0).
#include "adjoint3d_internal.cuh"

namespace svof3 {

namespace {

__constant__ double a3_gauss_p[2] = {-0.2886751345948129, +0.2886751345948129};
__constant__ double a3_gauss_w[2] = {+0.5, +0.5};
constexpr double kBeta3 = 1.;
constexpr double kVofMin3 = 1.e-8;

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
    const double nx_ = gx / norm, ny_ = gy / norm, nz_ = gz / norm;
    const double pr = nx_ * bx + ny_ * by + nz_ * bz;
    ox = (bx - nx_ * pr) / norm;
    oy = (by - ny_ * pr) / norm;
    oz = (bz - nz_ * pr) / norm;
  } else {
    ox = bx / kDblEpsilon;
    oy = by / kDblEpsilon;
    oz = bz / kDblEpsilon;
  }
}

// the unnormalised corner gradient of compute_gradient at corner (ic, jc, kc)
// (storage rows jc - 1, jc and planes kc - 1, kc)
__device__ __forceinline__ void corner_grad3(const double *__restrict__ vof, const Grid3 &g, int ic, int jc, int kc,
                                             double &gx, double &gy, double &gz) {
  double a[2][4];
  for (int q = 0; q < 2; q++) {
    const int kk = kc - 1 + q;
    a[q][0] = vof[ix_vof(g, ic - 1, jc - 1, kk)];
    a[q][1] = vof[ix_vof(g, ic, jc - 1, kk)];
    a[q][2] = vof[ix_vof(g, ic - 1, jc, kk)];
    a[q][3] = vof[ix_vof(g, ic, jc, kk)];
  }
  gx = 1. / g.dxc[ic - 1] * ((-a[0][0] + a[0][1] - a[0][2] + a[0][3]) + (-a[1][0] + a[1][1] - a[1][2] + a[1][3]));
  gy = 1. / g.dy * ((-a[0][0] - a[0][1] + a[0][2] + a[0][3]) + (-a[1][0] - a[1][1] + a[1][2] + a[1][3]));
  gz = 1. / g.dz * ((+a[1][0] + a[1][1] + a[1][2] + a[1][3]) - (+a[0][0] + a[0][1] + a[0][2] + a[0][3]));
}

__device__ __forceinline__ bool cell3(const Grid3 &g, int &i, int &j, int &k) {
  i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  k = 1 + blockIdx.z;
  return i <= g.nx && j <= g.ny && k <= g.nz;
}

}  // namespace

// ---------------------------------------------------------------------------
// psi_bar += (d p' / d psi)^T p_bar' (mode & 1), (d u' / d psi)^T u_bar'
// (mode & 2); u_bar and p_bar pass through (u' = u* - ..., p' = p + ...).
// update_pressure: p'(i) = p(i) + psi(i) - pre / dxf_i (-dm + dp) with the
// Neumann walls (dm = 0 at i = 1, dp = 0 at i = nx); correct: u' = u* - gdt
// grad psi, y and z periodic.
__global__ void k3_adj_project(const double *__restrict__ aux, const double *__restrict__ auy,
                               const double *__restrict__ auz, const double *__restrict__ ap,
                               double *__restrict__ apsi, double gdt, double pre, int mode, Grid3 g) {
  int i, j, k;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  double acc = 0.;
  if (mode & 1) {
    const double pb = ap[ix_src(g, i, j, k)];
    const double ci = pre / g.dxf[i - 1];
    double diag = 0.;
    if (i > 1) diag += 1. / g.dxc[i - 1];
    if (i < nx) diag += 1. / g.dxc[i];
    acc += pb + pb * ci * diag;
    if (i > 1) acc -= ap[ix_src(g, i - 1, j, k)] * (pre / g.dxf[i - 2]) / g.dxc[i - 1];
    if (i < nx) acc -= ap[ix_src(g, i + 1, j, k)] * (pre / g.dxf[i]) / g.dxc[i];
  }
  if (mode & 2) {
    if (i >= 2) acc -= gdt / g.dxc[i - 1] * aux[ix_srcx(g, i, j, k)];
    if (i + 1 <= nx) acc += gdt / g.dxc[i] * aux[ix_srcx(g, i + 1, j, k)];
    acc -= gdt / g.dy * auy[ix_src(g, i, j, k)];
    acc += gdt / g.dy * auy[ix_src(g, i, wrap(j + 1, ny), k)];
    acc -= gdt / g.dz * auz[ix_src(g, i, j, k)];
    acc += gdt / g.dz * auz[ix_src(g, i, j, wrap(k + 1, nz))];
  }
  apsi[ix_src(g, i, j, k)] += acc;
}

// b = psi_bar / dxf into the compact right-hand-side layout of the forward
// transforms (x fastest, nx ny per plane: the same as ix_src)
__global__ void k3_adj_scale(const double *__restrict__ apsi, double *__restrict__ b, Grid3 g) {
  int i, j, k;
  if (!cell3(g, i, j, k)) return;
  const long o = ix_src(g, i, j, k);
  b[o] = apsi[o] / g.dxf[i - 1];
}

// the transpose of the divergence right-hand side b = pre (dux/dxf + duy/dy +
// duz/dz) applied to the adjoint solve's output s (psi layout): b_bar =
// dxf s; also clears psi_bar (the forward overwrites psi)
__global__ void k3_adj_div(double *__restrict__ aux, double *__restrict__ auy, double *__restrict__ auz,
                           const double *__restrict__ s, double *__restrict__ apsi, double pre_p, Grid3 g) {
  int i, j, k;
  if (!cell3(g, i, j, k)) return;
  const int ny = g.ny, nz = g.nz;
  const double sc = s[ix_cc(g, i, j, k)];
  if (i >= 2) aux[ix_srcx(g, i, j, k)] += pre_p * (s[ix_cc(g, i - 1, j, k)] - sc);
  auy[ix_src(g, i, j, k)] += pre_p * (g.dxf[i - 1] / g.dy) * (s[ix_cc(g, i, wrap(j - 1, ny), k)] - sc);
  auz[ix_src(g, i, j, k)] += pre_p * (g.dxf[i - 1] / g.dz) * (s[ix_cc(g, i, j, wrap(k - 1, nz))] - sc);
  apsi[ix_src(g, i, j, k)] = 0.;
}

// ---------------------------------------------------------------------------
// delta_bar = T^-T u_bar* for every x line of ux, uy, uz, T = L U the
// forward's factorisation (k3_tdm_coef: per system s at coef + 3 s nx, L[i],
// R[i] = 1 / d_i (R[0] = d_0), V[i] = v_i; systems 0 ux, 1 uy and uz):
// U^T z = b (z_i = b_i - v_{i-1} z_{i-1}), then L^T y = z (y_i = (z_i -
// l_{i+1} y_{i+1}) / d_i).  Then the RK weights: src_a_bar = a dt delta_bar +
// pend, src_g_bar = g dt delta_bar, pend = b dt delta_bar.  A block owns R
// lines (j, k), staged in shared memory [3][R][nx].
__global__ void k3_adj_xsolve(const double *__restrict__ aux, const double *__restrict__ auy,
                              const double *__restrict__ auz, const double *__restrict__ coef,
                              double *__restrict__ sa_x, double *__restrict__ sg_x, double *__restrict__ sa_y,
                              double *__restrict__ sg_y, double *__restrict__ sa_z, double *__restrict__ sg_z,
                              double *__restrict__ pend_x, double *__restrict__ pend_y, double *__restrict__ pend_z,
                              double adt, double bdt, double gdt, int R, Grid3 g) {
  extern __shared__ double sm3[];
  const int nx = g.nx, ny = g.ny;
  const long nlines = (long)ny * g.nz;
  const long l0 = (long)blockIdx.x * R;
  const int nr = (int)min((long)R, nlines - l0);
  double *sq[3] = {sm3, sm3 + (size_t)R * nx, sm3 + 2 * (size_t)R * nx};
  const double *src[3] = {aux, auy, auz};
  for (int w = threadIdx.x; w < 3 * nr * nx; w += blockDim.x) {
    const int f = w / (nr * nx), rem = w - f * nr * nx, r = rem / nx, p = rem - r * nx;
    const long l = l0 + r;
    const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
    double v;
    if (0 == f) v = (p < nx - 1) ? src[0][ix_srcx(g, p + 2, j, k)] : 0.;
    else v = src[f][ix_src(g, p + 1, j, k)];
    sq[f][(size_t)r * nx + p] = v;
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < 3 * nr) {
    const int f = t / nr, r = t - f * nr;
    const int set = (0 == f) ? 0 : 1;
    const int n = (0 == f) ? nx - 1 : nx;
    double *q = sq[f] + (size_t)r * nx;
    const double *L = coef + (size_t)(3 * set + 0) * nx;
    const double *Rv = coef + (size_t)(3 * set + 1) * nx;
    const double *V = coef + (size_t)(3 * set + 2) * nx;
    double z = q[0];
    for (int p = 1; p < n; p++) {
      z = q[p] - V[p - 1] * z;
      q[p] = z;
    }
    double y = q[n - 1] * Rv[n - 1];
    q[n - 1] = y;
    for (int p = n - 2; p >= 1; p--) {
      y = Rv[p] * (q[p] - L[p + 1] * y);
      q[p] = y;
    }
    if (n > 1) q[0] = (q[0] - L[1] * y) / Rv[0];
  }
  __syncthreads();
  double *sa[3] = {sa_x, sa_y, sa_z}, *sg[3] = {sg_x, sg_y, sg_z}, *pd[3] = {pend_x, pend_y, pend_z};
  for (int w = threadIdx.x; w < 3 * nr * nx; w += blockDim.x) {
    const int f = w / (nr * nx), rem = w - f * nr * nx, r = rem / nx, p = rem - r * nx;
    if (0 == f && p >= nx - 1) continue;
    const long l = l0 + r;
    const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
    const long o = (0 == f) ? ix_srcx(g, p + 2, j, k) : ix_src(g, p + 1, j, k);
    const double d = sq[f][(size_t)r * nx + p];
    sa[f][o] = adt * d + pd[f][o];
    sg[f][o] = gdt * d;
    pd[f][o] = bdt * d;
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
// ux face i (i >= 2), uy, uz and p of the cell, and the three forces.

__global__ void k3_adj_rhs(Adj3RhsArgs a) {
  int i, j, k;
  const Grid3 g = a.g;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double dy = g.dy, dz = g.dz, nu = a.m_dif;
  const int jm = wrap(j - 1, ny), jp = wrap(j + 1, ny), km = wrap(k - 1, nz), kp = wrap(k + 1, nz);
  auto UX = [&](int ii, int jj, int kk) { return a.ux[ix_ux(g, ii, jj, kk)]; };
  auto V = [&](int ii, int jj, int kk) { return a.uy[ix_cc(g, ii, jj, kk)]; };
  auto W = [&](int ii, int jj, int kk) { return a.uz[ix_cc(g, ii, jj, kk)]; };
  // (jj, kk wrapped by the callers)
  auto SAX = [&](int ii, int jj, int kk) { return (ii >= 2 && ii <= nx) ? a.sa_x[ix_srcx(g, ii, jj, kk)] : 0.; };
  auto SGX = [&](int ii, int jj, int kk) { return (ii >= 2 && ii <= nx) ? a.sg_x[ix_srcx(g, ii, jj, kk)] : 0.; };
  auto SAY = [&](int ii, int jj, int kk) { return (ii >= 1 && ii <= nx) ? a.sa_y[ix_src(g, ii, jj, kk)] : 0.; };
  auto SGY = [&](int ii, int jj, int kk) { return (ii >= 1 && ii <= nx) ? a.sg_y[ix_src(g, ii, jj, kk)] : 0.; };
  auto SAZ = [&](int ii, int jj, int kk) { return (ii >= 1 && ii <= nx) ? a.sa_z[ix_src(g, ii, jj, kk)] : 0.; };
  auto SGZ = [&](int ii, int jj, int kk) { return (ii >= 1 && ii <= nx) ? a.sg_z[ix_src(g, ii, jj, kk)] : 0.; };
  const long oc = ix_src(g, i, j, k);
  // ---- ux face (i, j, k), i = 2..nx
  if (i >= 2) {
    const long o = ix_srcx(g, i, j, k);
    double acc = a.aux[o];
    const double uxc = UX(i, j, k);
    // advection x of ux: (0.25 / dxc_f) (ux(f-1)^2 - ux(f+1)^2) at faces f = i -+ 1
    if (i + 1 <= nx) acc += 2. * (0.25 / g.dxc[i]) * uxc * SAX(i + 1, j, k);
    if (i - 1 >= 2) acc -= 2. * (0.25 / g.dxc[i - 2]) * uxc * SAX(i - 1, j, k);
    const double w_xm = 0.5 * g.dxf[i - 2] / g.dxc[i - 1];
    const double w_xp = 0.5 * g.dxf[i - 1] / g.dxc[i - 1];
    {  // advection y of ux at rows j, j -+ 1, V(row) = w_xm uy(i-1, row) + w_xp uy(i, row)
      const double vj = w_xm * V(i - 1, j, k) + w_xp * V(i, j, k);
      const double vj1 = w_xm * V(i - 1, j + 1, k) + w_xp * V(i, j + 1, k);
      acc += (0.5 / dy) * (vj1 * SAX(i, jp, k) + (vj1 - vj) * SAX(i, j, k) - vj * SAX(i, jm, k));
    }
    {  // advection z of ux
      const double wk = w_xm * W(i - 1, j, k) + w_xp * W(i, j, k);
      const double wk1 = w_xm * W(i - 1, j, k + 1) + w_xp * W(i, j, k + 1);
      acc += (0.5 / dz) * (wk1 * SAX(i, j, kp) + (wk1 - wk) * SAX(i, j, k) - wk * SAX(i, j, km));
    }
    // diffusion y, z (src_a) and x (src_g)
    acc += nu * (a.ly0 * SAX(i, jp, k) + a.ly1 * SAX(i, j, k) + a.ly2 * SAX(i, jm, k));
    acc += nu * (a.lz0 * SAX(i, j, kp) + a.lz1 * SAX(i, j, k) + a.lz2 * SAX(i, j, km));
    {
      double d = a.lap_ux[3 * (i - 2) + 1] * SGX(i, j, k);
      if (i - 1 >= 2) d += a.lap_ux[3 * (i - 3) + 2] * SGX(i - 1, j, k);
      if (i + 1 <= nx) d += a.lap_ux[3 * (i - 1) + 0] * SGX(i + 1, j, k);
      acc += nu * d;
    }
    // advection x of uy and of uz: ux(i, j, k) is half of U_l of cell i and of
    // U_u of cell i - 1 at rows j, j + 1 (uy) and planes k, k + 1 (uz)
    for (int s = 0; s < 2; s++) {
      const int jq = j + s, jw = wrap(jq, ny);
      const double du = V(i - 1, jq, k) - V(i, jq, k);
      acc += 0.25 * du * (SAY(i, jw, k) / g.dxf[i - 1] + SAY(i - 1, jw, k) / g.dxf[i - 2]);
      const int kq = k + s, kw = wrap(kq, nz);
      const double dw = W(i - 1, j, kq) - W(i, j, kq);
      acc += 0.25 * dw * (SAZ(i, j, kw) / g.dxf[i - 1] + SAZ(i - 1, j, kw) / g.dxf[i - 2]);
    }
    a.aux[o] = acc;
    a.aifx[o] = SAX(i, j, k);
  }
  const double dxf = g.dxf[i - 1];
  // ---- uy cell (i, j, k)
  {
    double acc = a.auy[oc];
    const double uyc = V(i, j, k);
    acc += 2. * (0.25 / dy) * uyc * (SAY(i, jp, k) - SAY(i, jm, k));
    {  // advection x of uy (U of cells i, i -+ 1)
      const double ul = 0.5 * UX(i, j - 1, k) + 0.5 * UX(i, j, k);
      const double uu = 0.5 * UX(i + 1, j - 1, k) + 0.5 * UX(i + 1, j, k);
      acc += (0.5 / dxf) * (uu - ul) * SAY(i, j, k);
      if (i + 1 <= nx) acc += (0.5 / g.dxf[i]) * uu * SAY(i + 1, j, k);
      if (i - 1 >= 1) acc -= (0.5 / g.dxf[i - 2]) * ul * SAY(i - 1, j, k);
    }
    {  // advection z of uy (W(plane) = 0.5 uz(i, j-1, plane) + 0.5 uz(i, j, plane))
      const double wz = 0.5 * W(i, j - 1, k) + 0.5 * W(i, j, k);
      const double wz1 = 0.5 * W(i, j - 1, k + 1) + 0.5 * W(i, j, k + 1);
      acc += (0.5 / dz) * (wz1 * SAY(i, j, kp) + (wz1 - wz) * SAY(i, j, k) - wz * SAY(i, j, km));
    }
    // advection y of ux (V of faces i, i + 1 holds uy(i, j, k))
    for (int s = 0; s < 2; s++) {
      const int ip = i + s;
      if (ip < 2 || ip > nx) continue;
      const double w = 0.5 * dxf / g.dxc[ip - 1];
      const double du = UX(ip, j - 1, k) - UX(ip, j, k);
      acc += w * (0.5 / dy) * du * (SAX(ip, j, k) + SAX(ip, jm, k));
    }
    // advection y of uz (V(plane) = 0.5 uy(i, j, plane-1) + 0.5 uy(i, j, plane)
    // of uz cells (i, j, k), (i, j, k+1) and U_u of (i, j-1, .))
    for (int s = 0; s < 2; s++) {
      const int kq = k + s, kw = wrap(kq, nz);
      const double dw = W(i, j - 1, kq) - W(i, j, kq);
      acc += (0.25 / dy) * dw * (SAZ(i, j, kw) + SAZ(i, jm, kw));
    }
    acc += nu * (a.ly0 * SAY(i, jp, k) + a.ly1 * SAY(i, j, k) + a.ly2 * SAY(i, jm, k));
    acc += nu * (a.lz0 * SAY(i, j, kp) + a.lz1 * SAY(i, j, k) + a.lz2 * SAY(i, j, km));
    {
      double d = a.lap_cc[3 * (i - 1) + 1] * SGY(i, j, k);
      if (i - 1 >= 1) d += a.lap_cc[3 * (i - 2) + 2] * SGY(i - 1, j, k);
      if (i + 1 <= nx) d += a.lap_cc[3 * i + 0] * SGY(i + 1, j, k);
      acc += nu * d;
    }
    a.auy[oc] = acc;
    a.aify[oc] = SAY(i, j, k);
  }
  // ---- uz cell (i, j, k)
  {
    double acc = a.auz[oc];
    const double uzc = W(i, j, k);
    acc += 2. * (0.25 / dz) * uzc * (SAZ(i, j, kp) - SAZ(i, j, km));
    {  // advection x of uz
      const double ul = 0.5 * UX(i, j, k - 1) + 0.5 * UX(i, j, k);
      const double uu = 0.5 * UX(i + 1, j, k - 1) + 0.5 * UX(i + 1, j, k);
      acc += (0.5 / dxf) * (uu - ul) * SAZ(i, j, k);
      if (i + 1 <= nx) acc += (0.5 / g.dxf[i]) * uu * SAZ(i + 1, j, k);
      if (i - 1 >= 1) acc -= (0.5 / g.dxf[i - 2]) * ul * SAZ(i - 1, j, k);
    }
    {  // advection y of uz (V(row) = 0.5 uy(i, row, k-1) + 0.5 uy(i, row, k))
      const double vy = 0.5 * V(i, j, k - 1) + 0.5 * V(i, j, k);
      const double vy1 = 0.5 * V(i, j + 1, k - 1) + 0.5 * V(i, j + 1, k);
      acc += (0.5 / dy) * (vy1 * SAZ(i, jp, k) + (vy1 - vy) * SAZ(i, j, k) - vy * SAZ(i, jm, k));
    }
    // advection z of ux (W of faces i, i + 1 holds uz(i, j, k))
    for (int s = 0; s < 2; s++) {
      const int ip = i + s;
      if (ip < 2 || ip > nx) continue;
      const double w = 0.5 * dxf / g.dxc[ip - 1];
      const double du = UX(ip, j, k - 1) - UX(ip, j, k);
      acc += w * (0.5 / dz) * du * (SAX(ip, j, k) + SAX(ip, j, km));
    }
    // advection z of uy (W(row) = 0.5 uz(i, row-1, k) + 0.5 uz(i, row, k) of
    // uy cells (i, j, k), (i, j+1, k) and U_u of (., ., k-1))
    for (int s = 0; s < 2; s++) {
      const int jq = j + s, jw = wrap(jq, ny);
      const double dv = V(i, jq, k - 1) - V(i, jq, k);
      acc += (0.25 / dz) * dv * (SAY(i, jw, k) + SAY(i, jw, km));
    }
    acc += nu * (a.ly0 * SAZ(i, jp, k) + a.ly1 * SAZ(i, j, k) + a.ly2 * SAZ(i, jm, k));
    acc += nu * (a.lz0 * SAZ(i, j, kp) + a.lz1 * SAZ(i, j, k) + a.lz2 * SAZ(i, j, km));
    {
      double d = a.lap_cc[3 * (i - 1) + 1] * SGZ(i, j, k);
      if (i - 1 >= 1) d += a.lap_cc[3 * (i - 2) + 2] * SGZ(i - 1, j, k);
      if (i + 1 <= nx) d += a.lap_cc[3 * i + 0] * SGZ(i + 1, j, k);
      acc += nu * d;
    }
    a.auz[oc] = acc;
    a.aifz[oc] = SAZ(i, j, k);
  }
  // ---- pressure gradients of the three src_g
  double pb = -SGY(i, j, k) / dy + SGY(i, jp, k) / dy - SGZ(i, j, k) / dz + SGZ(i, j, kp) / dz;
  if (i >= 2) pb -= SGX(i, j, k) / g.dxc[i - 1];
  if (i + 1 <= nx) pb += SGX(i + 1, j, k) / g.dxc[i];
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

__global__ void k3_adj_interface(Adj3IfaceArgs a) {
  int i, j, k;
  const Grid3 g = a.g;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double dy = g.dy, dz = g.dz;
  const int jm = wrap(j - 1, ny), jp = wrap(j + 1, ny), km = wrap(k - 1, nz), kp = wrap(k + 1, nz);
  const long oc = ix_src(g, i, j, k);
  const double vofc = a.vof[ix_vof(g, i, j, k)];
  const bool inter = interfacial3(vofc);
  double vacc = a.avof_in[oc];
  double nb[4] = {0., 0., 0., 0.};
  if (a.mode & 1) {
    auto SRC = [&](int ii, int jj, int kk) {  // src_bar of cell (ii, jj, kk), 0 outside x
      if (ii < 1 || ii > nx) return 0.;
      const long q = ix_src(g, ii, jj, kk);
      return a.adt * a.avof_in[q] + a.pend_in[q];
    };
    const double sc = SRC(i, j, k);
    auto FX = [&](int f) { return SRC(f, j, k) / g.dxf[f - 1] - SRC(f - 1, j, k) / g.dxf[f - 2]; };
    const double fy_j = (sc - SRC(i, jm, k)) / dy, fy_jp = (SRC(i, jp, k) - sc) / dy;
    const double fz_k = (sc - SRC(i, j, km)) / dz, fz_kp = (SRC(i, j, kp) - sc) / dz;
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
      a.aux[ix_srcx(g, i, j, k)] += phi_of(neg ? i : i - 1, j, k, 0, neg ? -0.5 : +0.5) * FX(i);
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
      if (vel < 0.) upwind(vel, FX(i), 0, -0.5);
    }
    if (i + 1 <= nx) {
      const double vel = a.ux[ix_ux(g, i + 1, j, k)];
      if (!(vel < 0.)) upwind(vel, FX(i + 1), 0, +0.5);
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
      for (int m = 0; m < 4; m++) a.anrm[4 * oc + m] = nb[m];
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
      const double dx = g.dxc[f - 1];
      const double grad = 1. / dx * (-vof[ix_vof(g, f - 1, j, k)] + vof[ix_vof(g, f, j, k)]);
      const double kap = 0.5 * (+curv[ix_cc(g, f - 1, j, k)] + curv[ix_cc(g, f, j, k)]);
      vacc += (0 == s ? 1. : -1.) * sig * kap / dx * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    // y faces j (c above) and j + 1 (c below)
    for (int s = 0; s < 2; s++) {
      const int r = j + s;  // storage row of the face's upper cell
      const double ib = a.aify[ix_src(g, i, 0 == s ? j : jp, k)];
      const double grad = 1. / dy * (-vof[ix_vof(g, i, r - 1, k)] + vof[ix_vof(g, i, r, k)]);
      const double kap = 0.5 * (+curv[ix_cc(g, i, wrap(r - 1, ny), k)] + curv[ix_cc(g, i, wrap(r, ny), k)]);
      vacc += (0 == s ? 1. : -1.) * sig * kap / dy * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    // z faces k (c above) and k + 1 (c below)
    for (int s = 0; s < 2; s++) {
      const int r = k + s;
      const double ib = a.aifz[ix_src(g, i, j, 0 == s ? k : kp)];
      const double grad = 1. / dz * (-vof[ix_vof(g, i, j, r - 1)] + vof[ix_vof(g, i, j, r)]);
      const double kap = 0.5 * (+curv[ix_cc(g, i, j, wrap(r - 1, nz))] + curv[ix_cc(g, i, j, wrap(r, nz))]);
      vacc += (0 == s ? 1. : -1.) * sig * kap / dz * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    a.akap[oc] = kb;
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
        corner_grad3(a.vof, g, ic, jc, kc, gx, gy, gz);
        const double norm = sqrt(+gx * gx + gy * gy + gz * gz);
        const double ninv = 1. / fmax(norm, kDblEpsilon);
        mv[0] += gx * ninv;
        mv[1] += gy * ninv;
        mv[2] += gz * ninv;
      }
      mv[0] /= g.dxf[i - 1];
      mv[1] /= dy;
      mv[2] /= dz;
      unit_adj3(mv[0], mv[1], mv[2], nb[0], nb[1], nb[2], mb[0], mb[1], mb[2]);
    }
    for (int m = 0; m < 3; m++) a.am[3 * oc + m] = mb[m];
  }
  a.avof_out[oc] = vacc;
}

// ---------------------------------------------------------------------------
// k3_adj_cgrad: one thread per corner (ic, jc, kc), ic in [1, nx + 1], jc in
// [1, ny], kc in [1, nz] (the periodic corners once each): the corner normal's
// adjoint from the eight cells around it, cell (ic-1+dp, jc-1+dq, kc-1+dr):
// m_bar / (dxf, dy, dz) of the cell's mean normal and -+ kappa_bar / (4 dxf,
// 4 dy, 4 dz) of its curvature (+ for the cell's left / lower corner), then
// the normalisation's transpose; gbar[3 corner] = the corner gradient's
// adjoint, corner = (ic - 1) + (nx + 1) ((jc - 1) + ny (kc - 1)).
__global__ void k3_adj_cgrad(const double *__restrict__ vof, const double *__restrict__ am,
                             const double *__restrict__ akap, double *__restrict__ gbar, Grid3 g) {
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
        const double kap = akap[o];
        const double dxp = g.dxf[p - 1];
        b[0] += am[3 * o + 0] / dxp + (dp ? 1. : -1.) * kap * 0.25 / dxp;
        b[1] += am[3 * o + 1] / g.dy + (dq ? 1. : -1.) * kap * 0.25 / g.dy;
        b[2] += am[3 * o + 2] / g.dz + (dr ? 1. : -1.) * kap * 0.25 / g.dz;
      }
  double gx, gy, gz;
  corner_grad3(vof, g, ic, jc, kc, gx, gy, gz);
  double o0, o1, o2;
  unit_adj3(gx, gy, gz, b[0], b[1], b[2], o0, o1, o2);
  const long q = (long)(ic - 1) + (long)(nx + 1) * ((long)(jc - 1) + (long)ny * (kc - 1));
  gbar[3 * q + 0] = o0;
  gbar[3 * q + 1] = o1;
  gbar[3 * q + 2] = o2;
}

// k3_adj_cvof: one thread per cell: vof_bar += the corner gradients'
// transposes of its eight corners (ic in {i, i+1}, jc, kc wrapped): the cell is
// the corner's (ic-1+dp, jc-1+dq, kc-1+dr) cell, with coefficients
// -+1 / dxc(ic), -+1 / dy, -+1 / dz (+ for dp, dq, dr = 1)
__global__ void k3_adj_cvof(const double *__restrict__ gbar, double *__restrict__ avof, Grid3 g) {
  int i, j, k;
  if (!cell3(g, i, j, k)) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  double acc = 0.;
  for (int sr = 0; sr < 2; sr++)
    for (int sq = 0; sq < 2; sq++)
      for (int sp = 0; sp < 2; sp++) {
        const int ic = i + sp, jc = wrap(j + sq, ny), kc = wrap(k + sr, nz);
        const int dp = 1 - sp, dq = 1 - sq, dr = 1 - sr;  // the cell's place in the corner's stencil
        const long q = (long)(ic - 1) + (long)(nx + 1) * ((long)(jc - 1) + (long)ny * (kc - 1));
        acc += gbar[3 * q + 0] * (dp ? 1. : -1.) / g.dxc[ic - 1];
        acc += gbar[3 * q + 1] * (dq ? 1. : -1.) / g.dy;
        acc += gbar[3 * q + 2] * (dr ? 1. : -1.) / g.dz;
      }
  avof[ix_src(g, i, j, k)] += acc;
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

}  // namespace svof3
