// k_adjoint.cu -- adjoint kernels of one 2D time step (the differentiation
// form; no counterpart in the reference).
//
// Each kernel applies the transpose of the linearisation of one part of the
// step about the primal state at that part's input, in reverse order:
//
//   k_adj_project    fluid_update_pressure + fluid_correct_velocity
//                    (src/fluid/update_pressure.c:12-109,
//                    src/fluid/correct_velocity/{ux,uy}.c): psi_bar
//   (Poisson)        the potential's adjoint is a second Poisson solve of
//                    psi_bar / dxf with the forward kernels (L = D^-1 A with A
//                    symmetric and D = diag(dxf), so L^-T = D L^-1 D^-1)
//   k_adj_div        the divergence's transpose: psi's solve -> u_bar
//   k_adj_xsolve     the implicit-x systems transposed (src/fluid/predict/
//                    *.c, src/tdm.c:17-50), from the forward's LU table; the
//                    RK weights split delta_bar into src_a, src_b, src_g
//   k_adj_rhs        compute_rhs_ux / _uy transposed (advection, diffusion,
//                    pressure, surface force, vof buoyancy)
//   k_adj_interface  the THINC/QQ fluxes and RK update of vof
//                    (src/interface/update/*.c), the CSF force
//                    (src/interface/force.c:11-76) and the intercept and
//                    cell normal (src/interface/curvature_tensor.c:50-145)
//   k_adj_corners    the corner normals and the curvature
//                    (curvature_tensor.c:14-48, :147-176)
//
// Adjoint fields are compact: ux faces i = 2..nx ([j-1][i-2]), cells
// i = 1..nx ([j-1][i-1]); y is periodic, so an index j - 1 = 0 or j + 1 =
// ny + 1 wraps (a halo row holds a copy of an interior row, and every primal
// function reads the copy with the same arithmetic as the original).  Wall
// values are constants and carry no adjoint.  The primal fields are read in
// their storage layouts, halo rows included.  Branches follow the primal
// state (upwind side, interfacial test, eps clamps); the THINC intercept is
// differentiated through the implicit function theorem at the primal
// solution.  Every kernel gathers (each thread owns its outputs): no atomics,
// and the result does not depend on scheduling.
#include "adjoint_internal.cuh"

namespace svof {

namespace {

__constant__ double a_gauss_p[2] = {-0.2886751345948129, +0.2886751345948129};
__constant__ double a_gauss_w[2] = {+0.5, +0.5};
constexpr double kBeta = 1.;
constexpr double kVofMinA = 1.e-8;

__device__ __forceinline__ int wrapj(int j, int ny) { return j < 1 ? j + ny : (j > ny ? j - ny : j); }
__device__ __forceinline__ long axi(int nx, int i, int j) { return (long)(i - 2) + (long)(nx - 1) * (j - 1); }
__device__ __forceinline__ long aci(int nx, int i, int j) { return (long)(i - 1) + (long)nx * (j - 1); }

// H and H' of the THINC indicator 1 / (1 + exp(-2 beta z))
__device__ __forceinline__ void thinc_hh(double z, double &h, double &hp) {
  h = 1. / (1. + exp(-2. * kBeta * z));
  hp = 2. * kBeta * h * (1. - h);
}

__device__ __forceinline__ bool interfacial(double v) { return !(v < kVofMinA || 1. - kVofMinA < v); }

// corner normal (compute_gradient, curvature_tensor.c:14-48) at corner (ic, jc)
// from the storage-layout vof; g = the unnormalised gradient
__device__ __forceinline__ void corner_grad(const double *__restrict__ vof, const Grid2 &g, int ic, int jc,
                                            double &gx, double &gy) {
  const int nx = g.nx;
  const double dx = g.dxc[ic - 1];
  const double a = vof[ix_vof(nx, ic - 1, jc - 1)], b = vof[ix_vof(nx, ic, jc - 1)];
  const double c = vof[ix_vof(nx, ic - 1, jc)], d = vof[ix_vof(nx, ic, jc)];
  gx = 1. / dx * (-a + b - c + d);
  gy = 1. / g.dy * (-a - b + c + d);
}

// transpose of the derivative of g / max(|g|, eps) (a symmetric Jacobian)
__device__ __forceinline__ void unit_adj(double gx, double gy, double bx, double by, double &ox, double &oy) {
  const double norm = sqrt(gx * gx + gy * gy);
  if (norm > kDblEpsilon) {
    const double nx_ = gx / norm, ny_ = gy / norm;
    const double pr = nx_ * bx + ny_ * by;
    ox = (bx - nx_ * pr) / norm;
    oy = (by - ny_ * pr) / norm;
  } else {
    ox = bx / kDblEpsilon;
    oy = by / kDblEpsilon;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// k_adj_project: psi_bar += (d p' / d psi)^T p_bar' (mode & 1) and
// (d u' / d psi)^T u_bar' (mode & 2); one thread per cell.  u_bar and p_bar
// pass through unchanged (u' = u* - ..., p' = p + ...).
__global__ void k_adj_project(const double *__restrict__ aux, const double *__restrict__ auy,
                              const double *__restrict__ ap, double *__restrict__ apsi, double gdt, double pre,
                              int mode, Grid2 g) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j > ny) return;
  double acc = 0.;
  if (mode & 1) {
    // p'(i) = p(i) + psi(i) - c_i (dpsi_xp - dpsi_xm), c_i = pre / dxf_i,
    // Neumann ghosts (dpsi_xm = 0 at i = 1, dpsi_xp = 0 at i = nx)
    const double pb = ap[aci(nx, i, j)];
    const double ci = pre / g.dxf[i - 1];
    double diag = 0.;
    if (i > 1) diag += 1. / g.dxc[i - 1];
    if (i < nx) diag += 1. / g.dxc[i];
    acc += pb + pb * ci * diag;
    if (i > 1) acc -= ap[aci(nx, i - 1, j)] * (pre / g.dxf[i - 2]) / g.dxc[i - 1];
    if (i < nx) acc -= ap[aci(nx, i + 1, j)] * (pre / g.dxf[i]) / g.dxc[i];
  }
  if (mode & 2) {
    // ux'(i) = ux*(i) - gdt / dxc_i (psi(i) - psi(i-1)), i = 2..nx
    if (i >= 2) acc -= gdt / g.dxc[i - 1] * aux[axi(nx, i, j)];
    if (i + 1 <= nx) acc += gdt / g.dxc[i] * aux[axi(nx, i + 1, j)];
    // uy'(i, j) = uy*(i, j) - gdt / dy (psi(i, j) - psi(i, j-1))
    acc -= gdt / g.dy * auy[aci(nx, i, j)];
    acc += gdt / g.dy * auy[aci(nx, i, wrapj(j + 1, ny))];
  }
  apsi[aci(nx, i, j)] += acc;
}

// ---------------------------------------------------------------------------
// k_adj_div: the transpose of assign_input (dct.c:285-315, dft.c:315-345)
// applied to the adjoint solve's output s (psi storage layout): b_bar =
// dxf s, u_bar += pre_p div^T b_bar.  Also clears psi_bar (the forward
// overwrites psi).
__global__ void k_adj_div(double *__restrict__ aux, double *__restrict__ auy, const double *__restrict__ s,
                          double *__restrict__ apsi, double pre_p, Grid2 g) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j > ny) return;
  const double sc = s[ix_cc(nx, i, j)];
  if (i >= 2) aux[axi(nx, i, j)] += pre_p * (s[ix_cc(nx, i - 1, j)] - sc);
  auy[aci(nx, i, j)] += pre_p * (g.dxf[i - 1] / g.dy) * (s[ix_cc(nx, i, wrapj(j - 1, ny))] - sc);
  apsi[aci(nx, i, j)] = 0.;
}

// ---------------------------------------------------------------------------
// k_adj_xsolve: delta_bar = T^-T u_bar* for every x line of ux and uy, with
// T = L U the forward's factorisation (k_tdm_coef: L[i] = l_i, R[i] = 1 / d_i
// (R[0] = d_0), V[i] = v_i):  U^T z = b (z_i = b_i - v_{i-1} z_{i-1}), then
// L^T y = z (y_i = (z_i - l_{i+1} y_{i+1}) / d_i).  Then the RK weights:
// src_a_bar = a dt delta_bar + pend (the next substep's beta term), src_g_bar
// = g dt delta_bar, pend = b dt delta_bar (for the previous substep's src_a).
// A block owns R rows, staged in shared memory: [2][R][nx] line data.
__global__ void k_adj_xsolve(const double *__restrict__ aux, const double *__restrict__ auy,
                             const double *__restrict__ coef, double *__restrict__ sa_x, double *__restrict__ sg_x,
                             double *__restrict__ sa_y, double *__restrict__ sg_y, double *__restrict__ pend_x,
                             double *__restrict__ pend_y, double adt, double bdt, double gdt, int R, Grid2 g) {
  extern __shared__ double sm[];
  const int nx = g.nx, ny = g.ny;
  const int j0 = 1 + blockIdx.x * R;
  const int nrows = min(R, ny - j0 + 1);
  double *sx = sm;                   // [R][nx] ux lines (n = nx - 1)
  double *sy = sm + (size_t)R * nx;  // [R][nx] uy lines (n = nx)
  for (int w = threadIdx.x; w < nrows * nx; w += blockDim.x) {
    const int r = w / nx, k = w % nx;
    const int j = j0 + r;
    sx[r * nx + k] = (k < nx - 1) ? aux[axi(nx, k + 2, j)] : 0.;
    sy[r * nx + k] = auy[aci(nx, k + 1, j)];
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < 2 * nrows) {
    const int f = t / nrows, r = t % nrows;  // field 0: ux, 1: uy
    const int n = (0 == f) ? nx - 1 : nx;
    double *q = (0 == f ? sx : sy) + (size_t)r * nx;
    const double *L = coef + (size_t)(3 * f + 0) * nx;
    const double *Rv = coef + (size_t)(3 * f + 1) * nx;
    const double *V = coef + (size_t)(3 * f + 2) * nx;
    double z = q[0];
    for (int k = 1; k < n; k++) {
      z = q[k] - V[k - 1] * z;
      q[k] = z;
    }
    double y = q[n - 1] * Rv[n - 1];
    q[n - 1] = y;
    for (int k = n - 2; k >= 1; k--) {
      y = Rv[k] * (q[k] - L[k + 1] * y);
      q[k] = y;
    }
    if (n > 1) q[0] = (q[0] - L[1] * y) / Rv[0];
  }
  __syncthreads();
  for (int w = threadIdx.x; w < nrows * nx; w += blockDim.x) {
    const int r = w / nx, k = w % nx;
    const int j = j0 + r;
    if (k < nx - 1) {
      const long o = axi(nx, k + 2, j);
      const double d = sx[r * nx + k];
      sa_x[o] = adt * d + pend_x[o];
      sg_x[o] = gdt * d;
      pend_x[o] = bdt * d;
    }
    const long o = aci(nx, k + 1, j);
    const double d = sy[r * nx + k];
    sa_y[o] = adt * d + pend_y[o];
    sg_y[o] = gdt * d;
    pend_y[o] = bdt * d;
  }
}

// ---------------------------------------------------------------------------
// k_adj_rhs: transposes of compute_rhs_ux (ux.c:71-249) and compute_rhs_uy
// (uy.c:70-221): u_bar = u_bar* + (d src / d u)^T src_bar, p_bar +=
// (d src_g / d p)^T src_g_bar, ifrc_bar = src_a_bar, vof_bar += the vof
// buoyancy's transpose, grv_bar += its derivative in the coefficient.  The
// energy-consistent advection term l a + c b + u e with l = k (a + b),
// u = -k (b + e), c = -l - u equals k (a^2 - e^2): its derivatives are
// 2 k a, 0, -2 k e.  One thread per cell (i, j) writes ux face i (i >= 2),
// uy (i, j), p (i, j), vof (i, j), grv (i, j), the two forces.

__global__ void k_adj_rhs(AdjRhsArgs a) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const Grid2 g = a.g;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j > ny) return;
  const double dy = g.dy, nu = a.m_dif;
  const int jm = wrapj(j - 1, ny), jp = wrapj(j + 1, ny);
  const double *ux = a.ux, *uy = a.uy;
  auto SAX = [&](int ii, int jj) { return (ii >= 2 && ii <= nx) ? a.sa_x[axi(nx, ii, jj)] : 0.; };
  auto SGX = [&](int ii, int jj) { return (ii >= 2 && ii <= nx) ? a.sg_x[axi(nx, ii, jj)] : 0.; };
  auto SAY = [&](int ii, int jj) { return (ii >= 1 && ii <= nx) ? a.sa_y[aci(nx, ii, jj)] : 0.; };
  auto SGY = [&](int ii, int jj) { return (ii >= 1 && ii <= nx) ? a.sg_y[aci(nx, ii, jj)] : 0.; };
  // ---- ux face (i, j), i = 2..nx
  if (i >= 2) {
    const long o = axi(nx, i, j);
    double acc = a.aux[o];
    const double uxc = ux[ix_ux(nx, i, j)];
    // advection_x of ux: term(k) = k_k (ux(k-1)^2 - ux(k+1)^2), k_k = 0.25 / dxc_k
    if (i + 1 <= nx) acc += 2. * (0.25 / g.dxc[i]) * uxc * SAX(i + 1, j);
    if (i - 1 >= 2) acc -= 2. * (0.25 / g.dxc[i - 2]) * uxc * SAX(i - 1, j);
    // advection_y of ux at (i, j'): (0.5/dy) [V(j') a + (V(j'+1) - V(j')) b - V(j'+1) e],
    // V(j) = w_xm uy(i-1, j) + w_xp uy(i, j)
    {
      const double w_xm = 0.5 * g.dxf[i - 2] / g.dxc[i - 1];
      const double w_xp = 0.5 * g.dxf[i - 1] / g.dxc[i - 1];
      const double vj = w_xm * uy[ix_cc(nx, i - 1, j)] + w_xp * uy[ix_cc(nx, i, j)];
      const double vj1 = w_xm * uy[ix_cc(nx, i - 1, j + 1)] + w_xp * uy[ix_cc(nx, i, j + 1)];
      acc += (0.5 / dy) * (vj1 * SAX(i, jp) + (vj1 - vj) * SAX(i, j) - vj * SAX(i, jm));
    }
    // diffusion_y (src_a) and diffusion_x (src_g)
    acc += nu * (a.lapy0 * SAX(i, jp) + a.lapy1 * SAX(i, j) + a.lapy2 * SAX(i, jm));
    {
      double d = a.lap_ux[3 * (i - 2) + 1] * SGX(i, j);
      if (i - 1 >= 2) d += a.lap_ux[3 * (i - 3) + 2] * SGX(i - 1, j);
      if (i + 1 <= nx) d += a.lap_ux[3 * (i - 1) + 0] * SGX(i + 1, j);
      acc += nu * d;
    }
    // advection_x of uy: U_l(i, j') = 0.5 ux(i, j'-1) + 0.5 ux(i, j') of
    // cell i and U_u of cell i-1, both with derivative (0.5 / dxf) (uy(i-1, j') - uy(i, j'))
    for (int s = 0; s < 2; s++) {
      const int jq = (0 == s) ? j : j + 1;  // rows whose U holds ux(i, j)
      const int jw = wrapj(jq, ny);
      const double du = uy[ix_cc(nx, i - 1, jq)] - uy[ix_cc(nx, i, jq)];
      acc += 0.25 * du * (SAY(i, jw) / g.dxf[i - 1] + SAY(i - 1, jw) / g.dxf[i - 2]);
    }
    a.aux[o] = acc;
    a.aifx[o] = SAX(i, j);
  }
  // ---- uy cell (i, j)
  {
    const long o = aci(nx, i, j);
    double acc = a.auy[o];
    const double uyc = uy[ix_cc(nx, i, j)];
    // advection_y of uy: k (uy(j-1)^2 - uy(j+1)^2), k = 0.25 / dy
    acc += 2. * (0.25 / dy) * uyc * (SAY(i, jp) - SAY(i, jm));
    // advection_x of uy at (i', j): (0.5/dxf) [U_l a + (U_u - U_l) b - U_u e]
    {
      const double ul = 0.5 * ux[ix_ux(nx, i, j - 1)] + 0.5 * ux[ix_ux(nx, i, j)];
      const double uu = 0.5 * ux[ix_ux(nx, i + 1, j - 1)] + 0.5 * ux[ix_ux(nx, i + 1, j)];
      acc += (0.5 / g.dxf[i - 1]) * (uu - ul) * SAY(i, j);
      if (i + 1 <= nx) {
        const double ul1 = 0.5 * ux[ix_ux(nx, i + 1, j - 1)] + 0.5 * ux[ix_ux(nx, i + 1, j)];
        acc += (0.5 / g.dxf[i]) * ul1 * SAY(i + 1, j);
      }
      if (i - 1 >= 1) {
        const double uu1 = 0.5 * ux[ix_ux(nx, i, j - 1)] + 0.5 * ux[ix_ux(nx, i, j)];
        acc -= (0.5 / g.dxf[i - 2]) * uu1 * SAY(i - 1, j);
      }
    }
    // advection_y of ux: V(j) of faces i and i+1 holds uy(i, j); derivative
    // (0.5/dy)(ux(i', j-1) - ux(i', j)) times src_a_bar of (i', j) and (i', j-1)
    for (int s = 0; s < 2; s++) {
      const int ip = (0 == s) ? i : i + 1;
      if (ip < 2 || ip > nx) continue;
      const double w = (0 == s) ? 0.5 * g.dxf[i - 1] / g.dxc[ip - 1] : 0.5 * g.dxf[i - 1] / g.dxc[ip - 1];
      const double du = ux[ix_ux(nx, ip, j - 1)] - ux[ix_ux(nx, ip, j)];
      acc += w * (0.5 / dy) * du * (SAX(ip, j) + SAX(ip, jm));
    }
    acc += nu * (a.lapy0 * SAY(i, jp) + a.lapy1 * SAY(i, j) + a.lapy2 * SAY(i, jm));
    {
      double d = a.lap_uy[3 * (i - 1) + 1] * SGY(i, j);
      if (i - 1 >= 1) d += a.lap_uy[3 * (i - 2) + 2] * SGY(i - 1, j);
      if (i + 1 <= nx) d += a.lap_uy[3 * i + 0] * SGY(i + 1, j);
      acc += nu * d;
    }
    a.auy[o] = acc;
    a.aify[o] = SAY(i, j);
    // pressure gradients of src_g
    double pb = -SGY(i, j) / dy + SGY(i, jp) / dy;
    if (i >= 2) pb -= SGX(i, j) / g.dxc[i - 1];
    if (i + 1 <= nx) pb += SGX(i + 1, j) / g.dxc[i];
    a.ap[o] += pb;
    // vof buoyancy: grav_vof (0.5 vof(i, j-1) + 0.5 vof(i, j) - vof_ref) on uy (i, j);
    // its derivative in grav_vof is the bracket, for any grav_vof
    if (0. != a.grav_vof) a.avof[o] += a.grav_vof * 0.5 * (SAY(i, j) + SAY(i, jp));
    a.agrv[o] += SAY(i, j) * (0.5 * a.vof_post[ix_vof(nx, i, j - 1)] + 0.5 * a.vof_post[ix_vof(nx, i, j)] - a.vof_ref);
  }
}

// ---------------------------------------------------------------------------
// k_adj_interface: one thread per cell c = (i, j).
//  mode & 1 (update_vof): src_bar = a dt vof_bar' + pend; the face fluxes'
//    adjoints f_bar = div^T src_bar; u_bar of the faces c owns (x face i,
//    y face j) += (indicator sum or upwind vof) f_bar; for the faces where c
//    is upwind, vof_bar(c) += vel f_bar (single phase) or the normal's
//    adjoint n_bar(c) += vel f_bar sum_g w_g H'(z_g) (x_g, y_g, 1); pend =
//    b dt vof_bar' for the previous substep.
//  mode & 2 (force): vof_bar, kappa_bar and the tension's adjoint of the four
//    CSF faces of c.
//  mode & 4 (normal): the intercept (implicit function theorem) and the cell
//    normal's normalisation: n_bar -> vof_bar(c) and the adjoint m_bar of
//    the unnormalised mean corner normal.
// With mode & 1 but not & 4, n_bar goes to anrm; with & 4 but not & 1 it is
// read from there.

__global__ void k_adj_interface(AdjIfaceArgs a) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const Grid2 g = a.g;
  const int nx = g.nx, ny = g.ny;
  if (i > nx || j > ny) return;
  const double dy = g.dy;
  const int jm = wrapj(j - 1, ny), jp = wrapj(j + 1, ny);
  const long oc = aci(nx, i, j);
  const double vofc = a.vof[ix_vof(nx, i, j)];
  const bool inter = interfacial(vofc);
  double vacc = a.avof_in[oc];
  double nb0 = 0., nb1 = 0., nb2 = 0.;
  if (a.mode & 1) {
    auto SRC = [&](int ii, int jj) {  // src_bar of cell (ii, jj), 0 outside x
      if (ii < 1 || ii > nx) return 0.;
      const long q = aci(nx, ii, jj);
      return a.adt * a.avof_in[q] + a.pend_in[q];
    };
    const double sc = SRC(i, j);
    auto FX = [&](int k) { return SRC(k, j) / g.dxf[k - 1] - SRC(k - 1, j) / g.dxf[k - 2]; };  // face k, 2..nx
    const double fy_j = (sc - SRC(i, jm)) / dy;          // face j
    const double fy_jp = (SRC(i, jp) - sc) / dy;         // face j+1
    a.pend_out[oc] = a.bdt * a.avof_in[oc];
    // the faces c owns: x face i (i >= 2), y face j
    if (i >= 2) {
      const double vel = a.ux[ix_ux(nx, i, j)];
      const int ii = vel < 0. ? i : i - 1;
      const double x = vel < 0. ? -0.5 : +0.5;
      const double lvof = a.vof[ix_vof(nx, ii, j)];
      double phi;
      if (!interfacial(lvof)) {
        phi = lvof;
      } else {
        const double *n = a.normal + ix_nrm(nx, ii, j);
        phi = 0.;
        for (int q = 0; q < 2; q++) {
          double h, hp;
          thinc_hh(n[0] * x + n[1] * a_gauss_p[q] + n[2], h, hp);
          phi += a_gauss_w[q] * h;
        }
      }
      a.aux[axi(nx, i, j)] += phi * FX(i);
    }
    {
      const double vel = a.uy[ix_cc(nx, i, j)];
      const int jj = vel < 0. ? j : j - 1;
      const double y = vel < 0. ? -0.5 : +0.5;
      const double lvof = a.vof[ix_vof(nx, i, jj)];
      double phi;
      if (!interfacial(lvof)) {
        phi = lvof;
      } else {
        const double *n = a.normal + ix_nrm(nx, i, jj);
        phi = 0.;
        for (int q = 0; q < 2; q++) {
          double h, hp;
          thinc_hh(n[0] * a_gauss_p[q] + n[1] * y + n[2], h, hp);
          phi += a_gauss_w[q] * h;
        }
      }
      a.auy[oc] += phi * fy_j;
    }
    // the faces where c is upwind
    const double *nc = a.normal + ix_nrm(nx, i, j);
    auto upwind = [&](double vel, double fb, int xdir, double xf) {
      if (!inter) {
        vacc += vel * fb;
        return;
      }
      for (int q = 0; q < 2; q++) {
        const double x0 = xdir ? xf : a_gauss_p[q];
        const double x1 = xdir ? a_gauss_p[q] : xf;
        double h, hp;
        thinc_hh(nc[0] * x0 + nc[1] * x1 + nc[2], h, hp);
        const double c = vel * fb * a_gauss_w[q] * hp;
        nb0 += c * x0;
        nb1 += c * x1;
        nb2 += c;
      }
    };
    if (i >= 2) {
      const double vel = a.ux[ix_ux(nx, i, j)];
      if (vel < 0.) upwind(vel, FX(i), 1, -0.5);
    }
    if (i + 1 <= nx) {
      const double vel = a.ux[ix_ux(nx, i + 1, j)];
      if (!(vel < 0.)) upwind(vel, FX(i + 1), 1, +0.5);
    }
    {
      const double vel = a.uy[ix_cc(nx, i, j)];
      if (vel < 0.) upwind(vel, fy_j, 0, -0.5);
    }
    {
      const double vel = a.uy[ix_cc(nx, i, j + 1)];
      if (!(vel < 0.)) upwind(vel, fy_jp, 0, +0.5);
    }
    if (!(a.mode & 4)) {
      a.anrm[3 * oc + 0] = nb0;
      a.anrm[3 * oc + 1] = nb1;
      a.anrm[3 * oc + 2] = nb2;
    }
  }
  if (a.mode & 2) {
    const double sig = a.tension;
    const double *curv = a.curv, *vof = a.vof;
    double kb = 0., sb = 0.;
    // x faces k = i (c on the right) and k = i+1 (c on the left), 2..nx
    for (int s = 0; s < 2; s++) {
      const int k = i + s;
      if (k < 2 || k > nx) continue;
      const double ib = a.aifx[axi(nx, k, j)];
      const double dx = g.dxc[k - 1];
      const double grad = 1. / dx * (-vof[ix_vof(nx, k - 1, j)] + vof[ix_vof(nx, k, j)]);
      const double kap = 0.5 * (+curv[ix_cc(nx, k - 1, j)] + curv[ix_cc(nx, k, j)]);
      vacc += (0 == s ? 1. : -1.) * sig * kap / dx * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    // y faces j (c above) and j+1 (c below)
    for (int s = 0; s < 2; s++) {
      const int k = j + s;  // storage row of the face's upper cell
      const double ib = a.aify[aci(nx, i, 0 == s ? j : jp)];
      const double grad = 1. / dy * (-vof[ix_vof(nx, i, k - 1)] + vof[ix_vof(nx, i, k)]);
      const double kap = 0.5 * (+curv[ix_cc(nx, i, k - 1)] + curv[ix_cc(nx, i, k)]);
      vacc += (0 == s ? 1. : -1.) * sig * kap / dy * ib;
      kb += sig * grad * 0.5 * ib;
      if (0 == s) sb += grad * kap * ib;
    }
    a.akap[oc] = kb;
    a.asig[oc] += sb;
  }
  if (a.mode & 4) {
    if (!(a.mode & 1)) {
      nb0 = a.anrm[3 * oc + 0];
      nb1 = a.anrm[3 * oc + 1];
      nb2 = a.anrm[3 * oc + 2];
    }
    double mb0 = 0., mb1 = 0.;
    if (inter) {
      const double *nc = a.normal + ix_nrm(nx, i, j);
      double fd = 0., f0 = 0., f1 = 0.;
      for (int jj = 0; jj < 2; jj++) {
        for (int ii = 0; ii < 2; ii++) {
          const double w = a_gauss_w[ii] * a_gauss_w[jj];
          double h, hp;
          thinc_hh(nc[0] * a_gauss_p[ii] + nc[1] * a_gauss_p[jj] + nc[2], h, hp);
          fd += w * hp;
          f0 += w * hp * a_gauss_p[ii];
          f1 += w * hp * a_gauss_p[jj];
        }
      }
      // d = d(vof, n0, n1): dd = (dvof - f0 dn0 - f1 dn1) / fd
      const double r = nb2 / fd;
      vacc += r;
      nb0 -= f0 * r;
      nb1 -= f1 * r;
      // n = m / max(|m|, eps), m = (sum of the 4 corner normals / dxf, ... / dy)
      double mx = 0., my = 0.;
      for (int q = 0; q < 4; q++) {
        const int ic = i + (q & 1), jc = j + (q >> 1);
        double gx, gy;
        corner_grad(a.vof, g, ic, jc, gx, gy);
        const double norm = sqrt(gx * gx + gy * gy);
        const double ninv = 1. / fmax(norm, kDblEpsilon);
        mx += gx * ninv;
        my += gy * ninv;
      }
      mx /= g.dxf[i - 1];
      my /= dy;
      unit_adj(mx, my, nb0, nb1, mb0, mb1);
    }
    a.am[2 * oc + 0] = mb0;
    a.am[2 * oc + 1] = mb1;
  }
  a.avof_out[oc] = vacc;
}

// ---------------------------------------------------------------------------
// k_adj_corners: the corner normals' adjoints D_bar from the cells around
// each corner (m_bar / dxf, m_bar / dy of the mean normal; +-1 / (2 dxf),
// +-1 / (2 dy) of the curvature), through the normalisation's transpose to
// g_bar, and g_bar back to the four cells of each corner.  A block owns a
// CBX x CBY tile of cells; cells (tile + 1 ring) and corners in shared memory.
__global__ void __launch_bounds__(CBX * CBY) k_adj_corners(const double *__restrict__ vof,
                                                           const double *__restrict__ am,
                                                           const double *__restrict__ akap,
                                                           double *__restrict__ avof, Grid2 g) {
  __shared__ double s_m0[CBY + 2][CBX + 2], s_m1[CBY + 2][CBX + 2], s_k[CBY + 2][CBX + 2];
  __shared__ double s_gx[CBY + 1][CBX + 1], s_gy[CBY + 1][CBX + 1];
  const int nx = g.nx, ny = g.ny;
  const double dy = g.dy;
  const int i0 = 1 + blockIdx.x * CBX, j0 = 1 + blockIdx.y * CBY;
  const int tid = threadIdx.y * CBX + threadIdx.x;
  // cells [i0-1, i0+CBX] x [j0-1, j0+CBY] (x outside 1..nx: no cell)
  for (int t = tid; t < (CBX + 2) * (CBY + 2); t += CBX * CBY) {
    const int li = t % (CBX + 2), lj = t / (CBX + 2);
    const int ii = i0 - 1 + li, jj = wrapj(j0 - 1 + lj, ny);
    double m0 = 0., m1 = 0., k = 0.;
    if (ii >= 1 && ii <= nx && j0 - 1 + lj <= ny + 1) {
      const long o = aci(nx, ii, jj);
      m0 = am[2 * o];
      m1 = am[2 * o + 1];
      k = akap[o];
    }
    s_m0[lj][li] = m0;
    s_m1[lj][li] = m1;
    s_k[lj][li] = k;
  }
  __syncthreads();
  // corners (ic, jc) in [i0, i0+CBX] x [j0, j0+CBY]
  for (int t = tid; t < (CBX + 1) * (CBY + 1); t += CBX * CBY) {
    const int li = t % (CBX + 1), lj = t / (CBX + 1);
    const int ic = i0 + li, jc = j0 + lj;
    double bx = 0., by = 0.;
    if (ic <= nx + 1) {
      // cells around the corner: (ic-1, jc-1), (ic, jc-1), (ic-1, jc), (ic, jc);
      // s_*[lj + dq][li + dp] is cell (ic - 1 + dp, jc - 1 + dq)
      for (int dq = 0; dq < 2; dq++) {
        for (int dp = 0; dp < 2; dp++) {
          const int p = ic - 1 + dp;
          if (p < 1 || p > nx) continue;
          const double m0 = s_m0[lj + dq][li + dp], m1 = s_m1[lj + dq][li + dp], k = s_k[lj + dq][li + dp];
          const double dxp = g.dxf[p - 1];
          // corner on the cell's left (dp = 1) or right (dp = 0) side, bottom (dq = 1) or top (dq = 0)
          bx += m0 / dxp + (dp ? 1. : -1.) * k / (2. * dxp);
          by += m1 / dy + (dq ? 1. : -1.) * k / (2. * dy);
        }
      }
      double gx, gy;
      corner_grad(vof, g, ic, wrapj(jc, ny), gx, gy);
      double ox, oy;
      unit_adj(gx, gy, bx, by, ox, oy);
      bx = ox;
      by = oy;
    }
    s_gx[lj][li] = bx;
    s_gy[lj][li] = by;
  }
  __syncthreads();
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  if (i > nx || j > ny) return;
  const int li = threadIdx.x, lj = threadIdx.y;
  const double ixl = 1. / g.dxc[i - 1], ixr = 1. / g.dxc[i];
  // corner (i, j): c is its (ic, jc) cell; (i+1, j): (ic-1, jc); (i, j+1):
  // (ic, jc-1); (i+1, j+1): (ic-1, jc-1)
  double acc = s_gx[lj][li] * ixl + s_gy[lj][li] / dy;
  acc += -s_gx[lj][li + 1] * ixr + s_gy[lj][li + 1] / dy;
  acc += s_gx[lj + 1][li] * ixl - s_gy[lj + 1][li] / dy;
  acc += -s_gx[lj + 1][li + 1] * ixr - s_gy[lj + 1][li + 1] / dy;
  avof[aci(nx, i, j)] += acc;
}

// deterministic sum of n values (one block, fixed order of partial sums)
__global__ void k_adj_sum(const double *__restrict__ x, long n, double *__restrict__ out) {
  __shared__ double part[256];
  double s = 0.;
  for (long k = threadIdx.x; k < n; k += blockDim.x) s += x[k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (0 == threadIdx.x) *out = part[0];
}

__global__ void k_adj_set(double *dst, double v) { *dst = v; }

}  // namespace svof
