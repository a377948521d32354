// k_interface.cu -- interface (VOF) kernels of the FP64 2D path.
//
//   k_halo_bc     periodic y halo + x wall values      src/halo.c:18-76,
//                                                      src/fluid/boundary/*.c,
//                                                      src/interface/boundary.c:7-39
//   k_geom        corner normals, cell normal and     src/interface/curvature_tensor.c:14-186
//                 THINC intercept, curvature
//   k_force       CSF surface tension force           src/interface/force.c:11-76
//   k_vof_advect  THINC/QQ fluxes, divergence, RK     src/interface/update/{flxx,flxy,main}.c
//                 update of vof, its halo and walls
//
// Each thread evaluates the reference's expressions with the reference's
// association; tiles stage their stencil inputs in shared memory.
#include "svof_internal.cuh"

namespace svof {

// THINC/QQ constants, src/interface/common.c:4-14 and src/interface/internal.h:4
__constant__ double c_gauss_p[2] = {-0.2886751345948129, +0.2886751345948129};
__constant__ double c_gauss_w[2] = {+0.5, +0.5};
constexpr double kVofBeta = 1.;
constexpr double kVofMin = 1.e-8;

// ---------------------------------------------------------------------------
// halo + wall update of one field; one thread per storage cell of the grid
// (columns x blockIdx.y = storage row).  Both halo exchanges copy whole rows,
// x ghost cells included, before the wall values are assigned (src/halo.c:
// 51-74 followed by assign_boundary_conditions_in_x): interior columns copy
// their halo rows from the source rows; a wall cell of a source row first
// hands its pre-assignment value to the halo row, then takes its wall value.
__global__ void k_halo_bc(double *a, int width, int nh, int ny, int kind, double lo, double hi) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;  // storage row, 0 .. ny + 2 nh - 1
  if (c >= width) return;
  const long w = width;
  const bool left = (0 == c), right = (width - 1 == c);
  if (!left && !right) {
    if (r < nh) a[w * r + c] = a[w * (ny + r) + c];
    else if (r >= ny + nh) a[w * r + c] = a[w * (r - ny) + c];
    return;
  }
  if (BC_VOF == kind) {
    a[w * r + c] = 0.;
    return;
  }
  if (r < nh || r >= ny + nh) return;
  const double old = a[w * r + c];
  if (r >= ny) a[w * (r - ny) + c] = old;
  if (r < 2 * nh) a[w * (r + ny) + c] = old;
  double v;
  if (BC_ZERO_UX == kind) {
    v = 0.;
  } else if (BC_DIRICHLET == kind) {
    v = left ? lo : hi;
  } else {
    v = left ? a[w * r + 1] : a[w * r + width - 2];
  }
  a[w * r + c] = v;
}

// ---------------------------------------------------------------------------
// k_geom: cells i in [1, nx], j in [0, ny+1]; tile BX x BY cells, the vof
// tile (BX+2) x (BY+2) and the (BX+1) x (BY+1) corner normals in shared memory.
constexpr int GBX = 32, GBY = 8;

// compute_intercept, src/interface/curvature_tensor.c:50-92
__device__ __forceinline__ double thinc_intercept(const double vof, const double n0, const double n1) {
  const int cntmax = 8;
  const double resmax = 1.e-12;
  double exps[4];
#pragma unroll
  for (int jj = 0; jj < 2; jj++) {
#pragma unroll
    for (int ii = 0; ii < 2; ii++) {
      exps[jj * 2 + ii] = exp(-2. * kVofBeta * (+n0 * c_gauss_p[ii] + n1 * c_gauss_p[jj]));
    }
  }
  double val = 1. / vof - 1.;
  for (int cnt = 0; cnt < cntmax; cnt++) {
    double f0 = -1. * vof;
    double f1 = 0.;
#pragma unroll
    for (int jj = 0; jj < 2; jj++) {
#pragma unroll
      for (int ii = 0; ii < 2; ii++) {
        const double weight = c_gauss_w[ii] * c_gauss_w[jj];
        const double p = exps[jj * 2 + ii];
        const double denom = 1. / (1. + p * val);
        f0 += weight * denom;
        f1 -= weight * p * denom * denom;
      }
    }
    val -= f0 / f1;
    if (fabs(f0) < resmax) break;
  }
  return -0.5 / kVofBeta * log(val);
}

__global__ void __launch_bounds__(GBX * GBY) k_geom(const double *__restrict__ vof, double *__restrict__ normal,
                                                   double *__restrict__ curv, Grid2 g) {
  pdl_enter();
  __shared__ double sv[GBY + 2][GBX + 2];
  __shared__ double sdx[GBY + 1][GBX + 1];
  __shared__ double sdy[GBY + 1][GBX + 1];
  const int nx = g.nx, ny = g.ny;
  const int i0 = 1 + blockIdx.x * GBX;  // first cell of the tile
  const int j0 = blockIdx.y * GBY;
  const int tid = threadIdx.y * GBX + threadIdx.x;
  // vof for i in [i0-1, i0+GBX], j in [j0-1, j0+GBY]
  for (int t = tid; t < (GBX + 2) * (GBY + 2); t += GBX * GBY) {
    const int li = t % (GBX + 2), lj = t / (GBX + 2);
    const int i = i0 - 1 + li, j = j0 - 1 + lj;
    sv[lj][li] = (i <= nx + 1 && j <= ny + 2) ? vof[ix_vof(nx, i, j)] : 0.;
  }
  __syncthreads();
  // compute_gradient (:14-48) for corners ic in [i0, i0+GBX], jc in [j0, j0+GBY]
  for (int t = tid; t < (GBX + 1) * (GBY + 1); t += GBX * GBY) {
    const int li = t % (GBX + 1), lj = t / (GBX + 1);
    const int ic = i0 + li, jc = j0 + lj;
    double ddx = 0., ddy = 0.;
    if (ic <= nx + 1 && jc <= ny + 2) {
      const double dx = g.dxc[ic - 1];
      const double v00 = sv[lj][li], v10 = sv[lj][li + 1];
      const double v01 = sv[lj + 1][li], v11 = sv[lj + 1][li + 1];
      const double dvofdx = 1. / dx * (-v00 + v10 - v01 + v11);
      const double dvofdy = 1. / g.dy * (-v00 - v10 + v01 + v11);
      const double norm = sqrt(+dvofdx * dvofdx + dvofdy * dvofdy);
      const double norminv = 1. / fmax(norm, kDblEpsilon);
      ddx = dvofdx * norminv;
      ddy = dvofdy * norminv;
    }
    sdx[lj][li] = ddx;
    sdy[lj][li] = ddy;
  }
  __syncthreads();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  if (i > nx || j > ny + 1) return;
  const double dx = g.dxf[i - 1];
  // compute_normal (:94-145)
  const double lvof = sv[ty + 1][tx + 1];
  if (!(lvof < kVofMin || 1. - kVofMin < lvof)) {
    double nxv = (+sdx[ty][tx] + sdx[ty][tx + 1] + sdx[ty + 1][tx] + sdx[ty + 1][tx + 1]);
    double nyv = (+sdy[ty][tx] + sdy[ty][tx + 1] + sdy[ty + 1][tx] + sdy[ty + 1][tx + 1]);
    nxv /= dx;
    nyv /= g.dy;
    const double norm = sqrt(+nxv * nxv + nyv * nyv);
    const double norminv = 1. / fmax(norm, kDblEpsilon);
    nxv *= norminv;
    nyv *= norminv;
    const double seg = thinc_intercept(lvof, nxv, nyv);
    double *n = normal + ix_nrm(nx, i, j);
    n[0] = nxv;
    n[1] = nyv;
    n[2] = seg;
  }
  // compute_curvature (:147-176)
  const double dnxdx = 1. / dx * (-sdx[ty][tx] + sdx[ty][tx + 1] - sdx[ty + 1][tx] + sdx[ty + 1][tx + 1]);
  const double dnydy = 1. / g.dy * (-sdy[ty][tx] - sdy[ty][tx + 1] + sdy[ty + 1][tx] + sdy[ty + 1][tx + 1]);
  curv[ix_cc(nx, i, j)] = 0.5 * (-dnxdx - dnydy);
}

// ---------------------------------------------------------------------------
// k_force: one thread per cell i in [1, nx], j in [1, ny]
__global__ void k_force(const double *__restrict__ vof, const double *__restrict__ curv,
                        double *__restrict__ ifrcx, double *__restrict__ ifrcy, double tension, Grid2 g) {
  pdl_enter();
  const int nx = g.nx, ny = g.ny;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  const double vc = vof[ix_vof(nx, i, j)];
  const double cc = curv[ix_cc(nx, i, j)];
  if (i >= 2) {
    // compute_force_x, :11-38
    const double dx = g.dxc[i - 1];
    const double grad = 1. / dx * (-vof[ix_vof(nx, i - 1, j)] + vc);
    const double kappa = 0.5 * (+curv[ix_cc(nx, i - 1, j)] + cc);
    ifrcx[ix_srcx(nx, i, j)] = tension * grad * kappa;
  }
  // compute_force_y, :40-66
  const double grad = 1. / g.dy * (-vof[ix_vof(nx, i, j - 1)] + vc);
  const double kappa = 0.5 * (+curv[ix_cc(nx, i, j - 1)] + cc);
  ifrcy[ix_src(nx, i, j)] = tension * grad * kappa;
}

// ---------------------------------------------------------------------------
// k_vof_advect: tile of ABX x ABY interior cells.  Face fluxes of the tile are
// evaluated once into shared memory, then each cell takes their divergence
// and advances vof.  Reads vof (old buffer), writes vof_new (rows 1..ny, the
// two halo rows on each side and the zero wall columns).

// indicator, src/interface/update/main.c:16-26
__device__ __forceinline__ double thinc_indicator(const double *n, const double x0, const double x1) {
  return 1. / (1. + exp(-2. * kVofBeta * (+n[0] * x0 + n[1] * x1 + n[2])));
}

constexpr int ABX = 32, ABY = 8;

__global__ void __launch_bounds__(ABX * ABY) k_vof_advect(
    const double *__restrict__ vof, double *__restrict__ vof_new, const double *__restrict__ ux,
    const double *__restrict__ uy, const double *__restrict__ normal, double *__restrict__ src_a,
    const double *__restrict__ src_b, const double *__restrict__ dtp, RK rk, int use_b, Grid2 g) {
  pdl_enter();
  __shared__ double fx[ABY][ABX + 1];  // faces i0 .. i0+ABX of rows j0 .. j0+ABY-1
  __shared__ double fy[ABY + 1][ABX];  // faces j0 .. j0+ABY of columns i0 .. i0+ABX-1
  const int nx = g.nx, ny = g.ny;
  const int i0 = 1 + blockIdx.x * ABX, j0 = 1 + blockIdx.y * ABY;
  const int tid = threadIdx.y * ABX + threadIdx.x;
  // compute_flux_x, src/interface/update/flxx.c:11-44; faces i in [2, nx]
  // carry fluxes, the wall faces i = 1 and i = nx+1 carry zero.
  for (int t = tid; t < ABY * (ABX + 1); t += ABX * ABY) {
    const int li = t % (ABX + 1), lj = t / (ABX + 1);
    const int i = i0 + li, j = j0 + lj;
    double f = 0.;
    if (i >= 2 && i <= nx && j <= ny) {
      const double vel = ux[ix_ux(nx, i, j)];
      const int ii = vel < 0. ? i : i - 1;
      const double x = vel < 0. ? -0.5 : +0.5;
      const double lvof = vof[ix_vof(nx, ii, j)];
      if (lvof < kVofMin || 1. - kVofMin < lvof) {
        f = vel * lvof;
      } else {
        const double *n = normal + ix_nrm(nx, ii, j);
        double flux = 0.;
#pragma unroll
        for (int jj = 0; jj < 2; jj++) flux += c_gauss_w[jj] * thinc_indicator(n, x, c_gauss_p[jj]);
        f = vel * flux;
      }
    }
    fx[lj][li] = f;
  }
  // compute_flux_y, src/interface/update/flxy.c:11-44; faces j in [1, ny+1]
  for (int t = tid; t < (ABY + 1) * ABX; t += ABX * ABY) {
    const int li = t % ABX, lj = t / ABX;
    const int i = i0 + li, j = j0 + lj;
    double f = 0.;
    if (i <= nx && j <= ny + 1) {
      const double vel = uy[ix_cc(nx, i, j)];
      const int jj = vel < 0. ? j : j - 1;
      const double y = vel < 0. ? -0.5 : +0.5;
      const double lvof = vof[ix_vof(nx, i, jj)];
      if (lvof < kVofMin || 1. - kVofMin < lvof) {
        f = vel * lvof;
      } else {
        const double *n = normal + ix_nrm(nx, i, jj);
        double flux = 0.;
#pragma unroll
        for (int ii = 0; ii < 2; ii++) flux += c_gauss_w[ii] * thinc_indicator(n, c_gauss_p[ii], y);
        f = vel * flux;
      }
    }
    fy[lj][li] = f;
  }
  __syncthreads();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  if (i > nx || j > ny) return;
  const double dt = *dtp;
  // interface_compute_rhs, src/interface/update/main.c:47-78 (source starts zeroed)
  const double dx = g.dxf[i - 1];
  double s = 0.;
  s += 1. / dx * (+fx[ty][tx] - fx[ty][tx + 1]);
  s += 1. / g.dy * (+fy[ty][tx] - fy[ty + 1][tx]);
  src_a[ix_src(nx, i, j)] = s;
  // interface_advect_vof, src/interface/update/main.c:80-110
  double v = vof[ix_vof(nx, i, j)];
  v += dt * rk.a * s;
  if (use_b) v += dt * rk.b * src_b[ix_src(nx, i, j)];
  // interface_update_boundaries_vof: halo rows are copies, walls are zero
  vof_new[ix_vof(nx, i, j)] = v;
  if (j <= 2) vof_new[ix_vof(nx, i, ny + j)] = v;
  if (j >= ny - 1) vof_new[ix_vof(nx, i, j - ny)] = v;
  if (1 == i) {
    vof_new[ix_vof(nx, 0, j)] = 0.;
    if (j <= 2) vof_new[ix_vof(nx, 0, ny + j)] = 0.;
    if (j >= ny - 1) vof_new[ix_vof(nx, 0, j - ny)] = 0.;
  }
  if (nx == i) {
    vof_new[ix_vof(nx, nx + 1, j)] = 0.;
    if (j <= 2) vof_new[ix_vof(nx, nx + 1, ny + j)] = 0.;
    if (j >= ny - 1) vof_new[ix_vof(nx, nx + 1, j - ny)] = 0.;
  }
}

}  // namespace svof
