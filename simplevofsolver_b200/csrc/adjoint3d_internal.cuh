// adjoint3d_internal.cuh -- kernels of the 3D step's adjoint (k3_adjoint.cu)
// and their argument blocks, used by the host code in solver3d.cu.
#pragma once

#include "svof3d_internal.cuh"

namespace svof3 {

// the grid with the reciprocal spacings the adjoint kernels multiply by (the
// adjoint follows no reference rounding: no divisions in its kernels)
struct AGrid3 {
  Grid3 g;
  const double *rxf;  // [nx]   1 / dxf
  const double *rxc;  // [nx+1] 1 / dxc
  double rdy, rdz;
  // gradient floor tau: a corner whose gradient times its smallest spacing
  // is below tau (a vof variation below tau across a cell) counts as flat,
  // its normal's transpose zero; 0 = the exact transpose
  double tau;
};

// lines per block and points per shared-memory chunk of k3_adj_xsolve
constexpr int kAdjXLines = 128;
constexpr int kAdjXChunk = 16;

// psi_bar += (d p' / d psi)^T p_bar' (mode & 1), (d u' / d psi)^T u_bar' (mode & 2)
__global__ void k3_adj_project(const double *__restrict__ aux, const double *__restrict__ auy,
                               const double *__restrict__ auz, const double *__restrict__ ap,
                               double *__restrict__ apsi, double gdt, double pre, int mode, AGrid3 ag);
// b = psi_bar / dxf (compact)
__global__ void k3_adj_scale(const double *__restrict__ apsi, double *__restrict__ b, AGrid3 ag);
// u_bar += the divergence's transpose of pre_p dxf s; psi_bar = 0
__global__ void k3_adj_div(double *__restrict__ aux, double *__restrict__ auy, double *__restrict__ auz,
                           const double *__restrict__ s, double *__restrict__ apsi, double pre_p, AGrid3 ag);
// transposed implicit-x solves and the RK split: grid (lines / kAdjXLines,
// 3 fields), kAdjXLines threads, dynamic shared memory adj_xsolve_smem(nx)
__global__ void k3_adj_xsolve(const double *__restrict__ aux, const double *__restrict__ auy,
                              const double *__restrict__ auz, const double *__restrict__ coef,
                              double *__restrict__ sa_x, double *__restrict__ sg_x, double *__restrict__ sa_y,
                              double *__restrict__ sg_y, double *__restrict__ sa_z, double *__restrict__ sg_z,
                              double *__restrict__ pend_x, double *__restrict__ pend_y, double *__restrict__ pend_z,
                              double adt, double bdt, double gdt, Grid3 g);
inline size_t adj_xsolve_smem(int nx) {
  return sizeof(double) * (3 * (size_t)nx + 2 * (size_t)kAdjXLines * (kAdjXChunk + 1));
}

struct Adj3RhsArgs {
  const double *ux, *uy, *uz;                               // primal, storage layouts
  const double *sa_x, *sg_x, *sa_y, *sg_y, *sa_z, *sg_z;    // src_a_bar, src_g_bar
  double *aux, *auy, *auz, *ap, *aifx, *aify, *aifz;
  const double *lap_ux, *lap_cc;
  double m_dif, ly0, ly1, ly2, lz0, lz1, lz2;
  // the vof buoyancy extension (skipped while grav_vof == 0): vof_post the
  // primal vof after the substep's advection (storage layout), avof its
  // adjoint (+=), agrv the coefficient's adjoint per cell (+=)
  double grav_vof, vof_ref;
  const double *vof_post;
  double *avof, *agrv;
  AGrid3 ag;
};
__global__ void __launch_bounds__(256, 4) k3_adj_rhs(Adj3RhsArgs a);

struct Adj3IfaceArgs {
  const double *ux, *uy, *uz, *vof, *normal, *curv;  // primal, storage layouts
  const double *avof_in, *pend_in;                   // vof_bar' and pend (compact)
  double *avof_out, *pend_out;
  double *aux, *auy, *auz;                           // += flux terms of owned faces
  const double *aifx, *aify, *aifz;                  // force adjoints
  double *anrm;                                      // [4] per cell
  double *am;                                        // [3] per cell, m_bar
  double *akap;                                      // kappa_bar
  double *asig;                                      // tension adjoint, per cell, +=
  double adt, bdt, tension;
  int mode;
  AGrid3 ag;
};
__global__ void __launch_bounds__(256, 4) k3_adj_interface(Adj3IfaceArgs a);

// corner gradients' adjoints ([3] per corner, (nx + 1) ny nz corners)
__global__ void k3_adj_cgrad(const double *__restrict__ vof, const double *__restrict__ am,
                             const double *__restrict__ akap, double *__restrict__ gbar, AGrid3 ag);
// vof_bar += the corner gradients' transposes
__global__ void k3_adj_cvof(const double *__restrict__ gbar, double *__restrict__ avof, AGrid3 ag);
// deterministic sum (one block of 256 threads)
__global__ void k3_adj_sum(const double *__restrict__ x, long n, double *__restrict__ out);
// *dst = v in stream order
__global__ void k3_adj_set(double *dst, double v);

}  // namespace svof3
