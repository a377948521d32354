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
// S, the storage type of the adjoint's intermediates (the sources', forces',
// curvature's, normals' and corner gradients' adjoints): double, or float for
// the FP32 adjoint; accumulators, arithmetic, line recurrences and the
// Poisson solve are FP64 in both.

// dynamic shared memory of the x solves (kAdjXLines threads a block)
inline size_t adj_xsolve_smem(int nx) {
  return sizeof(double) * (3 * (size_t)nx + 2 * (size_t)kAdjXLines * (kAdjXChunk + 1));
}

template <class S>
struct Adj3RhsArgs {
  const double *ux, *uy, *uz;                               // primal, storage layouts
  const S *sa_x, *sg_x, *sa_y, *sg_y, *sa_z, *sg_z;         // src_a_bar, src_g_bar
  double *aux, *auy, *auz, *ap;
  S *aifx, *aify, *aifz;
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

template <class S>
struct Adj3IfaceArgs {
  const double *ux, *uy, *uz, *vof, *normal, *curv;  // primal, storage layouts
  const double *avof_in, *pend_in;                   // vof_bar' and pend (compact)
  double *avof_out, *pend_out;
  double *aux, *auy, *auz;                           // += flux terms of owned faces
  const S *aifx, *aify, *aifz;                       // force adjoints
  S *anrm;                                           // [4] per cell
  S *am;                                             // [3] per cell, m_bar
  S *akap;                                           // kappa_bar
  double *asig;                                      // tension adjoint, per cell, +=
  double adt, bdt, tension;
  int mode;
  AGrid3 ag;
};

// launchers of the templated kernels (defined beside them in k3_adjoint.cu):
// the x solves and RK split on `lines` lines (z_x, z_y, z_z: FP64 scratch of
// the forward sweep's values, src_g_bar itself when S is double), the
// right-hand-side and interface transposes on the cells, and the corner
// gradients (their normalisation's transpose, then back to vof_bar)
template <class S>
cudaError_t adj3_xsolve_launch(cudaStream_t st, long lines, size_t smem, const double *aux, const double *auy,
                               const double *auz, const double *coef, S *sa_x, S *sg_x, S *sa_y, S *sg_y, S *sa_z,
                               S *sg_z, S *pend_x, S *pend_y, S *pend_z, double *z_x, double *z_y, double *z_z,
                               double adt, double bdt, double gdt, Grid3 g);
template <class S>
cudaError_t adj3_xsolve_prepare(size_t smem);
template <class S>
cudaError_t adj3_rhs_launch(cudaStream_t st, const Adj3RhsArgs<S> &a);
template <class S>
cudaError_t adj3_interface_launch(cudaStream_t st, const Adj3IfaceArgs<S> &a);
template <class S>
cudaError_t adj3_corners_launch(cudaStream_t st, const double *vof, const S *am, const S *akap, S *gbar,
                                double *avof, AGrid3 ag);

// deterministic sum (one block of 256 threads)
__global__ void k3_adj_sum(const double *__restrict__ x, long n, double *__restrict__ out);
// *dst = v in stream order
__global__ void k3_adj_set(double *dst, double v);

}  // namespace svof3
