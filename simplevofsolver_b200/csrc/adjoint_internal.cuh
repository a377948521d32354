// adjoint_internal.cuh -- kernels of the 2D step's adjoint (k_adjoint.cu)
// and their argument blocks, used by the host code in adjoint.cu.
#pragma once

#include "svof_internal.cuh"

namespace svof {

// psi_bar += (d p' / d psi)^T p_bar' (mode & 1), (d u' / d psi)^T u_bar' (mode & 2)
__global__ void k_adj_project(const double *__restrict__ aux, const double *__restrict__ auy,
                              const double *__restrict__ ap, double *__restrict__ apsi, double gdt, double pre,
                              int mode, Grid2 g);
// u_bar += pre_p div^T (dxf s); psi_bar = 0
__global__ void k_adj_div(double *__restrict__ aux, double *__restrict__ auy, const double *__restrict__ s,
                          double *__restrict__ apsi, double pre_p, Grid2 g);
// transposed implicit-x solves and the RK split of delta_bar; dynamic shared
// memory 2 R nx doubles
__global__ void k_adj_xsolve(const double *__restrict__ aux, const double *__restrict__ auy,
                             const double *__restrict__ coef, double *__restrict__ sa_x, double *__restrict__ sg_x,
                             double *__restrict__ sa_y, double *__restrict__ sg_y, double *__restrict__ pend_x,
                             double *__restrict__ pend_y, double adt, double bdt, double gdt, int R, Grid2 g);

struct AdjRhsArgs {
  const double *ux, *uy;                     // primal, storage layouts
  const double *sa_x, *sg_x, *sa_y, *sg_y;   // src_a_bar, src_g_bar
  double *aux, *auy, *ap, *avof, *aifx, *aify;
  const double *lap_ux, *lap_uy;
  double m_dif, lapy0, lapy1, lapy2;
  double grav_vof, vof_ref;
  const double *vof_post;                    // primal vof after the substep's advection (storage layout)
  double *agrv;                              // buoyancy coefficient adjoint, per cell, +=
  Grid2 g;
};
__global__ void k_adj_rhs(AdjRhsArgs a);

struct AdjIfaceArgs {
  const double *ux, *uy, *vof, *normal, *curv;  // primal, storage layouts
  const double *avof_in, *pend_in;              // vof_bar' and pend (compact)
  double *avof_out, *pend_out;
  double *aux, *auy;                            // += flux terms of owned faces
  const double *aifx, *aify;                    // force adjoints
  double *anrm;                                 // [3] per cell
  double *am;                                   // [2] per cell, m_bar
  double *akap;                                 // kappa_bar
  double *asig;                                 // tension adjoint, per cell, +=
  double adt, bdt, tension;
  int mode;
  Grid2 g;
};
__global__ void k_adj_interface(AdjIfaceArgs a);

// tile of the corner kernel
constexpr int CBX = 32, CBY = 8;
__global__ void k_adj_corners(const double *__restrict__ vof, const double *__restrict__ am,
                              const double *__restrict__ akap, double *__restrict__ avof, Grid2 g);
// deterministic sum (one block of 256 threads)
__global__ void k_adj_sum(const double *__restrict__ x, long n, double *__restrict__ out);
// *dst = v in stream order
__global__ void k_adj_set(double *dst, double v);

}  // namespace svof
