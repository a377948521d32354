// svof_internal.cuh -- shared device helpers and kernel declarations of the
// FP64 2D path.  All kernels of this path are compiled with -fmad=false so
// that every multiply and add rounds separately, as the reference's C code
// does on x86-64; together with the reference's operation order this makes
// the device arithmetic reproduce the reference except where it calls libm
// exp/log (THINC intercept and indicator), whose CUDA versions may differ in
// the last bit.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/svof_b200.h"

namespace svof {

constexpr double kDblEpsilon = 2.220446049250313080847e-16;  // DBL_EPSILON
constexpr double kDblMax = 1.7976931348623157e308;          // DBL_MAX

// Programmatic dependent launch: on small grids the step graph launches its
// kernels with programmatic stream serialisation, so that a kernel is set up
// while its predecessor drains.  Every step kernel starts here and waits
// until the preceding kernels of its stream have completed and their memory
// is visible.  The successor is released when the blocks exit (an explicit
// early release measured slower from 256^2 cells up).  The wait does nothing
// for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// reference include/array_macros/**: index maps of the halo'd arrays
struct Grid2 {
  int nx, ny;
  double dy;
  const double *dxf;   // [nx]   DXF(i) = dxf[i-1]
  const double *dxc;   // [nx+1] DXC(i) = dxc[i-1]
};

__host__ __device__ __forceinline__ long ix_ux(int nx, int i, int j) { return (long)(i - 1) + (long)(nx + 1) * j; }
__host__ __device__ __forceinline__ long ix_cc(int nx, int i, int j) { return (long)i + (long)(nx + 2) * j; }
__host__ __device__ __forceinline__ long ix_vof(int nx, int i, int j) { return (long)i + (long)(nx + 2) * (j + 1); }
__host__ __device__ __forceinline__ long ix_nrm(int nx, int i, int j) { return 3L * ((long)(i - 1) + (long)nx * j); }
__host__ __device__ __forceinline__ long ix_srcx(int nx, int i, int j) { return (long)(i - 2) + (long)(nx - 1) * (j - 1); }
__host__ __device__ __forceinline__ long ix_src(int nx, int i, int j) { return (long)(i - 1) + (long)nx * (j - 1); }

// Runge-Kutta coefficients of one substep (src/runge_kutta.c:8-15)
struct RK {
  double a, b, g;
};

// boundary kinds of the halo / wall update
enum BcKind { BC_ZERO_UX = 0, BC_DIRICHLET = 1, BC_NEUMANN = 2, BC_VOF = 3 };

// ---- kernels (definitions in k_*.cu) ----
// periodic y halo then x wall values of one field (src/halo.c:18-76 and
// src/fluid/boundary/*.c, src/interface/boundary.c)
__global__ void k_halo_bc(double *a, int width, int nh, int ny, int kind, double lo, double hi);

// interface geometry: corner normals in shared memory, cell normal +
// intercept, curvature (src/interface/curvature_tensor.c:14-186)
__global__ void k_geom(const double *__restrict__ vof, double *__restrict__ normal,
                       double *__restrict__ curv, Grid2 g);
// CSF force (src/interface/force.c:11-76)
__global__ void k_force(const double *__restrict__ vof, const double *__restrict__ curv,
                        double *__restrict__ ifrcx, double *__restrict__ ifrcy, double tension, Grid2 g);
// THINC fluxes, flux divergence and RK update of vof
// (src/interface/update/*.c, src/interface/boundary.c)
__global__ void k_vof_advect(const double *__restrict__ vof, double *__restrict__ vof_new,
                             const double *__restrict__ ux, const double *__restrict__ uy,
                             const double *__restrict__ normal, double *__restrict__ src_a,
                             const double *__restrict__ src_b, const double *__restrict__ dtp,
                             RK rk, int use_b, Grid2 g);
// fused momentum / scalar right-hand sides, increments, implicit-x Thomas
// sweeps and field update (src/fluid/predict/*.c, src/tdm.c:17-50)
struct PredictArgs {
  const double *ux, *uy, *p, *t, *ifrcx, *ifrcy;
  double *ux_new, *uy_new, *t_new;
  double *sux_a, *suy_a, *st_a;
  const double *sux_b, *suy_b, *st_b;
  const double *lap_ux, *lap_uy, *lap_t;  // 3 per row
  const double *coef;                     // k_tdm_coef output, [3 fields][L, R, V][nx]
  const double *dtp;
  double m_dif, t_dif;
  double lapy0, lapy1, lapy2;
  RK rk;
  int use_b;
  int add_buoyancy;
  double uy_xm, uy_xp, t_xm, t_xp;
  // vof buoyancy on uy (an extension, absent from the reference; skipped
  // while grav_vof is 0): srcuy_a += grav_vof (vof at the uy face - vof_ref),
  // vof the field after this substep's advection
  const double *vof;
  double grav_vof, vof_ref;
  int rows_per_block;
  Grid2 g;
};
__global__ void k_predict(PredictArgs a);
// the Thomas tables of up to three substeps, one block each (block b uses
// gams.g[b] and writes coef_all + 9 nx b)
struct Gam3 {
  double g[3];
};
__global__ void k_tdm_coef(const double *__restrict__ lap_ux, const double *__restrict__ lap_uy,
                           const double *__restrict__ lap_t, const double *__restrict__ dtp, Gam3 gams,
                           double m_dif, double t_dif, int nx, double *__restrict__ coef_all);
size_t predict_smem_bytes(int nx, int rows_per_block);
// the line-streaming form of k_predict for large grids: right-hand sides of
// 32 x 32 tiles into the line array fw (3 fields, lines in blocks of 32,
// 3 nx 32 ceil(ny / 32) doubles), the x sweeps one warp per field and block of
// lines (3 ceil(ny / 32) blocks of 32 threads, dynamic shared memory
// predict_xsolve_smem(nx)), then u + delta' with halo rows and walls
__global__ void k_predict_rhs(PredictArgs a, double *__restrict__ fw);
__global__ void k_predict_xsolve(const double *__restrict__ coef, double *__restrict__ fw, int nx, int ny);
// (the three coefficient rows start at even offsets: nx rounded up to even)
inline size_t predict_xsolve_smem(int nx) {
  return sizeof(double) * ((size_t)4 * 64 * 32 + 3 * (size_t)((nx + 1) & ~1));
}
__global__ void k_predict_update(PredictArgs a, const double *__restrict__ fw);

// Poisson, DCT path (src/fluid/compute_potential/dct.c).  The row transforms
// (k_dct_fwd: divergence right-hand side + REDFT10; k_dct_fwd_rhs: the same
// on an array right-hand side r[j-1][i-1] / dxf[i-1], the adjoint's second
// solve; k_dct_inv: REDFT01 + psi rows with halo and walls) are compiled per
// length nx = 2^log2n, log2n in [kDctMinL2N, kDctMaxL2N]: dct_threads(log2n)
// threads, dct_rows(log2n) rows per block (grid ceil(ny / rows)),
// dct_smem(log2n, inverse) bytes of dynamic shared memory; dct_prepare raises
// those limits.
constexpr int kDctMinL2N = 2, kDctMaxL2N = 12;
using DctFwdKernel = void (*)(const double *, const double *, double *, const double *, const double *,
                              const double *, double, Grid2);
using DctFwdRhsKernel = void (*)(const double *, double *, const double *, const double *, Grid2);
using DctInvKernel = void (*)(const double *, double *, const double *, const double *, Grid2);
bool dct_length_ok(int log2n);
int dct_rows(int log2n);
int dct_threads(int log2n);
size_t dct_smem(int log2n, bool inverse);
DctFwdKernel dct_fwd_kernel(int log2n);
DctFwdRhsKernel dct_fwd_rhs_kernel(int log2n);
DctInvKernel dct_inv_kernel(int log2n);
cudaError_t dct_prepare(int log2n);
__global__ void k_dct_ysolve(double *__restrict__ spec, const double *__restrict__ vt,
                             const double *__restrict__ rvt, const double *__restrict__ q1t,
                             const double *__restrict__ ck, const double *__restrict__ lastf,
                             const double *__restrict__ den, double lap, int nx, int ny, int kt);
// Poisson, DFT path (src/fluid/compute_potential/dft.c)
__global__ void k_dft_fwd(const double *__restrict__ ux, const double *__restrict__ uy,
                          double *__restrict__ spec, const double *__restrict__ tw,
                          const double *__restrict__ dtp, double gam, int log2n, int cols, Grid2 g);
__global__ void k_dft_xsolve(double *__restrict__ spec, const double *__restrict__ vt,
                             const double *__restrict__ rvt, const double *__restrict__ pl,
                             const double *__restrict__ pu, const double *__restrict__ evals, int nx,
                             int nky, int kt);
__global__ void k_dft_inv(const double *__restrict__ spec, double *__restrict__ psi,
                          const double *__restrict__ tw, int log2n, int cols, Grid2 g);

// the DFT path's forward transform on a right-hand side r[j-1][i-1] /
// dxf[i-1] (the adjoint's second Poisson solve, with the grid-metric weights
// of the x grid); k_dft_fwd's launch shape
__global__ void k_dft_fwd_rhs(const double *__restrict__ r, double *__restrict__ spec, const double *__restrict__ tw,
                              int log2n, int cols, Grid2 g);

// projection and pressure update, in place (src/fluid/correct_velocity/*.c,
// src/fluid/update_pressure.c); do_vel / do_p select the two halves
__global__ void k_project(double *__restrict__ ux, double *__restrict__ uy, double *__restrict__ p,
                          const double *__restrict__ psi, const double *__restrict__ dtp, double gam,
                          double m_dif, double uy_xm, double uy_xp, int do_vel, int do_p, Grid2 g);

// time step (src/fluid/decide_dt.c)
// (status: bit 0 a non-finite velocity, bit 1 a time step that is not a
// positive finite number)
__global__ void k_cfl(const double *__restrict__ ux, const double *__restrict__ uy,
                      unsigned long long *__restrict__ minbits, unsigned *__restrict__ status, Grid2 g);
__global__ void k_dt_final(unsigned long long *minbits, double *dt, double coef_adv, double dif_m_y,
                           double dif_t_y, unsigned *status);
// diagnostics (src/logging/divergence.c, src/logging/interface.c)
__global__ void k_diag(const double *__restrict__ ux, const double *__restrict__ uy,
                       const double *__restrict__ vof, double *__restrict__ out, Grid2 g);
// logging reductions (src/logging/momentum.c, energy.c, nusselt/); one block
__global__ void k_logging(const double *__restrict__ ux, const double *__restrict__ uy,
                          const double *__restrict__ t, double m_dif, double t_dif, double ly,
                          double *__restrict__ out, Grid2 g);

// ---- engine internals shared by the C ABI front-ends (solver.cu, dropin.cu) ----
// svof_create with a choice of field memory: managed = CUDA managed memory,
// readable by a host program that holds the field pointers
int engine_create(const svof_params_t *prm, const double *xf, const double *xc, bool managed,
                  svof_solver_t **out);
// replace the run-time parameters (same grid); rebuilds the step graphs
int engine_update_params(svof_solver_t *s, const svof_params_t *prm);
// halo / wall update of field `field` stored at `ptr`, waited for
int engine_apply_bc(svof_solver_t *s, int field, double *ptr);
const svof_params_t *engine_params(const svof_solver_t *s);

}  // namespace svof
