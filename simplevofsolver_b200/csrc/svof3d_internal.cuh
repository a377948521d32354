// svof3d_internal.cuh -- device helpers and kernel declarations of the FP64
// 3D path.  Compiled with -fmad=false like the 2D path: every expression keeps
// the restatement's association (oracle/svof_oracle3d.c), so the device
// reproduces it except where CUDA's exp / log differ in the last bit (THINC).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/svof3d_b200.h"

namespace svof3 {

constexpr double kDblEpsilon = 2.220446049250313080847e-16;  // DBL_EPSILON
constexpr double kDblMax = 1.7976931348623157e308;          // DBL_MAX

struct Grid3 {
  int nx, ny, nz;
  double dy, dz;
  const double *dxf;  // [nx]   DXF(i) = dxf[i-1]
  const double *dxc;  // [nx+1] DXC(i) = dxc[i-1]
};

// index maps of the halo'd arrays (tools/define_arrays.py:192-229)
__host__ __device__ __forceinline__ long ix_ux(const Grid3 &g, int i, int j, int k) {
  return (long)(i - 1) + (long)(g.nx + 1) * ((long)j + (long)(g.ny + 2) * k);
}
__host__ __device__ __forceinline__ long ix_cc(const Grid3 &g, int i, int j, int k) {
  return (long)i + (long)(g.nx + 2) * ((long)j + (long)(g.ny + 2) * k);
}
__host__ __device__ __forceinline__ long ix_vof(const Grid3 &g, int i, int j, int k) {
  return (long)i + (long)(g.nx + 2) * ((long)(j + 1) + (long)(g.ny + 4) * (k + 1));
}
__host__ __device__ __forceinline__ long ix_nrm(const Grid3 &g, int i, int j, int k) {
  return 4L * ((long)(i - 1) + (long)g.nx * ((long)j + (long)(g.ny + 2) * k));
}
__host__ __device__ __forceinline__ long ix_srcx(const Grid3 &g, int i, int j, int k) {
  return (long)(i - 2) + (long)(g.nx - 1) * ((long)(j - 1) + (long)g.ny * (k - 1));
}
__host__ __device__ __forceinline__ long ix_src(const Grid3 &g, int i, int j, int k) {
  return (long)(i - 1) + (long)g.nx * ((long)(j - 1) + (long)g.ny * (k - 1));
}

// periodic images of an interior row (j, k): the row itself and the halo rows
// that copy it (one halo layer); returns the count, writes up to 4 (j, k)
__device__ __forceinline__ int halo_images(int j, int k, int ny, int nz, int *jj, int *kk) {
  int js[2], ks[2], nj = 1, nk = 1;
  js[0] = j;
  ks[0] = k;
  if (1 == j) js[nj++] = ny + 1;
  else if (ny == j) js[nj++] = 0;
  if (1 == k) ks[nk++] = nz + 1;
  else if (nz == k) ks[nk++] = 0;
  int n = 0;
  for (int a = 0; a < nk; a++)
    for (int b = 0; b < nj; b++) {
      jj[n] = js[b];
      kk[n] = ks[a];
      n++;
    }
  return n;
}

// the same, as a visitor: f(j', k') for the row itself (when `self`) and for
// each halo row that copies it; no local arrays
template <class F>
__device__ __forceinline__ void for_images(int j, int k, int ny, int nz, bool self, F f) {
  const int j2 = (1 == j) ? ny + 1 : ((ny == j) ? 0 : -1);
  const int k2 = (1 == k) ? nz + 1 : ((nz == k) ? 0 : -1);
  if (self) f(j, k);
  if (j2 >= 0) f(j2, k);
  if (k2 >= 0) {
    f(j, k2);
    if (j2 >= 0) f(j2, k2);
  }
}

// read-only global load through the non-coherent path
__device__ __forceinline__ double ldg(const double *p) { return __ldg(p); }
__device__ __forceinline__ float ldg(const float *p) { return __ldg(p); }

struct RK {
  double a, b, g;
};

enum BcKind3 { BC3_ZERO = 0, BC3_DIRICHLET = 1, BC3_NEUMANN = 2, BC3_VOF = 3 };

// ---- kernels ----
// periodic y then z halo and x wall values of one field (restatement of the
// 2D boundary update with z after y); one thread per storage cell of the
// interior rows
__global__ void k3_halo_bc(double *a, int width, int nh, int ny, int nz, int kind, double lo, double hi);

// interface kernels (k3_interface.cu), templates on R = double (FP64 path) or
// float (mixed path): R is the type of curv, normal, ifrc* and of the
// geometry / THINC arithmetic; vof, velocities and vof sources are FP64.
// geometry: corner normals, cell normals, curvature (clears and fills the
// interfacial-cell worklist), then the THINC intercepts of the listed cells
// (unconverged, when given: += the cells whose Newton iteration did not converge)
template <class R>
cudaError_t interface_geom(cudaStream_t st, const double *vof, R *normal, R *curv, unsigned *work,
                           unsigned *nwork, Grid3 g, unsigned long long *unconverged = nullptr);
// CSF force
template <class R>
cudaError_t interface_force(cudaStream_t st, const double *vof, const R *curv, R *ifrcx, R *ifrcy, R *ifrcz,
                            double tension, Grid3 g);
// opt-in shared memory of the interface kernels (once per device)
cudaError_t interface_prepare();
// THINC fluxes, divergence, RK update of vof with halo and walls
template <class R>
cudaError_t interface_advect(cudaStream_t st, const double *vof, double *vof_new, const double *ux,
                             const double *uy, const double *uz, const R *normal, double *src_a,
                             const double *src_b, const double *dtp, RK rk, int use_b, Grid3 g);

// momentum / scalar predictor: right-hand sides, increments and the forward
// Thomas sweep in x-chunks, then the backward sweep and the update.  R is the
// storage type of the forces, the momentum sources and the sweep scratch; the
// arithmetic is FP64 in both precisions.
template <class R>
struct Predict3Args {
  const double *ux, *uy, *uz, *p, *t;
  const R *ifrcx, *ifrcy, *ifrcz;
  double *ux_new, *uy_new, *uz_new, *t_new;
  R *sa[4];        // src_a of ux, uy, uz, t
  const R *sb[4];  // src_b
  R *fw;           // forward-sweep scratch, [4][ny nz][nx]
  const double *lap_ux, *lap_cc;  // 3 per row
  const double *coef;   // [3 sets (ux, uy/uz, t)][L, R, V][nx]
  const double *dtp;
  double m_dif, t_dif;
  double lapy[3], lapz[3];
  RK rk;
  int use_b, add_buoyancy;
  double uy_xm, uy_xp, uz_xm, uz_xp, t_xm, t_xp;
  // extension (off while grav_vof == 0): srcuy += grav_vof (vof_face -
  // vof_ref), vof the field after this substep's advection (storage layout)
  const double *vof;
  double grav_vof, vof_ref;
  Grid3 g;
};
template <class R>
cudaError_t predict_launch(cudaStream_t st, const Predict3Args<R> &a);
// opt-in shared memory of the right-hand-side kernel (once per device)
cudaError_t predict_prepare();
// Thomas coefficients of one substep for the three distinct systems
__global__ void k3_tdm_coef(const double *__restrict__ lap_ux, const double *__restrict__ lap_cc,
                            const double *__restrict__ dtp, double gam, double m_dif, double t_dif, int nx,
                            double *__restrict__ coef);

// Poisson: spectral array S[kz][ky][i] (complex, i fastest)
// Poisson stages (k3_poisson.cu), templates on R, the type of the spectrum,
// the twiddles and the transform arithmetic; the FP64 and the mixed path
// use R = double, the defect-corrected mixed form R = float.  The x line
// solve is FP64.  The transforms are compiled for each length 2^1 .. 2^11
// (log2n outside that range is an invalid value).
template <class R>
cudaError_t pois_prepare(int log2ny, int log2nz);
// (b: scratch of nx ny nz doubles for the right-hand side)
template <class R>
cudaError_t pois_fwd_y(cudaStream_t st, const double *ux, const double *uy, const double *uz, double *b, R *spec,
                       const R *tw, const double *dtp, double gam, int log2n, Grid3 g);
template <class R>
cudaError_t pois_z(cudaStream_t st, R *spec, const R *tw, int log2n, Grid3 g);
template <class R>
// (gauge0: the ky = kz = 0 line takes the gauge psi_hat(last) = 0, for FP32 storage;
// small_pivots, when given: += the lines other than ky = kz = 0 that met a
// pivot of magnitude at most DBL_EPSILON)
cudaError_t pois_x(cudaStream_t st, R *spec, R *scratch, const double *pl, const double *pu, const double *evy,
                   const double *evz, Grid3 g, bool gauge0 = false, unsigned long long *small_pivots = nullptr);
// acc: psi += the result (the correction pass), the walls' halo images kept
template <class R>
cudaError_t pois_inv_y(cudaStream_t st, const R *spec, double *psi, const R *tw, int log2n, Grid3 g,
                       bool acc = false);
// the forward y transform of a right-hand side given as a compact array
template <class R>
cudaError_t pois_fwd_y_array(cudaStream_t st, const double *b, R *spec, const R *tw, int log2n, Grid3 g);
// r = b - L psi / (ny nz), compact arrays of nx ny nz doubles (FP64)
// the mixed path's y transforms with two columns packed into one complex
// line (FP64; the right-hand side as pois_fwd_y; a block covers 2 COLS columns)
cudaError_t pois_fwd_y_packed(cudaStream_t st, const double *ux, const double *uy, const double *uz, double *b,
                              double *spec, const double *tw, const double *dtp, double gam, int log2n, Grid3 g);
cudaError_t pois_inv_y_packed(cudaStream_t st, const double *spec, double *psi, const double *tw, int log2n,
                              Grid3 g);
cudaError_t pois_resid(cudaStream_t st, const double *b, const double *psi, double *r, const double *pl,
                       const double *pu, Grid3 g);

// projection and pressure update, in place
__global__ void k3_project(double *__restrict__ ux, double *__restrict__ uy, double *__restrict__ uz,
                           double *__restrict__ p, const double *__restrict__ psi, const double *__restrict__ dtp,
                           double gam, double m_dif, double uy_xm, double uy_xp, double uz_xm, double uz_xp,
                           int do_vel, int do_p, Grid3 g);

// time step (status: bit 0 a non-finite velocity, bit 1 a time step that is
// not a positive finite number)
__global__ void k3_cfl(const double *__restrict__ ux, const double *__restrict__ uy, const double *__restrict__ uz,
                       unsigned long long *__restrict__ minbits, unsigned *__restrict__ status, Grid3 g);
__global__ void k3_dt_final(unsigned long long *minbits, double *dt, double coef_adv, double l0, double l1,
                            double l2, double l3, unsigned *status);
// diagnostics, deterministic two-stage reduction: blocks of 32 x 8 threads
// over kDiagPlanes planes write 5 partials each; out = {max |div u|, vof min,
// vof max, sum vof dx dy dz (compensated)}
constexpr int kDiagPlanes = 8, kDiagThreads = 1024;
__global__ void k3_diag_part(const double *__restrict__ ux, const double *__restrict__ uy,
                             const double *__restrict__ uz, const double *__restrict__ vof,
                             double *__restrict__ part, Grid3 g);
__global__ void k3_diag_final(const double *__restrict__ part, long nparts, double *__restrict__ out);

// launch constants shared by the kernels and the host
constexpr int kPredLines = 32;  // lines per predictor block
constexpr int kPredChunk = 32;  // x positions per chunk
constexpr int kProjectPlanes = 4;  // z planes per thread of k3_project
constexpr int kCflPlanes = 8;      // z planes per thread of k3_cfl (blocks of 32 x 8)

}  // namespace svof3
