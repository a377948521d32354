// k3_predict.cu -- momentum / scalar predictor of the 3D path.
//
// ux, uy, uz and t each take delta = dt (alpha src_a + beta src_b + gamma
// src_g), solve (1 - gamma dt nu / 2 Lx) delta' = delta along x, and update
// u += delta' (src/fluid/predict/{ux,uy,t}.c in 2D, carried to z by the
// restatement oracle/svof_oracle3d.c).  Two kernels:
//
//   k3_rhs     all right-hand sides and increments: a 2.5D stencil that
//              marches along z with the state planes staged in shared memory
//              by cp.async one plane ahead; writes src_a and the increments
//              in a line layout
//   k3_xsolve  the x lines (ny nz of them, serial recurrences): a block owns
//              32 lines, walks them in 32-cell chunks forward and backward
//              with one line per lane of four sweeping warps, and writes the
//              updated fields with their halo images and walls
//
// The Thomas coefficients depend on the substep only (k3_tdm_coef: three
// distinct systems, ux, uy/uz, t).  The right-hand sides compute in FP64
// with the restatement's association in both precisions, the x sweeps in FP64
// (FP64 path: bit for bit) or FP32 (mixed path, whose increments are stored
// in FP32); R is the storage type of forces, sources and increments.
#include <cuda_pipeline.h>

#include <type_traits>

#include "svof3d_internal.cuh"
#include "smem_limit.cuh"

// Precision split as in k3_interface.cu: SVOF3_PRECISION=64 builds the FP64
// instantiations and the shared code (no FMA contraction), =32 the FP32
// instantiations only (FMA on); unset builds both.
#if !defined(SVOF3_PRECISION) || SVOF3_PRECISION == 64
#define SVOF3_WITH_F64 1
#else
#define SVOF3_WITH_F64 0
#endif
#if !defined(SVOF3_PRECISION) || SVOF3_PRECISION == 32
#define SVOF3_WITH_F32 1
#else
#define SVOF3_WITH_F32 0
#endif

namespace svof3 {

// Layout per system s at coef + 3 s nx:  L[i] = tdm_l[i];  R[0] = tdm_c[0],
// R[i] = 1 / (c_i - l_i v_{i-1}) for 0 < i < n-1, R[n-1] = 1 / (c - l v) of
// the last row or 0 when that row is zeroed (src/tdm.c:17-50);  V[i] = v_i.
#if SVOF3_WITH_F64
__global__ void k3_tdm_coef(const double *__restrict__ lap_ux, const double *__restrict__ lap_cc,
                            const double *__restrict__ dtp, double gam, double m_dif, double t_dif, int nx,
                            double *__restrict__ coef) {
  extern __shared__ double slap[];  // [2][3 nx]
  for (int w = threadIdx.x; w < 3 * nx; w += blockDim.x) {
    slap[w] = (w < 3 * (nx - 1)) ? lap_ux[w] : 0.;
    slap[3 * nx + w] = lap_cc[w];
  }
  __syncthreads();
  const int f = threadIdx.x;
  if (f >= 3) return;
  const double *lap = slap + ((0 == f) ? 0 : 3 * nx);
  const double dif = (2 == f) ? t_dif : m_dif;
  const int n = (0 == f) ? nx - 1 : nx;
  double *L = coef + (size_t)(3 * f + 0) * nx;
  double *R = coef + (size_t)(3 * f + 1) * nx;
  double *V = coef + (size_t)(3 * f + 2) * nx;
  const double dt = *dtp;
  const double pf = 0.5 * gam * dt * dif;
  const double c0 = 1. - pf * lap[1];
  double v = (-pf * lap[2]) / c0;
  L[0] = -pf * lap[0];
  R[0] = c0;
  V[0] = v;
  for (int i = 1; i < n - 1; i++) {
    const double l = -pf * lap[3 * i + 0];
    const double c = 1. - pf * lap[3 * i + 1];
    const double u = -pf * lap[3 * i + 2];
    const double val = 1. / (c - l * v);
    v = val * (u);
    L[i] = l;
    R[i] = val;
    V[i] = v;
  }
  {
    const double l = -pf * lap[3 * (n - 1) + 0];
    const double c = 1. - pf * lap[3 * (n - 1) + 1];
    const double val = c - l * v;
    L[n - 1] = l;
    R[n - 1] = fabs(val) > kDblEpsilon ? 1. / val : 0.;
  }
}
#endif

// The stencil values one cell's right-hand sides read: uy, uz, t at cell i
// and ux at the face iu = i + 1 (names: u = ux, v = uy, w = uz, t, p; 0 / 1
// / 2 the x offset from i, s / n the row j -+ 1, b / t the plane k -+ 1).
struct Stencil4 {
  double u00, u10, u20, u0s, u1s, u1n, u0b, u1b, u1t;
  double vc, vxm, vxp, vs, vn, vb, vt, vnb, v1n;
  double wc, wxm, wxp, ws, wn, wb, wt, wst, w1t;
  double tc, txm, txp, ts, tn, tb, tt;
  double gv;  // the vof buoyancy's face value (the GRAV instantiation only)
  double pc, ps, pb, pxp;
  double ifx, ify, ifz;
  double dxf_i, dxf_i1, dxc_i1;
  double lu0, lu1, lu2, lc0, lc1, lc2;
};

// The quotients of grid spacings the right-hand sides use, each evaluated
// once (per column for the x ones) with the expression the restatement
// evaluates per cell, hence the same values: h.. = +-0.5 / d., r.. = 1 / d.,
// w_xm / w_xp the x interpolation weights of the ux face.
struct RhsCoef {
  double hxc0, hxc1, w_xm, w_xp, rdxc;  // face iu = i + 1
  double hxf0, hxf1;                    // cell i
  double hy0, hy1, hz0, hz1, rdy, rdz;
};

__device__ __forceinline__ RhsCoef rhs_coef(double dxf_i, double dxf_i1, double dxc_i1, double dy, double dz) {
  RhsCoef c;
  c.hxc0 = +0.5 / dxc_i1;
  c.hxc1 = -0.5 / dxc_i1;
  c.w_xm = 0.5 * dxf_i / dxc_i1;
  c.w_xp = 0.5 * dxf_i1 / dxc_i1;
  c.rdxc = 1. / dxc_i1;
  c.hxf0 = +0.5 / dxf_i;
  c.hxf1 = -0.5 / dxf_i;
  c.hy0 = +0.5 / dy;
  c.hy1 = -0.5 / dy;
  c.hz0 = +0.5 / dz;
  c.hz1 = -0.5 / dz;
  c.rdy = 1. / dy;
  c.rdz = 1. / dz;
  return c;
}

// Right-hand sides of one cell (src/fluid/predict/{ux,uy,t}.c compute_rhs_*
// in 2D, carried to z by the restatement): the explicit part into sa[f], the
// x-implicit diffusion and the pressure gradient into sg[f], in the
// restatement's order (advection x, y, z; diffusion x, y, z; pressure;
// buoyancy; surface).  Fields 0 ux (do_ux: the face exists), 1 uy, 2 uz, 3 t.
template <class R, bool GRAV>
__device__ __forceinline__ void rhs4_values(const Predict3Args<R> &a, const Grid3 &g, const Stencil4 &S,
                                            const RhsCoef &K, bool do_ux, double *sa, double *sg) {
  const double u00 = S.u00, u10 = S.u10, u20 = S.u20, u0s = S.u0s, u1s = S.u1s, u1n = S.u1n, u0b = S.u0b,
               u1b = S.u1b, u1t = S.u1t;
  const double vc = S.vc, vxm = S.vxm, vxp = S.vxp, vs = S.vs, vn = S.vn, vb = S.vb, vt = S.vt, vnb = S.vnb,
               v1n = S.v1n;
  const double wc = S.wc, wxm = S.wxm, wxp = S.wxp, ws = S.ws, wn = S.wn, wb = S.wb, wt = S.wt, wst = S.wst,
               w1t = S.w1t;
  const double tc = S.tc, txm = S.txm, txp = S.txp, ts = S.ts, tn = S.tn, tb = S.tb, tt = S.tt;
  const double pc = S.pc, ps = S.ps, pb = S.pb, pxp = S.pxp;
  const double ifx = S.ifx, ify = S.ify, ifz = S.ifz;
  const double lu0 = S.lu0, lu1 = S.lu1, lu2 = S.lu2, lc0 = S.lc0, lc1 = S.lc1, lc2 = S.lc2;
  const double md = a.m_dif, td = a.t_dif;
  const double *ly = a.lapy, *lz = a.lapz;
  // ---- ux at the face iu = i + 1: xm = UX(iu-1), xc = UX(iu), xp = UX(iu+1)
  if (do_ux) {
    const double xm = u00, xc = u10, xp = u20, ys = u1s, yn = u1n, zs = u1b, zn = u1t;
    double ra = 0., rg = 0.;
    {
      const double ul = +0.5 * xm + 0.5 * xc, uu = +0.5 * xc + 0.5 * xp;
      const double l = K.hxc0 * ul, u = K.hxc1 * uu, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    const double w_xm = K.w_xm, w_xp = K.w_xp;
    {
      const double ul = w_xm * vc + w_xp * vxp;
      const double uu = w_xm * vn + w_xp * v1n;
      const double l = K.hy0 * ul, u = K.hy1 * uu, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double ul = w_xm * wc + w_xp * wxp;
      const double uu = w_xm * wt + w_xp * w1t;
      const double l = K.hz0 * ul, u = K.hz1 * uu, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += md * (+lu0 * xm + lu1 * xc + lu2 * xp);
    ra += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    rg -= K.rdxc * (-pc + pxp);
    if (a.add_buoyancy) ra += +0.5 * tc + 0.5 * txp;
    ra += ifx;
    sa[0] = ra;
    sg[0] = rg;
  }
  // ---- uy at cell i
  {
    const double xm = vxm, xc = vc, xp = vxp, ys = vs, yn = vn, zs = vb, zn = vt;
    double ra = 0., rg = 0.;
    {
      const double ul = +0.5 * u0s + 0.5 * u00;
      const double uu = +0.5 * u1s + 0.5 * u10;
      const double l = K.hxf0 * ul, u = K.hxf1 * uu, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    {
      const double ul = +0.5 * ys + 0.5 * xc, uu = +0.5 * xc + 0.5 * yn;
      const double l = K.hy0 * ul, u = K.hy1 * uu, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double ul = +0.5 * ws + 0.5 * wc;
      const double uu = +0.5 * wst + 0.5 * wt;
      const double l = K.hz0 * ul, u = K.hz1 * uu, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += md * (+lc0 * xm + lc1 * xc + lc2 * xp);
    ra += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    rg -= K.rdy * (-ps + pc);
    ra += ify;
    // extension: buoyancy of the volume fraction (not in the reference)
    if (GRAV) ra += a.grav_vof * (S.gv - a.vof_ref);
    sa[1] = ra;
    sg[1] = rg;
  }
  // ---- uz at cell i
  {
    const double xm = wxm, xc = wc, xp = wxp, ys = ws, yn = wn, zs = wb, zn = wt;
    double ra = 0., rg = 0.;
    {
      const double ul = +0.5 * u0b + 0.5 * u00;
      const double uu = +0.5 * u1b + 0.5 * u10;
      const double l = K.hxf0 * ul, u = K.hxf1 * uu, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    {
      const double ul = +0.5 * vb + 0.5 * vc;
      const double uu = +0.5 * vnb + 0.5 * vn;
      const double l = K.hy0 * ul, u = K.hy1 * uu, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double ul = +0.5 * zs + 0.5 * xc, uu = +0.5 * xc + 0.5 * zn;
      const double l = K.hz0 * ul, u = K.hz1 * uu, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += md * (+lc0 * xm + lc1 * xc + lc2 * xp);
    ra += md * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += md * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    rg -= K.rdz * (-pb + pc);
    ra += ifz;
    sa[2] = ra;
    sg[2] = rg;
  }
  // ---- t at cell i
  {
    const double xm = txm, xc = tc, xp = txp, ys = ts, yn = tn, zs = tb, zn = tt;
    double ra = 0., rg = 0.;
    {
      const double l = K.hxf0 * u00, u = K.hxf1 * u10, cc = -l - u;
      ra += +l * xm + cc * xc + u * xp;
    }
    {
      const double l = K.hy0 * vc, u = K.hy1 * vn, cc = -l - u;
      ra += +l * ys + cc * xc + u * yn;
    }
    {
      const double l = K.hz0 * wc, u = K.hz1 * wt, cc = -l - u;
      ra += +l * zs + cc * xc + u * zn;
    }
    rg += td * (+lc0 * xm + lc1 * xc + lc2 * xp);
    ra += td * (+ly[0] * ys + ly[1] * xc + ly[2] * yn);
    ra += td * (+lz[0] * zs + lz[1] * xc + lz[2] * zn);
    sa[3] = ra;
    sg[3] = rg;
  }
}

// ---------------------------------------------------------------------------
// k3_rhs: the right-hand sides and increments of all cells.  A block owns a
// 32 x 8 tile of (i, j) and marches along z over RZ planes.  The five state
// fields ux, uy, uz, t, p live in a ring of four shared-memory planes (a
// 34 x 10 window each, the tile with its x and y neighbours): planes k - 1,
// k, k + 1 are read by the stencil while plane k + 2 arrives by cp.async.
// Writes src_a and the increment delta = dt (alpha src_a + beta src_b +
// gamma src_g) in the line layout [field][j - 1 + ny (k - 1)][x position]
// that the line solver reads.
constexpr int RX = 32, RY = 8, RZ = 64;
constexpr int WX = RX + 2, WY = RY + 2, NSLOT = 4, NFLD = 5, NCEN = 7;
// the state windows (FP64) and the per-cell inputs ifrcx / ifrcy / ifrcz and
// src_b of the four fields (R-sized: 83 KB per mixed block instead of 112 KB,
// which measured 3 % faster on the mixed step at 512^3)
// FP64: the per-cell inputs are read straight from global memory (they are
// used by their own thread only, and the FP64 kernel runs faster without
// their ring); FP32 (mixed): they ride the ring with the state planes
template <class R>
constexpr bool kRhsDirect = 8 == sizeof(R);
template <class R>
constexpr size_t kRhsSmem =
    sizeof(double) * NFLD * NSLOT * WY * WX + (kRhsDirect<R> ? 0 : sizeof(R) * NCEN * NSLOT * RY * RX);

// GRAV: the instantiation with the vof buoyancy extension (grav_vof != 0);
// the other one is the reference's right-hand side alone
template <class R, bool GRAV>
__global__ void __launch_bounds__(RX * RY, 2) k3_rhs(Predict3Args<R> a) {
  extern __shared__ double ring[];  // [NFLD][NSLOT][WY][WX]
  const Grid3 g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tid = threadIdx.x, tx = tid % RX, ty = tid / RX;
  const int i0 = 1 + blockIdx.x * RX, j0 = 1 + blockIdx.y * RY, k0 = 1 + blockIdx.z * RZ;
  const int kend = min(k0 + RZ, nz + 1);  // cells k in [k0, kend)
  const int i = i0 + tx, j = j0 + ty;
  const bool mine = i <= nx && j <= ny;
  const bool do_ux = i < nx;
  const double *fld[NFLD] = {a.ux, a.uy, a.uz, a.t, a.p};
  const long width[NFLD] = {nx + 1, nx + 2, nx + 2, nx + 2, nx + 2};
  const long plane_rows = ny + 2;
  // window column c <-> storage x = i0 - 1 + c; row r <-> j = j0 - 1 + r
  R *cen = reinterpret_cast<R *>(ring + (size_t)NFLD * NSLOT * WY * WX);  // [NCEN][NSLOT][RY][RX]
  const R *cen_src[NCEN] = {a.ifrcx, a.ifrcy, a.ifrcz, a.sb[0], a.sb[1], a.sb[2], a.sb[3]};
  const int ncen = a.use_b ? NCEN : 3;
  auto load_plane = [&](int kk) {
    const int slot = kk & (NSLOT - 1);
    // per-cell inputs of the interior planes: thread (tx, ty) copies its own
    if (!kRhsDirect<R> && kk >= k0 && kk < kend && mine) {
      const long is = ix_src(g, i, j, kk);
      const long isx = (long)(i - 1) + (long)(nx - 1) * ((long)(j - 1) + (long)ny * (kk - 1));  // face i + 1
      for (int q = 0; q < ncen; q++) {
        const bool xface = (0 == q || 3 == q);
        if (xface && !do_ux) continue;
        __pipeline_memcpy_async(cen + ((size_t)(q * NSLOT + slot) * RY + ty) * RX + tx,
                                cen_src[q] + (xface ? isx : is), sizeof(R));
      }
    }
    for (int f = 0; f < NFLD; f++) {
      double *dst = ring + ((size_t)f * NSLOT + slot) * WY * WX;
      const double *src = fld[f] + width[f] * plane_rows * kk;
      for (int e = tid; e < WY * WX; e += RX * RY) {
        const int r = e / WX, c = e - r * WX;
        const long x = i0 - 1 + c;
        const int jj = j0 - 1 + r;
        if (x < width[f] && jj <= ny + 1) {
          __pipeline_memcpy_async(dst + e, src + x + width[f] * jj, sizeof(double));
        } else {
          dst[e] = 0.;
        }
      }
    }
    __pipeline_commit();
  };
  load_plane(k0 - 1);
  load_plane(k0);
  load_plane(k0 + 1);
  __pipeline_wait_prior(0);
  __syncthreads();
  const double dt = ldg(a.dtp);
  const double ca = a.rk.a * dt, cb = a.rk.b * dt, cg = a.rk.g * dt;
  const size_t fstride = (size_t)ny * nz * nx;
  // per-column constants
  double dxf_i = 1., dxf_i1 = 1., dxc_i1 = 1., lu0 = 0., lu1 = 0., lu2 = 0., lc0 = 0., lc1 = 0., lc2 = 0.;
  if (mine) {
    dxf_i = ldg(g.dxf + i - 1);
    lc0 = ldg(a.lap_cc + 3 * (i - 1) + 0);
    lc1 = ldg(a.lap_cc + 3 * (i - 1) + 1);
    lc2 = ldg(a.lap_cc + 3 * (i - 1) + 2);
    if (do_ux) {
      dxf_i1 = ldg(g.dxf + i);
      dxc_i1 = ldg(g.dxc + i);
      lu0 = ldg(a.lap_ux + 3 * (i - 1) + 0);
      lu1 = ldg(a.lap_ux + 3 * (i - 1) + 1);
      lu2 = ldg(a.lap_ux + 3 * (i - 1) + 2);
    }
  }
  const RhsCoef K = rhs_coef(dxf_i, dxf_i1, dxc_i1, g.dy, g.dz);
  for (int k = k0; k < kend; k++) {
    if (k + 2 <= min(kend, nz + 1)) load_plane(k + 2);
    if (mine) {
      // FP64: the per-cell inputs from global memory, issued first
      double ifx_v = 0., ify_v = 0., ifz_v = 0., sbv[4] = {0., 0., 0., 0.};
      if constexpr (kRhsDirect<R>) {
        const long is_ = ix_src(g, i, j, k), isx_ = ix_srcx(g, i + 1, j, k);
        ifx_v = do_ux ? (double)__ldg(a.ifrcx + isx_) : 0.;
        ify_v = (double)__ldg(a.ifrcy + is_);
        ifz_v = (double)__ldg(a.ifrcz + is_);
        if (a.use_b) {
          sbv[0] = do_ux ? (double)__ldg(a.sb[0] + isx_) : 0.;
          sbv[1] = (double)__ldg(a.sb[1] + is_);
          sbv[2] = (double)__ldg(a.sb[2] + is_);
          sbv[3] = (double)__ldg(a.sb[3] + is_);
        }
      }
      const int sm = (k - 1) & (NSLOT - 1), s0 = k & (NSLOT - 1), sp = (k + 1) & (NSLOT - 1);
#define RING(f, slot, r, c) ring[(((size_t)(f) * NSLOT + (slot)) * WY + (r)) * WX + (c)]
      Stencil4 S;
      // ux (f 0): face iu <-> column iu - i0, i.e. face i <-> tx
      S.u00 = RING(0, s0, ty + 1, tx);
      S.u10 = RING(0, s0, ty + 1, tx + 1);
      S.u20 = RING(0, s0, ty + 1, tx + 2);
      S.u0s = RING(0, s0, ty, tx);
      S.u1s = RING(0, s0, ty, tx + 1);
      S.u1n = RING(0, s0, ty + 2, tx + 1);
      S.u0b = RING(0, sm, ty + 1, tx);
      S.u1b = RING(0, sm, ty + 1, tx + 1);
      S.u1t = RING(0, sp, ty + 1, tx + 1);
      // cell-centred fields: cell i <-> column tx + 1
      S.vc = RING(1, s0, ty + 1, tx + 1);
      S.vxm = RING(1, s0, ty + 1, tx);
      S.vxp = RING(1, s0, ty + 1, tx + 2);
      S.vs = RING(1, s0, ty, tx + 1);
      S.vn = RING(1, s0, ty + 2, tx + 1);
      S.vb = RING(1, sm, ty + 1, tx + 1);
      S.vt = RING(1, sp, ty + 1, tx + 1);
      S.vnb = RING(1, sm, ty + 2, tx + 1);
      S.v1n = RING(1, s0, ty + 2, tx + 2);
      S.wc = RING(2, s0, ty + 1, tx + 1);
      S.wxm = RING(2, s0, ty + 1, tx);
      S.wxp = RING(2, s0, ty + 1, tx + 2);
      S.ws = RING(2, s0, ty, tx + 1);
      S.wn = RING(2, s0, ty + 2, tx + 1);
      S.wb = RING(2, sm, ty + 1, tx + 1);
      S.wt = RING(2, sp, ty + 1, tx + 1);
      S.wst = RING(2, sp, ty, tx + 1);
      S.w1t = RING(2, sp, ty + 1, tx + 2);
      S.tc = RING(3, s0, ty + 1, tx + 1);
      S.txm = RING(3, s0, ty + 1, tx);
      S.txp = RING(3, s0, ty + 1, tx + 2);
      S.ts = RING(3, s0, ty, tx + 1);
      S.tn = RING(3, s0, ty + 2, tx + 1);
      S.tb = RING(3, sm, ty + 1, tx + 1);
      S.tt = RING(3, sp, ty + 1, tx + 1);
      S.pc = RING(4, s0, ty + 1, tx + 1);
      S.ps = RING(4, s0, ty, tx + 1);
      S.pb = RING(4, sm, ty + 1, tx + 1);
      S.gv = 0.;
      if (GRAV) S.gv = 0.5 * ldg(a.vof + ix_vof(g, i, j - 1, k)) + 0.5 * ldg(a.vof + ix_vof(g, i, j, k));
      S.pxp = RING(4, s0, ty + 1, tx + 2);
#undef RING
      const long is = ix_src(g, i, j, k);
#define CEN(q) (double)cen[((size_t)((q) * NSLOT + s0) * RY + ty) * RX + tx]
      if constexpr (kRhsDirect<R>) {
        S.ify = ify_v;
        S.ifz = ifz_v;
        S.ifx = ifx_v;
      } else {
        S.ify = CEN(1);
        S.ifz = CEN(2);
        S.ifx = do_ux ? CEN(0) : 0.;
      }
      S.dxf_i = dxf_i;
      S.dxf_i1 = dxf_i1;
      S.dxc_i1 = dxc_i1;
      S.lu0 = lu0;
      S.lu1 = lu1;
      S.lu2 = lu2;
      S.lc0 = lc0;
      S.lc1 = lc1;
      S.lc2 = lc2;
      double sa[4], sg[4];
      rhs4_values<R, GRAV>(a, g, S, K, do_ux, sa, sg);
      const size_t line = (size_t)(j - 1) + (size_t)ny * (k - 1);
      R *dl = a.fw + line * nx + (i - 1);
      if (do_ux) {
        const long isx = ix_srcx(g, i + 1, j, k);
        a.sa[0][isx] = R(sa[0]);
        const double sb = a.use_b ? cb * (kRhsDirect<R> ? sbv[0] : CEN(3)) : 0.;
        dl[0] = R(+ca * sa[0] + sb + cg * sg[0]);
      }
#pragma unroll
      for (int q = 1; q < 4; q++) {
        a.sa[q][is] = R(sa[q]);
        const double sb = a.use_b ? cb * (kRhsDirect<R> ? sbv[q] : CEN(3 + q)) : 0.;
        dl[q * fstride] = R(+ca * sa[q] + sb + cg * sg[q]);
      }
#undef CEN
    }
    __pipeline_wait_prior(0);
    __syncthreads();
  }
}

constexpr int PL = kPredLines, PC = kPredChunk;

// ---------------------------------------------------------------------------
// k3_xsolve: the implicit-x Thomas sweeps of the four fields and the update.
// A block owns 32 lines, walked in 32-cell x-chunks staged by cp.async:
// forward (the increments come in from the line array, warps 0..3 continue
// the recurrence with the carry in a register in FP64, one field per warp and
// one line per lane, the swept values go back), then backward in reverse
// chunk order with the update u + delta' into the other buffer of the
// ping-pong pair, halo images included, then the walls.  The tile holds the
// storage type R (in the mixed path the swept increments are FP32, as in the
// line array).
// chunk buffers: the FP32 tile (mixed path) is double-buffered, so that the
// copies of chunk c + 1 are in flight while chunk c is swept (a 4-byte copy
// carries half the bytes of an FP64 one); the FP64 tile stays single, within
// the 48 KB of static shared memory
template <class R>
constexpr int kXsBufs = 4 == sizeof(R) ? 2 : 1;

// the arithmetic type of the sweeps: FP64 in the FP64 path (the restatement's
// roundings, bit for bit), FP32 in the mixed path (its increments are FP32
// already; an FP32 chain is a tenth of the FP64 one's latency)
template <class R>
using SweepT = typename std::conditional<4 == sizeof(R), float, double>::type;

template <class R>
__global__ void __launch_bounds__(256) k3_xsolve(Predict3Args<R> a) {
  constexpr int NB = kXsBufs<R>;
  using T = SweepT<R>;
  __shared__ R sd[NB][4][PL][PC + 1];  // the four fields' values of one tile
  __shared__ T sco[NB][9][PC];         // L, R, V of the three systems, one chunk
  const Grid3 g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long nlines = (long)ny * nz;
  const long l0 = (long)blockIdx.x * PL;
  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  const int nchunks = (nx + PC - 1) / PC;
  // the sweeping warps: warp f < 4 owns field f, lane = line of the block
  const int f = ty;
  const bool sweeper = f < 4 && (l0 + tx < nlines);
  const int set = (0 == f) ? 0 : (3 == f ? 2 : 1);
  const int nf = (0 == f) ? nx - 1 : nx;
  const size_t fstride = (size_t)nlines * nx;  // line array per field
  // coefficients of chunk c into buffer b: all nine rows (forward) or the
  // three V rows (backward)
  auto load_coef = [&](int c, int b, bool fwd) {
    const int p0 = c * PC;
    for (int w = tid; w < (fwd ? 9 : 3) * PC; w += 256) {
      const int r = w / PC, q = w - r * PC;
      const int row = fwd ? r : 3 * r + 2;
      sco[b][row][q] = (p0 + q < nx) ? T(ldg(a.coef + (size_t)row * nx + p0 + q)) : T(0.);
    }
  };
  // the four fields of chunk c of the block's lines into buffer b, one commit group
  auto load_tile = [&](int c, int b) {
    const int p0 = c * PC;
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l >= nlines || p >= nx) continue;
      const R *fw = a.fw + (size_t)l * nx + p;
      if (p < nx - 1) __pipeline_memcpy_async(&sd[b][0][ll][tx], fw, sizeof(R));
      else sd[b][0][ll][tx] = R(0.);
      __pipeline_memcpy_async(&sd[b][1][ll][tx], fw + fstride, sizeof(R));
      __pipeline_memcpy_async(&sd[b][2][ll][tx], fw + 2 * fstride, sizeof(R));
      __pipeline_memcpy_async(&sd[b][3][ll][tx], fw + 3 * fstride, sizeof(R));
    }
    __pipeline_commit();
  };
  // chunk c (position `it` of the walk) in place: with two buffers the next
  // chunk of the walk is requested first and one group may stay in flight
  auto stage = [&](int it, int c, int cnext, bool fwd) {
    if (NB > 1 && it + 1 < nchunks) {
      load_coef(cnext, (it + 1) % NB, fwd);
      load_tile(cnext, (it + 1) % NB);
      __pipeline_wait_prior(1);
    } else {
      if (NB == 1 && it > 0) {
        load_coef(c, 0, fwd);
        load_tile(c, 0);
      }
      __pipeline_wait_prior(0);
    }
    __syncthreads();
  };
  T carry = T(0.);

  // ------------------------------------------------------------ forward
  load_coef(0, 0, true);
  load_tile(0, 0);
  for (int c = 0; c < nchunks; c++) {
    const int b = c % NB;
    const int p0 = c * PC;
    stage(c, c, c + 1, true);
    if (sweeper) {
      R *q = sd[b][f][tx];
      const T *L = sco[b][3 * set], *Rr = sco[b][3 * set + 1];
      const int smax = min(PC, nf - p0);
#pragma unroll 4
      for (int s = 0; s < smax; s++) {
        const int pp = p0 + s;
        const T x = T(q[s]);
        if (0 == pp) {
          carry = x / Rr[s];
        } else if (pp < nf - 1) {
          carry = Rr[s] * (x - L[s] * carry);
        } else {
          carry = (T(0.) != Rr[s]) ? Rr[s] * (x - L[s] * carry) : T(0.);
        }
        q[s] = R(carry);
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l >= nlines || p >= nx) continue;
      R *fw = a.fw + (size_t)l * nx + p;
      if (p < nx - 1) fw[0] = R(sd[b][0][ll][tx]);
      fw[fstride] = R(sd[b][1][ll][tx]);
      fw[2 * fstride] = R(sd[b][2][ll][tx]);
      fw[3 * fstride] = R(sd[b][3][ll][tx]);
    }
    __syncthreads();
  }

  // ------------------------------------------------------------ backward
  T nxt = T(0.);
  load_coef(nchunks - 1, 0, false);
  load_tile(nchunks - 1, 0);
  for (int it = 0; it < nchunks; it++) {
    const int c = nchunks - 1 - it;
    const int b = it % NB;
    const int p0 = c * PC;
    stage(it, c, c - 1, false);
    if (sweeper) {
      R *q = sd[b][f][tx];
      const T *V = sco[b][3 * set + 2];
      const int smax = min(PC, nf - p0);
#pragma unroll 4
      for (int s = smax - 1; s >= 0; s--) {
        const int pp = p0 + s;
        if (nf - 1 == pp) {
          nxt = T(q[s]);
        } else {
          nxt = T(q[s]) - V[s] * nxt;
          q[s] = R(nxt);
        }
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int m = 0; m < 4; m++) {
      const int ll = ty + 8 * m;
      const long l = l0 + ll;
      const int p = p0 + tx;
      if (l >= nlines || p >= nx) continue;
      const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
      if (p < nx - 1) {
        const int i = p + 2;
        const double v = ldg(a.ux + ix_ux(g, i, j, k)) + sd[b][0][ll][tx];
        for_images(j, k, ny, nz, true, [&](int jj, int kk) { a.ux_new[ix_ux(g, i, jj, kk)] = v; });
      }
      {
        const int i = p + 1;
        const long ic = ix_cc(g, i, j, k);
        const double vy = ldg(a.uy + ic) + sd[b][1][ll][tx];
        const double vz = ldg(a.uz + ic) + sd[b][2][ll][tx];
        const double vt = ldg(a.t + ic) + sd[b][3][ll][tx];
        for_images(j, k, ny, nz, true, [&](int jj, int kk) {
          const long o = ix_cc(g, i, jj, kk);
          a.uy_new[o] = vy;
          a.uz_new[o] = vz;
          a.t_new[o] = vt;
        });
      }
    }
    __syncthreads();
  }

  // ------------------------------------------------------------ walls
  // each interior row's wall cell takes its wall value; its halo images take
  // the value it held before (halo copy before the wall assignment)
  for (int w = tid; w < 2 * PL; w += 256) {
    const int ll = w % PL, side = w / PL;
    const long l = l0 + ll;
    if (l >= nlines) continue;
    const int j = 1 + (int)(l % ny), k = 1 + (int)(l / ny);
    {
      const int i = side ? nx + 1 : 1;
      const double old = ldg(a.ux + ix_ux(g, i, j, k));
      a.ux_new[ix_ux(g, i, j, k)] = 0.;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) { a.ux_new[ix_ux(g, i, jj, kk)] = old; });
    }
    {
      const int i = side ? nx + 1 : 0;
      const long ic = ix_cc(g, i, j, k);
      const double oy = ldg(a.uy + ic), oz = ldg(a.uz + ic), ot = ldg(a.t + ic);
      a.uy_new[ic] = side ? a.uy_xp : a.uy_xm;
      a.uz_new[ic] = side ? a.uz_xp : a.uz_xm;
      a.t_new[ic] = side ? a.t_xp : a.t_xm;
      for_images(j, k, ny, nz, false, [&](int jj, int kk) {
        const long o = ix_cc(g, i, jj, kk);
        a.uy_new[o] = oy;
        a.uz_new[o] = oz;
        a.t_new[o] = ot;
      });
    }
  }
}

template <class R>
cudaError_t predict_launch(cudaStream_t st, const Predict3Args<R> &a) {
  const Grid3 &g = a.g;
  dim3 gr((g.nx + RX - 1) / RX, (g.ny + RY - 1) / RY, (g.nz + RZ - 1) / RZ);
  if (0. != a.grav_vof) k3_rhs<R, true><<<gr, RX * RY, kRhsSmem<R>, st>>>(a);
  else k3_rhs<R, false><<<gr, RX * RY, kRhsSmem<R>, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (cudaSuccess != e) return e;
  const long nlines = (long)g.ny * g.nz;
  k3_xsolve<R><<<(unsigned)((nlines + PL - 1) / PL), 256, 0, st>>>(a);
  return cudaGetLastError();
}

template <class R>
cudaError_t predict_prepare_t() {
  const cudaError_t e = raise_smem_limit(k3_rhs<R, false>, kRhsSmem<R>);
  if (cudaSuccess != e) return e;
  return raise_smem_limit(k3_rhs<R, true>, kRhsSmem<R>);
}
#if SVOF3_WITH_F64
template cudaError_t predict_launch<double>(cudaStream_t, const Predict3Args<double> &);
template cudaError_t predict_prepare_t<double>();
#endif
#if SVOF3_WITH_F32
template cudaError_t predict_launch<float>(cudaStream_t, const Predict3Args<float> &);
template cudaError_t predict_prepare_t<float>();
#endif

#if SVOF3_WITH_F64
#if !SVOF3_WITH_F32
extern template cudaError_t predict_prepare_t<float>();
#endif
cudaError_t predict_prepare() {
  cudaError_t e = predict_prepare_t<double>();
  if (cudaSuccess != e) return e;
  return predict_prepare_t<float>();
}
#endif

}  // namespace svof3
