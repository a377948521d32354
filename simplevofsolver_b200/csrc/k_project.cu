// k_project.cu -- projection, pressure update, time-step and diagnostics
// kernels of the FP64 2D path.
//
//   k_project   u -= gamma dt grad psi (src/fluid/correct_velocity/{ux,uy}.c)
//               and p += psi - gamma dt nu / 2 Lx psi (src/fluid/update_pressure.c),
//               in place, with the halo rows and walls of
//               fluid_update_boundaries_{ux,uy,p}
//   k_cfl       min over faces of dx / (|u| + 1e-8) (src/fluid/decide_dt.c:28-64)
//   k_dt_final  safety factor and explicit-diffusion limits (:66-146)
//   k_diag      max |div u|, vof min / max / volume (src/logging/divergence.c:36-50,
//               src/logging/interface.c:22-39)
#include "svof_internal.cuh"

namespace svof {

// one thread per cell i in [1, nx], j in [1, ny]; the thread at i = nx also
// owns the ux column i = nx + 1
__global__ void k_project(double *__restrict__ ux, double *__restrict__ uy, double *__restrict__ p,
                          const double *__restrict__ psi, const double *__restrict__ dtp, double gam,
                          double m_dif, double uy_xm, double uy_xp, int do_vel, int do_p, Grid2 g) {
  pdl_enter();
  const int nx = g.nx, ny = g.ny;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i > nx || j > ny) return;
  const double dt = *dtp;
  const bool top = (1 == j), bottom = (ny == j);
  if (do_vel) {
    const double prefactor = gam * dt;  // correct_velocity/main.c:21-23
    // ux, correct_velocity/ux.c:16-41
    if (i >= 2) {
      const double dx = g.dxc[i - 1];
      const double psi_xm = psi[ix_cc(nx, i - 1, j)];
      const double psi_xp = psi[ix_cc(nx, i, j)];
      double v = ux[ix_ux(nx, i, j)];
      v -= prefactor / dx * (+psi_xp - psi_xm);
      ux[ix_ux(nx, i, j)] = v;
      if (bottom) ux[ix_ux(nx, i, 0)] = v;
      if (top) ux[ix_ux(nx, i, ny + 1)] = v;
    } else {
      // wall i = 1: halo rows take the value before the wall assignment
      const double w = ux[ix_ux(nx, 1, j)];
      if (bottom) ux[ix_ux(nx, 1, 0)] = w;
      if (top) ux[ix_ux(nx, 1, ny + 1)] = w;
      ux[ix_ux(nx, 1, j)] = 0.;
    }
    if (nx == i) {
      const double w = ux[ix_ux(nx, nx + 1, j)];
      if (bottom) ux[ix_ux(nx, nx + 1, 0)] = w;
      if (top) ux[ix_ux(nx, nx + 1, ny + 1)] = w;
      ux[ix_ux(nx, nx + 1, j)] = 0.;
    }
    // uy, correct_velocity/uy.c:15-39
    {
      const double psi_ym = psi[ix_cc(nx, i, j - 1)];
      const double psi_yp = psi[ix_cc(nx, i, j)];
      double v = uy[ix_cc(nx, i, j)];
      v -= prefactor / g.dy * (+psi_yp - psi_ym);
      uy[ix_cc(nx, i, j)] = v;
      if (bottom) uy[ix_cc(nx, i, 0)] = v;
      if (top) uy[ix_cc(nx, i, ny + 1)] = v;
    }
    if (1 == i) {
      const double w = uy[ix_cc(nx, 0, j)];
      if (bottom) uy[ix_cc(nx, 0, 0)] = w;
      if (top) uy[ix_cc(nx, 0, ny + 1)] = w;
      uy[ix_cc(nx, 0, j)] = uy_xm;
    }
    if (nx == i) {
      const double w = uy[ix_cc(nx, nx + 1, j)];
      if (bottom) uy[ix_cc(nx, nx + 1, 0)] = w;
      if (top) uy[ix_cc(nx, nx + 1, ny + 1)] = w;
      uy[ix_cc(nx, nx + 1, j)] = uy_xp;
    }
  }
  if (do_p) {
    // update_pressure.c:12-109 (x implicit)
    const double psi_c = psi[ix_cc(nx, i, j)];
    double v = p[ix_cc(nx, i, j)];
    v += psi_c;
    const double prefactor = 0.5 * gam * dt * m_dif;
    const double dpsidx_xm = (-psi[ix_cc(nx, i - 1, j)] + psi_c) / g.dxc[i - 1];
    const double dpsidx_xp = (-psi_c + psi[ix_cc(nx, i + 1, j)]) / g.dxc[i];
    v -= prefactor / g.dxf[i - 1] * (-dpsidx_xm + dpsidx_xp);
    p[ix_cc(nx, i, j)] = v;
    if (bottom) p[ix_cc(nx, i, 0)] = v;
    if (top) p[ix_cc(nx, i, ny + 1)] = v;
    // Neumann walls, boundary/p.c:7-20
    if (1 == i) {
      const double w = p[ix_cc(nx, 0, j)];
      if (bottom) p[ix_cc(nx, 0, 0)] = w;
      if (top) p[ix_cc(nx, 0, ny + 1)] = w;
      p[ix_cc(nx, 0, j)] = v;
    }
    if (nx == i) {
      const double w = p[ix_cc(nx, nx + 1, j)];
      if (bottom) p[ix_cc(nx, nx + 1, 0)] = w;
      if (top) p[ix_cc(nx, nx + 1, ny + 1)] = w;
      p[ix_cc(nx, nx + 1, j)] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// k_cfl: grid-stride over the ux faces i in [2, nx] and the uy faces
// i in [1, nx] of rows 1..ny.  All candidates are positive, so the minimum
// of their IEEE bit patterns (as unsigned integers) is the bit pattern of
// the minimum; NaN candidates sort above every finite value and are ignored,
// like fmin ignores them in the reference.  A non-finite velocity (NaN or
// Inf) sets bit 0 of *status (the failure detection the reference lacks:
// the host reports it at its next synchronisation).
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

__global__ void k_cfl(const double *__restrict__ ux, const double *__restrict__ uy,
                      unsigned long long *__restrict__ minbits, unsigned *__restrict__ status, Grid2 g) {
  pdl_enter();
  const int nx = g.nx, ny = g.ny;
  const double small = 1.e-8;
  unsigned long long best = 0x7ff0000000000000ull;  // +inf
  bool bad = false;
  const long nfx = (long)(nx - 1) * ny, nfy = (long)nx * ny;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < nfx + nfy; w += stride) {
    double cand;
    if (w < nfx) {
      const int i = 2 + (int)(w % (nx - 1));
      const int j = 1 + (int)(w / (nx - 1));
      const double dx = g.dxc[i - 1];
      const double au = fabs(ux[ix_ux(nx, i, j)]);
      bad |= !(au <= kDblMax);
      const double vel = au + small;
      cand = dx / vel;
    } else {
      const long v = w - nfx;
      const int i = 1 + (int)(v % nx);
      const int j = 1 + (int)(v / nx);
      const double av = fabs(uy[ix_cc(nx, i, j)]);
      bad |= !(av <= kDblMax);
      const double vel = av + small;
      cand = g.dy / vel;
    }
    const unsigned long long b = (unsigned long long)__double_as_longlong(cand);
    best = b < best ? b : best;
  }
  if (__any_sync(0xffffffffu, bad) && 0 == (threadIdx.x & 31)) atomicOr(status, 1u);
  best = warp_min_u64(best);
  __shared__ unsigned long long sbest[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (0 == lane) sbest[warp] = best;
  __syncthreads();
  if (0 == warp) {
    best = lane < (int)(blockDim.x >> 5) ? sbest[lane] : 0x7ff0000000000000ull;
    best = warp_min_u64(best);
    if (0 == lane) atomicMin(minbits, best);
  }
}

// decide_dt_adv tail and fluid_decide_dt (src/fluid/decide_dt.c:61-63, 129-143);
// dif_m_y, dif_t_y are decide_dt_dif's y limits, computed on the host.
// Resets the accumulator to the bit pattern of 1.0 (the initial *dt = 1.).
// A time step that is not a positive finite number sets bit 1 of *status.
__global__ void k_dt_final(unsigned long long *minbits, double *dt, double coef_adv, double dif_m_y,
                           double dif_t_y, unsigned *status) {
  pdl_enter();
  double dta = fmin(1., __longlong_as_double((long long)*minbits));
  dta *= coef_adv;
  double r = dta;
  r = fmin(r, dif_m_y);
  r = fmin(r, dif_t_y);
  *dt = r;
  if (!(r > 0. && r <= kDblMax)) atomicOr(status, 2u);
  *minbits = (unsigned long long)__double_as_longlong(1.);
}

// ---------------------------------------------------------------------------
// k_diag: one block, deterministic order; out = {divmax, vofmin, vofmax,
// sum vof dx dy, sum dx dy}.  Sums use a TwoSum-compensated accumulation.
__device__ __forceinline__ void two_sum_acc(double &s, double &c, double x) {
  const double t = s + x;
  const double bp = t - s;
  const double err = (s - (t - bp)) + (x - bp);
  s = t;
  c += err;
}

__global__ void k_diag(const double *__restrict__ ux, const double *__restrict__ uy,
                       const double *__restrict__ vof, double *__restrict__ out, Grid2 g) {
  const int nx = g.nx, ny = g.ny;
  double dmax = 0., vmin = 1., vmax = 0., s0 = 0., c0 = 0., s1 = 0., c1 = 0.;
  for (long w = threadIdx.x; w < (long)nx * ny; w += blockDim.x) {
    const int i = 1 + (int)(w % nx), j = 1 + (int)(w / nx);
    const double dx = g.dxf[i - 1];
    const double div = +(ux[ix_ux(nx, i + 1, j)] - ux[ix_ux(nx, i, j)]) / dx +
                       (uy[ix_cc(nx, i, j + 1)] - uy[ix_cc(nx, i, j)]) / g.dy;
    dmax = fmax(dmax, fabs(div));
    const double lv = vof[ix_vof(nx, i, j)];
    vmin = fmin(vmin, lv);
    vmax = fmax(vmax, lv);
    two_sum_acc(s0, c0, lv * (dx * g.dy));
    two_sum_acc(s1, c1, dx * g.dy);
  }
  __shared__ double red[5][1024];
  red[0][threadIdx.x] = dmax;
  red[1][threadIdx.x] = vmin;
  red[2][threadIdx.x] = vmax;
  red[3][threadIdx.x] = s0 + c0;
  red[4][threadIdx.x] = s1 + c1;
  __syncthreads();
  if (0 == threadIdx.x) {
    double a = 0., b = 1., c = 0., ss0 = 0., cc0 = 0., ss1 = 0., cc1 = 0.;
    for (int t = 0; t < (int)blockDim.x; t++) {
      a = fmax(a, red[0][t]);
      b = fmin(b, red[1][t]);
      c = fmax(c, red[2][t]);
      two_sum_acc(ss0, cc0, red[3][t]);
      two_sum_acc(ss1, cc1, red[4][t]);
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
    out[3] = ss0 + cc0;
    out[4] = ss1 + cc1;
  }
}

// ---------------------------------------------------------------------------
// k_logging: the logging reductions of src/logging/momentum.c:38-54,
// energy.c:41-65 and nusselt/{heat_flux,kinetic_energy_injection,
// kinetic_energy_dissipation,thermal_energy_dissipation}.c on the device,
// every term with the reference's expression and association; the sums are
// TwoSum-compensated, thread partials folded over a warp by a fixed
// butterfly and over the block in warp order (deterministic).  One block of
// kLogThreads threads walks the positions (i, j), i in [1, nx+1], j in
// [1, ny].  out = {momentum x, y; energy ux, uy, t; Nusselt from the wall
// heat flux, kinetic energy injection, kinetic and thermal energy
// dissipation}.
namespace {
constexpr int kLogThreads = 1024, kLogSums = 13;
struct CSum {
  double s = 0., c = 0.;
  __device__ __forceinline__ void add(double x) { two_sum_acc(s, c, x); }
  __device__ __forceinline__ void add(const CSum &o) {
    two_sum_acc(s, c, o.s);
    c += o.c;
  }
};
}  // namespace

__global__ void __launch_bounds__(kLogThreads) k_logging(const double *__restrict__ ux, const double *__restrict__ uy,
                                                         const double *__restrict__ t, double m_dif, double t_dif,
                                                         double ly, double *__restrict__ out, Grid2 g) {
  const int nx = g.nx, ny = g.ny;
  const double dy = g.dy, md = m_dif, td = t_dif;
  auto UX = [&](int i, int j) { return ux[ix_ux(nx, i, j)]; };
  auto UY = [&](int i, int j) { return uy[ix_cc(nx, i, j)]; };
  auto TT = [&](int i, int j) { return t[ix_cc(nx, i, j)]; };
  auto DXF = [&](int i) { return g.dxf[i - 1]; };
  auto DXC = [&](int i) { return g.dxc[i - 1]; };
  // 0 mx, 1 my, 2 ex, 3 ey, 4 et, 5 heat flux, 6 injection, 7..10 kinetic
  // dissipation (ux-x, ux-y, uy-x, uy-y), 11..12 thermal dissipation (x, y)
  CSum sum[kLogSums];
  const int npos = (nx + 1) * ny;
  for (int w = threadIdx.x; w < npos; w += kLogThreads) {
    const int i = 1 + w % (nx + 1), j = 1 + w / (nx + 1);
    // ---- ux faces i in [1, nx+1]
    {
      const double cs = DXC(i) * dy;
      if (2 <= i && i <= nx) {
        const double u = UX(i, j);
        sum[0].add(u * (DXC(i) * dy));
        sum[2].add(0.5 * (u * u) * (DXC(i) * dy));
        const double t_ = +0.5 * TT(i - 1, j) + 0.5 * TT(i, j);
        sum[6].add(u * t_ * (DXC(i) * dy));
      }
      if (1 != i) {
        const double d = 1. / DXF(i - 1) * (UX(i, j) - UX(i - 1, j));
        const double wt = DXF(i - 1) / DXC(i);
        sum[7].add(md * 0.5 * wt * (d * d) * cs);
      }
      if (nx + 1 != i) {
        const double d = 1. / DXF(i) * (UX(i + 1, j) - UX(i, j));
        const double wt = DXF(i) / DXC(i);
        sum[7].add(md * 0.5 * wt * (d * d) * cs);
      }
      const double dm = 1. / dy * (UX(i, j) - UX(i, j - 1));
      sum[8].add(md * 0.5 * (dm * dm) * cs);
      const double dp = 1. / dy * (UX(i, j + 1) - UX(i, j));
      sum[8].add(md * 0.5 * (dp * dp) * cs);
    }
    // ---- cells i in [1, nx]
    if (i <= nx) {
      const double cs = DXF(i) * dy;
      const double v = UY(i, j), tc = TT(i, j);
      sum[1].add(v * (DXF(i) * dy));
      sum[3].add(0.5 * (v * v) * (DXF(i) * dy));
      sum[4].add(0.5 * (tc * tc) * (DXF(i) * dy));
      const double w1m = 1 == i ? 2. : 1., w1p = nx == i ? 2. : 1.;
      {
        const double d = 1. / DXC(i) * (v - UY(i - 1, j));
        sum[9].add(md * 0.5 * (DXC(i) / DXF(i)) * w1m * (d * d) * cs);
      }
      {
        const double d = 1. / DXC(i + 1) * (UY(i + 1, j) - v);
        sum[9].add(md * 0.5 * (DXC(i + 1) / DXF(i)) * w1p * (d * d) * cs);
      }
      {
        const double dm = 1. / dy * (v - UY(i, j - 1));
        sum[10].add(md * 0.5 * (dm * dm) * cs);
        const double dp = 1. / dy * (UY(i, j + 1) - v);
        sum[10].add(md * 0.5 * (dp * dp) * cs);
      }
      {
        const double d = 1. / DXC(i) * (tc - TT(i - 1, j));
        sum[11].add(td * 0.5 * (DXC(i) / DXF(i)) * w1m * (d * d) * cs);
      }
      {
        const double d = 1. / DXC(i + 1) * (TT(i + 1, j) - tc);
        sum[11].add(td * 0.5 * (DXC(i + 1) / DXF(i)) * w1p * (d * d) * cs);
      }
      {
        const double dm = 1. / dy * (tc - TT(i, j - 1));
        sum[12].add(td * 0.5 * (dm * dm) * cs);
        const double dp = 1. / dy * (TT(i, j + 1) - tc);
        sum[12].add(td * 0.5 * (dp * dp) * cs);
      }
    }
    // ---- the wall heat flux of row j
    if (1 == i) {
      const double dtdx_xm = (+TT(1, j) - TT(0, j)) / DXC(1);
      const double dtdx_xp = (+TT(nx + 1, j) - TT(nx, j)) / DXC(nx + 1);
      sum[5].add(-(0.5 * td * (dtdx_xm + dtdx_xp) * dy));
    }
  }
  // warp butterfly, then warp order
#pragma unroll
  for (int q = 0; q < kLogSums; q++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      CSum x;
      x.s = __shfl_xor_sync(0xffffffffu, sum[q].s, o);
      x.c = __shfl_xor_sync(0xffffffffu, sum[q].c, o);
      sum[q].add(x);
    }
  }
  __shared__ CSum red[kLogSums][kLogThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (0 == lane) {
#pragma unroll
    for (int q = 0; q < kLogSums; q++) red[q][warp] = sum[q];
  }
  __syncthreads();
  if (threadIdx.x < kLogSums) {
    const int q = threadIdx.x;
    CSum r = red[q][0];
    for (int w = 1; w < kLogThreads / 32; w++) r.add(red[q][w]);
    red[q][0] = r;
  }
  __syncthreads();
  if (0 == threadIdx.x) {
    auto v = [&](int q) { return red[q][0].s + red[q][0].c; };
    const double ref = td * ly;  // laminar heat flux (nusselt/reference.c:4-12)
    out[0] = v(0);
    out[1] = v(1);
    out[2] = v(2);
    out[3] = v(3);
    out[4] = v(4);
    out[5] = v(5) / ref;
    out[6] = v(6) / ref + 1.;
    out[7] = (((v(7) + v(8)) + v(9)) + v(10)) / ref + 1.;
    out[8] = (v(11) + v(12)) / ref;
  }
}

}  // namespace svof
