// k3_interface.cu -- boundary and interface (VOF) kernels of the 3D path.
//
// The kernels are templates on R, the type of the interface intermediates
// (curvature, normals, forces) and of the geometry and THINC arithmetic:
// R = double is the FP64 path, which follows the restatement bit for bit
// except for exp / log; R = float is the mixed path, where vof, the
// velocities and the vof sources stay FP64, the geometry and the THINC flux
// evaluations run in FP32 and the intercept's Newton iteration in FP64.
//
//   k3_halo_bc     periodic y and z halos + x wall values of one field
//   k3_geom        corner normals (2x2x2 differences), cell normal and THINC
//                  intercept (2x2x2 Gauss points), curvature
//   k3_force       CSF surface-tension force in x, y, z
//   k3_vof_advect  THINC/QQ face fluxes, flux divergence, RK update of vof
//                  with its two-layer halo and zero walls
//
// The arithmetic is that of oracle/svof_oracle3d.c, which carries the
// reference's 2D expressions (src/interface/curvature_tensor.c:14-186,
// force.c:11-76, update/{flxx,flxy,main}.c) to z.  Geometry and advection
// march along z through a 32 x 4 tile: each plane's inputs are read once,
// the corner normals of the plane below and the z-face flux of the cell below
// are kept from the previous plane.
#include <cuda_pipeline.h>

#include "svof3d_internal.cuh"
#include "smem_limit.cuh"

// Precision split of this translation unit: built twice, once with
// SVOF3_PRECISION=64 (the FP64 instantiations and the shared non-template
// code, FMA contraction off as for every FP64 kernel) and once with
// SVOF3_PRECISION=32 (the mixed path's FP32 instantiations only, FMA on).
// Without the macro both are built in one pass.
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

static __constant__ double c3_gauss_p[2] = {-0.2886751345948129, +0.2886751345948129};
static __constant__ double c3_gauss_w[2] = {+0.5, +0.5};
constexpr double kVofBeta = 1.;
constexpr double kVofMin = 1.e-8;

// ---------------------------------------------------------------------------
// k3_halo_bc: one thread per storage cell c of an interior row (j, k).  The
// restatement copies the y halo rows of every interior plane, then whole z
// halo planes, then assigns the x wall values of the interior rows; vof walls
// are zero in every row.  A halo row therefore holds the values its source
// row had before the wall assignment.
#if SVOF3_WITH_F64
__global__ void k3_halo_bc(double *a, int width, int nh, int ny, int nz, int kind, double lo, double hi) {
  const long w = width;
  const long tot = w * ny * nz;
  const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= tot) return;
  const int c = (int)(id % w);
  const long row = id / w;
  const int r = nh + (int)(row % ny);  // stored y index of the interior row
  const int q = nh + (int)(row / ny);  // stored z index
  const long rows = ny + 2 * nh;
  auto at = [&](int rr, int qq) -> double & { return a[w * (rr + rows * qq) + c]; };
  const double old = at(r, q);
  int rs[2], qs[2], nr = 1, nq = 1;
  rs[0] = r;
  qs[0] = q;
  if (r - ny >= 0 && r - ny < nh) rs[nr++] = r - ny;
  if (r + ny >= ny + nh && r + ny < ny + 2 * nh) rs[nr++] = r + ny;
  if (q - nz >= 0 && q - nz < nh) qs[nq++] = q - nz;
  if (q + nz >= nz + nh && q + nz < nz + 2 * nh) qs[nq++] = q + nz;
  const bool left = (0 == c), right = (width - 1 == c);
  double val = old, img = old;
  if (BC3_VOF == kind) {
    if (left || right) val = img = 0.;
  } else if (left || right) {
    if (BC3_ZERO == kind) val = 0.;
    else if (BC3_DIRICHLET == kind) val = left ? lo : hi;
    else val = left ? a[w * (r + rows * q) + 1] : a[w * (r + rows * q) + width - 2];
  }
  for (int x = 0; x < nq; x++)
    for (int y = 0; y < nr; y++) {
      if (0 == x && 0 == y) continue;
      at(rs[y], qs[x]) = img;
    }
  at(r, q) = val;
}
#endif

template <class T>
__device__ __forceinline__ T plane_dx(T v00, T v10, T v01, T v11) {
  return -v00 + v10 - v01 + v11;
}
template <class T>
__device__ __forceinline__ T plane_dy(T v00, T v10, T v01, T v11) {
  return -v00 - v10 + v01 + v11;
}
template <class T>
__device__ __forceinline__ T plane_sum(T v00, T v10, T v01, T v11) {
  return +v00 + v10 + v01 + v11;
}

// 1 / max(|v|, eps) for |v|^2 = s: the restatement's form in FP64; in FP32 a
// reciprocal square root of max(s, eps^2), which stays on the fast path for
// the vanishing gradients of the vof tails
__device__ __forceinline__ double rnorm(double s, double eps) { return 1. / fmax(sqrt(s), eps); }
__device__ __forceinline__ float rnorm(float s, float eps) { return rsqrtf(fmaxf(s, eps * eps)); }
// x / y: a division in FP64, a multiplication by the reciprocal in FP32
__device__ __forceinline__ double div_by(double x, double y) { return x / y; }
__device__ __forceinline__ float div_by(float x, float y) { return x * (1.f / y); }

// THINC intercept with 2 x 2 x 2 Gauss points (compute_intercept3 of the
// restatement; src/interface/curvature_tensor.c:50-92 in 2D), Newton
// tolerance 1e-12.  `converged` tells whether the residual fell below the
// tolerance within the 8 iterations (the value is the last iterate either way).
template <class R>
__device__ __forceinline__ R thinc_intercept3(const R vof, const R n0, const R n1, const R n2, bool &converged) {
  const int cntmax = 8;
  const R resmax = R(1.e-12);
  const R gp0 = R(c3_gauss_p[0]), gp1 = R(c3_gauss_p[1]), gw = R(c3_gauss_w[0]);
  const R gp[2] = {gp0, gp1};
  R exps[8];
#pragma unroll
  for (int kk = 0; kk < 2; kk++)
#pragma unroll
    for (int jj = 0; jj < 2; jj++)
#pragma unroll
      for (int ii = 0; ii < 2; ii++)
        exps[(kk * 2 + jj) * 2 + ii] = exp(R(-2.) * R(kVofBeta) * (+n0 * gp[ii] + n1 * gp[jj] + n2 * gp[kk]));
  R val = R(1.) / vof - R(1.);
  for (int cnt = 0; cnt < cntmax; cnt++) {
    R f0 = R(-1.) * vof;
    R f1 = R(0.);
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
#pragma unroll
      for (int jj = 0; jj < 2; jj++) {
#pragma unroll
        for (int ii = 0; ii < 2; ii++) {
          const R weight = gw * gw * gw;
          const R p = exps[(kk * 2 + jj) * 2 + ii];
          const R denom = R(1.) / (R(1.) + p * val);
          f0 += weight * denom;
          f1 -= weight * p * denom * denom;
        }
      }
    }
    val -= f0 / f1;
    if (fabs(f0) < resmax) {
      converged = true;
      break;
    }
  }
  return R(-0.5) / R(kVofBeta) * log(val);
}

// four normal components per cell: two double2 / one float4
__device__ __forceinline__ void store_normal3(double *o, double n0, double n1, double n2) {
  reinterpret_cast<double2 *>(o)[0] = make_double2(n0, n1);
  o[2] = n2;
}
__device__ __forceinline__ void store_normal3(float *o, float n0, float n1, float n2) {
  reinterpret_cast<float2 *>(o)[0] = make_float2(n0, n1);
  o[2] = n2;
}
__device__ __forceinline__ void load_normal(const double *__restrict__ normal, long idx, double *n) {
  const double2 *p = reinterpret_cast<const double2 *>(normal + idx);
  const double2 a = __ldg(p), b = __ldg(p + 1);
  n[0] = a.x;
  n[1] = a.y;
  n[2] = b.x;
  n[3] = b.y;
}
__device__ __forceinline__ void load_normal(const float *__restrict__ normal, long idx, float *n) {
  const float4 a = __ldg(reinterpret_cast<const float4 *>(normal + idx));
  n[0] = a.x;
  n[1] = a.y;
  n[2] = a.z;
  n[3] = a.w;
}

// ---------------------------------------------------------------------------
// k3_geom: cells i in [1, nx], j in [0, ny+1], k in [0, nz+1] (halo cells
// included, as the restatement computes them).  Block: 32 x 4 cells of one
// plane, marching over G3Z planes; shared memory holds a ring of vof planes
// (34 x 6, FP64), G3D planes in flight ahead of the two being read, and two
// planes of corner normals (33 x 5 x 3, R).  The vof differences are taken
// in FP64 and then carried in R.
constexpr int G3X = 32, G3Y = 4, G3Z = 32, G3D = 4, G3S = G3D + 2;

template <class R>
__global__ void __launch_bounds__(G3X * G3Y) k3_geom(const double *__restrict__ vof, R *__restrict__ normal,
                                                    R *__restrict__ curv, unsigned *__restrict__ work,
                                                    unsigned *__restrict__ nwork, Grid3 g) {
  __shared__ double sv[G3S][G3Y + 2][G3X + 2];  // vof planes, plane p in slot (p - k0 + 1) % G3S
  __shared__ R sc[2][3][G3Y + 1][G3X + 1];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int i0 = 1 + blockIdx.x * G3X;
  const int j0 = blockIdx.y * G3Y;
  const int k0 = blockIdx.z * G3Z;
  const int kend = min(k0 + G3Z, nz + 2);  // cells k in [k0, kend)
  const int tid = threadIdx.x;
  const int tx = tid % G3X, ty = tid / G3X;
  const R eps = R(kDblEpsilon);
  const R rdy = R(1.) / R(g.dy), rdz = R(1.) / R(g.dz);
  // cp.async: planes arrive G3D ahead of the one being processed; the window
  // elements a thread copies are the same on every plane, their in-plane
  // offsets computed once (-1: zero fill, -2: no element).  Every thread
  // commits one group per plane slot (empty past the block's last plane), so
  // that a plane's group is always a fixed number of groups behind the newest
  constexpr int NT = G3X * G3Y, NW = ((G3X + 2) * (G3Y + 2) + NT - 1) / NT;
  const long vplane = (long)(nx + 2) * (ny + 4);
  int woff[NW];
#pragma unroll
  for (int q = 0; q < NW; q++) {
    const int t = tid + NT * q, li = t % (G3X + 2), lj = t / (G3X + 2);
    const int i = i0 - 1 + li, j = j0 - 1 + lj;
    woff[q] = (t >= (G3X + 2) * (G3Y + 2)) ? -2 : ((i <= nx + 1 && j <= ny + 2) ? i + (nx + 2) * (j + 1) : -1);
  }
  auto load_plane = [&](int k) {
    const int buf = (k - k0 + 1) % G3S;
    const double *vp = vof + vplane * (k + 1);
    double *d = &sv[buf][0][0];
#pragma unroll
    for (int q = 0; q < NW; q++) {
      if (woff[q] >= 0) __pipeline_memcpy_async(d + tid + NT * q, vp + woff[q], 8);
      else if (-1 == woff[q]) d[tid + NT * q] = 0.;
    }
    __pipeline_commit();
  };
  for (int p = k0 - 1; p < k0 + G3D; p++) {
    if (p <= kend) load_plane(p);
    else __pipeline_commit();
  }
  // 1 / dxc of the (up to two) corner columns this thread handles and 1 / dxf
  // of its cell column, once (the same values as per corner / cell)
  R rdxc[2] = {R(0.), R(0.)};
  for (int t = tid, q = 0; t < (G3X + 1) * (G3Y + 1) && q < 2; t += G3X * G3Y, q++) {
    const int ic = i0 + t % (G3X + 1);
    if (ic <= nx + 1) rdxc[q] = R(1.) / R(ldg(g.dxc + ic - 1));
  }
  const R rdxf = (i0 + tx <= nx) ? R(1.) / R(ldg(g.dxf + i0 + tx - 1)) : R(0.);
  // whether this thread's window elements of a plane (its own copies and zero
  // fills, complete after its wait) are all +0: the block's vote, taken at a
  // barrier, tells whether the whole window of the plane is +0
  auto my_zero = [&](int buf) {
    const double *d = &sv[buf][0][0];
    int z = 1;
#pragma unroll
    for (int q = 0; q < NW; q++)
      if (woff[q] >= -1 && 0 != __double_as_longlong(d[tid + NT * q])) z = 0;
    return z;
  };
  __pipeline_wait_prior(G3D - 1);             // planes k0 - 1 and k0
  int z_lo = __syncthreads_and(my_zero(0));  // plane kc - 1 all +0
  int z_hi = __syncthreads_and(my_zero(1));  // plane kc all +0
  R l_dx0 = R(0.), l_dy1 = R(0.), l_s0 = R(0.), l_s1 = R(0.), l_s2 = R(0.);  // lower corner plane
  for (int kc = k0; kc <= kend; kc++) {
    const int bcur = (kc - k0 + 1) % G3S, bprev = (kc - k0) % G3S;
    const int ccur = (kc - k0) & 1;
    // plane kc + G3D into the slot of plane kc - 2 (read last in the
    // previous iteration, before its closing barrier)
    if (kc + G3D <= kend) load_plane(kc + G3D);
    else __pipeline_commit();
    // both vof planes of the corner plane kc all +0 (the gas bulk, most of
    // the domain): every corner is flat, every corner normal +0 and so every
    // 2 x 2 stencil sum below; the corner pass and its barrier are skipped
    // (block-uniform), the cells take the +0 sums
    const bool flat_tile = z_lo && z_hi;
    // compute_gradient at corners (ic, jc, kc): planes kc-1 (bprev) and kc (bcur)
    if (!flat_tile) {
      for (int t = tid, q = 0; t < (G3X + 1) * (G3Y + 1); t += G3X * G3Y, q++) {
        const int li = t % (G3X + 1), lj = t / (G3X + 1);
        const int ic = i0 + li, jc = j0 + lj;
        R d0 = R(0.), d1 = R(0.), d2 = R(0.);
        if (ic <= nx + 1 && jc <= ny + 2) {
          const double a00 = sv[bprev][lj][li], a10 = sv[bprev][lj][li + 1];
          const double a01 = sv[bprev][lj + 1][li], a11 = sv[bprev][lj + 1][li + 1];
          const double b00 = sv[bcur][lj][li], b10 = sv[bcur][lj][li + 1];
          const double b01 = sv[bcur][lj + 1][li], b11 = sv[bcur][lj + 1][li + 1];
          // eight bit-identical values (the bulk outside the droplets): every
          // difference is +0, so the normal is +0 (+0 times 1 / eps) without
          // the square root and division
          const long long r = __double_as_longlong(a00);
          const bool flat = r == __double_as_longlong(a10) && r == __double_as_longlong(a01) &&
                            r == __double_as_longlong(a11) && r == __double_as_longlong(b00) &&
                            r == __double_as_longlong(b10) && r == __double_as_longlong(b01) &&
                            r == __double_as_longlong(b11);
          if (!flat) {
            const R dvofdx = rdxc[q] * R(plane_dx(a00, a10, a01, a11) + plane_dx(b00, b10, b01, b11));
            const R dvofdy = rdy * R(plane_dy(a00, a10, a01, a11) + plane_dy(b00, b10, b01, b11));
            const R dvofdz = rdz * R(plane_sum(b00, b10, b01, b11) - plane_sum(a00, a10, a01, a11));
            const R norminv = rnorm(+dvofdx * dvofdx + dvofdy * dvofdy + dvofdz * dvofdz, eps);
            d0 = dvofdx * norminv;
            d1 = dvofdy * norminv;
            d2 = dvofdz * norminv;
          }
        }
        sc[ccur][0][lj][li] = d0;
        sc[ccur][1][lj][li] = d1;
        sc[ccur][2][lj][li] = d2;
      }
      __syncthreads();
    }
    // the corner plane kc's 2 x 2 stencils of this thread's cell column: the
    // upper plane of cell k = kc - 1 now, the lower plane of cell kc next
    // (carried in registers, so each is formed once, with the same operands
    // in the same order)
    const int i = i0 + tx, j = j0 + ty;
    const bool cell = i <= nx && j <= ny + 1;
    R u_dx0 = R(0.), u_dy1 = R(0.), u_s0 = R(0.), u_s1 = R(0.), u_s2 = R(0.);
    if (cell && !flat_tile) {
#define CU(m, a, b) sc[ccur][m][ty + (b)][tx + (a)]
      u_dx0 = plane_dx(CU(0, 0, 0), CU(0, 1, 0), CU(0, 0, 1), CU(0, 1, 1));
      u_dy1 = plane_dy(CU(1, 0, 0), CU(1, 1, 0), CU(1, 0, 1), CU(1, 1, 1));
      u_s0 = plane_sum(CU(0, 0, 0), CU(0, 1, 0), CU(0, 0, 1), CU(0, 1, 1));
      u_s1 = plane_sum(CU(1, 0, 0), CU(1, 1, 0), CU(1, 0, 1), CU(1, 1, 1));
      u_s2 = plane_sum(CU(2, 0, 0), CU(2, 1, 0), CU(2, 0, 1), CU(2, 1, 1));
#undef CU
    }
    if (kc > k0) {
      // cells of plane k = kc - 1: corners kc - 1 (lower, carried) and kc (upper)
      const int k = kc - 1;
      bool inter = false;
      if (cell) {
        const R dxf = R(ldg(g.dxf + i - 1));
        const R dnxdx = rdxf * (l_dx0 + u_dx0);
        const R dnydy = rdy * (l_dy1 + u_dy1);
        const R dnzdz = rdz * (u_s2 - l_s2);
        curv[ix_cc(g, i, j, k)] = R(0.25) * (-dnxdx - dnydy - dnzdz);
        const double lvof = sv[bprev][ty + 1][tx + 1];
        if (!(lvof < kVofMin || 1. - kVofMin < lvof)) {
          R n0 = l_s0 + u_s0;
          R n1 = l_s1 + u_s1;
          R n2 = l_s2 + u_s2;
          n0 = div_by(n0, dxf);
          n1 = div_by(n1, R(g.dy));
          n2 = div_by(n2, R(g.dz));
          const R norminv = rnorm(+n0 * n0 + n1 * n1 + n2 * n2, eps);
          n0 *= norminv;
          n1 *= norminv;
          n2 *= norminv;
          store_normal3(normal + ix_nrm(g, i, j, k), n0, n1, n2);
          inter = true;
        }
      }
      // the intercept's Newton iteration runs in k3_intercept over a compacted
      // list of the interfacial cells (warp-aggregated append)
      const unsigned mask = __ballot_sync(0xffffffffu, inter);
      if (mask) {
        const int lane = tid & 31;
        unsigned base = 0;
        if (lane == __ffs(mask) - 1) base = atomicAdd(nwork, (unsigned)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
        if (inter) {
          const unsigned rank = __popc(mask & ((1u << lane) - 1u));
          work[base + rank] = (unsigned)(ix_nrm(g, i, j, k) >> 2);
        }
      }
    }
    l_dx0 = u_dx0;
    l_dy1 = u_dy1;
    l_s0 = u_s0;
    l_s1 = u_s1;
    l_s2 = u_s2;
    __pipeline_wait_prior(G3D - 1);  // plane kc + 1
    const int zn = __syncthreads_and(kc + 1 <= kend ? my_zero((kc - k0 + 2) % G3S) : 1);
    z_lo = z_hi;
    z_hi = zn;
  }
}

// k3_intercept: THINC intercept of every listed interfacial cell (the normal
// vector is already stored); one thread per cell, grid-stride over the list.
// The Newton iteration runs in FP64 in both precisions: near-full cells
// (1 - vof below FP32 resolution) have no FP32 solution, and the list holds
// only the interfacial cells.  With `unconverged` given, the cells whose
// iteration did not converge are added to it (one atomic per warp).
template <class R>
__global__ void __launch_bounds__(256) k3_intercept(const double *__restrict__ vof, R *__restrict__ normal,
                                                   const unsigned *__restrict__ work,
                                                   const unsigned *__restrict__ nwork, Grid3 g,
                                                   unsigned long long *__restrict__ unconverged) {
  const unsigned n = *nwork;
  const int nx = g.nx, rows = g.ny + 2;
  unsigned missed = 0;
  for (unsigned w = blockIdx.x * blockDim.x + threadIdx.x; w < n; w += gridDim.x * blockDim.x) {
    const unsigned c = work[w];
    const int i = 1 + (int)(c % (unsigned)nx);
    const unsigned r = c / (unsigned)nx;
    const int j = (int)(r % (unsigned)rows), k = (int)(r / (unsigned)rows);
    R *o = normal + 4L * c;
    bool converged = false;
    o[3] = R(thinc_intercept3<double>(ldg(vof + ix_vof(g, i, j, k)), (double)o[0], (double)o[1], (double)o[2],
                                      converged));
    missed += converged ? 0u : 1u;
  }
  // every thread of the block reaches this point (no early return)
  missed = __reduce_add_sync(0xffffffffu, missed);
  if (unconverged && missed && 0 == (threadIdx.x & 31)) atomicAdd(unconverged, (unsigned long long)missed);
}

// ---------------------------------------------------------------------------
// k3_force: one thread per interior (i, j) and kForcePlanes planes k (vof and
// curvature at k - 1 carried from the previous plane, the loads of the
// thread's planes issued before its arithmetic); FP64 arithmetic, R output
constexpr int kForcePlanes = 8;
template <class R>
__global__ void __launch_bounds__(256) k3_force(const double *__restrict__ vof, const R *__restrict__ curv,
                                                R *__restrict__ ifrcx, R *__restrict__ ifrcy, R *__restrict__ ifrcz,
                                                double tension, Grid3 g) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = 1 + blockIdx.z * kForcePlanes;
  if (i > g.nx || j > g.ny || k0 > g.nz) return;
  const double rdxc = (i >= 2) ? 1. / ldg(g.dxc + i - 1) : 0., rdy = 1. / g.dy, rdz = 1. / g.dz;
  double vc[kForcePlanes], vxm[kForcePlanes], vym[kForcePlanes], cc[kForcePlanes], cxm[kForcePlanes],
      cym[kForcePlanes];
#pragma unroll
  for (int h = 0; h < kForcePlanes; h++) {
    const int k = min(k0 + h, g.nz);
    vc[h] = ldg(vof + ix_vof(g, i, j, k));
    vxm[h] = ldg(vof + ix_vof(g, i - 1, j, k));
    vym[h] = ldg(vof + ix_vof(g, i, j - 1, k));
    cc[h] = (double)__ldg(curv + ix_cc(g, i, j, k));
    cxm[h] = (double)__ldg(curv + ix_cc(g, i - 1, j, k));
    cym[h] = (double)__ldg(curv + ix_cc(g, i, j - 1, k));
  }
  double vzm = ldg(vof + ix_vof(g, i, j, k0 - 1)), czm = (double)__ldg(curv + ix_cc(g, i, j, k0 - 1));
#pragma unroll
  for (int h = 0; h < kForcePlanes; h++) {
    const int k = k0 + h;
    if (k > g.nz) break;
    if (i >= 2) {
      const double grad = rdxc * (-vxm[h] + vc[h]);
      const double kappa = 0.5 * (+cxm[h] + cc[h]);
      ifrcx[ix_srcx(g, i, j, k)] = R(tension * grad * kappa);
    }
    {
      const double grad = rdy * (-vym[h] + vc[h]);
      const double kappa = 0.5 * (+cym[h] + cc[h]);
      ifrcy[ix_src(g, i, j, k)] = R(tension * grad * kappa);
    }
    {
      const double grad = rdz * (-vzm + vc[h]);
      const double kappa = 0.5 * (+czm + cc[h]);
      ifrcz[ix_src(g, i, j, k)] = R(tension * grad * kappa);
    }
    vzm = vc[h];
    czm = cc[h];
  }
}

// ---------------------------------------------------------------------------
// THINC/QQ flux helpers (indicator3 and the face fluxes of the restatement):
// the indicator sums run in R, the flux vel * sum in FP64
__device__ __forceinline__ double indicator3(const double *n, double x0, double x1, double x2) {
  return 1. / (1. + exp(-2. * kVofBeta * (+n[0] * x0 + n[1] * x1 + n[2] * x2 + n[3])));
}
__device__ __forceinline__ float indicator3(const float *n, float x0, float x1, float x2) {
  return __fdividef(1.f, 1.f + expf(-2.f * (float)kVofBeta * (+n[0] * x0 + n[1] * x1 + n[2] * x2 + n[3])));
}

// flux through one face given its velocity and the vof of the cells below
// (lo) and above (hi) it along the face normal, AXIS 0 / 1 / 2 = x / y / z
// (update/flx{x,y}.c and the restatement's z face): the upwind cell's
// vof times the velocity outside the interface, else the velocity times the
// 2 x 2 Gauss-point THINC indicator of the upwind cell on the face
template <class R, int AXIS>
__device__ __forceinline__ double face_flux(double vel, double vlo, double vhi, const R *__restrict__ normal,
                                            long nrm_lo, long nrm_hi) {
  const bool neg = vel < 0.;
  const double lvof = neg ? vhi : vlo;
  if (lvof < kVofMin || 1. - kVofMin < lvof) return vel * lvof;
  const R c = neg ? R(-0.5) : R(+0.5);
  R n[4];
  load_normal(normal, neg ? nrm_hi : nrm_lo, n);
  R flux = R(0.);
#pragma unroll
  for (int b = 0; b < 2; b++)
#pragma unroll
    for (int a = 0; a < 2; a++) {
      const R pa = R(c3_gauss_p[a]), pb = R(c3_gauss_p[b]);
      const R wgt = R(c3_gauss_w[a]) * R(c3_gauss_w[b]);
      if (0 == AXIS) flux += wgt * indicator3(n, c, pa, pb);
      else if (1 == AXIS) flux += wgt * indicator3(n, pa, c, pb);
      else flux += wgt * indicator3(n, pa, pb, c);
    }
  return vel * (double)flux;
}

// k3_vof_advect: cells i in [1, nx], j in [1, ny], k in [1, nz].  A block
// owns a 32 x 8 tile of (i, j) and marches along z over AZ planes; vof (34 x
// 10 windows), the x and y face velocities of the tile, the z face velocities
// and src_b live in a ring of four shared-memory planes that cp.async fills
// two planes ahead.  The x and y face fluxes of a plane are staged in shared
// memory; the z-face flux below a cell is the one above it in the previous
// plane.  Writes vof_new with its halo images (two layers) and zero x walls,
// and src_a.  The flux divergence and the update are FP64 in both
// precisions, so that the update conserves volume to FP64 round-off.
constexpr int AX = 32, AY = 8, AZ = 32, AWX = AX + 2, AWY = AY + 2, ASLOT = 4;
constexpr int kVofRing = ASLOT * AWY * AWX, kUxRing = ASLOT * AY * (AX + 1), kUyRing = ASLOT * (AY + 1) * AX;
constexpr int kUzRing = ASLOT * AY * AX, kSbRing = ASLOT * AY * AX;
constexpr size_t kAdvectSmem =
    sizeof(double) * (kVofRing + kUxRing + kUyRing + kUzRing + kSbRing + AY * (AX + 1) + (AY + 1) * AX);

template <class R>
__global__ void __launch_bounds__(AX * AY, 4) k3_vof_advect(const double *__restrict__ vof, double *__restrict__ vof_new,
                                                        const double *__restrict__ ux, const double *__restrict__ uy,
                                                        const double *__restrict__ uz, const R *__restrict__ normal,
                                                        double *__restrict__ src_a, const double *__restrict__ src_b,
                                                        const double *__restrict__ dtp, RK rk, int use_b, Grid3 g) {
  extern __shared__ double sm[];
  double *vr = sm;                  // [ASLOT][AWY][AWX]  vof, rows j0-1.., cols i0-1..
  double *xr = vr + kVofRing;       // [ASLOT][AY][AX+1]  ux faces i0 .. i0+32
  double *yr = xr + kUxRing;        // [ASLOT][AY+1][AX]  uy faces j0 .. j0+8
  double *zr = yr + kUyRing;        // [ASLOT][AY][AX]    uz face k (plane k)
  double *br = zr + kUzRing;        // [ASLOT][AY][AX]    src_b
  double *fx = br + kSbRing;        // [AY][AX+1]
  double *fy = fx + AY * (AX + 1);  // [AY+1][AX]
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tid = threadIdx.x, tx = tid % AX, ty = tid / AX;
  const int i0 = 1 + blockIdx.x * AX, j0 = 1 + blockIdx.y * AY, k0 = 1 + blockIdx.z * AZ;
  const int kend = min(k0 + AZ, nz + 1);  // cells k in [k0, kend)
  const int i = i0 + tx, j = j0 + ty;
  const bool mine = (i <= nx && j <= ny);
  const long vw = nx + 2, vrows = ny + 4, uw = nx + 1, crow = ny + 2;
  const long vplane = vw * vrows, uplane = uw * crow, cplane = vw * crow, splane = (long)nx * ny;
  const long nplane = 4L * nx * crow;  // normal array, per plane k
  auto cp = [](double *dst, const double *src) { __pipeline_memcpy_async(dst, src, sizeof(double)); };
  // The copies and faces a thread handles are the same on every plane: their
  // in-plane offsets are computed once (-1: zero fill, -2: no element).
  constexpr int NT = AX * AY;
  constexpr int NV = (AWY * AWX + NT - 1) / NT, NXF = (AY * (AX + 1) + NT - 1) / NT,
                NYF = ((AY + 1) * AX + NT - 1) / NT;
  int vsrc[NV], xsrc[NXF], ysrc[NYF];
#pragma unroll
  for (int q = 0; q < NV; q++) {
    const int e = tid + NT * q, r = e / AWX, c = e - r * AWX;
    const int x = i0 - 1 + c, jj = j0 - 1 + r;
    vsrc[q] = (e >= AWY * AWX) ? -2 : ((x <= nx + 1 && jj <= ny + 2) ? (int)(x + vw * (jj + 1)) : -1);
  }
#pragma unroll
  for (int q = 0; q < NXF; q++) {
    const int e = tid + NT * q, r = e / (AX + 1), c = e - r * (AX + 1);
    const int fi = i0 + c, jj = j0 + r;  // face fi, storage fi - 1
    xsrc[q] = (e >= AY * (AX + 1)) ? -2 : ((fi <= nx + 1 && jj <= ny) ? (int)((fi - 1) + uw * jj) : -1);
  }
#pragma unroll
  for (int q = 0; q < NYF; q++) {
    const int e = tid + NT * q, r = e / AX, c = e - r * AX;
    const int ii = i0 + c, fj = j0 + r;
    ysrc[q] = (e >= (AY + 1) * AX) ? -2 : ((ii <= nx && fj <= ny + 1) ? (int)(ii + vw * fj) : -1);
  }
  const int zsrc = (int)(i + vw * j), bsrc = (i - 1) + nx * (j - 1);
  auto load_plane = [&](int kk) {
    const int sl = kk & (ASLOT - 1);
    // vof window, planes k0 - 1 .. kend + 1
    const double *vp = vof + vplane * (kk + 1);
    double *vd = vr + (size_t)sl * AWY * AWX;
#pragma unroll
    for (int q = 0; q < NV; q++) {
      if (vsrc[q] >= 0) cp(vd + tid + NT * q, vp + vsrc[q]);
      else if (-1 == vsrc[q]) vd[tid + NT * q] = 0.;
    }
    // z face velocities of planes k0 .. kend (the top face of the last cell)
    if (kk >= k0 && kk <= kend && mine) cp(zr + (size_t)sl * AY * AX + tid, uz + cplane * kk + zsrc);
    if (kk >= k0 && kk < kend) {
      const double *up = ux + uplane * kk;
      double *xd = xr + (size_t)sl * AY * (AX + 1);
#pragma unroll
      for (int q = 0; q < NXF; q++) {
        if (xsrc[q] >= 0) cp(xd + tid + NT * q, up + xsrc[q]);
        else if (-1 == xsrc[q]) xd[tid + NT * q] = 0.;
      }
      const double *yp = uy + cplane * kk;
      double *yd = yr + (size_t)sl * (AY + 1) * AX;
#pragma unroll
      for (int q = 0; q < NYF; q++) {
        if (ysrc[q] >= 0) cp(yd + tid + NT * q, yp + ysrc[q]);
        else if (-1 == ysrc[q]) yd[tid + NT * q] = 0.;
      }
      if (use_b && mine) cp(br + (size_t)sl * AY * AX + tid, src_b + splane * (kk - 1) + bsrc);
    }
    __pipeline_commit();
  };
  // faces: window offsets of the two cells and in-plane normal offsets
  int xface[NXF], yface[NYF];  // window offset of the lower cell, -1 outside the domain
  int xnrm[NXF], ynrm[NYF];
#pragma unroll
  for (int q = 0; q < NXF; q++) {
    const int e = tid + NT * q, r = e / (AX + 1), c = e - r * (AX + 1);
    const int fi = i0 + c, fj = j0 + r;
    const bool ok = e < AY * (AX + 1) && fi >= 2 && fi <= nx && fj <= ny;
    xface[q] = ok ? (r + 1) * AWX + c : -1;
    xnrm[q] = ok ? 4 * ((fi - 2) + nx * fj) : 0;  // normal of cell fi - 1; cell fi is 4 further
  }
#pragma unroll
  for (int q = 0; q < NYF; q++) {
    const int e = tid + NT * q, r = e / AX, c = e - r * AX;
    const int fi = i0 + c, fj = j0 + r;
    const bool ok = e < (AY + 1) * AX && fi <= nx && fj <= ny + 1;
    yface[q] = ok ? r * AWX + c + 1 : -1;
    ynrm[q] = ok ? 4 * ((fi - 1) + nx * (fj - 1)) : 0;  // normal of row fj - 1; row fj is 4 nx further
  }
  load_plane(k0 - 1);
  load_plane(k0);
  load_plane(k0 + 1);
  __pipeline_wait_prior(0);
  __syncthreads();
  const double dt = ldg(dtp);
  // 1 / dx of the flux divergence, once per thread (same values)
  const double rdx = mine ? 1. / ldg(g.dxf + i - 1) : 0., rdy = 1. / g.dy, rdz = 1. / g.dz;
#define VR(sl, r, c) vr[((size_t)(sl) * AWY + (r)) * AWX + (c)]
  double fz_lo = 0.;
  if (mine) {
    const int sm1 = (k0 - 1) & (ASLOT - 1), s0 = k0 & (ASLOT - 1);
    fz_lo = face_flux<R, 2>(zr[(size_t)s0 * AY * AX + tid], VR(sm1, ty + 1, tx + 1), VR(s0, ty + 1, tx + 1), normal,
                            ix_nrm(g, i, j, k0 - 1), ix_nrm(g, i, j, k0));
  }
  for (int k = k0; k < kend; k++) {
    if (k + 2 <= kend + 1) load_plane(k + 2);
    const int s0 = k & (ASLOT - 1), sp = (k + 1) & (ASLOT - 1);
    const double *vs = vr + (size_t)s0 * AWY * AWX;
    const long nk = nplane * k;
#pragma unroll
    for (int q = 0; q < NXF; q++) {
      const int e = tid + NT * q;
      if (e >= AY * (AX + 1)) break;
      double f = 0.;
      if (xface[q] >= 0)
        f = face_flux<R, 0>(xr[(size_t)s0 * AY * (AX + 1) + e], vs[xface[q]], vs[xface[q] + 1], normal,
                            nk + xnrm[q], nk + xnrm[q] + 4);
      fx[e] = f;
    }
#pragma unroll
    for (int q = 0; q < NYF; q++) {
      const int e = tid + NT * q;
      if (e >= (AY + 1) * AX) break;
      double f = 0.;
      if (yface[q] >= 0)
        f = face_flux<R, 1>(yr[(size_t)s0 * (AY + 1) * AX + e], vs[yface[q]], vs[yface[q] + AWX], normal,
                            nk + ynrm[q], nk + ynrm[q] + 4L * nx);
      fy[e] = f;
    }
    double fz_hi = 0.;
    if (mine)
      fz_hi = face_flux<R, 2>(zr[(size_t)sp * AY * AX + tid], VR(s0, ty + 1, tx + 1), VR(sp, ty + 1, tx + 1), normal,
                              ix_nrm(g, i, j, k), ix_nrm(g, i, j, k + 1));
    __syncthreads();
    if (mine) {
      double s = 0.;
      s += rdx * (+fx[ty * (AX + 1) + tx] - fx[ty * (AX + 1) + tx + 1]);
      s += rdy * (+fy[ty * AX + tx] - fy[(ty + 1) * AX + tx]);
      s += rdz * (+fz_lo - fz_hi);
      const long is = ix_src(g, i, j, k);
      src_a[is] = s;
      double v = VR(s0, ty + 1, tx + 1);
      v += dt * rk.a * s;
      if (use_b) v += dt * rk.b * br[(size_t)s0 * AY * AX + tid];
      // images: two halo layers in y and z
      const bool hj = (j >= ny - 1) || (j <= 2), hk = (k >= nz - 1) || (k <= 2);
      const int j2 = (j >= ny - 1) ? j - ny : j + ny;
      const int k2 = (k >= nz - 1) ? k - nz : k + nz;
      auto put = [&](int jj, int kk) {
        vof_new[ix_vof(g, i, jj, kk)] = v;
        if (1 == i) vof_new[ix_vof(g, 0, jj, kk)] = 0.;
        if (nx == i) vof_new[ix_vof(g, nx + 1, jj, kk)] = 0.;
      };
      put(j, k);
      if (hj) put(j2, k);
      if (hk) {
        put(j, k2);
        if (hj) put(j2, k2);
      }
    }
    fz_lo = fz_hi;
    // plane k + 2 (issued at the top of this iteration) complete: the next
    // iteration reads it as its upper plane sp (the z-face flux above each
    // cell); waiting for all but the newest group would leave it in flight
    __pipeline_wait_prior(0);
    __syncthreads();
  }
#undef VR
}

// ---- host-side launchers
template <class R>
cudaError_t interface_geom(cudaStream_t st, const double *vof, R *normal, R *curv, unsigned *work,
                           unsigned *nwork, Grid3 g, unsigned long long *unconverged) {
  cudaError_t e = cudaMemsetAsync(nwork, 0, sizeof(unsigned), st);
  if (cudaSuccess != e) return e;
  dim3 gr((g.nx + G3X - 1) / G3X, (g.ny + 2 + G3Y - 1) / G3Y, (g.nz + 2 + G3Z - 1) / G3Z);
  k3_geom<R><<<gr, G3X * G3Y, 0, st>>>(vof, normal, curv, work, nwork, g);
  if (cudaSuccess != (e = cudaGetLastError())) return e;
  k3_intercept<R><<<148 * 8, 256, 0, st>>>(vof, normal, work, nwork, g, unconverged);
  return cudaGetLastError();
}

template <class R>
cudaError_t interface_force(cudaStream_t st, const double *vof, const R *curv, R *ifrcx, R *ifrcy, R *ifrcz,
                            double tension, Grid3 g) {
  dim3 b(32, 8), gr((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kForcePlanes - 1) / kForcePlanes);
  k3_force<R><<<gr, b, 0, st>>>(vof, curv, ifrcx, ifrcy, ifrcz, tension, g);
  return cudaGetLastError();
}

template <class R>
cudaError_t interface_advect(cudaStream_t st, const double *vof, double *vof_new, const double *ux,
                             const double *uy, const double *uz, const R *normal, double *src_a,
                             const double *src_b, const double *dtp, RK rk, int use_b, Grid3 g) {
  dim3 gr((g.nx + AX - 1) / AX, (g.ny + AY - 1) / AY, (g.nz + AZ - 1) / AZ);
  k3_vof_advect<R><<<gr, AX * AY, kAdvectSmem, st>>>(vof, vof_new, ux, uy, uz, normal, src_a, src_b, dtp, rk, use_b, g);
  return cudaGetLastError();
}

template <class R>
cudaError_t interface_prepare_t() {
  return raise_smem_limit(k3_vof_advect<R>, kAdvectSmem);
}

#define SVOF3_INTERFACE_INST(R)                                                                                \
  template cudaError_t interface_geom<R>(cudaStream_t, const double *, R *, R *, unsigned *, unsigned *, Grid3, \
                                          unsigned long long *);                                         \
  template cudaError_t interface_force<R>(cudaStream_t, const double *, const R *, R *, R *, R *, double, Grid3); \
  template cudaError_t interface_advect<R>(cudaStream_t, const double *, double *, const double *, const double *, \
                                           const double *, const R *, double *, const double *, const double *,   \
                                           RK, int, Grid3);
#if SVOF3_WITH_F64
SVOF3_INTERFACE_INST(double)
template cudaError_t interface_prepare_t<double>();
#endif
#if SVOF3_WITH_F32
SVOF3_INTERFACE_INST(float)
template cudaError_t interface_prepare_t<float>();
#endif
#undef SVOF3_INTERFACE_INST

#if SVOF3_WITH_F64
#if !SVOF3_WITH_F32
extern template cudaError_t interface_prepare_t<float>();
#endif
cudaError_t interface_prepare() {
  cudaError_t e = interface_prepare_t<double>();
  if (cudaSuccess != e) return e;
  return interface_prepare_t<float>();
}
#endif

}  // namespace svof3
