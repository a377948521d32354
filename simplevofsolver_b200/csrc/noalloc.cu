// noalloc.cu -- pressure Poisson solve (uniform-x, DCT path) that allocates
// no device memory.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// owned by a pool or budget it does not control, code that runs while device
// allocation is forbidden or would synchronise the device at the wrong time,
// or a plug-in loaded into a process that hands it only input and output
// buffers.  For them svof_poisson_dct_noalloc() runs the same three kernels as
// svof_fluid_compute_potential_dct() (k_dct_fwd, k_dct_ysolve, k_dct_inv) but
// keeps the spectrum and the line-solve tables in one file-scope
// `static __device__` array of fixed size instead of memory from cudaMalloc.
// Every GPU that loads this library holds that array (about 2.2 MB) until the
// process exits.
//
// Limits: nx a power of two, nx * ny <= 65536, 4 <= nx, ny <= 1024.  The
// array is shared by all calls and keeps the last call's contents (the tables
// are reused while the grid is unchanged; dt and the spectrum are overwritten
// by every call), so calls that overlap on the GPU race.  The host part of a
// call (grid metrics, tables, their upload) holds a process-wide lock, so
// host threads may call concurrently; their GPU work must still not overlap.
// A call on a grid other than the previous call's on that device builds and
// uploads new tables and waits for the stream; any other call only enqueues
// work (dt is written into the array by a one-thread kernel in stream order).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/svof_b200.h"
#include "smem_limit.cuh"
#include "svof_internal.cuh"

using namespace svof;

namespace {

constexpr size_t kMaxCells = 65536;
constexpr int kMaxN = 1024;
// scratch layout, in doubles
constexpr size_t kSpec = 0;                       // nx*ny spectrum
constexpr size_t kVt = kSpec + kMaxCells;         // nx*ny  gtsv v
constexpr size_t kRvt = kVt + kMaxCells;          // nx*ny  gtsv val
constexpr size_t kQ1t = kRvt + kMaxCells;         // nx*ny  Sherman-Morrison q1
constexpr size_t kCk = kQ1t + kMaxCells;          // nx     diagonal
constexpr size_t kDen = kCk + kMaxN;              // nx     Sherman-Morrison denominator
constexpr size_t kLastf = kDen + kMaxN;           // nx     1 / last pivot or 0
constexpr size_t kDxf = kLastf + kMaxN;           // nx     face-to-face distances
constexpr size_t kTwf = kDxf + kMaxN;             // nx     forward twiddles (n/2 pairs)
constexpr size_t kTwb = kTwf + kMaxN;             // nx     backward twiddles
constexpr size_t kCs = kTwb + kMaxN;              // 2 nx   DCT pre/post twiddles
constexpr size_t kDt = kCs + 2 * kMaxN;           // 1      dt
constexpr size_t kTotal = kDt + 32;

static __device__ __align__(256) double g_noalloc_scratch[kTotal];

constexpr int kMaxDevices = 64;
struct DeviceState {
  bool ready = false;
  double *scratch = nullptr;  // device address of g_noalloc_scratch on this device
  // grid whose tables are currently in the scratch array
  int nx = 0, ny = 0;
  double lx = 0., ly = 0.;
  uint64_t dxf_hash = 0;
};
DeviceState g_dev[kMaxDevices];

// guards g_dev and the host staging below (the host part of every call)
std::mutex g_mu;

// host staging of the tables (static: no allocation on the call path)
double h_vt[kMaxCells], h_rvt[kMaxCells], h_q1t[kMaxCells];
double h_ck[kMaxN], h_den[kMaxN], h_lastf[kMaxN], h_dxf[kMaxN], h_twf[kMaxN], h_twb[kMaxN], h_cs[2 * kMaxN];
double h_l[kMaxN], h_c[kMaxN], h_u[kMaxN], h_v[kMaxN], h_q1[kMaxN];

// dt of this call, written in stream order (no host staging, no wait)
__global__ void k_noalloc_set_dt(double *dst, double dt) { *dst = dt; }

// failures are reported on stderr (the reference's convention) and by the
// non-zero return value
int nfail(const char *m, cudaError_t e = cudaSuccess) {
  if (cudaSuccess != e) {
    fprintf(stderr, "svof_poisson_dct_noalloc: %s: %s\n", m, cudaGetErrorString(e));
  } else {
    fprintf(stderr, "svof_poisson_dct_noalloc: %s\n", m);
  }
  return 1;
}

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return ((1 << l) == n) ? l : -1;
}

uint64_t fnv1a(const void *p, size_t n) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; i++) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

// gtsv of src/tdm.c:17-50 (table set-up, same expressions as svof_create)
void host_gtsv(int n, const double *l, const double *c, const double *u, double *v, double *q) {
  v[0] = u[0] / c[0];
  q[0] = q[0] / c[0];
  for (int i = 1; i < n - 1; i++) {
    const double val = 1. / (c[i] - l[i] * v[i - 1]);
    v[i] = val * (u[i]);
    q[i] = val * (q[i] - l[i] * q[i - 1]);
  }
  const double val = c[n - 1] - l[n - 1] * v[n - 2];
  q[n - 1] = std::fabs(val) > kDblEpsilon ? 1. / val * (q[n - 1] - l[n - 1] * q[n - 2]) : 0.;
  for (int i = n - 2; i >= 0; i--) q[i] -= v[i] * q[i + 1];
}

// the DCT-path tables of svof_create (src/fluid/compute_potential/dct.c:142-261)
void build_tables(int nx, int ny, double lx, double dy) {
  constexpr double kPi = 3.14159265358979323846;
  constexpr double kGPi = 3.14159265358979324;
  const int n = ny;
  const double lap = 1. / dy / dy;
  for (int j = 0; j < n; j++) {
    h_l[j] = lap;
    h_u[j] = lap;
  }
  const double signal_length = 2. * nx;
  const double gridsize = lx / nx;
  for (size_t k = 0; k < (size_t)nx; k++) {
    const double ev = -4. / std::pow(gridsize, 2.) * std::pow(std::sin(kGPi * k / signal_length), 2.);
    for (int r = 0; r < n; r++) h_c[r] = -h_l[r] - h_u[r] + ev;
    for (int i = 0; i < n - 1; i++) h_q1[i] = i == 0 ? -h_l[i] : i == n - 2 ? -h_u[i] : 0.;
    host_gtsv(n - 1, h_l, h_c, h_u, h_v, h_q1);
    for (int i = 0; i < n; i++) {
      h_vt[(size_t)i * nx + k] = (i < n - 1) ? h_v[i] : 0.;
      h_q1t[(size_t)i * nx + k] = (i < n - 1) ? h_q1[i] : 0.;
      h_rvt[(size_t)i * nx + k] = (i >= 1 && i < n - 2) ? 1. / (h_c[i] - h_l[i] * h_v[i - 1]) : 0.;
    }
    const double val = h_c[n - 2] - h_l[n - 2] * h_v[n - 3];
    h_lastf[k] = std::fabs(val) > kDblEpsilon ? 1. / val : 0.;
    h_ck[k] = h_c[0];
    h_den[k] = h_c[n - 1] + h_u[n - 1] * h_q1[0] + h_l[n - 1] * h_q1[n - 2];
  }
  for (int m = 0; m < nx / 2; m++) {
    const double ang = 2.0 * kPi * (double)m / (double)nx;
    h_twf[2 * m] = std::cos(ang);
    h_twf[2 * m + 1] = -std::sin(ang);
    h_twb[2 * m] = std::cos(ang);
    h_twb[2 * m + 1] = std::sin(ang);
  }
  for (int k = 0; k < nx; k++) {
    const double ang = kPi * (double)k / (2.0 * (double)nx);
    h_cs[2 * k] = std::cos(ang);
    h_cs[2 * k + 1] = std::sin(ang);
  }
}

}  // namespace

extern "C" int svof_poisson_dct_noalloc(const svof_params_t *prm, const double *xf, const double *ux,
                                        const double *uy, double *psi, size_t rkstep, double dt, void *stream) {
  if (!prm || !xf || !ux || !uy || !psi) return nfail("null argument");
  const int nx = prm->nx, ny = prm->ny;
  if (nx < 4 || ny < 4 || nx > kMaxN || ny > kMaxN || (size_t)nx * ny > kMaxCells)
    return nfail("grid exceeds the static scratch (nx, ny in [4, 1024], nx * ny <= 65536)");
  const int log2n = ilog2_exact(nx);
  if (log2n < 1) return nfail("nx must be a power of two");
  if (rkstep > 2) return nfail("rkstep out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  // grid metrics as src/domain.c:107-121 and the uniformity test :75-98
  double mn = 1.7976931348623157e308, mx = -1.7976931348623157e308;
  for (int i = 1; i <= nx; i++) {
    h_dxf[i - 1] = xf[i] - xf[i - 1];
    mn = std::fmin(mn, h_dxf[i - 1]);
    mx = std::fmax(mx, h_dxf[i - 1]);
  }
  if (!(std::fabs(mx - mn) < 1.e-15)) return nfail("the x grid is not uniform (the DCT path needs it)");
  const double dy = prm->ly / ny;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (cudaSuccess != e) return nfail("cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return nfail("device index out of range");
  DeviceState &st = g_dev[dev];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // once per device: the device address of the scratch array (the symbol's
  // name in host code is only a host-side stand-in)
  if (!st.ready) {
    void *addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (cudaSuccess != e) return nfail("cudaGetSymbolAddress", e);
    st.scratch = static_cast<double *>(addr);
    st.ready = true;
  }
  double *S = st.scratch;
  // tables: rebuilt and uploaded only when the grid changes
  const uint64_t hsh = fnv1a(h_dxf, sizeof(double) * nx);
  if (st.nx != nx || st.ny != ny || st.lx != prm->lx || st.ly != prm->ly || st.dxf_hash != hsh) {
    st.nx = 0;  // the array holds no valid tables until the upload has completed
    build_tables(nx, ny, prm->lx, dy);
    const size_t nn = (size_t)nx * ny;
    struct { size_t off; const double *src; size_t n; } up[] = {
        {kVt, h_vt, nn}, {kRvt, h_rvt, nn}, {kQ1t, h_q1t, nn}, {kCk, h_ck, (size_t)nx},
        {kDen, h_den, (size_t)nx}, {kLastf, h_lastf, (size_t)nx}, {kDxf, h_dxf, (size_t)nx},
        {kTwf, h_twf, (size_t)nx}, {kTwb, h_twb, (size_t)nx}, {kCs, h_cs, 2 * (size_t)nx}};
    for (auto &u : up) {
      e = cudaMemcpyAsync(S + u.off, u.src, sizeof(double) * u.n, cudaMemcpyHostToDevice, s);
      if (cudaSuccess != e) return nfail("table upload", e);
    }
    e = cudaStreamSynchronize(s);
    if (cudaSuccess != e) return nfail("table upload", e);
    st.nx = nx;
    st.ny = ny;
    st.lx = prm->lx;
    st.ly = prm->ly;
    st.dxf_hash = hsh;
  }
  k_noalloc_set_dt<<<1, 1, 0, s>>>(S + kDt, dt);
  // the three kernels of the DCT path, on the scratch array
  const double gam = (rkstep == 0 ? 32. / 60. + 0. / 60.
                                  : rkstep == 1 ? 25. / 60. + -17. / 60. : 45. / 60. + -25. / 60.);
  const Grid2 g{nx, ny, dy, S + kDxf, S + kDxf};
  // (the row transforms' shared-memory limits: raised once per length, as the
  // allocating solver does)
  e = dct_prepare(log2n);
  if (cudaSuccess != e) return nfail("shared-memory limit of the row transforms", e);
  const dim3 rows_grid((ny + dct_rows(log2n) - 1) / dct_rows(log2n));
  dct_fwd_kernel(log2n)<<<rows_grid, dct_threads(log2n), dct_smem(log2n, false), s>>>(ux, uy, S + kSpec, S + kTwf, S + kCs,
                                                                              S + kDt, gam, g);
  int kt = 32;
  while (kt > 4 && nx / kt < 148) kt >>= 1;
  while (kt > 1 && sizeof(double) * 3 * (size_t)ny * kt > 48 * 1024) kt >>= 1;
  // the default 48 KB limit counts the kernel's static shared memory as well:
  // raise the dynamic limit for every size, as the allocating solver does
  e = raise_smem_limit(k_dct_ysolve, sizeof(double) * 3 * kt * ny);
  if (cudaSuccess != e) return nfail("shared-memory limit of the y solve", e);
  k_dct_ysolve<<<(nx + kt - 1) / kt, 128, sizeof(double) * 3 * kt * ny, s>>>(
      S + kSpec, S + kVt, S + kRvt, S + kQ1t, S + kCk, S + kLastf, S + kDen, 1. / dy / dy, nx, ny, kt);
  dct_inv_kernel(log2n)<<<rows_grid, dct_threads(log2n), dct_smem(log2n, true), s>>>(S + kSpec, psi, S + kTwb, S + kCs, g);
  e = cudaGetLastError();
  if (cudaSuccess != e) return nfail("kernel launch", e);
  return 0;
}
