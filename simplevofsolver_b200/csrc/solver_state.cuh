// solver_state.cuh -- the 2D engine's state and the helpers that issue its
// kernels, shared by solver.cu (the step functions and their C ABI) and
// adjoint.cu (the differentiation form).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/svof_b200.h"
#include "svof_internal.cuh"

namespace svof {

struct DevBuf {
  double *p = nullptr;
  size_t n = 0;
};

struct AdjointState;  // adjoint.cu

}  // namespace svof

struct svof_solver {
  svof_params_t prm{};
  bool managed = false;     // field buffers in CUDA managed memory
  int nx = 0, ny = 0;
  double dy = 0.;
  bool uniform = false;
  int log2fft = 0;          // log2 of the FFT length (nx for DCT, ny for DFT)
  cudaStream_t stream = nullptr;
  // fields (two buffers where a kernel writes a new copy)
  svof::DevBuf ux[2], uy[2], t[2], vof[2];
  svof::DevBuf p, psi, curv, normal, ifrcx, ifrcy;
  svof::DevBuf sux[2], suy[2], st[2], svof[2];
  int cur_u = 0;   // which of ux/uy/t[] is current
  int cur_v = 0;   // which of vof[] is current
  int sa_f = 0;    // which of sux/suy/st[] is src[rk_a]
  int sa_v = 0;    // which of svof[] is src[rk_a]
  // grid tables
  svof::DevBuf dxf, dxc, lap_ux, lap_uy, lap_t;
  double lapy[3] = {0., 0., 0.};
  double dif_m_y = 0., dif_t_y = 0.;
  // Poisson
  svof::DevBuf spec, twf, twb, cs, vt, rvt, q1t, ck, lastf, den, pl, pu, evals;
  int ysolve_kt = 32;       // wavenumber lines per block of the DCT y solve
  // predictor Thomas coefficients, one table per substep (k_tdm_coef)
  svof::DevBuf coef;
  // side stream of the step graph: the coefficient kernel runs beside the
  // interface kernels
  cudaStream_t side = nullptr;
  // the branch of the three substeps' Thomas tables (computed at the start
  // of a step) and its join event
  cudaStream_t side2 = nullptr;
  cudaEvent_t ev_coef = nullptr;
  cudaEvent_t ev_fork[3] = {nullptr, nullptr, nullptr}, ev_join[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_geom[3] = {nullptr, nullptr, nullptr};
  // predict launch shape
  // large grids: the line-streaming predictor (k_predict_rhs, _xsolve,
  // _update) with its line array
  bool pred_lines = false;
  svof::DevBuf fw;
  int pred_rows = 1;
  int pred_threads = 256;
  size_t pred_smem = 0;
  int xsolve_kt = 8;        // ky lines per block of the DFT x solve
  int dft_cols = 1;
  // time step
  double *d_dt = nullptr;
  unsigned long long *d_minbits = nullptr;
  // failure detection: bits set on the device (k_cfl: a non-finite velocity;
  // k_dt_final: a time step that is not a positive finite number), read and
  // cleared by the host at its synchronisations (check_status)
  unsigned *d_status = nullptr;
  double *h_dt = nullptr;   // pinned, many slots for svof_run
  int h_dt_slots = 0;
  svof::DevBuf diag;
  // set while the step graph of a small grid is captured: its kernels are
  // launched with programmatic stream serialisation (each starts with
  // pdl_enter)
  bool pdl = false;
  // time-averaged statistics: accumulators (made on the first collection),
  // row-sum scratch, samples so far
  svof::DevBuf stat[SVOF_NSTATS], stat_part;
  size_t stat_num = 0;
  std::vector<double> xf, xc, dxf_h, dxc_h;
  // graphs keyed by the buffer state at the start of a step
  std::map<int, cudaGraphExec_t> graphs;
  // vof buoyancy on uy (an extension, absent from the reference; off while
  // grav_vof is 0): srcuy_a += grav_vof (vof at the uy face - vof_ref)
  double grav_vof = 0., vof_ref = 0.;
  // the differentiation form's buffers, made on first use (adjoint.cu)
  svof::AdjointState *adj = nullptr;

  svof::Grid2 grid() const { return svof::Grid2{nx, ny, dy, dxf.p, dxc.p}; }
};

namespace svof {

// the last error message of this thread (svof_last_error)
extern thread_local std::string g_err;
// records a message for svof_last_error and returns 1
int fail(const char *fmt, ...);

#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (cudaSuccess != e_) return fail("%s: %s", #x, cudaGetErrorString(e_));  \
  } while (0)

#define CK_LAUNCH() CK(cudaGetLastError())

// src/runge_kutta.c:8-15
constexpr double RK_A[3] = {32. / 60., 25. / 60., 45. / 60.};
constexpr double RK_B[3] = {0. / 60., -17. / 60., -25. / 60.};

// managed: CUDA managed memory, so that a host program holding the pointer
// can read the field
int dalloc(DevBuf &b, size_t n, bool managed = false);
void dfree(DevBuf &b);

// launch k on st; with pdl, as a programmatic dependent of the stream's
// previous kernel
template <typename... KArgs, typename... Args>
cudaError_t launch_k(bool pdl, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args... args) {
  if (!pdl) {
    k<<<grid, block, smem, st>>>(args...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

// each issues the kernels of one reference function on the solver's stream
int launch_halo_bc(svof_solver *s, double *a, int field);
int launch_dt(svof_solver *s);
int check_status(svof_solver *s, const char *who);
int launch_coef(svof_solver *s, int rk, cudaStream_t st);
// the predictor's Thomas table of substep rk (k_tdm_coef layout)
double *coef_table(svof_solver *s, int rk);
int launch_geom(svof_solver *s);
int launch_force(svof_solver *s, cudaStream_t st = nullptr);
int launch_vof(svof_solver *s, int rk);
// with_coef: launch k_tdm_coef first on the same stream
int launch_predict(svof_solver *s, int rk, bool with_coef = true);
int launch_potential(svof_solver *s, int rk, int want_dct);
int launch_project(svof_solver *s, int rk, int do_vel, int do_p);

// frees the differentiation form's buffers (adjoint.cu)
void adjoint_free(svof_solver *s);

}  // namespace svof
