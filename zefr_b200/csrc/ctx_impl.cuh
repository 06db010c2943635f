// Device context shared by the forward (context.cu) and adjoint (adjoint.cu)
// translation units: buffers, launch helpers and profiling scopes.
#pragma once
#include <cstring>
#include <cmath>
#include <mutex>
#include <type_traits>

#include "context.hpp"
#include "dfr_kernels.cuh"

namespace zb {

using dev::Args;
using dev::LineOpsT;
using dev::Shape;
using dev::TW;

#define CK(x)                                                                                  \
  do                                                                                           \
  {                                                                                            \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct StageCfg
{
  unsigned stage;
  int rk_mode;      // 0 none, 1 stage update, 2 final combination
  int save_ini;
  int extrap_next;
  int want_dU = 0;     // write the physical gradient (NS)
  int grad_only = 0;   // NS: stop after the gradient kernel
  int face_only = 0;   // NS: the face kernel alone (the gradient kernel ran before)
};

// RK44 tables (src/solver.cpp:722-735)
static const double kRkAlpha[3] = {0.5, 0.5, 1.0};
static const double kRkBeta[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

struct Ctx
{
  Plan plan;
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int prec = ZB_FP64;
  size_t tsz = 8;  // storage type size
  size_t asz = 8;  // arithmetic type size
  int D = 0, N = 0, S = 0, Fp = 0, V = 0, nstages = 4;
  int64_t ntiles = 0;
  void *U = nullptr, *U_ini = nullptr, *divF[4] = {nullptr, nullptr, nullptr, nullptr};
  void *divF_vol = nullptr, *Ufp[2] = {nullptr, nullptr}, *Fvn = nullptr, *Fcom = nullptr, *mets = nullptr,
       *fgeo = nullptr;
  void *Ucomp = nullptr;
  void *dops = nullptr;  // triangles: dense operators in the arithmetic type
  double *dwall = nullptr;  // wall force: FP64 oppE, face weights, flux point coordinates
  int *nbr = nullptr;
  double *dtmp = nullptr;
  size_t dtmp_bytes = 0;
  double *dred = nullptr;
  int cur = 0;
  bool ufp_valid = false;
  bool need_fvn = false;  // the next stage launch must store the viscous normal flux
  bool fused_traces = false;  // hexahedral NS with one-sided LDG: residuals read no trace buffer
  // split residual (zb_compute_residual_start/mid/finish, zb_rk_stage_*):
  // phase 0 idle, 1 after start, 2 after mid; the stage and kind being split
  int split_phase = 0;
  unsigned split_stage = 0;
  int split_rk = 0;
  double dt = 0.0;
  // mixed form: reference state (FP32-representable values) the stored state
  // deviates from; zero for the FP64 form
  double uref[5] = {0, 0, 0, 0, 0};
  double *dref = nullptr;  // device copy for the conversion kernels
  void *dU = nullptr;          // physical gradient side output (functionals)
  double *dweights = nullptr;  // quadrature weights of the solution points
  double *dfun = nullptr;      // functional reduction buffer
  int64_t launches = 0;
  // per-kernel CUDA-event timing (zb_profile_*)
  bool profiling = false;
  struct Rec { int kid; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double prof_ms[ZB_NKERNELS] = {0};
  int64_t prof_n[ZB_NKERNELS] = {0};
  // adjoint (plain FP64 form), allocated on first use
  double *lam = nullptr, *Lfp = nullptr, *Ubfp = nullptr, *dUbfp = nullptr, *UCb = nullptr, *Ubar = nullptr;
  double *Ubx = nullptr;  // NS: Riemann-flux adjoint a left side leaves at its right partner
  double *pbar = nullptr;
  double *mbar = nullptr, *gbar = nullptr, *nbx = nullptr;  // geometry adjoint
  double *mbar_acc = nullptr, *gbar_acc = nullptr;          // its device-side sums
  double *rkv = nullptr;  // step adjoint: stage states, residuals and adjoints (tile layout)
  double *rkfvn = nullptr;  // step adjoint: the four stages' forward viscous normal fluxes
  // geometry from node coordinates (geometry.cu): shape tables, face pairing, scratch
  double *geo_tab = nullptr;
  int64_t *geo_pair = nullptr;
  double *geo_work = nullptr;
  size_t geo_work_bytes = 0;
  // time integration (zb_set_time_scheme; time_scheme.cu); the RK54 and CFL
  // buffers are allocated on first use
  zb_time_scheme ts{ZB_RK44, 0, 1, 1.0, 0, 1e-5, 1e-5, 0.7, 0.4, 0.8, 2.5, 0.3, 100.0};
  double prev_err = 1.0, flow_time = 0.0;
  int64_t rejected = 0;
  double *d_dt = nullptr;     // [0] CFL step (global minimum), [1] error maximum, [2] flow time of CFL steps
  double *dt_ele = nullptr;   // [ntiles * TW] per-element CFL step
  double *h_ref = nullptr;    // [ntiles][Fp][TW] CFL_type 2 line lengths
  double *evol = nullptr;     // [ntiles * TW] element volumes
  double *dfw = nullptr;      // face-point quadrature weights [Fp / faces]
  void *U_til = nullptr, *rk_err = nullptr;
  bool use_dt_dev = false, use_dt_ele = false;  // stage kernels read the step from d_dt / dt_ele
  // residuals of host-resident states with overlapped copies
  // (ctx_residuals_host): two input and two output staging buffers, a copy
  // stream per direction, and the events that hand the buffers over
  double *pipe_in[2] = {nullptr, nullptr}, *pipe_out[2] = {nullptr, nullptr};
  cudaStream_t pipe_h2d = nullptr, pipe_d2h = nullptr;
  cudaEvent_t pipe_ev[8] = {};
  // tensor-core kernels' timeout flag: mapped pinned host memory (host and
  // device addresses), checked before each stage launch
  volatile int *tc_err_host = nullptr;
  int *tc_err_dev = nullptr;
  void (*launch_extrap)(Ctx &) = nullptr;
  void (*launch_stage)(Ctx &, const StageCfg &) = nullptr;
  void (*launch_vjp)(Ctx &, bool, bool) = nullptr;
  void (*launch_dt)(Ctx &) = nullptr;  // CFL estimate from the current traces
};

static cudaEvent_t take_event(Ctx &c)
{
  if (!c.pool.empty())
  {
    cudaEvent_t e = c.pool.back();
    c.pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}

// Brackets one kernel launch with events when profiling is on.
struct ProfScope
{
  Ctx &c;
  int kid;
  cudaEvent_t a = nullptr;
  ProfScope(Ctx &cc, int k) : c(cc), kid(k)
  {
    if (c.profiling)
    {
      a = take_event(c);
      CK(cudaEventRecord(a, c.stream));
    }
  }
  ~ProfScope()
  {
    if (c.profiling && a)
    {
      cudaEvent_t b = take_event(c);
      cudaEventRecord(b, c.stream);
      c.recs.push_back({kid, a, b});
    }
  }
};

template <typename T, int N>
static LineOpsT<T, N> line_ops(const Plan &p)
{
  LineOpsT<T, N> o;
  for (int i = 0; i < N * N; i++) o.Dm[i] = (T)p.ops.D[i];
  for (int i = 0; i < N; i++)
  {
    o.Em[i] = (T)p.ops.Em[i];
    o.Ep[i] = (T)p.ops.Ep[i];
    o.Dbm[i] = (T)p.ops.Dbm[i];
    o.Dbp[i] = (T)p.ops.Dbp[i];
  }
  return o;
}

template <typename T>
static dev::Phys<T> phys_of(const zb_params &p, const double *uref, int ndims, bool deviations)
{
  dev::Phys<T> ph;
  std::memset(&ph, 0, sizeof(ph));
  ph.dev = deviations ? 1 : 0;
  // perturbation-form constants of the reference state (FP64, then rounded)
  const int V = ndims + 2;
  double m2 = 0.0;
  for (int d = 0; d < ndims; d++) m2 += uref[d + 1] * uref[d + 1];
  for (int v = 0; v < V; v++) ph.Ur[v] = (T)uref[v];
  if (uref[0] != 0.0)
  {
    const double Pr = (p.gamma - 1.0) * (uref[V - 1] - 0.5 * m2 / uref[0]);
    ph.Pr = (T)Pr;
    ph.er = (T)(uref[V - 1] + Pr);
    ph.inv_rr = (T)(1.0 / uref[0]);
    ph.mr2 = (T)m2;
  }
  ph.gamma = (T)p.gamma;
  ph.prandtl = (T)p.prandtl;
  ph.mu = (T)p.mu;
  ph.rt = (T)p.rt;
  ph.c_sth = (T)p.c_sth;
  ph.rus_k = (T)p.rus_k;
  ph.ldg_b = (T)p.ldg_b;
  ph.ldg_tau = (T)p.ldg_tau;
  ph.rho_fs = (T)p.rho_fs;
  ph.P_fs = (T)p.P_fs;
  ph.T_wall = (T)p.T_wall;
  ph.R_ref = (T)p.R_ref;
  for (int d = 0; d < 3; d++)
  {
    ph.V_fs[d] = (T)p.V_fs[d];
    ph.V_wall[d] = (T)p.V_wall[d];
  }
  ph.fix_vis = p.fix_vis;
  ph.fconv = p.fconv;
  return ph;
}

static int grid_for(int64_t work, int threads)
{
  int64_t b = (work + threads - 1) / threads;
  if (b > 148 * 64) b = 148 * 64;
  if (b < 1) b = 1;
  return (int)b;
}

template <typename K>
static void set_smem(K kernel, size_t bytes)
{
  CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// kernel arguments of one stage of a context
template <typename T, typename A>
static Args<T, A> make_args(Ctx &c, const StageCfg &sc)
{
  Args<T, A> a;
  std::memset(&a, 0, sizeof(a));
  a.U = (const T *)c.U;
  a.Ufp = (const T *)c.Ufp[c.cur];
  a.Ufp_next = (T *)c.Ufp[c.cur ^ 1];
  a.mets = (const T *)c.mets;
  a.fgeo = (const T *)c.fgeo;
  a.nbr = c.nbr;
  a.divF = (T *)c.divF[sc.stage];
  a.divF_vol = (A *)c.divF_vol;
  if (c.Fcom && (c.plan.params.ldg_b == 0.5 || c.plan.params.ldg_b == -0.5)) a.Fcom = (T *)c.Fcom;
  // with the one-sided common flux the face kernel does not read the viscous
  // normal flux; only the geometry adjoint does (need_fvn)
  a.Fvn = (a.Fcom && !c.need_fvn) ? nullptr : (T *)c.Fvn;
  a.rk_mode = sc.rk_mode;
  a.save_ini = sc.save_ini;
  // the one-sided form keeps no trace buffer: the gradient kernel forms the
  // traces from the state, so the next stage's extrapolation is not stored
  a.extrap_next = a.Fcom ? 0 : sc.extrap_next;
  a.Uout = (T *)c.U;
  a.U_ini = (T *)c.U_ini;
  a.Ucomp = nullptr;
  a.dt = (A)c.dt;
  a.dt_dev = c.use_dt_dev ? c.d_dt : nullptr;
  a.dt_ele = c.use_dt_ele ? c.dt_ele : nullptr;
  a.ntiles = c.ntiles;
  a.dU_out = sc.want_dU ? (T *)c.dU : nullptr;
  a.dops = (const A *)c.dops;
  a.err = c.tc_err_dev;
  a.ph = phys_of<A>(c.plan.params, c.uref, c.D, sizeof(T) < sizeof(double));
  if (sc.rk_mode == 1)
    a.rk_coef[0] = (A)kRkAlpha[sc.stage];
  else if (sc.rk_mode == 2)
  {
    a.nprev = (int)sc.stage;
    for (unsigned s = 0; s <= sc.stage; s++) a.rk_coef[s] = (A)kRkBeta[s];
    for (unsigned s = 0; s < sc.stage; s++) a.divF_prev[s] = (const T *)c.divF[s];
    if (c.Ucomp) a.Ucomp = (T *)c.Ucomp;
  }
  return a;
}

// selects the adjoint kernels of the context (plain FP64 form; adjoint.cu)
void bind_vjp(Ctx &c);

}  // namespace zb
