// Time integration around the residual: the five-stage low-storage RK54 of
// FRSolver::step_LSRK with the embedded error estimate and PI step
// controller of step_adaptive (reference src/solver.cpp:2663-2757,
// 3100-3255), and RK44 steps whose dt is the CFL estimate of
// compute_element_dt (src/solver.cpp:2864-3097, 4105-4272).
#include "time_kernels.cuh"

namespace zb {

// RK54 coefficients (src/solver.cpp:749-777): Kennedy-Carpenter 2N-storage
// pair, stage weights b, embedded weights bhat, stage increments a.
static const double kLsA[4] = {970286171893. / 4311952581923., 6584761158862. / 12103376702013.,
                               2251764453980. / 15575788980749., 26877169314380. / 34165994151039.};
static const double kLsB[5] = {1153189308089. / 22510343858157., 1772645290293. / 4653164025191.,
                               -1672844663538. / 4480602732383., 2114624349019. / 3568978502595.,
                               5198255086312. / 14908931495163.};
static const double kLsBhat[5] = {1016888040809. / 7410784769900., 11231460423587. / 58533540763752.,
                                  -1563879915014. / 6823010717585., 606302364029. / 971179775848.,
                                  1097981568119. / 3980877426909.};

// CFL limits per order (src/funcs.cpp:435-560): upwinded advection; LDG
// diffusion centred (beta = 0) or upwinded.
double cfl_limit_adv(int order)
{
  static const double t[] = {1.392, 0.4642, 0.2351, 0.1453, 0.1000, 0.07363,
                             0.05678, 0.04530, 0.03709, 0.03101, 0.02635};
  if (order < 0 || order > 10) ZB_THROW(ZB_ERR_UNSUPPORTED, "no CFL limit for this order");
  return t[order];
}

double cfl_limit_diff(int order, double beta)
{
  static const double centred[] = {2.785, 0.1740, 0.04264, 0.01580, 0.007193, 0.003730,
                                   0.002120, 0.001292, 0.0008314, 0.0005586, 0.0003890};
  static const double upwind[] = {0.6963, 0.07736, 0.01878, 0.006345, 0.002664, 0.001299,
                                  0.0007060, 0.0004153, 0.0002599, 0.0001708, 0.0001168};
  if (order < 0 || order > 10) ZB_THROW(ZB_ERR_UNSUPPORTED, "no CFL limit for this order");
  return beta == 0.0 ? centred[order] : upwind[order];
}

namespace dev {

// One RK54 stage update per point (step_LSRK, src/solver.cpp:3164-3226):
//   err -= (b - bhat) dt/|J| R                       (adaptive)
//   U = U_til - a dt/|J| R;  U_til = U - (b - a) dt/|J| R   (stages 0-3)
//   U = U_til - b dt/|J| R                           (stage 4)
// FP64 arithmetic on the stored values (deviations from the reference state in
// the mixed form, which the update is linear in).
template <typename T>
__global__ void k_lsrk_update(T *__restrict__ U, T *__restrict__ Util, T *__restrict__ err,
                              const T *__restrict__ R, const T *__restrict__ mets, int64_t ntiles, int S, int V,
                              int NM, int D, double dt, double ai, double bi, double bhi, int last, int adapt)
{
  const int64_t total = ntiles * S * V * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int64_t ps = i / ((int64_t)TW * V);  // tile * S + s
    const double detJ = (double)mets[(ps * NM + D * D) * TW + l];
    const double r = (double)R[i];
    if (adapt) err[i] = (T)((double)err[i] - (bi - bhi) * dt / detJ * r);
    if (!last)
    {
      const double u = (double)Util[i] - ai * dt / detJ * r;
      U[i] = (T)u;
      Util[i] = (T)(u - (bi - ai) * dt / detJ * r);
    }
    else
      U[i] = (T)((double)Util[i] - bi * dt / detJ * r);
  }
}

// max over real elements of |err| / (atol + rtol max(|U|, |U_ini|)) as the bit
// pattern of a non-negative double; NaN counts as infinite (the reference's
// GPU path, src/solver.cpp:2702-2706)
template <typename T>
__global__ void k_rk_error(const T *__restrict__ U, const T *__restrict__ Uini, const T *__restrict__ err,
                           const double *__restrict__ ref, int64_t neles, int64_t ntiles, int S, int V, double atol,
                           double rtol, unsigned long long *out)
{
  const int64_t total = ntiles * S * V * TW;
  double m = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int v = (int)((i / TW) % V);
    const int64_t t = i / ((int64_t)TW * V * S);
    if (t * TW + l >= neles) continue;
    const double r = ref ? ref[v] : 0.0;
    const double u = (double)U[i] + r, u0 = (double)Uini[i] + r;
    double x = fabs((double)err[i]) / (atol + rtol * fmax(fabs(u), fabs(u0)));
    if (!(x <= 1.7976931348623157e308)) x = __longlong_as_double(0x7ff0000000000000LL);
    m = fmax(m, x);
  }
  for (int o = 16; o > 0; o /= 2) m = fmax(m, __shfl_down_sync(0xffffffff, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// mixed form: fold the compensated-summation remainder of RK44 into the stored
// state (value = U - comp) before steps that do not carry it
template <typename T>
__global__ void k_fold_comp(T *__restrict__ U, T *__restrict__ comp, int64_t total)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    U[i] = (T)((double)U[i] - (double)comp[i]);
    comp[i] = T(0);
  }
}

}  // namespace dev

static void *talloc(size_t bytes)
{
  void *p = nullptr;
  const cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  return p;
}

// element volumes (src/elements.cpp:878-883), face-point weights
// (weights_fpts, src/quads.cpp:64-66, src/hexas.cpp:72-75) and, for CFL_type
// 2, the line lengths h_ref between paired flux points of opposite faces
// (src/elements.cpp:408-483), in the tile layout
static void upload_cfl_geometry(Ctx *c)
{
  const Plan &p = c->plan;
  const int64_t E = p.neles, nt = c->ntiles;
  const int S = p.nspts, Fp = p.nfpts, D = p.ndims, N = p.N, NF = p.nfpts_face;
  if (!c->evol)
  {
    std::vector<double> vol((size_t)nt * TW, 0.0);
    for (int64_t e = 0; e < E; e++)
    {
      double v = 0.0;
      for (int s = 0; s < S; s++) v += p.weights_spts[s] * p.jaco_det_spts[(size_t)s * E + e];
      vol[e] = v;
    }
    const std::vector<double> w1 = gauss_legendre_weights(N);
    std::vector<double> wf(NF);
    for (int k = 0; k < NF; k++) wf[k] = (D == 2) ? w1[k] : w1[k / N] * w1[k % N];
    c->evol = (double *)talloc(vol.size() * sizeof(double));
    c->dfw = (double *)talloc(wf.size() * sizeof(double));
    CK(cudaMemcpy(c->evol, vol.data(), vol.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->dfw, wf.data(), wf.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (c->ts.cfl_type == 2 && !c->h_ref)
  {
    std::vector<double> h((size_t)nt * Fp * TW, 1.0);
    auto X = [&](int f, int d, int64_t e) { return p.coord_fpts[((size_t)f * D + d) * E + e]; };
    auto put = [&](int f, int64_t e, double v) { h[((size_t)(e / TW) * Fp + f) * TW + e % TW] = v; };
    for (int64_t e = 0; e < E; e++)
    {
      if (D == 2)
      {
        // face 0 point i pairs with face 2 point N-1-i, face 1 with face 3
        for (int f1 = 0; f1 < Fp / 2; f1++)
        {
          const int i = f1 % N, f2 = (f1 / N + 3) * N - i - 1;
          const double dx = X(f1, 0, e) - X(f2, 0, e), dy = X(f1, 1, e) - X(f2, 1, e);
          const double dist = std::sqrt(dx * dx + dy * dy);
          put(f1, e, dist);
          put(f2, e, dist);
        }
      }
      else
      {
        // the point of the opposite face at the same face-tangential
        // position; the length keeps the reference's expression
        // sqrt(dx^2 + dy^2 * dz^2) (src/elements.cpp:474)
        const int N2 = N * N;
        for (int a = 0; a < N; a++)
          for (int b = 0; b < N; b++)
          {
            const int pairs[3][2] = {{b * N + a, N2 + b * N + (N - 1 - a)},
                                     {2 * N2 + a * N + b, 3 * N2 + a * N + (N - 1 - b)},
                                     {4 * N2 + b * N + (N - 1 - a), 5 * N2 + b * N + a}};
            for (auto &pr : pairs)
            {
              double dx[3];
              for (int d = 0; d < 3; d++) dx[d] = X(pr[0], d, e) - X(pr[1], d, e);
              const double dist = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] * dx[2] * dx[2]);
              put(pr[0], e, dist);
              put(pr[1], e, dist);
            }
          }
      }
    }
    c->h_ref = (double *)talloc(h.size() * sizeof(double));
    CK(cudaMemcpy(c->h_ref, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (!c->dt_ele) c->dt_ele = (double *)talloc((size_t)nt * TW * sizeof(double));
}

// volumes and line lengths again from the (moved) geometry
void ctx_refresh_cfl_geometry(Ctx *c)
{
  double **bufs[] = {&c->evol, &c->dfw, &c->h_ref};
  for (double **b : bufs)
    if (*b)
    {
      cudaFree(*b);
      *b = nullptr;
    }
  if (c->ts.dt_type != 0) upload_cfl_geometry(c);
}

void ctx_set_time_scheme(Ctx *c, const zb_time_scheme *ts)
{
  if (!ts) ZB_THROW(ZB_ERR_ARG, "null time scheme");
  if (ts->scheme != ZB_RK44 && ts->scheme != ZB_RK54) ZB_THROW(ZB_ERR_ARG, "unknown time scheme");
  if (ts->dt_type < 0 || ts->dt_type > 2) ZB_THROW(ZB_ERR_ARG, "dt_type must be 0, 1 or 2");
  if (ts->dt_type != 0 && ts->cfl_type != 1 && ts->cfl_type != 2) ZB_THROW(ZB_ERR_ARG, "CFL_type must be 1 or 2");
  if (ts->adapt_dt && ts->scheme != ZB_RK54)
    ZB_THROW(ZB_ERR_UNSUPPORTED, "adaptive time stepping needs an embedded pair (RK54)");
  if (ts->dt_type != 0 && ts->scheme != ZB_RK44)
    ZB_THROW(ZB_ERR_UNSUPPORTED, "the CFL time step is computed in RK44 steps (step_RK)");
  if (ts->dt_type != 0 && c->plan.etype == ET_TRI)
    ZB_THROW(ZB_ERR_UNSUPPORTED, "the CFL time step is built for quadrilaterals and hexahedra");
  if (ts->dt_type != 0) cfl_limit_adv(c->plan.order);  // order check
  c->ts = *ts;
  if (!c->d_dt)
  {
    c->d_dt = (double *)talloc(4 * sizeof(double));
    CK(cudaMemsetAsync(c->d_dt, 0, 4 * sizeof(double), c->stream));
  }
  if (ts->dt_type != 0) upload_cfl_geometry(c);
  if (ts->scheme == ZB_RK54)
  {
    const size_t nU = (size_t)c->ntiles * c->S * c->V * TW * c->tsz;
    if (!c->U_til) c->U_til = talloc(nU);
    if (!c->rk_err) c->rk_err = talloc(nU);
  }
  c->prev_err = 1.0;
}

void ctx_time_state(Ctx *c, double *dt, double *prev_err, int64_t *rejected, double *flow_time)
{
  CK(cudaStreamSynchronize(c->stream));
  double dd[4] = {0, 0, 0, 0};
  if (c->d_dt) CK(cudaMemcpy(dd, c->d_dt, sizeof(dd), cudaMemcpyDeviceToHost));
  const bool cfl = c->ts.scheme == ZB_RK44 && c->ts.dt_type != 0;
  if (cfl && c->ts.dt_type == 2) CK(cudaMemcpy(&dd[0], c->dt_ele, sizeof(double), cudaMemcpyDeviceToHost));
  if (dt) *dt = cfl ? dd[0] : c->dt;
  if (prev_err) *prev_err = c->prev_err;
  if (rejected) *rejected = c->rejected;
  if (flow_time) *flow_time = c->flow_time + dd[2];
}

void ctx_get_element_dt(Ctx *c, double *out)
{
  if (!out) ZB_THROW(ZB_ERR_ARG, "null output");
  if (!c->dt_ele) ZB_THROW(ZB_ERR_ARG, "no CFL time step has been computed (dt_type 0)");
  std::vector<double> t((size_t)c->ntiles * TW);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(t.data(), c->dt_ele, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
  std::memcpy(out, t.data(), (size_t)c->plan.neles * sizeof(double));
}

template <typename T>
static void lsrk_step(Ctx *c)
{
  const int64_t total = c->ntiles * c->S * c->V * TW;
  const size_t bytes = (size_t)total * sizeof(T);
  const unsigned grid = grid_for(total, 256);
  const bool adapt = c->ts.adapt_dt != 0;
  if (c->Ucomp)
  {
    dev::k_fold_comp<T><<<grid, 256, 0, c->stream>>>((T *)c->U, (T *)c->Ucomp, total);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(c->U_ini, c->U, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->U_til, c->U, bytes, cudaMemcpyDeviceToDevice, c->stream));
  if (adapt) CK(cudaMemsetAsync(c->rk_err, 0, bytes, c->stream));
  for (int st = 0; st < 5; st++)
  {
    ctx_compute_residual(c, 0);
    dev::k_lsrk_update<T><<<grid, 256, 0, c->stream>>>(
        (T *)c->U, (T *)c->U_til, (T *)c->rk_err, (const T *)c->divF[0], (const T *)c->mets, c->ntiles, c->S, c->V,
        c->D * c->D + 1, c->D, c->dt, st < 4 ? kLsA[st] : 0.0, kLsB[st], kLsBhat[st], st == 4, adapt);
    c->launches++;
    CK(cudaGetLastError());
    c->ufp_valid = false;
  }
}

template <typename T>
static double rk_error(Ctx *c)
{
  const int64_t total = c->ntiles * c->S * c->V * TW;
  CK(cudaMemsetAsync(c->d_dt + 1, 0, sizeof(double), c->stream));
  dev::k_rk_error<T><<<grid_for(total, 256), 256, 0, c->stream>>>(
      (const T *)c->U, (const T *)c->U_ini, (const T *)c->rk_err, c->prec == ZB_FP64 ? nullptr : c->dref,
      c->plan.neles, c->ntiles, c->S, c->V, c->ts.atol, c->ts.rtol,
      reinterpret_cast<unsigned long long *>(c->d_dt + 1));
  c->launches++;
  CK(cudaGetLastError());
  double m = 0.0;
  CK(cudaMemcpyAsync(&m, c->d_dt + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return m;
}

// step_adaptive (src/solver.cpp:2663-2757): a rejected step restarts from its
// start state with the reduced dt until one is accepted
template <typename T>
static void adaptive_step(Ctx *c)
{
  const double p = 4.0;  // order of the RK54 pair
  const double expa = c->ts.pi_alpha / p, expb = c->ts.pi_beta / p;
  for (;;)
  {
    const double dt_used = c->dt;
    lsrk_step<T>(c);
    const double max_err = rk_error<T>(c);
    double fac = std::pow(max_err, -expa) * std::pow(c->prev_err, expb);
    fac = std::min(c->ts.max_factor, std::max(c->ts.min_factor, c->ts.safety * fac));
    c->dt = std::min(c->dt * fac, c->ts.max_dt);
    if (c->dt < 1e-14) ZB_THROW(ZB_ERR_NONFINITE, "dt approaching 0 - quitting simulation");
    if (max_err < 1.0)
    {
      c->prev_err = max_err;
      c->flow_time += dt_used;
      return;
    }
    const size_t bytes = (size_t)c->ntiles * c->S * c->V * TW * sizeof(T);
    CK(cudaMemcpyAsync(c->U, c->U_ini, bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->ufp_valid = false;
    c->rejected++;
  }
}

void ctx_step_scheme(Ctx *c, int n)
{
  if (n < 0) ZB_THROW(ZB_ERR_ARG, "negative step count");
  const zb_time_scheme &ts = c->ts;
  if (ts.scheme == ZB_RK44)
  {
    const bool cfl = ts.dt_type != 0;
    for (int i = 0; i < n; i++)
    {
      if (cfl)
      {
        // compute_element_dt after the stage-0 residual, i.e. from the
        // state at the start of the step (src/solver.cpp:2903-2909)
        c->ufp_valid = false;
        c->launch_extrap(*c);
        c->ufp_valid = true;
        c->launch_dt(*c);
        c->use_dt_dev = ts.dt_type == 1;
        c->use_dt_ele = ts.dt_type == 2;
      }
      for (int s = 0; s < c->nstages; s++) ctx_rk_stage(c, (unsigned)s);
      if (cfl)
      {
        dev::k_dt_advance<<<1, 1, 0, c->stream>>>(c->d_dt, c->dt_ele, ts.dt_type == 2);
        CK(cudaGetLastError());
        c->use_dt_dev = c->use_dt_ele = false;
      }
      else
        c->flow_time += c->dt;
    }
    return;
  }
  for (int i = 0; i < n; i++)
  {
    if (ts.adapt_dt)
    {
      if (c->prec == ZB_FP64)
        adaptive_step<double>(c);
      else
        adaptive_step<float>(c);
    }
    else
    {
      if (c->prec == ZB_FP64)
        lsrk_step<double>(c);
      else
        lsrk_step<float>(c);
      c->flow_time += c->dt;
    }
  }
}

}  // namespace zb
