// CFL time-step estimate of FRSolver::compute_element_dt (reference
// src/solver.cpp:4105-4272) from the traces of the state at the start of a
// step.  The reference takes the face wave speed and diffusion coefficient
// that its Rusanov and LDG fluxes store per face point (src/faces.cpp:
// 1308-1316, 1572-1577); here the same quantities are formed from the traces
// directly, since the fused face kernels keep no per-point side outputs.
#pragma once

#include "ctx_impl.cuh"

namespace zb {
namespace dev {

// inviscid wave speed |Vn| + a of one absolute state
// (compute_Fconv_EulerNS pressure, src/faces.cpp:1296-1313)
template <int D>
__device__ __forceinline__ double wave_speed(const double U[D + 2], const double n[D], double gamma)
{
  double momF = 0.0;
#pragma unroll
  for (int d = 0; d < D; d++) momF += U[d + 1] * U[d + 1];
  momF /= U[0];
  const double P = (gamma - 1.0) * (U[D + 1] - 0.5 * momF);
  const double a = sqrt(gamma * P / U[0]);
  double Vn = 0.0;
#pragma unroll
  for (int d = 0; d < D; d++) Vn += U[d + 1] / U[0] * n[d];
  return fabs(Vn) + a;
}

// LDG diffusion coefficient of one side (src/faces.cpp:1575-1576)
__device__ __forceinline__ double diff_coef(double rho, const Phys<double> &ph)
{
  return fmax(ph.mu / rho, ph.gamma * ph.mu / (ph.prandtl * rho));
}

// One thread per element.  cfl_type 1: dt = 2 CFL c_adv vol / sum_f w dA ws;
// cfl_type 2: per face max of ws / (c_adv h) (+ dc / (c_diff h^2)), summed
// over directions.  dt_ele gets every element's step (0 for padding lanes),
// dt_min the minimum as the bit pattern of a non-negative double.
template <typename T, int D, int N>
__global__ void __launch_bounds__(128) k_element_dt(const T *__restrict__ Ufp, const T *__restrict__ fgeo,
                                                    const int *__restrict__ nbr, const double *__restrict__ h_ref,
                                                    const double *__restrict__ evol, const double *__restrict__ wf,
                                                    int64_t ntiles, int64_t neles, const Phys<double> ph, int visc,
                                                    int cfl_type, double cfl, double c_adv, double c_diff,
                                                    double *__restrict__ dt_ele,
                                                    unsigned long long *__restrict__ dt_min)
{
  using G = Shape<D, N>;
  constexpr int Fp = G::Fp, V = G::V, NF = G::NF;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ntiles * TW) return;
  if (e >= neles)
  {
    dt_ele[e] = 0.0;
    return;
  }
  const int64_t tile = e / TW;
  const int l = (int)(e % TW);
  double int_ws = 0.0;
  double dtinv[2 * D];
#pragma unroll
  for (int k = 0; k < 2 * D; k++) dtinv[k] = 0.0;
#pragma unroll 1
  for (int f = 0; f < Fp; f++)
  {
    const int64_t pf = tile * Fp + f;
    double n[D], Us[V], Ua[V], UR[V], UB[V];
    const T *g = fgeo + pf * (D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = (double)g[d * TW];
    const double dA = (double)g[D * TW];
    const int code = nbr[pf * TW + l];
#pragma unroll
    for (int v = 0; v < V; v++) Us[v] = (double)Ufp[(pf * V + v) * TW + l];
    to_abs<double, D>(Us, Ua, ph);
    if (code >= 0)
    {
      double Un[V];
      gather_fpt<T, double, V>(Ufp, code >> 1, Un);
      to_abs<double, D>(Un, UR, ph);
#pragma unroll
      for (int v = 0; v < V; v++) UB[v] = UR[v];
    }
    else
      ghost_state<double, D>(-code - 1, Ua, n, UR, UB, ph);
    const double ws = fmax(wave_speed<D>(Ua, n, ph.gamma), wave_speed<D>(UR, n, ph.gamma));
    if (cfl_type == 1)
      int_ws += wf[f % NF] * ws * dA;
    else
    {
      const double h = h_ref[pf * TW + l];
      double t = ws / (c_adv * h);
      if (visc) t += fmax(diff_coef(Ua[0], ph), diff_coef(UB[0], ph)) / (c_diff * h * h);
      dtinv[f / NF] = fmax(dtinv[f / NF], t);
    }
  }
  double dt;
  if (cfl_type == 1)
    dt = 2.0 * cfl * c_adv * evol[e] / int_ws;
  else if constexpr (D == 2)
    dt = cfl / (fmax(dtinv[0], dtinv[2]) + fmax(dtinv[1], dtinv[3]));  // quad faces: 0/2 and 1/3 opposite
  else
    dt = cfl / (fmax(dtinv[0], dtinv[1]) + fmax(dtinv[2], dtinv[3]) + fmax(dtinv[4], dtinv[5]));
  dt_ele[e] = dt;
  atomicMin(dt_min, (unsigned long long)__double_as_longlong(dt));
}

static __global__ void k_dt_reset(double *d_dt)
{
  d_dt[0] = __longlong_as_double(0x7ff0000000000000LL);  // +inf
}

// after a CFL-stepped RK44 step: flow time += dt(0) (the global step, or
// element 0's under local stepping, as the reference's prev_time + dt(0))
static __global__ void k_dt_advance(double *d_dt, const double *dt_ele, int local)
{
  d_dt[2] += local ? dt_ele[0] : d_dt[0];
}

}  // namespace dev

template <typename T, typename A, int D, int N>
static void launch_dt_impl(Ctx &c)
{
  const Args<T, A> a = make_args<T, A>(c, StageCfg{0, 0, 0, 0});
  const dev::Phys<double> ph = phys_of<double>(c.plan.params, c.uref, c.D, c.prec != ZB_FP64);
  const int P = c.plan.order;
  dev::k_dt_reset<<<1, 1, 0, c.stream>>>(c.d_dt);
  const int64_t n = c.ntiles * TW;
  dev::k_element_dt<T, D, N><<<(unsigned)((n + 127) / 128), 128, 0, c.stream>>>(
      a.Ufp, a.fgeo, a.nbr, c.h_ref, c.evol, c.dfw, c.ntiles, c.plan.neles, ph, c.plan.params.viscous,
      c.ts.cfl_type, c.ts.cfl, cfl_limit_adv(P), cfl_limit_diff(P, c.plan.params.ldg_b), c.dt_ele,
      reinterpret_cast<unsigned long long *>(c.d_dt));
  c.launches += 2;
  CK(cudaGetLastError());
}

}  // namespace zb
