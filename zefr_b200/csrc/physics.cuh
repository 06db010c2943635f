// Pointwise Euler / Navier-Stokes physics of the DFR residual, templated on the
// arithmetic type T (double for the plain form, float for the mixed form) and
// the dimension D.  Each function restates a reference routine; the reference
// location is given beside it.  Grid velocity is zero (static meshes).
#pragma once

#include <cuda_runtime.h>

namespace zb {
namespace dev {

template <typename T>
struct Phys
{
  T gamma, prandtl, mu, rt, c_sth;
  T rus_k, ldg_b, ldg_tau;
  T rho_fs, V_fs[3], P_fs, T_wall, R_ref, V_wall[3];
  int fix_vis, fconv;
};

template <typename T> __device__ __forceinline__ T dsqrt(T x);
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <typename T> __device__ __forceinline__ T dpow(T x, T y);
template <> __device__ __forceinline__ double dpow<double>(double x, double y) { return pow(x, y); }
template <> __device__ __forceinline__ float dpow<float>(float x, float y) { return powf(x, y); }
template <typename T> __device__ __forceinline__ T dabs(T x) { return x < T(0) ? -x : x; }
template <typename T> __device__ __forceinline__ T dmax(T a, T b) { return a > b ? a : b; }

// Inviscid flux F[var][dim] and pressure (include/flux.hpp:11-63, Vg = 0).
template <typename T, int D>
__device__ __forceinline__ void flux_conv(const T U[D + 2], T F[D + 2][D], T &P, T gamma)
{
  const T invrho = T(1) / U[0];
  T momF = U[1] * U[1];
#pragma unroll
  for (int d = 1; d < D; d++) momF += U[d + 1] * U[d + 1];
  momF *= invrho;
  P = (gamma - T(1)) * (U[D + 1] - T(0.5) * momF);
  const T H = (U[D + 1] + P) * invrho;
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    F[0][d] = U[d + 1];
#pragma unroll
    for (int k = 0; k < D; k++) F[k + 1][d] = U[d + 1] * U[k + 1] * invrho + (k == d ? P : T(0));
    F[D + 1][d] = U[d + 1] * H;
  }
}

// Viscous flux added to F (include/flux.hpp:71-202): F -= tau / heat flux.
template <typename T, int D>
__device__ __forceinline__ void flux_visc_add(const T U[D + 2], const T dU[D + 2][D], T F[D + 2][D],
                                              const Phys<T> &ph)
{
  const T invrho = T(1) / U[0];
  T vel[D];
#pragma unroll
  for (int d = 0; d < D; d++) vel[d] = U[d + 1] * invrho;
  T vsq = vel[0] * vel[0];
#pragma unroll
  for (int d = 1; d < D; d++) vsq += vel[d] * vel[d];
  const T e_int = U[D + 1] * invrho - T(0.5) * vsq;
  T mu;
  if (ph.fix_vis)
    mu = ph.mu;
  else
  {
    const T rt_ratio = (ph.gamma - T(1)) * e_int / ph.rt;
    mu = ph.mu * dpow<T>(rt_ratio, T(1.5)) * (T(1) + ph.c_sth) / (rt_ratio + ph.c_sth);
  }
  // dvel[i][j] = d u_i / d x_j
  T dvel[D][D];
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++) dvel[i][j] = (dU[i + 1][j] - dU[0][j] * vel[i]) * invrho;
  T de[D];
#pragma unroll
  for (int j = 0; j < D; j++)
  {
    T s = vel[0] * dvel[0][j];
#pragma unroll
    for (int i = 1; i < D; i++) s += vel[i] * dvel[i][j];
    const T dke = T(0.5) * vsq * dU[0][j] + U[0] * s;
    de[j] = (dU[D + 1][j] - dke - dU[0][j] * e_int) * invrho;
  }
  T div = dvel[0][0];
#pragma unroll
  for (int d = 1; d < D; d++) div += dvel[d][d];
  const T diag = div / T(3);
  T tau[D][D];
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++)
      tau[i][j] = (i == j) ? T(2) * mu * (dvel[i][i] - diag) : mu * (dvel[i][j] + dvel[j][i]);
  const T kappa = (mu / ph.prandtl) * ph.gamma;
#pragma unroll
  for (int j = 0; j < D; j++)
  {
#pragma unroll
    for (int i = 0; i < D; i++) F[i + 1][j] -= tau[i][j];
    T w = vel[0] * tau[0][j];
#pragma unroll
    for (int i = 1; i < D; i++) w += vel[i] * tau[i][j];
    F[D + 1][j] -= (w + kappa * de[j]);
  }
}

// Normal viscous flux from one side: (F_visc(U, dU)) . n
template <typename T, int D>
__device__ __forceinline__ void visc_normal(const T U[D + 2], const T dU[D + 2][D], const T n[D],
                                            T Fn[D + 2], const Phys<T> &ph)
{
  T F[D + 2][D];
#pragma unroll
  for (int v = 0; v < D + 2; v++)
#pragma unroll
    for (int d = 0; d < D; d++) F[v][d] = T(0);
  flux_visc_add<T, D>(U, dU, F, ph);
#pragma unroll
  for (int v = 0; v < D + 2; v++)
  {
    T s = F[v][0] * n[0];
#pragma unroll
    for (int d = 1; d < D; d++) s += F[v][d] * n[d];
    Fn[v] = s;
  }
}

// Rusanov common normal flux, upwinded form (src/faces.cpp:1243-1364, rus_bias 0).
template <typename T, int D>
__device__ __forceinline__ void rusanov(const T UL[D + 2], const T UR[D + 2], const T n[D], T Fc[D + 2],
                                        const Phys<T> &ph)
{
  T FL[D + 2][D], FR[D + 2][D], PL, PR;
  flux_conv<T, D>(UL, FL, PL, ph.gamma);
  flux_conv<T, D>(UR, FR, PR, ph.gamma);
  const T aL = dsqrt<T>(ph.gamma * PL / UL[0]);
  const T aR = dsqrt<T>(ph.gamma * PR / UR[0]);
  T VnL = UL[1] / UL[0] * n[0], VnR = UR[1] / UR[0] * n[0];
#pragma unroll
  for (int d = 1; d < D; d++)
  {
    VnL += UL[d + 1] / UL[0] * n[d];
    VnR += UR[d + 1] / UR[0] * n[d];
  }
  const T eig = dmax<T>(dabs<T>(VnL) + aL, dabs<T>(VnR) + aR);
  const T diss = T(0.5) * eig * (T(1) - ph.rus_k);
#pragma unroll
  for (int v = 0; v < D + 2; v++)
  {
    T fl = FL[v][0] * n[0], fr = FR[v][0] * n[0];
#pragma unroll
    for (int d = 1; d < D; d++)
    {
      fl += FL[v][d] * n[d];
      fr += FR[v][d] * n[d];
    }
    Fc[v] = T(0.5) * (fr + fl) - diss * (UR[v] - UL[v]);
  }
}

// Roe approximate Riemann solver (Roe 1981, J. Comput. Phys. 43:357) in the
// eigen-decomposition form of Toro, "Riemann Solvers and Numerical Methods",
// sec. 11.3, with Harten's entropy fix (Harten & Hyman 1983): an eigenvalue
// |l| below delta = 0.1 * (|u_n| + a) of the Roe state is replaced by
// (l^2 + delta^2) / (2 delta).  No reference counterpart.
template <typename T, int D>
__device__ __forceinline__ void roe(const T UL[D + 2], const T UR[D + 2], const T n[D], T Fc[D + 2],
                                    const Phys<T> &ph)
{
  const T g = ph.gamma;
  T FL[D + 2][D], FR[D + 2][D], PL, PR;
  flux_conv<T, D>(UL, FL, PL, g);
  flux_conv<T, D>(UR, FR, PR, g);
  const T rL = UL[0], rR = UR[0];
  const T sL = dsqrt<T>(rL), sR = dsqrt<T>(rR);
  const T inv = T(1) / (sL + sR);
  T u[D];
  T unL = T(0), unR = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    const T uL = UL[d + 1] / rL, uR = UR[d + 1] / rR;
    u[d] = (sL * uL + sR * uR) * inv;
    unL += uL * n[d];
    unR += uR * n[d];
  }
  const T HL = (UL[D + 1] + PL) / rL, HR = (UR[D + 1] + PR) / rR;
  const T H = (sL * HL + sR * HR) * inv;
  T q2 = T(0), un = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    q2 += u[d] * u[d];
    un += u[d] * n[d];
  }
  T a2 = (g - T(1)) * (H - T(0.5) * q2);
  a2 = dmax<T>(a2, T(1e-30));
  const T a = dsqrt<T>(a2);
  const T rho = sL * sR;
  const T dp = PR - PL, dr = rR - rL, dun = unR - unL;
  // wave strengths
  const T a1 = (dp - rho * a * dun) / (T(2) * a2);
  const T a3 = (dp + rho * a * dun) / (T(2) * a2);
  const T a2w = dr - dp / a2;
  T l1 = dabs<T>(un - a), l2 = dabs<T>(un), l3 = dabs<T>(un + a);
  const T delta = T(0.1) * (dabs<T>(un) + a);
  if (l1 < delta) l1 = (l1 * l1 + delta * delta) / (T(2) * delta);
  if (l2 < delta) l2 = (l2 * l2 + delta * delta) / (T(2) * delta);
  if (l3 < delta) l3 = (l3 * l3 + delta * delta) / (T(2) * delta);
  // |A| dU = l1 a1 r1 + l2 (a2w r2 + rho dv_t) + l3 a3 r3
  T diss[D + 2];
  diss[0] = l1 * a1 + l2 * a2w + l3 * a3;
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    const T uLd = UL[d + 1] / rL, uRd = UR[d + 1] / rR;
    const T dvt = (uRd - uLd) - dun * n[d];
    diss[d + 1] = l1 * a1 * (u[d] - a * n[d]) + l2 * (a2w * u[d] + rho * dvt) + l3 * a3 * (u[d] + a * n[d]);
  }
  T udvt = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    const T uLd = UL[d + 1] / rL, uRd = UR[d + 1] / rR;
    udvt += u[d] * ((uRd - uLd) - dun * n[d]);
  }
  diss[D + 1] = l1 * a1 * (H - a * un) + l2 * (a2w * T(0.5) * q2 + rho * udvt) + l3 * a3 * (H + a * un);
#pragma unroll
  for (int v = 0; v < D + 2; v++)
  {
    T fl = FL[v][0] * n[0], fr = FR[v][0] * n[0];
#pragma unroll
    for (int d = 1; d < D; d++)
    {
      fl += FL[v][d] * n[d];
      fr += FR[v][d] * n[d];
    }
    Fc[v] = T(0.5) * (fl + fr) - T(0.5) * diss[v];
  }
}

// Boundary ghost states (src/faces.cpp:123-506, explicit time stepping so
// rus_bias = 0: Rusanov uses the ghost state UR, LDG the prescribed state UB).
// Returns false for a boundary code with no ghost state.
template <typename T, int D>
__device__ __forceinline__ void ghost_state(int bc, const T UL[D + 2], const T n[D], T UR[D + 2], T UB[D + 2],
                                            const Phys<T> &ph)
{
  const T g = ph.gamma;
  switch (bc)
  {
    case 3:  // SUP_IN / farfield
    {
      T vsq = T(0);
      UR[0] = ph.rho_fs;
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        UR[d + 1] = ph.rho_fs * ph.V_fs[d];
        vsq += ph.V_fs[d] * ph.V_fs[d];
      }
      UR[D + 1] = ph.P_fs / (g - T(1)) + T(0.5) * ph.rho_fs * vsq;
#pragma unroll
      for (int v = 0; v < D + 2; v++) UB[v] = UR[v];
      break;
    }
    case 4:  // SUP_OUT
    {
#pragma unroll
      for (int v = 0; v < D + 2; v++) UR[v] = UB[v] = UL[v];
      break;
    }
    case 2:  // CHAR (Riemann invariants)
    {
      T VnL = T(0), VnR = T(0), momF = T(0);
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        VnL += UL[d + 1] / UL[0] * n[d];
        VnR += ph.V_fs[d] * n[d];
      }
#pragma unroll
      for (int d = 0; d < D; d++) momF += UL[d + 1] * UL[d + 1];
      momF /= UL[0];
      const T PL = (g - T(1)) * (UL[D + 1] - T(0.5) * momF);
      T PR = ph.P_fs;
      const T cL = dsqrt<T>(g * PL / UL[0]);
      const T cR = dsqrt<T>(g * PR / ph.rho_fs);
      T RL, RB;
      if (dabs<T>(VnR) >= cR && VnL >= T(0))
        RL = VnR + T(2) / (g - T(1)) * cR;
      else
        RL = VnL + T(2) / (g - T(1)) * cL;
      if (dabs<T>(VnR) >= cR && VnL < T(0))
        RB = VnL - T(2) / (g - T(1)) * cL;
      else
        RB = VnR - T(2) / (g - T(1)) * cR;
      const T cstar = T(0.25) * (g - T(1)) * (RL - RB);
      const T ustarn = T(0.5) * (RL + RB);
      T rhoR = cstar * cstar / g;
      T VR[D];
      if (VnL < T(0))
      {
        rhoR *= dpow<T>(ph.rho_fs, g) / PR;
#pragma unroll
        for (int d = 0; d < D; d++) VR[d] = ph.V_fs[d] + (ustarn - VnR) * n[d];
      }
      else
      {
        rhoR *= dpow<T>(UL[0], g) / PL;
#pragma unroll
        for (int d = 0; d < D; d++) VR[d] = UL[d + 1] / UL[0] + (ustarn - VnL) * n[d];
      }
      rhoR = dpow<T>(rhoR, T(1) / (g - T(1)));
      UR[0] = rhoR;
#pragma unroll
      for (int d = 0; d < D; d++) UR[d + 1] = rhoR * VR[d];
      PR = rhoR / g * cstar * cstar;
      UR[D + 1] = PR / (g - T(1));
#pragma unroll
      for (int d = 0; d < D; d++) UR[D + 1] += T(0.5) * rhoR * VR[d] * VR[d];
#pragma unroll
      for (int v = 0; v < D + 2; v++) UB[v] = UR[v];
      break;
    }
    case 5:   // SLIP_WALL
    case 11:  // SYMMETRY: reflected normal momentum
    {
      T momN = T(0);
#pragma unroll
      for (int d = 0; d < D; d++) momN += UL[d + 1] * n[d];
      UR[0] = UL[0];
#pragma unroll
      for (int d = 0; d < D; d++) UR[d + 1] = UL[d + 1] - T(2) * momN * n[d];
      UR[D + 1] = UL[D + 1];
#pragma unroll
      for (int v = 0; v < D + 2; v++) UB[v] = UR[v];
      break;
    }
    case 6:  // ISOTHERMAL_NOSLIP (static wall)
    case 8:  // ISOTHERMAL_NOSLIP_MOVING
    {
      const T rhoL = UL[0];
      const bool moving = (bc == 8);
      UR[0] = rhoL;
      UB[0] = rhoL;
      T vsq = T(0), vwsq = T(0);
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        const T vw = moving ? ph.V_wall[d] : T(0);
        const T VL = UL[d + 1] / rhoL;
        const T V = -VL + T(2) * vw;
        UR[d + 1] = rhoL * V;
        vsq += V * V;
        UB[d + 1] = moving ? rhoL * vw : vw;
        vwsq += vw * vw;
      }
      const T cp_over_gam = ph.R_ref / (g - T(1));
      UR[D + 1] = rhoL * (cp_over_gam * ph.T_wall + T(0.5) * vsq);
      UB[D + 1] = moving ? rhoL * (cp_over_gam * ph.T_wall + T(0.5) * vwsq) : rhoL * cp_over_gam * ph.T_wall;
      break;
    }
    case 7:  // ADIABATIC_NOSLIP
    case 9:  // ADIABATIC_NOSLIP_MOVING
    {
      const T rhoL = UL[0];
      const bool moving = (bc == 9);
      UR[0] = rhoL;
      UB[0] = rhoL;
      T vsq = T(0), vlsq = T(0), vwsq = T(0);
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        const T vw = moving ? ph.V_wall[d] : T(0);
        const T VL = UL[d + 1] / rhoL;
        const T V = -VL + T(2) * vw;
        UR[d + 1] = rhoL * V;
        UB[d + 1] = rhoL * vw;
        vsq += V * V;
        vlsq += VL * VL;
        vwsq += vw * vw;
      }
      const T EL = UL[D + 1];
      UR[D + 1] = EL + T(0.5) * rhoL * (vsq - vlsq);
      UB[D + 1] = moving ? EL - T(0.5) * rhoL * (vlsq + vwsq) : EL + T(0.5) * rhoL * (vwsq - vlsq);
      break;
    }
    default:
    {
#pragma unroll
      for (int v = 0; v < D + 2; v++) UR[v] = UB[v] = UL[v];
      break;
    }
  }
}

// Boundary gradient (src/faces.cpp:508-710): copy, except adiabatic walls
// remove the wall-normal temperature gradient from the energy gradient.
template <typename T, int D>
__device__ __forceinline__ void ghost_grad(int bc, const T UL[D + 2], const T dUL[D + 2][D], const T n[D],
                                           T dUR[D + 2][D])
{
#pragma unroll
  for (int v = 0; v < D + 2; v++)
#pragma unroll
    for (int d = 0; d < D; d++) dUR[v][d] = dUL[v][d];
  if (bc == 7 || bc == 9)
  {
    const T rho = UL[0], E = UL[D + 1];
    T vel[D];
#pragma unroll
    for (int d = 0; d < D; d++) vel[d] = UL[d + 1] / rho;
    T dTn = T(0);
#pragma unroll
    for (int j = 0; j < D; j++)
    {
      T s = T(0);
#pragma unroll
      for (int i = 0; i < D; i++) s += vel[i] * ((dUL[i + 1][j] - dUL[0][j] * vel[i]) / rho);
      const T dT = dUL[D + 1][j] - dUL[0][j] * E / rho - rho * s;
      dTn += dT * n[j];
    }
#pragma unroll
    for (int j = 0; j < D; j++) dUR[D + 1][j] = dUL[D + 1][j] - dTn * n[j];
  }
}

}  // namespace dev
}  // namespace zb
