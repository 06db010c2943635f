// Pointwise Euler / Navier-Stokes physics of the DFR residual, templated on the
// arithmetic type T (double for the plain form, float for the mixed form) and
// the dimension D.  Each function restates a reference routine; the reference
// location is given beside it.  Grid velocity is zero (static meshes).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

// Pointwise functions compile for the host too (unit tests of the adjoint
// algebra run them on the CPU).
#ifndef ZB_HD
#define ZB_HD __host__ __device__ __forceinline__
#endif

namespace zb {
namespace dev {

template <typename T>
struct Phys
{
  T gamma, prandtl, mu, rt, c_sth;
  T rus_k, ldg_b, ldg_tau;
  T rho_fs, V_fs[3], P_fs, T_wall, R_ref, V_wall[3];
  int fix_vis, fconv;
  // Reference state of the perturbation form (mixed precision): the stored
  // state is U' = U - Ur.  Pr = p(Ur), er = Er + Pr, inv_rr = 1/rho_r,
  // mr2 = |m_r|^2.
  T Ur[5], Pr, er, inv_rr, mr2;
  int dev;  // 1: stored states are deviations from Ur (FP32 storage)
};

// Arithmetic of the perturbation form: FP32 stores deviations from Ur.
template <typename T> struct Pert { static constexpr bool on = false; };
template <> struct Pert<float> { static constexpr bool on = true; };
// plain FP64 arithmetic (not the perturbation form, not dual numbers)
template <typename T> struct IsF64 { static constexpr bool on = false; };
template <> struct IsF64<double> { static constexpr bool on = true; };

template <typename T> ZB_HD T dsqrt(T x);
template <> ZB_HD double dsqrt<double>(double x) { return sqrt(x); }
template <> ZB_HD float dsqrt<float>(float x) { return sqrtf(x); }
template <typename T> ZB_HD T dpow(T x, T y);
template <> ZB_HD double dpow<double>(double x, double y) { return pow(x, y); }
template <> ZB_HD float dpow<float>(float x, float y) { return powf(x, y); }
// reciprocal square root: CUDA's rsqrt on the device (max 1 ulp error), the
// quotient on the host
template <typename T> ZB_HD T drsqrt(T x);
template <> ZB_HD double drsqrt<double>(double x)
{
#ifdef __CUDA_ARCH__
  return rsqrt(x);
#else
  return 1.0 / sqrt(x);
#endif
}
template <typename T> ZB_HD T dabs(T x) { return x < T(0) ? -x : x; }
template <typename T> ZB_HD T dmax(T a, T b) { return a > b ? a : b; }

// Inviscid flux F[var][dim] and pressure (include/flux.hpp:11-63, Vg = 0).
template <typename T, int D>
ZB_HD void flux_conv(const T U[D + 2], T F[D + 2][D], T &P, T gamma)
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

// Inviscid flux deviation F(Ur + Up) - F(Ur), absolute pressure P and its
// deviation Pp, written so no O(1) constant cancels (the flux of
// include/flux.hpp:11-63 expanded about the reference state Ur):
//   |m|^2/rho - |mr|^2/rho_r = (2 mr.m' + |m'|^2)/rho - |mr|^2 rho'/(rho rho_r)
//   m_k m_d/rho - mr_k mr_d/rho_r = (mr_k m'_d + m'_k mr_d + m'_k m'_d)/rho
//                                   - mr_k mr_d rho'/(rho rho_r)
//   m_d e/rho - mr_d er/rho_r = (m'_d er + mr_d e' + m'_d e')/rho - mr_d er rho'/(rho rho_r)
// with e = E + P the total enthalpy per volume.
template <typename T, int D>
ZB_HD void flux_conv_pert(const T Up[D + 2], T F[D + 2][D], T &P, T &Pp, const Phys<T> &ph)
{
  const T *Ur = ph.Ur;
  const T rho = Ur[0] + Up[0];
  const T invr = T(1) / rho;
  const T c = Up[0] * invr * ph.inv_rr;  // rho' / (rho rho_r)
  T mrmp = Ur[1] * Up[1], mpmp = Up[1] * Up[1];
#pragma unroll
  for (int d = 1; d < D; d++)
  {
    mrmp += Ur[d + 1] * Up[d + 1];
    mpmp += Up[d + 1] * Up[d + 1];
  }
  const T dke2 = (T(2) * mrmp + mpmp) * invr - ph.mr2 * c;
  Pp = (ph.gamma - T(1)) * (Up[D + 1] - T(0.5) * dke2);
  P = ph.Pr + Pp;
  const T ep = Up[D + 1] + Pp;
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    F[0][d] = Up[d + 1];
#pragma unroll
    for (int k = 0; k < D; k++)
      F[k + 1][d] = (Ur[k + 1] * Up[d + 1] + Up[k + 1] * Ur[d + 1] + Up[k + 1] * Up[d + 1]) * invr -
                    Ur[k + 1] * Ur[d + 1] * c + (k == d ? Pp : T(0));
    F[D + 1][d] = (Up[d + 1] * ph.er + Ur[d + 1] * ep + Up[d + 1] * ep) * invr - Ur[d + 1] * ph.er * c;
  }
}

// absolute state from a stored one (identity outside the perturbation form)
template <typename T, int D>
ZB_HD void to_abs(const T Us[D + 2], T Ua[D + 2], const Phys<T> &ph)
{
#pragma unroll
  for (int v = 0; v < D + 2; v++) Ua[v] = ph.dev ? ph.Ur[v] + Us[v] : Us[v];
}

template <typename T, int D>
ZB_HD void to_stored(const T Ua[D + 2], T Us[D + 2], const Phys<T> &ph)
{
#pragma unroll
  for (int v = 0; v < D + 2; v++) Us[v] = ph.dev ? Ua[v] - ph.Ur[v] : Ua[v];
}

// Inviscid flux of a stored state (deviation from Ur in the perturbation form)
// and the absolute pressure.
template <typename T, int D>
ZB_HD void flux_conv_stored(const T Us[D + 2], T F[D + 2][D], T &P, T &Pp, const Phys<T> &ph)
{
  if constexpr (Pert<T>::on)
    flux_conv_pert<T, D>(Us, F, P, Pp, ph);
  else
  {
    // FP64 arithmetic: absolute flux (a stored deviation is added back exactly)
    T Ua[D + 2];
    to_abs<T, D>(Us, Ua, ph);
    flux_conv<T, D>(Ua, F, P, ph.gamma);
    Pp = P;
  }
}

// Viscous flux added to F (include/flux.hpp:71-202): F -= tau / heat flux.
template <typename T, int D>
ZB_HD void flux_visc_add(const T U[D + 2], const T dU[D + 2][D], T F[D + 2][D],
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
  const T diag = div * (T(1) / T(3));
  T tau[D][D];
#pragma unroll
  for (int i = 0; i < D; i++)
#pragma unroll
    for (int j = 0; j < D; j++)
      tau[i][j] = (i == j) ? T(2) * mu * (dvel[i][i] - diag) : mu * (dvel[i][j] + dvel[j][i]);
  const T kappa = mu * (ph.gamma / ph.prandtl);  // gamma / Pr is loop-invariant
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
ZB_HD void visc_normal(const T U[D + 2], const T dU[D + 2][D], const T n[D],
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
// UL, UR are stored states (deviations from Ur in the perturbation form); the
// result is the common flux of the stored form (minus F(Ur).n).
template <typename T, int D>
ZB_HD void rusanov(const T UL[D + 2], const T UR[D + 2], const T n[D], T Fc[D + 2],
                                        const Phys<T> &ph)
{
  T FL[D + 2][D], FR[D + 2][D], PL, PR, QL, QR;
  flux_conv_stored<T, D>(UL, FL, PL, QL, ph);
  flux_conv_stored<T, D>(UR, FR, PR, QR, ph);
  T AL[D + 2], AR[D + 2];
  to_abs<T, D>(UL, AL, ph);
  to_abs<T, D>(UR, AR, ph);
  const T irL = T(1) / AL[0], irR = T(1) / AR[0];
  const T aL = dsqrt<T>(ph.gamma * PL * irL);
  const T aR = dsqrt<T>(ph.gamma * PR * irR);
  T VnL = AL[1] * irL * n[0], VnR = AR[1] * irR * n[0];
#pragma unroll
  for (int d = 1; d < D; d++)
  {
    VnL += AL[d + 1] * irL * n[d];
    VnR += AR[d + 1] * irR * n[d];
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
ZB_HD void roe_plain(const T SL[D + 2], const T SR[D + 2], const T n[D], T Fc[D + 2], const Phys<T> &ph);

template <typename T, int D>
ZB_HD void roe(const T SL[D + 2], const T SR[D + 2], const T n[D], T Fc[D + 2],
                                    const Phys<T> &ph)
{
  if constexpr (IsF64<T>::on)
  {
    roe_plain<T, D>(SL, SR, n, Fc, ph);
    return;
  }
  const T g = ph.gamma;
  T FL[D + 2][D], FR[D + 2][D], PL, PR, QL, QR;
  flux_conv_stored<T, D>(SL, FL, PL, QL, ph);
  flux_conv_stored<T, D>(SR, FR, PR, QR, ph);
  T UL[D + 2], UR[D + 2];
  to_abs<T, D>(SL, UL, ph);
  to_abs<T, D>(SR, UR, ph);
  const T rL = UL[0], rR = UR[0];
  const T sL = dsqrt<T>(rL), sR = dsqrt<T>(rR);
  const T inv = T(1) / (sL + sR);
  // one reciprocal per state: velocities and enthalpies by multiplication
  const T irL = T(1) / rL, irR = T(1) / rR;
  T u[D], uL[D], uR[D];
  T unL = T(0), unR = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    uL[d] = UL[d + 1] * irL;
    uR[d] = UR[d + 1] * irR;
    u[d] = (sL * uL[d] + sR * uR[d]) * inv;
    unL += uL[d] * n[d];
    unR += uR[d] * n[d];
  }
  const T HL = (UL[D + 1] + PL) * irL, HR = (UR[D + 1] + PR) * irR;
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
  const T ia2 = T(1) / a2;
  const T rho = sL * sR;
  const T dp = QR - QL, dr = SR[0] - SL[0], dun = unR - unL;
  // wave strengths
  const T a1 = (dp - rho * a * dun) * (T(0.5) * ia2);
  const T a3 = (dp + rho * a * dun) * (T(0.5) * ia2);
  const T a2w = dr - dp * ia2;
  T l1 = dabs<T>(un - a), l2 = dabs<T>(un), l3 = dabs<T>(un + a);
  const T delta = T(0.1) * (dabs<T>(un) + a);
  const T i2d = T(0.5) / delta;
  if (l1 < delta) l1 = (l1 * l1 + delta * delta) * i2d;
  if (l2 < delta) l2 = (l2 * l2 + delta * delta) * i2d;
  if (l3 < delta) l3 = (l3 * l3 + delta * delta) * i2d;
  // |A| dU = l1 a1 r1 + l2 (a2w r2 + rho dv_t) + l3 a3 r3
  T diss[D + 2];
  diss[0] = l1 * a1 + l2 * a2w + l3 * a3;
  T udvt = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    const T dvt = (uR[d] - uL[d]) - dun * n[d];
    diss[d + 1] = l1 * a1 * (u[d] - a * n[d]) + l2 * (a2w * u[d] + rho * dvt) + l3 * a3 * (u[d] + a * n[d]);
    udvt += u[d] * dvt;
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

// The same Roe flux in FP64 arithmetic on absolute states: the normal fluxes
// F(U).n = [m.n, m u.n + p n, (E + p) u.n] directly, and 1/rho, sqrt(rho),
// the sound speed and 1/a^2 from reciprocal square roots (three rsqrt and
// two divisions per face in place of three square roots and seven
// divisions); equal to the form above to a few ulp.
template <typename T, int D>
ZB_HD void roe_plain(const T SL[D + 2], const T SR[D + 2], const T n[D], T Fc[D + 2], const Phys<T> &ph)
{
  const T g = ph.gamma;
  T UL[D + 2], UR[D + 2];
  to_abs<T, D>(SL, UL, ph);
  to_abs<T, D>(SR, UR, ph);
  const T rL = UL[0], rR = UR[0];
  const T rsL = drsqrt<T>(rL), rsR = drsqrt<T>(rR);
  const T sL = rL * rsL, sR = rR * rsR;      // sqrt(rho)
  const T irL = rsL * rsL, irR = rsR * rsR;  // 1 / rho
  const T inv = T(1) / (sL + sR);
  T u[D], uL[D], uR[D];
  T unL = T(0), unR = T(0), kL = T(0), kR = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    uL[d] = UL[d + 1] * irL;
    uR[d] = UR[d + 1] * irR;
    u[d] = (sL * uL[d] + sR * uR[d]) * inv;
    unL += uL[d] * n[d];
    unR += uR[d] * n[d];
    kL += UL[d + 1] * uL[d];  // |m|^2 / rho
    kR += UR[d + 1] * uR[d];
  }
  const T PL = (g - T(1)) * (UL[D + 1] - T(0.5) * kL), PR = (g - T(1)) * (UR[D + 1] - T(0.5) * kR);
  const T HL = (UL[D + 1] + PL) * irL, HR = (UR[D + 1] + PR) * irR;
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
  const T ra = drsqrt<T>(a2);
  const T a = a2 * ra, ia2 = ra * ra;
  const T rho = sL * sR;
  const T dp = PR - PL, dr = UR[0] - UL[0], dun = unR - unL;
  const T a1 = (dp - rho * a * dun) * (T(0.5) * ia2);
  const T a3 = (dp + rho * a * dun) * (T(0.5) * ia2);
  const T a2w = dr - dp * ia2;
  T l1 = dabs<T>(un - a), l2 = dabs<T>(un), l3 = dabs<T>(un + a);
  const T delta = T(0.1) * (dabs<T>(un) + a);
  const T i2d = T(0.5) / delta;
  if (l1 < delta) l1 = (l1 * l1 + delta * delta) * i2d;
  if (l2 < delta) l2 = (l2 * l2 + delta * delta) * i2d;
  if (l3 < delta) l3 = (l3 * l3 + delta * delta) * i2d;
  T diss[D + 2];
  diss[0] = l1 * a1 + l2 * a2w + l3 * a3;
  T udvt = T(0);
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    const T dvt = (uR[d] - uL[d]) - dun * n[d];
    diss[d + 1] = l1 * a1 * (u[d] - a * n[d]) + l2 * (a2w * u[d] + rho * dvt) + l3 * a3 * (u[d] + a * n[d]);
    udvt += u[d] * dvt;
  }
  diss[D + 1] = l1 * a1 * (H - a * un) + l2 * (a2w * T(0.5) * q2 + rho * udvt) + l3 * a3 * (H + a * un);
  const T mnL = rL * unL, mnR = rR * unR;
  Fc[0] = T(0.5) * (mnL + mnR) - T(0.5) * diss[0];
#pragma unroll
  for (int d = 0; d < D; d++)
    Fc[d + 1] = T(0.5) * ((UL[d + 1] * unL + PL * n[d]) + (UR[d + 1] * unR + PR * n[d])) - T(0.5) * diss[d + 1];
  Fc[D + 1] = T(0.5) * (mnL * HL + mnR * HR) - T(0.5) * diss[D + 1];
}

// Boundary ghost states (src/faces.cpp:123-506, explicit time stepping so
// rus_bias = 0: Rusanov uses the ghost state UR, LDG the prescribed state UB).
// Returns false for a boundary code with no ghost state.
template <typename T, int D>
ZB_HD void ghost_state(int bc, const T UL[D + 2], const T n[D], T UR[D + 2], T UB[D + 2],
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
ZB_HD void ghost_grad(int bc, const T UL[D + 2], const T dUL[D + 2][D], const T n[D],
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
