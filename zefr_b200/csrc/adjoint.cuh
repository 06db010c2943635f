// Adjoint (vector-Jacobian product) of the DFR residual, plain FP64 form.
//
// For a weight lam on the residual divF(U) of FRSolver::compute_residual
// (src/solver.cpp:1494-1645) the kernels return Ubar = (d divF / d U)^T lam.
// The reverse pass mirrors the forward kernels of dfr_kernels.cuh:
//   - every line operator is applied transposed (Dm^T, Em^T, the surface
//     lifting coefficients -Dbm / Dbp transposed into a flux point weight);
//   - face coupling is gathered, never scattered: both elements of a face pair
//     evaluate the vector-Jacobian product of the common flux with the summed
//     weight of both sides and keep the part for their own trace, so no
//     atomics are needed and the result is deterministic;
//   - pointwise Jacobian-transpose products are hand-written reverse mode for
//     the fluxes and Riemann solvers (flux_conv_vjp, flux_visc_vjp,
//     rusanov_vjp, roe_vjp) and forward-mode dual numbers (dual.cuh) for the
//     boundary ghost states and gradients, which run on boundary faces only.
// Navier-Stokes needs three passes because the LDG common solution couples the
// gradient of one element to the trace of its neighbour.
#pragma once

#include "dfr_kernels.cuh"
#include "dual.cuh"

// Boundary-face functions run on few flux points and hold many dual numbers.
// In 3D they are called out of line, so their registers do not weigh on the
// interior path; in 2D they are inlined (their frames are small, and a call
// from the register-bound 2D kernels costs more than the registers).
#define ZB_HD_COLD __host__ __device__ __noinline__
#define ZB_HD_INLINE __host__ __device__ __forceinline__

namespace zb {
namespace dev {

// ---------------------------------------------------------------------------
// Pointwise reverse mode (restating the forward functions of physics.cuh)
// ---------------------------------------------------------------------------

// Ub += (d F / d U)^T Fb for the inviscid flux F[var][dim] of flux_conv.
template <int D>
ZB_HD void flux_conv_vjp(const double U[D + 2], const double Fb[D + 2][D], double gamma, double Ub[D + 2])
{
  constexpr int V = D + 2;
  const double ir = 1.0 / U[0];
  double u[D], m2 = 0.0;
  for (int k = 0; k < D; k++)
  {
    u[k] = U[k + 1] * ir;
    m2 += U[k + 1] * U[k + 1];
  }
  const double q = 0.5 * m2 * ir;
  const double P = (gamma - 1.0) * (U[V - 1] - q);
  const double H = (U[V - 1] + P) * ir;
  double mb[D], ub[D], Pb = 0.0, Hb = 0.0;
  for (int d = 0; d < D; d++)
  {
    double s = Fb[0][d] + Fb[V - 1][d] * H;
    for (int k = 0; k < D; k++) s += Fb[k + 1][d] * u[k];
    mb[d] = s;
    Hb += Fb[V - 1][d] * U[d + 1];
    Pb += Fb[d + 1][d];
  }
  for (int k = 0; k < D; k++)
  {
    double s = 0.0;
    for (int d = 0; d < D; d++) s += Fb[k + 1][d] * U[d + 1];
    ub[k] = s;
  }
  double Eb = Hb * ir;
  Pb += Hb * ir;
  double irb = Hb * (U[V - 1] + P);
  Eb += (gamma - 1.0) * Pb;
  const double qb = -(gamma - 1.0) * Pb;
  irb += qb * 0.5 * m2;
  for (int k = 0; k < D; k++)
  {
    mb[k] += qb * u[k] + ub[k] * ir;
    irb += ub[k] * U[k + 1];
  }
  Ub[0] += -irb * ir * ir;
  for (int k = 0; k < D; k++) Ub[k + 1] += mb[k];
  Ub[V - 1] += Eb;
}

// (Ub, dUb) += (d F / d (U, dU))^T Fb for the viscous contribution that
// flux_visc_add adds to F (include/flux.hpp:71-202).
template <int D>
ZB_HD void flux_visc_vjp(const double U[D + 2], const double dU[D + 2][D], const double Fb[D + 2][D],
                         const Phys<double> &ph, double Ub[D + 2], double dUb[D + 2][D])
{
  constexpr int V = D + 2;
  const double g = ph.gamma;
  // forward recomputation
  const double ir = 1.0 / U[0];
  double vel[D], vsq = 0.0;
  for (int d = 0; d < D; d++)
  {
    vel[d] = U[d + 1] * ir;
    vsq += vel[d] * vel[d];
  }
  const double e_int = U[V - 1] * ir - 0.5 * vsq;
  double mu, rr = 0.0;
  if (ph.fix_vis)
    mu = ph.mu;
  else
  {
    rr = (g - 1.0) * e_int / ph.rt;
    mu = ph.mu * pow(rr, 1.5) * (1.0 + ph.c_sth) / (rr + ph.c_sth);
  }
  double dvel[D][D];
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) dvel[i][j] = (dU[i + 1][j] - dU[0][j] * vel[i]) * ir;
  double sj[D], dke[D], de[D];
  for (int j = 0; j < D; j++)
  {
    double s = 0.0;
    for (int i = 0; i < D; i++) s += vel[i] * dvel[i][j];
    sj[j] = s;
    dke[j] = 0.5 * vsq * dU[0][j] + U[0] * s;
    de[j] = (dU[V - 1][j] - dke[j] - dU[0][j] * e_int) * ir;
  }
  double div = 0.0;
  for (int d = 0; d < D; d++) div += dvel[d][d];
  // constant reciprocals: an FP64 division is a multi-instruction sequence
  const double third = 1.0 / 3.0, ipr = 1.0 / ph.prandtl;
  const double diag = div * third;
  double tau[D][D];
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++)
      tau[i][j] = (i == j) ? 2.0 * mu * (dvel[i][i] - diag) : mu * (dvel[i][j] + dvel[j][i]);
  const double kappa = (mu * ipr) * g;
  // reverse
  double taub[D][D], velb[D], dvelb[D][D], deb[D];
  double mub = 0.0, kappab = 0.0, diagb = 0.0, irb = 0.0, rhob = 0.0, e_intb = 0.0, vsqb = 0.0;
  for (int i = 0; i < D; i++)
  {
    velb[i] = 0.0;
    for (int j = 0; j < D; j++)
    {
      taub[i][j] = -Fb[i + 1][j] - Fb[V - 1][j] * vel[i];
      velb[i] -= Fb[V - 1][j] * tau[i][j];
      dvelb[i][j] = 0.0;
    }
  }
  for (int j = 0; j < D; j++)
  {
    kappab -= Fb[V - 1][j] * de[j];
    deb[j] = -Fb[V - 1][j] * kappa;
  }
  mub += kappab * g * ipr;
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++)
    {
      if (i == j)
      {
        mub += taub[i][i] * 2.0 * (dvel[i][i] - diag);
        dvelb[i][i] += 2.0 * mu * taub[i][i];
        diagb -= 2.0 * mu * taub[i][i];
      }
      else
      {
        mub += taub[i][j] * (dvel[i][j] + dvel[j][i]);
        dvelb[i][j] += mu * taub[i][j];
        dvelb[j][i] += mu * taub[i][j];
      }
    }
  for (int d = 0; d < D; d++) dvelb[d][d] += diagb * third;
  for (int j = 0; j < D; j++)
  {
    const double X = dU[V - 1][j] - dke[j] - dU[0][j] * e_int;
    const double Xb = deb[j] * ir;
    irb += deb[j] * X;
    dUb[V - 1][j] += Xb;
    const double dkeb = -Xb;
    dUb[0][j] -= Xb * e_int;
    e_intb -= Xb * dU[0][j];
    vsqb += 0.5 * dkeb * dU[0][j];
    dUb[0][j] += 0.5 * vsq * dkeb;
    rhob += dkeb * sj[j];
    const double sb = dkeb * U[0];
    for (int i = 0; i < D; i++)
    {
      velb[i] += sb * dvel[i][j];
      dvelb[i][j] += sb * vel[i];
    }
  }
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++)
    {
      const double Y = dU[i + 1][j] - dU[0][j] * vel[i];
      const double Yb = dvelb[i][j] * ir;
      irb += dvelb[i][j] * Y;
      dUb[i + 1][j] += Yb;
      dUb[0][j] -= Yb * vel[i];
      velb[i] -= Yb * dU[0][j];
    }
  if (!ph.fix_vis)
  {
    // d mu / d r = mu (1.5 / r - 1 / (r + c))
    const double rb = mub * mu * (1.5 / rr - 1.0 / (rr + ph.c_sth));
    e_intb += rb * (g - 1.0) / ph.rt;
  }
  Ub[V - 1] += e_intb * ir;
  irb += e_intb * U[V - 1];
  vsqb -= 0.5 * e_intb;
  for (int i = 0; i < D; i++)
  {
    velb[i] += 2.0 * vsqb * vel[i];
    Ub[i + 1] += velb[i] * ir;
    irb += velb[i] * U[i + 1];
  }
  rhob -= irb * ir * ir;
  Ub[0] += rhob;
}

// Ub += (dP/dU)^T Pb for the pressure P = (gamma-1)(E - |m|^2 / 2 rho).
template <int D>
ZB_HD void pressure_vjp(const double U[D + 2], double Pb, double gamma, double Ub[D + 2])
{
  const double g1 = (gamma - 1.0) * Pb, ir = 1.0 / U[0];
  double m2 = 0.0;
  for (int d = 0; d < D; d++)
  {
    m2 += U[d + 1] * U[d + 1];
    Ub[d + 1] -= g1 * U[d + 1] * ir;
  }
  Ub[0] += g1 * 0.5 * m2 * ir * ir;
  Ub[D + 1] += g1;
}

// (UbL, UbR) += (d Fc / d (UL, UR))^T w for the Rusanov flux of physics.cuh
// (absolute FP64 states).  The wave-speed max and |Vn| take the derivative of
// the branch the forward evaluation takes.
template <int D>
ZB_HD void rusanov_vjp(const double UL[D + 2], const double UR[D + 2], const double n[D], const double w[D + 2],
                       const Phys<double> &ph, double UbL[D + 2], double UbR[D + 2])
{
  constexpr int V = D + 2;
  const double g = ph.gamma;
  double m2L = 0.0, m2R = 0.0, VnL = 0.0, VnR = 0.0;
  for (int d = 0; d < D; d++)
  {
    m2L += UL[d + 1] * UL[d + 1];
    m2R += UR[d + 1] * UR[d + 1];
    VnL += UL[d + 1] / UL[0] * n[d];
    VnR += UR[d + 1] / UR[0] * n[d];
  }
  const double PL = (g - 1.0) * (UL[V - 1] - 0.5 * m2L / UL[0]);
  const double PR = (g - 1.0) * (UR[V - 1] - 0.5 * m2R / UR[0]);
  const double aL = sqrt(g * PL / UL[0]), aR = sqrt(g * PR / UR[0]);
  const double sL = fabs(VnL) + aL, sR = fabs(VnR) + aR;
  const double eig = sL > sR ? sL : sR;
  const double diss = 0.5 * eig * (1.0 - ph.rus_k);
  double FbL[V][D], FbR[V][D], dissb = 0.0;
  for (int v = 0; v < V; v++)
  {
    for (int d = 0; d < D; d++) FbL[v][d] = FbR[v][d] = 0.5 * w[v] * n[d];
    UbR[v] -= diss * w[v];
    UbL[v] += diss * w[v];
    dissb -= w[v] * (UR[v] - UL[v]);
  }
  flux_conv_vjp<D>(UL, FbL, g, UbL);
  flux_conv_vjp<D>(UR, FbR, g, UbR);
  const double eigb = 0.5 * (1.0 - ph.rus_k) * dissb;
  const bool left = sL > sR;
  const double *U = left ? UL : UR;
  double *Ub = left ? UbL : UbR;
  const double Vn = left ? VnL : VnR, a = left ? aL : aR, P = left ? PL : PR;
  // |Vn| + a
  const double Vnb = (Vn < 0.0) ? -eigb : eigb;
  const double qb = eigb / (2.0 * a);  // a = sqrt(q), q = g P / rho
  const double ir = 1.0 / U[0];
  pressure_vjp<D>(U, qb * g * ir, g, Ub);
  Ub[0] -= qb * g * P * ir * ir;
  for (int d = 0; d < D; d++) Ub[d + 1] += Vnb * n[d] * ir;
  Ub[0] -= Vnb * Vn * ir;
}

// (UbL, UbR) += (d Fc / d (UL, UR))^T w for the Roe flux with Harten's
// entropy fix of physics.cuh (absolute FP64 states).
template <int D>
ZB_HD void roe_vjp(const double UL[D + 2], const double UR[D + 2], const double n[D], const double w[D + 2],
                   const Phys<double> &ph, double UbL[D + 2], double UbR[D + 2])
{
  constexpr int V = D + 2;
  const double g = ph.gamma;
  // ---- forward recomputation ----
  const double rL = UL[0], rR = UR[0];
  // 1/rho and sqrt(rho) from one reciprocal square root per state (the FP64
  // division and square root are multi-instruction sequences)
  const double rsL = drsqrt<double>(rL), rsR = drsqrt<double>(rR);
  const double irL = rsL * rsL, irR = rsR * rsR;
  double m2L = 0.0, m2R = 0.0;
  for (int d = 0; d < D; d++)
  {
    m2L += UL[d + 1] * UL[d + 1];
    m2R += UR[d + 1] * UR[d + 1];
  }
  const double PL = (g - 1.0) * (UL[V - 1] - 0.5 * m2L * irL);
  const double PR = (g - 1.0) * (UR[V - 1] - 0.5 * m2R * irR);
  const double sL = rL * rsL, sR = rR * rsR;
  const double inv = 1.0 / (sL + sR);
  double uL[D], uR[D], u[D], unL = 0.0, unR = 0.0;
  for (int d = 0; d < D; d++)
  {
    uL[d] = UL[d + 1] * irL;
    uR[d] = UR[d + 1] * irR;
    u[d] = (sL * uL[d] + sR * uR[d]) * inv;
    unL += uL[d] * n[d];
    unR += uR[d] * n[d];
  }
  const double HL = (UL[V - 1] + PL) * irL, HR = (UR[V - 1] + PR) * irR;
  const double H = (sL * HL + sR * HR) * inv;
  double q2 = 0.0, un = 0.0;
  for (int d = 0; d < D; d++)
  {
    q2 += u[d] * u[d];
    un += u[d] * n[d];
  }
  double c2 = (g - 1.0) * (H - 0.5 * q2);
  const bool clamped = !(c2 > 1e-30);
  if (clamped) c2 = 1e-30;
  const double ia = drsqrt<double>(c2);
  const double a = c2 * ia, ic2 = ia * ia;
  const double rho = sL * sR;
  const double dp = PR - PL, dr = rR - rL, dun = unR - unL;
  const double t2 = 0.5 * ic2;
  const double a1 = (dp - rho * a * dun) * t2;
  const double a3 = (dp + rho * a * dun) * t2;
  const double a2w = dr - dp * ic2;
  const double x[3] = {un - a, un, un + a};
  const double delta = 0.1 * (fabs(un) + a);
  const double idelta = 1.0 / delta;
  double l[3];
  bool fixed[3];
  for (int i = 0; i < 3; i++)
  {
    const double ax = fabs(x[i]);
    fixed[i] = ax < delta;
    l[i] = fixed[i] ? (ax * ax + delta * delta) * (0.5 * idelta) : ax;
  }
  double dvt[D], udvt = 0.0;
  for (int d = 0; d < D; d++)
  {
    dvt[d] = (uR[d] - uL[d]) - dun * n[d];
    udvt += u[d] * dvt[d];
  }
  // ---- reverse ----
  double FbL[V][D], FbR[V][D], dsb[V];
  for (int v = 0; v < V; v++)
  {
    for (int d = 0; d < D; d++) FbL[v][d] = FbR[v][d] = 0.5 * w[v] * n[d];
    dsb[v] = -0.5 * w[v];
  }
  flux_conv_vjp<D>(UL, FbL, g, UbL);
  flux_conv_vjp<D>(UR, FbR, g, UbR);
  double lb[3] = {0.0, 0.0, 0.0};
  double a1b = 0.0, a3b = 0.0, a2wb = 0.0, Hb = 0.0, ab = 0.0, unb = 0.0, q2b = 0.0, rhob = 0.0, udvtb = 0.0;
  double ub[D], dvtb[D];
  for (int d = 0; d < D; d++) ub[d] = dvtb[d] = 0.0;
  {
    const double X = dsb[V - 1];
    lb[0] += X * a1 * (H - a * un);
    a1b += X * l[0] * (H - a * un);
    Hb += X * (l[0] * a1 + l[2] * a3);
    ab += X * (-l[0] * a1 * un + l[2] * a3 * un);
    unb += X * (-l[0] * a1 * a + l[2] * a3 * a);
    lb[1] += X * (a2w * 0.5 * q2 + rho * udvt);
    a2wb += X * l[1] * 0.5 * q2;
    q2b += X * l[1] * a2w * 0.5;
    rhob += X * l[1] * udvt;
    udvtb += X * l[1] * rho;
    lb[2] += X * a3 * (H + a * un);
    a3b += X * l[2] * (H + a * un);
  }
  for (int d = 0; d < D; d++)
  {
    ub[d] += udvtb * dvt[d];
    dvtb[d] += udvtb * u[d];
    const double X = dsb[d + 1];
    lb[0] += X * a1 * (u[d] - a * n[d]);
    a1b += X * l[0] * (u[d] - a * n[d]);
    ub[d] += X * (l[0] * a1 + l[1] * a2w + l[2] * a3);
    ab += X * (-l[0] * a1 * n[d] + l[2] * a3 * n[d]);
    lb[1] += X * (a2w * u[d] + rho * dvt[d]);
    a2wb += X * l[1] * u[d];
    rhob += X * l[1] * dvt[d];
    dvtb[d] += X * l[1] * rho;
    lb[2] += X * a3 * (u[d] + a * n[d]);
    a3b += X * l[2] * (u[d] + a * n[d]);
  }
  {
    const double X = dsb[0];
    lb[0] += X * a1;
    a1b += X * l[0];
    lb[1] += X * a2w;
    a2wb += X * l[1];
    lb[2] += X * a3;
    a3b += X * l[2];
  }
  double uLb[D], uRb[D], dunb = 0.0;
  for (int d = 0; d < D; d++)
  {
    uRb[d] = dvtb[d];
    uLb[d] = -dvtb[d];
    dunb -= dvtb[d] * n[d];
  }
  // entropy fix and |x|
  double deltab = 0.0;
  for (int i = 0; i < 3; i++)
  {
    const double ax = fabs(x[i]);
    double axb = lb[i];
    if (fixed[i])
    {
      axb = lb[i] * ax * idelta;
      deltab += lb[i] * (delta * delta - ax * ax) * (0.5 * idelta * idelta);
    }
    const double xb = (x[i] < 0.0) ? -axb : axb;
    unb += xb;
    if (i == 0) ab -= xb;
    if (i == 2) ab += xb;
  }
  unb += 0.1 * deltab * ((un < 0.0) ? -1.0 : 1.0);
  ab += 0.1 * deltab;
  // wave strengths
  double dpb = 0.0, drb = 0.0, c2b = 0.0;
  dpb += a1b * t2;
  rhob -= a1b * a * dun * t2;
  ab -= a1b * rho * dun * t2;
  dunb -= a1b * rho * a * t2;
  c2b -= a1b * a1 * ic2;
  dpb += a3b * t2;
  rhob += a3b * a * dun * t2;
  ab += a3b * rho * dun * t2;
  dunb += a3b * rho * a * t2;
  c2b -= a3b * a3 * ic2;
  drb += a2wb;
  dpb -= a2wb * ic2;
  c2b += a2wb * dp * (ic2 * ic2);
  c2b += ab * (0.5 * ia);
  if (!clamped)
  {
    Hb += (g - 1.0) * c2b;
    q2b -= 0.5 * (g - 1.0) * c2b;
  }
  double sLb = rhob * sR, sRb = rhob * sL;
  double PLb = -dpb, PRb = dpb;
  double rLb = -drb, rRb = drb;
  double unLb = -dunb, unRb = dunb;
  for (int d = 0; d < D; d++) ub[d] += 2.0 * q2b * u[d] + unb * n[d];
  double invb = 0.0;
  {
    const double HLb = Hb * sL * inv, HRb = Hb * sR * inv;
    sLb += Hb * HL * inv;
    sRb += Hb * HR * inv;
    invb += Hb * (sL * HL + sR * HR);
    UbL[V - 1] += HLb * irL;
    PLb += HLb * irL;
    rLb -= HLb * HL * irL;
    UbR[V - 1] += HRb * irR;
    PRb += HRb * irR;
    rRb -= HRb * HR * irR;
  }
  for (int d = 0; d < D; d++)
  {
    uLb[d] += ub[d] * sL * inv + unLb * n[d];
    uRb[d] += ub[d] * sR * inv + unRb * n[d];
    sLb += ub[d] * uL[d] * inv;
    sRb += ub[d] * uR[d] * inv;
    invb += ub[d] * (sL * uL[d] + sR * uR[d]);
  }
  sLb -= invb * inv * inv;
  sRb -= invb * inv * inv;
  for (int d = 0; d < D; d++)
  {
    UbL[d + 1] += uLb[d] * irL;
    rLb -= uLb[d] * uL[d] * irL;
    UbR[d + 1] += uRb[d] * irR;
    rRb -= uRb[d] * uR[d] * irR;
  }
  rLb += sLb * (0.5 * sL * irL);  // d sqrt(r) / dr = 1 / (2 sqrt(r)) = sqrt(r) / (2 r)
  rRb += sRb * (0.5 * sR * irR);
  UbL[0] += rLb;
  UbR[0] += rRb;
  pressure_vjp<D>(UL, PLb, g, UbL);
  pressure_vjp<D>(UR, PRb, g, UbR);
}

// Common convective flux of a face as a function of (UL, UR); boundary faces
// (bc >= 0) take UR from the ghost state of UL.
template <int D, typename X>
ZB_HD void conv_face(int bc, const X UL[D + 2], const X URin[D + 2], const X n[D], X Fc[D + 2], const Phys<X> &ph)
{
  X UR[D + 2];
  if (bc >= 0)
  {
    X UB[D + 2];
    ghost_state<X, D>(bc, UL, n, UR, UB, ph);
  }
  else
    for (int v = 0; v < D + 2; v++) UR[v] = URin[v];
  if (ph.fconv == 2)
    roe<X, D>(UL, UR, n, Fc, ph);
  else
    rusanov<X, D>(UL, UR, n, Fc, ph);
}

// Ub_own += (d Fc / d U_own)^T w for an interior face (own = left or right),
// by the hand-written reverse of the Riemann solver.
template <int D>
ZB_HD void conv_face_vjp_side(const double UL[D + 2], const double UR[D + 2], const double n[D], const double w[D + 2],
                              bool own_left, const Phys<double> &ph, double Ub[D + 2])
{
  constexpr int V = D + 2;
  double bL[V], bR[V];
  for (int v = 0; v < V; v++) bL[v] = bR[v] = 0.0;
  if (ph.fconv == 2)
    roe_vjp<D>(UL, UR, n, w, ph, bL, bR);
  else
    rusanov_vjp<D>(UL, UR, n, w, ph, bL, bR);
  for (int v = 0; v < V; v++) Ub[v] += own_left ? bL[v] : bR[v];
}

// Viscous normal flux of one trace (visc_normal) and its reverse:
// (Ub, dUb) += (d (F_visc(U, dU) . n) / d (U, dU))^T w.
template <int D>
ZB_HD void visc_normal_vjp(const double U[D + 2], const double dU[D + 2][D], const double n[D], const double w[D + 2],
                           const Phys<double> &ph, double Ub[D + 2], double dUb[D + 2][D])
{
  double Fb[D + 2][D];
  for (int v = 0; v < D + 2; v++)
    for (int d = 0; d < D; d++) Fb[v][d] = w[v] * n[d];
  flux_visc_vjp<D>(U, dU, Fb, ph, Ub, dUb);
}

// Boundary face, everything the own trace (U, dU) feeds:
//   convective common flux with the ghost state, plus for viscous runs
//   F_visc(UB, ghost_grad(U, dU)) . n + tau (U - UB).
template <int D, bool VISC>
ZB_HD_INLINE void bnd_face_vjp_body(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                    const double w[D + 2], const Phys<Dual<double>> &pd,
                                    double Ub[D + 2], double dUb[D + 2][D])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  constexpr int NI = VISC ? V + V * D : V;
  DD nd[D];
  for (int d = 0; d < D; d++) nd[d] = DD(n[d]);
  for (int k = 0; k < NI; k++)
  {
    DD L[V], dL[V][D], F[V];
    for (int v = 0; v < V; v++)
    {
      L[v] = DD(U[v], v == k ? 1.0 : 0.0);
      for (int d = 0; d < D; d++) dL[v][d] = DD(dU[v][d], (k == V + v * D + d) ? 1.0 : 0.0);
    }
    conv_face<D, DD>(bc, L, L, nd, F, pd);
    if (VISC)
    {
      DD UR[V], UB[V], dUB[V][D], Fn[V];
      ghost_state<DD, D>(bc, L, nd, UR, UB, pd);
      ghost_grad<DD, D>(bc, L, dL, nd, dUB);
      visc_normal<DD, D>(UB, dUB, nd, Fn, pd);
      for (int v = 0; v < V; v++) F[v] += Fn[v] + pd.ldg_tau * (L[v] - UB[v]);
    }
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * F[v].d;
    if (k < V)
      Ub[k] += acc;
    else
      dUb[(k - V) / D][(k - V) % D] += acc;
  }
}
template <int D, bool VISC>
ZB_HD_COLD void bnd_face_vjp_cold(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                  const double w[D + 2], const Phys<Dual<double>> &pd,
                                  double Ub[D + 2], double dUb[D + 2][D])
{
  bnd_face_vjp_body<D, VISC>(bc, U, dU, n, w, pd, Ub, dUb);
}
template <int D, bool VISC>
ZB_HD_INLINE void bnd_face_vjp(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                               const double w[D + 2], const Phys<Dual<double>> &pd,
                               double Ub[D + 2], double dUb[D + 2][D])
{
  if constexpr (D == 2)
    bnd_face_vjp_body<D, VISC>(bc, U, dU, n, w, pd, Ub, dUb);
  else
    bnd_face_vjp_cold<D, VISC>(bc, U, dU, n, w, pd, Ub, dUb);
}

// Ub += (d UB / d U)^T w for the prescribed boundary state UB of the LDG
// common solution.
template <int D>
ZB_HD_INLINE void bnd_ucomm_vjp_body(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                     const Phys<Dual<double>> &pd, double Ub[D + 2])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  DD nd[D];
  for (int d = 0; d < D; d++) nd[d] = DD(n[d]);
  for (int k = 0; k < V; k++)
  {
    DD L[V], UR[V], UB[V];
    for (int v = 0; v < V; v++) L[v] = DD(U[v], v == k ? 1.0 : 0.0);
    ghost_state<DD, D>(bc, L, nd, UR, UB, pd);
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * UB[v].d;
    Ub[k] += acc;
  }
}
template <int D>
ZB_HD_COLD void bnd_ucomm_vjp_cold(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                   const Phys<Dual<double>> &pd, double Ub[D + 2])
{
  bnd_ucomm_vjp_body<D>(bc, U, n, w, pd, Ub);
}
template <int D>
ZB_HD_INLINE void bnd_ucomm_vjp(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                const Phys<Dual<double>> &pd, double Ub[D + 2])
{
  if constexpr (D == 2)
    bnd_ucomm_vjp_body<D>(bc, U, n, w, pd, Ub);
  else
    bnd_ucomm_vjp_cold<D>(bc, U, n, w, pd, Ub);
}

// Free-stream parameters a boundary state depends on: k = 0 rho_fs,
// 1..3 V_fs[k-1], 4 P_fs.  Only far-field (3) and characteristic (2) faces.
ZB_HD bool bc_uses_freestream(int bc) { return bc == 2 || bc == 3; }

ZB_HD void seed_param(Phys<Dual<double>> &q, int k)
{
  if (k == 0)
    q.rho_fs.d = 1.0;
  else if (k <= 3)
    q.V_fs[k - 1].d = 1.0;
  else
    q.P_fs.d = 1.0;
}

// pb[k] += d (w . phi) / d param_k for the boundary face function of
// bnd_face_vjp.
template <int D, bool VISC>
ZB_HD_INLINE void bnd_face_param_vjp_body(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                          const double w[D + 2], const Phys<Dual<double>> &pd, double pb[5])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  if (!bc_uses_freestream(bc)) return;
  DD nd[D], L[V], dL[V][D];
  for (int d = 0; d < D; d++) nd[d] = DD(n[d]);
  for (int v = 0; v < V; v++)
  {
    L[v] = DD(U[v]);
    for (int d = 0; d < D; d++) dL[v][d] = DD(dU[v][d]);
  }
  for (int k = 0; k < 5; k++)
  {
    if (k >= 1 && k <= 3 && k > D) continue;
    Phys<DD> q = pd;
    seed_param(q, k);
    DD F[V];
    conv_face<D, DD>(bc, L, L, nd, F, q);
    if (VISC)
    {
      DD UR[V], UB[V], dUB[V][D], Fn[V];
      ghost_state<DD, D>(bc, L, nd, UR, UB, q);
      ghost_grad<DD, D>(bc, L, dL, nd, dUB);
      visc_normal<DD, D>(UB, dUB, nd, Fn, q);
      for (int v = 0; v < V; v++) F[v] += Fn[v] + q.ldg_tau * (L[v] - UB[v]);
    }
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * F[v].d;
    pb[k] += acc;
  }
}
template <int D, bool VISC>
ZB_HD_COLD void bnd_face_param_vjp_cold(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                        const double w[D + 2], const Phys<Dual<double>> &pd, double pb[5])
{
  bnd_face_param_vjp_body<D, VISC>(bc, U, dU, n, w, pd, pb);
}
template <int D, bool VISC>
ZB_HD_INLINE void bnd_face_param_vjp(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                     const double w[D + 2], const Phys<Dual<double>> &pd, double pb[5])
{
  if constexpr (D == 2)
    bnd_face_param_vjp_body<D, VISC>(bc, U, dU, n, w, pd, pb);
  else
    bnd_face_param_vjp_cold<D, VISC>(bc, U, dU, n, w, pd, pb);
}

// pb[k] += d (w . UB) / d param_k for the LDG boundary common solution.
template <int D>
ZB_HD_INLINE void bnd_ucomm_param_vjp_body(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                           const Phys<Dual<double>> &pd, double pb[5])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  if (!bc_uses_freestream(bc)) return;
  DD nd[D], L[V];
  for (int d = 0; d < D; d++) nd[d] = DD(n[d]);
  for (int v = 0; v < V; v++) L[v] = DD(U[v]);
  for (int k = 0; k < 5; k++)
  {
    if (k >= 1 && k <= 3 && k > D) continue;
    Phys<DD> q = pd;
    seed_param(q, k);
    DD UR[V], UB[V];
    ghost_state<DD, D>(bc, L, nd, UR, UB, q);
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * UB[v].d;
    pb[k] += acc;
  }
}
template <int D>
ZB_HD_COLD void bnd_ucomm_param_vjp_cold(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                         const Phys<Dual<double>> &pd, double pb[5])
{
  bnd_ucomm_param_vjp_body<D>(bc, U, n, w, pd, pb);
}
template <int D>
ZB_HD_INLINE void bnd_ucomm_param_vjp(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                      const Phys<Dual<double>> &pd, double pb[5])
{
  if constexpr (D == 2)
    bnd_ucomm_param_vjp_body<D>(bc, U, n, w, pd, pb);
  else
    bnd_ucomm_param_vjp_cold<D>(bc, U, n, w, pd, pb);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// ---- geometry adjoint: derivatives with respect to the face normal ----

// nb += d (w . Fc(UL, UR, n)) / d n for an interior face (dual-number seeds on n)
template <int D>
ZB_HD_INLINE void conv_face_n_vjp_body(const double UL[D + 2], const double UR[D + 2], const double n[D],
                                       const double w[D + 2], const Phys<double> &ph, double nb[D])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  const Phys<DD> pd = dual_phys(ph);
  DD L[V], R[V];
  for (int v = 0; v < V; v++)
  {
    L[v] = DD(UL[v]);
    R[v] = DD(UR[v]);
  }
  for (int k = 0; k < D; k++)
  {
    DD nd[D], F[V];
    for (int d = 0; d < D; d++) nd[d] = DD(n[d], d == k ? 1.0 : 0.0);
    conv_face<D, DD>(-1, L, R, nd, F, pd);
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * F[v].d;
    nb[k] += acc;
  }
}
template <int D>
ZB_HD_COLD void conv_face_n_vjp_cold(const double UL[D + 2], const double UR[D + 2], const double n[D],
                                     const double w[D + 2], const Phys<double> &ph, double nb[D])
{
  conv_face_n_vjp_body<D>(UL, UR, n, w, ph, nb);
}
template <int D>
ZB_HD_INLINE void conv_face_n_vjp(const double UL[D + 2], const double UR[D + 2], const double n[D],
                                  const double w[D + 2], const Phys<double> &ph, double nb[D])
{
  if constexpr (D == 2)
    conv_face_n_vjp_body<D>(UL, UR, n, w, ph, nb);
  else
    conv_face_n_vjp_cold<D>(UL, UR, n, w, ph, nb);
}

// nb += d (w . phi) / d n for the boundary face function of bnd_face_vjp
template <int D, bool VISC>
ZB_HD_INLINE void bnd_face_n_vjp_body(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                      const double w[D + 2], const Phys<double> &ph, double nb[D])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  const Phys<DD> pd = dual_phys(ph);
  DD L[V], dL[V][D];
  for (int v = 0; v < V; v++)
  {
    L[v] = DD(U[v]);
    for (int d = 0; d < D; d++) dL[v][d] = DD(dU[v][d]);
  }
  for (int k = 0; k < D; k++)
  {
    DD nd[D], F[V];
    for (int d = 0; d < D; d++) nd[d] = DD(n[d], d == k ? 1.0 : 0.0);
    conv_face<D, DD>(bc, L, L, nd, F, pd);
    if (VISC)
    {
      DD UR[V], UB[V], dUB[V][D], Fn[V];
      ghost_state<DD, D>(bc, L, nd, UR, UB, pd);
      ghost_grad<DD, D>(bc, L, dL, nd, dUB);
      visc_normal<DD, D>(UB, dUB, nd, Fn, pd);
      for (int v = 0; v < V; v++) F[v] += Fn[v] + pd.ldg_tau * (L[v] - UB[v]);
    }
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * F[v].d;
    nb[k] += acc;
  }
}
template <int D, bool VISC>
ZB_HD_COLD void bnd_face_n_vjp_cold(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                    const double w[D + 2], const Phys<double> &ph, double nb[D])
{
  bnd_face_n_vjp_body<D, VISC>(bc, U, dU, n, w, ph, nb);
}
template <int D, bool VISC>
ZB_HD_INLINE void bnd_face_n_vjp(int bc, const double U[D + 2], const double dU[D + 2][D], const double n[D],
                                 const double w[D + 2], const Phys<double> &ph, double nb[D])
{
  if constexpr (D == 2)
    bnd_face_n_vjp_body<D, VISC>(bc, U, dU, n, w, ph, nb);
  else
    bnd_face_n_vjp_cold<D, VISC>(bc, U, dU, n, w, ph, nb);
}

// nb += d (w . UB(U, n)) / d n for the LDG boundary common solution
template <int D>
ZB_HD_INLINE void bnd_ucomm_n_vjp_body(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                       const Phys<double> &ph, double nb[D])
{
  constexpr int V = D + 2;
  using DD = Dual<double>;
  const Phys<DD> pd = dual_phys(ph);
  DD L[V];
  for (int v = 0; v < V; v++) L[v] = DD(U[v]);
  for (int k = 0; k < D; k++)
  {
    DD nd[D], UR[V], UB[V];
    for (int d = 0; d < D; d++) nd[d] = DD(n[d], d == k ? 1.0 : 0.0);
    ghost_state<DD, D>(bc, L, nd, UR, UB, pd);
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += w[v] * UB[v].d;
    nb[k] += acc;
  }
}
template <int D>
ZB_HD_COLD void bnd_ucomm_n_vjp_cold(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                     const Phys<double> &ph, double nb[D])
{
  bnd_ucomm_n_vjp_body<D>(bc, U, n, w, ph, nb);
}
template <int D>
ZB_HD_INLINE void bnd_ucomm_n_vjp(int bc, const double U[D + 2], const double n[D], const double w[D + 2],
                                  const Phys<double> &ph, double nb[D])
{
  if constexpr (D == 2)
    bnd_ucomm_n_vjp_body<D>(bc, U, n, w, ph, nb);
  else
    bnd_ucomm_n_vjp_cold<D>(bc, U, n, w, ph, nb);
}

// Viscous flux matrix F_visc[var][dim] of one trace (the part flux_visc_add adds)
template <int D>
ZB_HD void visc_matrix(const double U[D + 2], const double dU[D + 2][D], const Phys<double> &ph,
                       double F[D + 2][D])
{
  for (int v = 0; v < D + 2; v++)
    for (int d = 0; d < D; d++) F[v][d] = 0.0;
  flux_visc_add<double, D>(U, dU, F, ph);
}

// Deterministic block sum of pb[5] into out[5] (fixed shuffle and warp order).
__device__ __forceinline__ void block_sum5(double pb[5], double *out)
{
  __shared__ double red[32][5];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 5; k++)
  {
    double x = pb[k];
    for (int o = 16; o > 0; o /= 2) x += __shfl_down_sync(0xffffffff, x, o);
    if (lane == 0) red[warp][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < 5)
  {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

struct AdjArgs
{
  const double *U;     // [tile][S][V][TW] state the residual is linearised at
  const double *Ufp;   // [tile][Fp][V][TW] its extrapolation
  const double *mets;  // [tile][S][NM][TW]
  const double *fgeo;  // [tile][Fp][D+1][TW]
  const int *nbr;      // [tile][Fp][TW]
  const double *lam;   // [tile][S][V][TW] weight on the residual
  double *Lfp;         // [tile][Fp][V][TW] weight on the own-side surface flux
  double *Ubfp;        // [tile][Fp][V][TW] adjoint of the own trace U_fpts
  double *dUbfp;       // NS: [tile][Fp][V][D][TW] adjoint of the own gradient trace
  double *Ubx;         // NS: [tile][Fp][V][TW] Riemann-flux adjoint of a right side's trace,
                       // written by its left partner, added in the trace pass
  double *UCb;         // NS: [tile][Fp][V][TW] adjoint of the own common solution
  double *Ubar;        // [tile][S][V][TW] result
  double *pbar;        // [ntiles][5] per-tile free-stream adjoint (nullptr: off)
  // geometry adjoint (nullptr: off)
  double *mbar;        // [tile][S][NM][TW] adjoint of the adjugate and |J|
  double *gbar;        // [tile][Fp][D+1][TW] adjoint of the face normal (whole face, kept at the
                       // left side or the boundary; zero at right sides) and of the own dA
  double *nbx;         // NS: [tile][Fp][D][TW] right side's part of its face's normal adjoint
  const double *Fvn;   // NS: forward viscous normal flux at own flux points
  const double *dops;  // triangles: the dense operators (TriShape layout)
  int64_t ntiles;
  Phys<double> ph;
};

// Geometry adjoint of F~_d = sum_k adj[d][k] F_k at one solution point:
// mbar(adj[d][k]) = sum_v Ft[d][v] F[v][k]; |J| gets 0 here (written, not added).
template <int D>
__device__ __forceinline__ void geo_adj_bar(const AdjArgs &a, int64_t tile, int s, int l, const double Ft[D][D + 2],
                                            const double F[D + 2][D], int S)
{
  constexpr int NM = D * D + 1;
  double *mb = a.mbar + (tile * S + s) * (int64_t)NM * TW + l;
#pragma unroll
  for (int d = 0; d < D; d++)
#pragma unroll
    for (int k = 0; k < D; k++)
    {
      double acc = 0.0;
#pragma unroll
      for (int v = 0; v < D + 2; v++) acc += Ft[d][v] * F[v][k];
      mb[(d * D + k) * TW] = acc;
    }
  mb[D * D * TW] = 0.0;
}

// Geometry adjoint at an own flux point: the own surface term is
// +-phi dA_own (minus on the right side), so dA_own_bar = +-Lfp . phi; the
// normal's adjoint nb (the whole face's, or zero on a right side) is stored
// beside it.
template <int D, int N>
__device__ __forceinline__ void geo_face_bar(const AdjArgs &a, int64_t tile, int f, int l, int code,
                                             const double phi[D + 2], const double nb[D])
{
  constexpr int Fp = Shape<D, N>::Fp, V = D + 2;
  const double *lo = a.Lfp + (tile * Fp + f) * (int64_t)V * TW + l;
  double acc = 0.0;
#pragma unroll
  for (int v = 0; v < V; v++) acc += lo[v * TW] * phi[v];
  const bool right = (code >= 0) && (code & 1);
  double *g = a.gbar + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
  for (int d = 0; d < D; d++) g[d * TW] = nb[d];
  g[D * TW] = right ? -acc : acc;
}

// Weight of the own surface flux point: the transpose of the surface
// correction of finish_point, Lfp(f) = sum over the line of f of
// (-Dbm | +Dbp)[m] lam(spt m).
template <int D, int N>
__global__ void __launch_bounds__(256) k_adj_lift(const __grid_constant__ AdjArgs a,
                                                  const __grid_constant__ LineOpsT<double, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V;
  const int64_t total = a.ntiles * Fp * TW;
  for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(gid % TW);
    const int f = (int)((gid / TW) % Fp);
    const int64_t tile = gid / ((int64_t)TW * Fp);
    int dim, side, base, stride;
    fpt_line<D, N>(f, dim, side, base, stride);
    const double *Lt = a.lam + tile * (int64_t)S * V * TW;
    double *out = a.Lfp + (tile * Fp + f) * (int64_t)V * TW;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < N; m++)
        acc += (side < 0 ? -ops.Dbm[m] : ops.Dbp[m]) * Lt[((base + m * stride) * V + v) * TW + l];
      out[v * TW + l] = acc;
    }
  }
}

// Adjoint of the volume flux divergence at solution point s:
// Fb[v][k] = sum_d adj[d][k] (Dm^T lam)_d[v].
template <int D, int N>
__device__ __forceinline__ void vol_weight(const AdjArgs &a, const LineOpsT<double, N> &ops, int64_t tile, int s, int l,
                                           double Fb[D + 2][D], double Ft[D][D + 2])
{
  using G = Shape<D, N>;
  constexpr int S = G::S, V = G::V, NM = G::NM;
  const double *Lt = a.lam + tile * (int64_t)S * V * TW;
#pragma unroll
  for (int d = 0; d < D; d++)
  {
    int i, fm, fp;
    spt_ends<D, N>(s, d, i, fm, fp);
    const int st = pow_n<N>(d);
    const int b = s - i * st;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < N; m++) acc += ops.Dm[m * N + i] * Lt[((b + m * st) * V + v) * TW + l];
      Ft[d][v] = acc;
    }
  }
  const double *mt = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
#pragma unroll
  for (int v = 0; v < V; v++)
#pragma unroll
    for (int k = 0; k < D; k++)
    {
      double acc = 0.0;
#pragma unroll
      for (int d = 0; d < D; d++) acc += mt[(d * D + k) * TW] * Ft[d][v];
      Fb[v][k] = acc;
    }
}

// Summed weight on the common flux of the face of own flux point f (both
// sides' surface terms) and the own-side bookkeeping.
template <int D, int N>
__device__ __forceinline__ void face_weight(const AdjArgs &a, int64_t tile, int f, int l, int code, double n[D],
                                            double w[D + 2])
{
  using G = Shape<D, N>;
  constexpr int Fp = G::Fp, V = G::V;
  const double *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
  for (int d = 0; d < D; d++) n[d] = g[d * TW];
  const double dA = g[D * TW];
  double Lo[V];
  const double *lo = a.Lfp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
  for (int v = 0; v < V; v++) Lo[v] = lo[v * TW];
  if (code < 0)
  {
#pragma unroll
    for (int v = 0; v < V; v++) w[v] = dA * Lo[v];
    return;
  }
  const int pidx = code >> 1;
  const bool own_left = !(code & 1);
  double Ln[V];
  gather_fpt<double, double, V>(a.Lfp, pidx, Ln);
  const double dAn = a.fgeo[((int64_t)(pidx / TW) * (D + 1) + D) * TW + pidx % TW];
  const double so = own_left ? dA : -dA, sn = own_left ? -dAn : dAn;
#pragma unroll
  for (int v = 0; v < V; v++) w[v] = so * Lo[v] + sn * Ln[v];
}

// Navier-Stokes geometry adjoint at an own flux point: the face value
// phi = Fc + Fv (Fv from the forward viscous normal fluxes), dA_own_bar, and
// the normal's adjoint: the left side (or the boundary) takes the Riemann
// part and its own viscous part; a right side leaves its viscous part in nbx
// for the left side to collect in the second pass.
template <int D, int N>
__device__ __forceinline__ void geo_face_ns(const AdjArgs &a, int64_t tile, int f, int l, int code, const double n[D],
                                            const double w[D + 2], const double Uo[D + 2],
                                            const double dUo[D + 2][D])
{
  constexpr int Fp = Shape<D, N>::Fp, V = D + 2;
  const double beta = a.ph.ldg_b, tau = a.ph.ldg_tau;
  double phi[V], nb[D];
#pragma unroll
  for (int d = 0; d < D; d++) nb[d] = 0.0;
  const double *fo = a.Fvn + (tile * Fp + f) * (int64_t)V * TW + l;
  if (code >= 0)
  {
    double Un[V];
    gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
    const bool own_left = !(code & 1);
    const double *UL = own_left ? Uo : Un, *UR = own_left ? Un : Uo;
    conv_face<D, double>(-1, UL, UR, n, phi, a.ph);
    const double cL = 0.5 + beta, cR = 0.5 - beta;
    double Fx[V];
    if ((own_left && cR != 0.0) || (!own_left && cL != 0.0)) gather_fpt<double, double, V>(a.Fvn, code >> 1, Fx);
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double fv = tau * (UL[v] - UR[v]);
      if (cL != 0.0) fv += cL * (own_left ? fo[v * TW] : Fx[v]);
      if (cR != 0.0) fv += cR * (own_left ? Fx[v] : fo[v * TW]);
      phi[v] += fv;
    }
    const double c_own = own_left ? cL : cR;
    double own[D];
#pragma unroll
    for (int d = 0; d < D; d++) own[d] = 0.0;
    if (c_own != 0.0)
    {
      double Fv[V][D];
      visc_matrix<D>(Uo, dUo, a.ph, Fv);
#pragma unroll
      for (int d = 0; d < D; d++)
#pragma unroll
        for (int v = 0; v < V; v++) own[d] += c_own * w[v] * Fv[v][d];
    }
    if (own_left)
    {
      conv_face_n_vjp<D>(UL, UR, n, w, a.ph, nb);
#pragma unroll
      for (int d = 0; d < D; d++) nb[d] += own[d];
    }
    else
    {
      double *x = a.nbx + (tile * Fp + f) * (int64_t)D * TW + l;
#pragma unroll
      for (int d = 0; d < D; d++) x[d * TW] = own[d];
    }
  }
  else
  {
    const int bc = -code - 1;
    double UR[V], UB[V];
    conv_face<D, double>(bc, Uo, Uo, n, phi, a.ph);
    ghost_state<double, D>(bc, Uo, n, UR, UB, a.ph);
#pragma unroll
    for (int v = 0; v < V; v++) phi[v] += fo[v * TW] + tau * (Uo[v] - UB[v]);
    bnd_face_n_vjp<D, true>(bc, Uo, dUo, n, w, a.ph, nb);
  }
  geo_face_bar<D, N>(a, tile, f, l, code, phi, nb);
}

// ---------------------------------------------------------------------------
// Euler: one kernel after k_adj_lift
// ---------------------------------------------------------------------------
template <int D, int N, bool GEO>
__global__ void __launch_bounds__(Shape<D, N>::NT) k_adj_euler(const __grid_constant__ AdjArgs a,
                                                               const __grid_constant__ LineOpsT<double, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sUb = reinterpret_cast<double *>(smem_raw);  // [S][V][TW]
  double *sUbfp = sUb + S * V * TW;                     // [Fp][V][TW]
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  double pb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double Fb[V][D], U[V], Ub[V];
    double Ft[D][V];
    vol_weight<D, N>(a, ops, tile, s, l, Fb, Ft);
    const double *ut = a.U + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      U[v] = ut[v * TW];
      Ub[v] = 0.0;
    }
    flux_conv_vjp<D>(U, Fb, a.ph.gamma, Ub);
#pragma unroll
    for (int v = 0; v < V; v++) sUb[(s * V + v) * TW + l] = Ub[v];
    if (GEO && a.mbar)
    {
      // F~_d = sum_k adj[d][k] F_k: adj_bar[d][k] = sum_v F~bar_d[v] F[v][k]
      double F[V][D], P;
      flux_conv<double, D>(U, F, P, a.ph.gamma);
      geo_adj_bar<D>(a, tile, s, l, Ft, F, S);
    }
  }
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    double n[D], w[V], Uo[V], Ub[V];
    face_weight<D, N>(a, tile, f, l, code, n, w);
    const double *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      Uo[v] = uo[v * TW];
      Ub[v] = 0.0;
    }
    if (code >= 0)
    {
      double Un[V];
      gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
      const bool own_left = !(code & 1);
      conv_face_vjp_side<D>(own_left ? Uo : Un, own_left ? Un : Uo, n, w, own_left, a.ph, Ub);
    }
    else
    {
      double dUz[V][D], dUbz[V][D];
#pragma unroll
      for (int v = 0; v < V; v++)
#pragma unroll
        for (int d = 0; d < D; d++) dUz[v][d] = dUbz[v][d] = 0.0;
      bnd_face_vjp<D, false>(-code - 1, Uo, dUz, n, w, dual_phys(a.ph), Ub, dUbz);
      if (a.pbar) bnd_face_param_vjp<D, false>(-code - 1, Uo, dUz, n, w, dual_phys(a.ph), pb);
    }
#pragma unroll
    for (int v = 0; v < V; v++) sUbfp[(f * V + v) * TW + l] = Ub[v];
    if (GEO && a.gbar)
    {
      // face value phi = Fc; sFc = +-phi dA_own
      double Fc[V], nb[D], Un[V], dUz[V][D];
#pragma unroll
      for (int d = 0; d < D; d++) nb[d] = 0.0;
#pragma unroll
      for (int v = 0; v < V; v++)
#pragma unroll
        for (int d = 0; d < D; d++) dUz[v][d] = 0.0;
      if (code >= 0)
      {
        gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
        const bool own_left = !(code & 1);
        conv_face<D, double>(-1, own_left ? Uo : Un, own_left ? Un : Uo, n, Fc, a.ph);
        if (own_left) conv_face_n_vjp<D>(Uo, Un, n, w, a.ph, nb);
      }
      else
      {
        conv_face<D, double>(-code - 1, Uo, Uo, n, Fc, a.ph);
        bnd_face_n_vjp<D, false>(-code - 1, Uo, dUz, n, w, a.ph, nb);
      }
      geo_face_bar<D, N>(a, tile, f, l, code, Fc, nb);
    }
  }
  if (a.pbar) block_sum5(pb, a.pbar + tile * 5);
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double acc[V];
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = sUb[(s * V + v) * TW + l];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      int i, fm, fp;
      spt_ends<D, N>(s, d, i, fm, fp);
#pragma unroll
      for (int v = 0; v < V; v++)
        acc[v] += ops.Em[i] * sUbfp[(fm * V + v) * TW + l] + ops.Ep[i] * sUbfp[(fp * V + v) * TW + l];
    }
    double *out = a.Ubar + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = acc[v];
  }
}

// ---------------------------------------------------------------------------
// Navier-Stokes pass 1: recompute the common solution and gradient, adjoint of
// the volume flux, of the face fluxes and of the gradient; writes the partial
// solution-point result, the trace adjoint and the common-solution adjoint.
// ---------------------------------------------------------------------------
// Item order of the face pass: face pairs in turn, with the pair's two faces
// swapped on every other pair, so the items a thread takes (stride NT) mix
// both sides of the faces -- the Riemann VJP runs on the left side only,
// usually the + face -- and each warp's lanes stay on one face.
template <int D, int N>
__device__ __forceinline__ void face_item(int it, int &f, int &l)
{
  constexpr int NF = Shape<D, N>::NF;
  const int pair = it / (2 * NF * TW), within = it % (2 * NF * TW);
  const int face = 2 * pair + ((within / (NF * TW)) ^ (pair & 1));
  const int rest = within % (NF * TW);
  f = face * NF + rest / TW;
  l = rest % TW;
}

template <int D, int N, bool GEO>
__global__ void __launch_bounds__(Shape<D, N>::NT) k_adj_ns1(const __grid_constant__ AdjArgs a,
                                                                           const __grid_constant__ LineOpsT<double, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, NM = G::NM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sU = reinterpret_cast<double *>(smem_raw);  // [S][V][TW]
  double *sUC = sU + S * V * TW;                       // [Fp][V][TW]
  double *sdU = sUC + Fp * V * TW;                     // [D][S][V][TW] physical gradient
  // The state adjoint reuses the common solution's array for the volume
  // flux's U adjoint [S][V][TW] and the gradient's for the gradient adjoint
  // [D][S][V][TW] (each dead by then), which leaves more of the SM's L1 to
  // cache the gathers; the geometry variant reads both again later and keeps
  // all five apart.
  double *sUb = GEO ? sdU + D * S * V * TW : sUC;
  double *sG = GEO ? sUb + S * V * TW : sdU;
  // State adjoint: the face pass's inputs per own flux point -- weight w,
  // own and partner traces, normal -- gathered once in the common-solution
  // pass, where the same traces are loaded, so the register-heavy face pass
  // runs on shared-memory reads ([Fp][FK][TW]; FK = 3V + D).
  constexpr int FK = 3 * V + D;
  static_assert(FK >= V * D, "staging slots hold the gradient-trace adjoint");
  double *sFace = sdU + D * S * V * TW;
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  // this tile's metrics (gradient, volume and gradient-adjoint passes) and
  // the inputs of the tile one wave of resident CTAs (one per SM) ahead on
  // their way to L2
  if (threadIdx.x == 0)
  {
    prefetch_l2(a.mets + tile * (int64_t)S * NM * TW, S * NM * TW * sizeof(double));
    const int64_t ahead = tile + 148;
    if (ahead < a.ntiles)
    {
      prefetch_l2(a.Ufp + ahead * (int64_t)Fp * V * TW, Fp * V * TW * sizeof(double));
      prefetch_l2(a.Lfp + ahead * (int64_t)Fp * V * TW, Fp * V * TW * sizeof(double));
      prefetch_l2(a.fgeo + ahead * (int64_t)Fp * (D + 1) * TW, Fp * (D + 1) * TW * sizeof(double));
      prefetch_l2(a.nbr + ahead * (int64_t)Fp * TW, Fp * TW * sizeof(int));
      prefetch_l2(a.U + ahead * (int64_t)S * V * TW, S * V * TW * sizeof(double));
    }
  }
  const double beta = a.ph.ldg_b, tau = a.ph.ldg_tau;
  double pb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  {
    const double *src = a.U + tile * (int64_t)S * V * TW;
    for (int i = threadIdx.x; i < S * V * TW; i += blockDim.x) sU[i] = src[i];
  }
  // common solution (as k_ns_grad); unrolled over a thread's items so their
  // gathers are in flight together
#pragma unroll
  for (int k = 0; k < (Fp * TW + G::NT - 1) / G::NT; k++)
  {
    const int it = (int)threadIdx.x + k * G::NT;
    if (it >= Fp * TW) break;
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    double Uo[V], UC[V];
    const double *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (!GEO)
    {
      double n[D], w[V];
      face_weight<D, N>(a, tile, f, l, code, n, w);
      double *sf = sFace + f * FK * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        sf[v * TW] = w[v];
        sf[(V + v) * TW] = Uo[v];
      }
#pragma unroll
      for (int d = 0; d < D; d++) sf[(3 * V + d) * TW] = n[d];
    }
    if (code >= 0)
    {
      double Un[V];
      gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
      if (!GEO)
      {
#pragma unroll
        for (int v = 0; v < V; v++) sFace[(f * FK + 2 * V + v) * TW + l] = Un[v];
      }
      const int slot = code & 1;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        const double ul = slot ? Un[v] : Uo[v];
        const double ur = slot ? Uo[v] : Un[v];
        if (beta == 0.5)
          UC[v] = ur;
        else if (beta == -0.5)
          UC[v] = ul;
        else
          UC[v] = 0.5 * (ul + ur) - beta * (ul - ur);
      }
    }
    else
    {
      double n[D], UR[V];
      const double *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
      for (int d = 0; d < D; d++) n[d] = g[d * TW];
      ghost_state<double, D>(-code - 1, Uo, n, UR, UC, a.ph);
    }
#pragma unroll
    for (int v = 0; v < V; v++) sUC[(f * V + v) * TW + l] = UC[v];
  }
  __syncthreads();
  // physical gradient (as k_ns_grad)
#pragma unroll
  for (int k = 0; k < (S * TW + G::NT - 1) / G::NT; k++)
  {
    const int it = (int)threadIdx.x + k * G::NT;
    if (it >= S * TW) break;
    const int s = it / TW, l = it % TW;
    double tdU[V][D];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      int i, fm, fp;
      spt_ends<D, N>(s, d, i, fm, fp);
      const int st = pow_n<N>(d);
      const int b = s - i * st;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        double acc = 0.0;
#pragma unroll
        for (int m = 0; m < N; m++) acc += ops.Dm[i * N + m] * sU[((b + m * st) * V + v) * TW + l];
        const double cm = ops.Dbm[i] * sUC[(fm * V + v) * TW + l];
        const double cp = ops.Dbp[i] * sUC[(fp * V + v) * TW + l];
        tdU[v][d] = acc + ((fm < fp) ? (cm + cp) : (cp + cm));
      }
    }
    const double *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    const double inv_det = 1.0 / m[D * D * TW];
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d1 = 0; d1 < D; d1++)
      {
        double g = tdU[v][0] * m[(0 * D + d1) * TW];
#pragma unroll
        for (int d2 = 1; d2 < D; d2++) g += tdU[v][d2] * m[(d2 * D + d1) * TW];
        sdU[((d1 * S + s) * V + v) * TW + l] = g * inv_det;
      }
  }
  __syncthreads();
  // adjoint of the face fluxes at own flux points
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    int f, l;
    face_item<D, N>(it, f, l);
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    double n[D], w[V], Uo[V], dUo[V][D], Ub[V], dUb[V][D];
    const double *sf = sFace + f * FK * TW + l;
    if (GEO)
      face_weight<D, N>(a, tile, f, l, code, n, w);
    else
    {
#pragma unroll
      for (int v = 0; v < V; v++) w[v] = sf[v * TW];
#pragma unroll
      for (int d = 0; d < D; d++) n[d] = sf[(3 * V + d) * TW];
    }
    const double *uo = GEO ? a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l : sf + V * TW;
    SOps<double, N> o(reinterpret_cast<const double *>(&ops));
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      Uo[v] = uo[v * TW];
      Ub[v] = 0.0;
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        dUo[v][d] = extrap_smem<double, D, N>(sdU + d * S * V * TW, o, f, v, l, V);
        dUb[v][d] = 0.0;
      }
    }
    if (code >= 0)
    {
      const bool own_left = !(code & 1);
      if (own_left)
      {
        // one reverse sweep of the shared Riemann flux gives both sides'
        // adjoints (the right side forms the same weight w bitwise): keep
        // the left's, leave the right's at the partner's flux point
        double Un[V], bL[V], bR[V];
        if (GEO)
          gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
        else
        {
#pragma unroll
          for (int v = 0; v < V; v++) Un[v] = sf[(2 * V + v) * TW];
        }
#pragma unroll
        for (int v = 0; v < V; v++) bL[v] = bR[v] = 0.0;
        if (a.ph.fconv == 2)
          roe_vjp<D>(Uo, Un, n, w, a.ph, bL, bR);
        else
          rusanov_vjp<D>(Uo, Un, n, w, a.ph, bL, bR);
        const int pidx = code >> 1;
        double *px = a.Ubx + (int64_t)(pidx / TW) * V * TW + pidx % TW;
#pragma unroll
        for (int v = 0; v < V; v++)
        {
          Ub[v] += bL[v];
          px[v * TW] = bR[v];
        }
      }
      // LDG: (1/2 + beta) FnL + (1/2 - beta) FnR + tau (UL - UR)
      const double c = own_left ? 0.5 + beta : 0.5 - beta;
      if (c != 0.0)
      {
        double wc[V];
#pragma unroll
        for (int v = 0; v < V; v++) wc[v] = c * w[v];
        visc_normal_vjp<D>(Uo, dUo, n, wc, a.ph, Ub, dUb);
      }
#pragma unroll
      for (int v = 0; v < V; v++) Ub[v] += own_left ? tau * w[v] : -tau * w[v];
    }
    else
    {
      bnd_face_vjp<D, true>(-code - 1, Uo, dUo, n, w, dual_phys(a.ph), Ub, dUb);
      if (a.pbar) bnd_face_param_vjp<D, true>(-code - 1, Uo, dUo, n, w, dual_phys(a.ph), pb);
    }
    if (GEO && a.gbar) geo_face_ns<D, N>(a, tile, f, l, code, n, w, Uo, dUo);
    double *ub = a.Ubfp + (tile * Fp + f) * (int64_t)V * TW + l;
    // the gradient-trace adjoint stays in this tile: the state adjoint keeps
    // it in the item's staging slots (read above, FK >= V D), the geometry
    // variant in global memory
    double *dub = GEO ? a.dUbfp + (tile * Fp + f) * (int64_t)V * D * TW + l : sFace + f * FK * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      ub[v * TW] = Ub[v];
#pragma unroll
      for (int d = 0; d < D; d++) dub[(v * D + d) * TW] = dUb[v][d];
    }
  }
  __syncthreads();  // the face pass reads sdU, which the volume pass may overwrite
  // adjoint of the volume flux: U and gradient parts
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double Fb[V][D], U[V], dU[V][D], Ub[V], dUb[V][D];
    double Ft[D][V];
    vol_weight<D, N>(a, ops, tile, s, l, Fb, Ft);
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      U[v] = sU[(s * V + v) * TW + l];
      Ub[v] = 0.0;
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        dU[v][d] = sdU[((d * S + s) * V + v) * TW + l];
        dUb[v][d] = 0.0;
      }
    }
    flux_conv_vjp<D>(U, Fb, a.ph.gamma, Ub);
    flux_visc_vjp<D>(U, dU, Fb, a.ph, Ub, dUb);
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      sUb[(s * V + v) * TW + l] = Ub[v];
#pragma unroll
      for (int d = 0; d < D; d++) sG[((d * S + s) * V + v) * TW + l] = dUb[v][d];
    }
    if (GEO && a.mbar)
    {
      double F[V][D], P;
      flux_conv<double, D>(U, F, P, a.ph.gamma);
      flux_visc_add<double, D>(U, dU, F, a.ph);
      geo_adj_bar<D>(a, tile, s, l, Ft, F, S);
    }
  }
  __syncthreads();
  // gradient adjoint: add the transposed trace extrapolation, then map to
  // the reference gradient: tdUb[v][d2] = sum_d1 adj[d2][d1] dUb[v][d1] / |J|
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double g[V][D];
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d = 0; d < D; d++) g[v][d] = sG[((d * S + s) * V + v) * TW + l];
#pragma unroll
    for (int dl = 0; dl < D; dl++)
    {
      int i, fm, fp;
      spt_ends<D, N>(s, dl, i, fm, fp);
      const double *bm = GEO ? a.dUbfp + (tile * Fp + fm) * (int64_t)V * D * TW + l : sFace + fm * FK * TW + l;
      const double *bp = GEO ? a.dUbfp + (tile * Fp + fp) * (int64_t)V * D * TW + l : sFace + fp * FK * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++)
#pragma unroll
        for (int d = 0; d < D; d++) g[v][d] += ops.Em[i] * bm[(v * D + d) * TW] + ops.Ep[i] * bp[(v * D + d) * TW];
    }
    const double *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    const double inv_det = 1.0 / m[D * D * TW];
    if (GEO && a.mbar)
    {
      // dU[v][d1] = sum_d2 tdU[v][d2] adj[d2][d1] / |J|
      double *mb = a.mbar + (tile * S + s) * (int64_t)NM * TW + l;
      double detb = 0.0;
#pragma unroll
      for (int d2 = 0; d2 < D; d2++)
      {
        int i, fm, fp;
        spt_ends<D, N>(s, d2, i, fm, fp);
        const int st = pow_n<N>(d2);
        const int b = s - i * st;
        double ab[D];
#pragma unroll
        for (int d1 = 0; d1 < D; d1++) ab[d1] = 0.0;
#pragma unroll
        for (int v = 0; v < V; v++)
        {
          double acc = 0.0;
#pragma unroll
          for (int mm = 0; mm < N; mm++) acc += ops.Dm[i * N + mm] * sU[((b + mm * st) * V + v) * TW + l];
          const double cm = ops.Dbm[i] * sUC[(fm * V + v) * TW + l];
          const double cp = ops.Dbp[i] * sUC[(fp * V + v) * TW + l];
          const double tdu = acc + ((fm < fp) ? (cm + cp) : (cp + cm));
#pragma unroll
          for (int d1 = 0; d1 < D; d1++) ab[d1] += g[v][d1] * tdu;
        }
#pragma unroll
        for (int d1 = 0; d1 < D; d1++) mb[(d2 * D + d1) * TW] += ab[d1] * inv_det;
      }
#pragma unroll
      for (int v = 0; v < V; v++)
#pragma unroll
        for (int d1 = 0; d1 < D; d1++) detb -= g[v][d1] * sdU[((d1 * S + s) * V + v) * TW + l];
      mb[D * D * TW] += detb * inv_det;
    }
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d2 = 0; d2 < D; d2++)
      {
        double acc = 0.0;
#pragma unroll
        for (int d1 = 0; d1 < D; d1++) acc += m[(d2 * D + d1) * TW] * g[v][d1];
        sG[((d2 * S + s) * V + v) * TW + l] = acc * inv_det;
      }
  }
  __syncthreads();
  // U part of the reference gradient: Ub += Dm^T tdUb along each line
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double acc[V];
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = sUb[(s * V + v) * TW + l];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      int i, fm, fp;
      spt_ends<D, N>(s, d, i, fm, fp);
      const int st = pow_n<N>(d);
      const int b = s - i * st;
#pragma unroll
      for (int m = 0; m < N; m++)
      {
        const double c = ops.Dm[m * N + i];
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] += c * sG[((d * S + b + m * st) * V + v) * TW + l];
      }
    }
    double *out = a.Ubar + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = acc[v];
  }
  // common solution part: UCb(f) = sum over the line of (Dbm | Dbp)[m] tdUb
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    int dim, side, base, stride;
    fpt_line<D, N>(f, dim, side, base, stride);
    double ucb[V];
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < N; m++)
        acc += (side < 0 ? ops.Dbm[m] : ops.Dbp[m]) * sG[((dim * S + base + m * stride) * V + v) * TW + l];
      ucb[v] = acc;
    }
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    if (code >= 0)
    {
      double *out = a.UCb + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++) out[v * TW] = ucb[v];
    }
    else
    {
      double n[D], Uo[V], Ub[V];
      const double *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
      for (int d = 0; d < D; d++) n[d] = g[d * TW];
      const double *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
      double *ub = a.Ubfp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        Uo[v] = uo[v * TW];
        Ub[v] = 0.0;
      }
      bnd_ucomm_vjp<D>(-code - 1, Uo, n, ucb, dual_phys(a.ph), Ub);
      if (a.pbar) bnd_ucomm_param_vjp<D>(-code - 1, Uo, n, ucb, dual_phys(a.ph), pb);
      if (GEO && a.gbar)
      {
        double nb[D];
#pragma unroll
        for (int d = 0; d < D; d++) nb[d] = 0.0;
        bnd_ucomm_n_vjp<D>(-code - 1, Uo, n, ucb, a.ph, nb);
        double *gg = a.gbar + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
        for (int d = 0; d < D; d++) gg[d * TW] += nb[d];
      }
#pragma unroll
      for (int v = 0; v < V; v++) ub[v * TW] += Ub[v];
    }
  }
  if (a.pbar) block_sum5(pb, a.pbar + tile * 5);
}

// ---------------------------------------------------------------------------
// Navier-Stokes pass 2: both sides' common-solution adjoints reach the own
// trace, then the transposed extrapolation finishes Ubar.
// ---------------------------------------------------------------------------
template <int D, int N, bool GEO>
__global__ void __launch_bounds__(Shape<D, N>::NT) k_adj_ns2(const __grid_constant__ AdjArgs a,
                                                             const __grid_constant__ LineOpsT<double, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sUbfp = reinterpret_cast<double *>(smem_raw);  // [Fp][V][TW]
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  const double beta = a.ph.ldg_b;
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    const double *ub = a.Ubfp + (tile * Fp + f) * (int64_t)V * TW + l;
    double Ub[V];
#pragma unroll
    for (int v = 0; v < V; v++) Ub[v] = ub[v * TW];
    if (code >= 0 && (code & 1))
    {
      // the Riemann-flux adjoint the left partner formed for this trace
      const double *ux = a.Ubx + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++) Ub[v] += ux[v * TW];
    }
    if (GEO && a.gbar && code >= 0 && !(code & 1))
    {
      // collect the right side's viscous part of this face's normal adjoint
      const int pidx = code >> 1;
      double *gg = a.gbar + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
      for (int d = 0; d < D; d++)
        gg[d * TW] += a.nbx[((int64_t)(pidx / TW) * D + d) * TW + pidx % TW];
    }
    if (code >= 0)
    {
      // UC = (1/2 - beta) UL + (1/2 + beta) UR, shared by both sides
      const bool own_left = !(code & 1);
      const double c = own_left ? 0.5 - beta : 0.5 + beta;
      if (c != 0.0)
      {
        double Co[V], Cn[V];
        const double *co = a.UCb + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
        for (int v = 0; v < V; v++) Co[v] = co[v * TW];
        gather_fpt<double, double, V>(a.UCb, code >> 1, Cn);
#pragma unroll
        for (int v = 0; v < V; v++) Ub[v] += c * (Co[v] + Cn[v]);
      }
    }
#pragma unroll
    for (int v = 0; v < V; v++) sUbfp[(f * V + v) * TW + l] = Ub[v];
  }
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double *out = a.Ubar + (tile * S + s) * (int64_t)V * TW + l;
    double acc[V];
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = out[v * TW];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      int i, fm, fp;
      spt_ends<D, N>(s, d, i, fm, fp);
#pragma unroll
      for (int v = 0; v < V; v++)
        acc[v] += ops.Em[i] * sUbfp[(fm * V + v) * TW + l] + ops.Ep[i] * sUbfp[(fp * V + v) * TW + l];
    }
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = acc[v];
  }
}

}  // namespace dev
}  // namespace zb
