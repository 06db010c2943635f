// Host-side check of the hand-written reverse-mode pointwise functions of the
// adjoint against forward-mode dual numbers through the forward physics
// (both compiled for the CPU).  Prints the worst relative error and exits
// non-zero above 1e-12.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "../../zefr_b200/csrc/adjoint.cuh"

using namespace zb::dev;
using DD = Dual<double>;

static double g_worst = 0.0;

static void record(const char *what, double a, double b)
{
  const double e = std::fabs(a - b) / (1e-300 + std::fmax(1.0, std::fmax(std::fabs(a), std::fabs(b))));
  if (e > g_worst) g_worst = e;
  if (e > 1e-12) std::printf("MISMATCH %s: %.17g vs %.17g\n", what, a, b);
}

static Phys<double> phys(bool sutherland)
{
  Phys<double> p;
  std::memset(&p, 0, sizeof(p));
  p.gamma = 1.4;
  p.prandtl = 0.71;
  p.mu = 3.1e-3;
  p.rt = 0.7;
  p.c_sth = 0.37;
  p.fix_vis = sutherland ? 0 : 1;
  return p;
}

template <int D>
static void check_point(std::mt19937_64 &rng, bool sutherland)
{
  constexpr int V = D + 2;
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  double U[V], dU[V][D], Fb[V][D];
  U[0] = 1.0 + 0.3 * u(rng);
  double m2 = 0.0;
  for (int d = 0; d < D; d++)
  {
    U[d + 1] = 0.4 * u(rng);
    m2 += U[d + 1] * U[d + 1];
  }
  U[V - 1] = 2.5 + 0.5 * m2 / U[0] + 0.2 * u(rng);
  for (int v = 0; v < V; v++)
    for (int d = 0; d < D; d++)
    {
      dU[v][d] = u(rng);
      Fb[v][d] = u(rng);
    }
  const Phys<double> ph = phys(sutherland);
  const Phys<DD> pd = dual_phys(ph);
  // hand reverse
  double Ub[V] = {0}, dUb[V][D] = {{0}}, Ubc[V] = {0};
  flux_conv_vjp<D>(U, Fb, ph.gamma, Ubc);
  flux_visc_vjp<D>(U, dU, Fb, ph, Ub, dUb);
  // dual forward, one seed per input
  for (int k = 0; k < V + V * D; k++)
  {
    DD Ud[V], dUd[V][D], Fc[V][D], Fv[V][D], P;
    for (int v = 0; v < V; v++)
    {
      Ud[v] = DD(U[v], v == k ? 1.0 : 0.0);
      for (int d = 0; d < D; d++)
      {
        dUd[v][d] = DD(dU[v][d], (k == V + v * D + d) ? 1.0 : 0.0);
        Fv[v][d] = DD(0.0);
      }
    }
    flux_conv<DD, D>(Ud, Fc, P, pd.gamma);
    flux_visc_add<DD, D>(Ud, dUd, Fv, pd);
    double sc = 0.0, sv = 0.0;
    for (int v = 0; v < V; v++)
      for (int d = 0; d < D; d++)
      {
        sc += Fb[v][d] * Fc[v][d].d;
        sv += Fb[v][d] * Fv[v][d].d;
      }
    if (k < V)
    {
      record("conv dU", Ubc[k], sc);
      record("visc dU", Ub[k], sv);
    }
    else
    {
      record("conv d(grad)", 0.0, sc);
      record("visc d(grad)", dUb[(k - V) / D][(k - V) % D], sv);
    }
  }
  // dual against a central difference of the forward flux
  const double h = 1e-6;
  for (int k = 0; k < V; k++)
  {
    double Up[V], Um[V], Fp[V][D], Fm[V][D], Pp, Pm;
    for (int v = 0; v < V; v++) Up[v] = Um[v] = U[v];
    Up[k] += h;
    Um[k] -= h;
    flux_conv<double, D>(Up, Fp, Pp, ph.gamma);
    flux_conv<double, D>(Um, Fm, Pm, ph.gamma);
    double s = 0.0;
    for (int v = 0; v < V; v++)
      for (int d = 0; d < D; d++) s += Fb[v][d] * (Fp[v][d] - Fm[v][d]) / (2 * h);
    const double e = std::fabs(s - Ubc[k]) / std::fmax(1.0, std::fabs(s));
    if (e > 1e-7)
    {
      std::printf("FD MISMATCH conv %d: %.12g vs %.12g\n", k, s, Ubc[k]);
      g_worst = std::fmax(g_worst, 1.0);
    }
  }
}

// Riemann solvers: hand reverse (both sides) against dual numbers.  near0
// puts the normal velocity near zero so Roe's entropy fix is active.
template <int D>
static void check_riemann(std::mt19937_64 &rng, int fconv, bool near0)
{
  constexpr int V = D + 2;
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  double UL[V], UR[V], n[D], w[V];
  double nn = 0.0;
  for (int d = 0; d < D; d++)
  {
    n[d] = u(rng);
    nn += n[d] * n[d];
  }
  for (int d = 0; d < D; d++) n[d] /= std::sqrt(nn);
  for (double *U : {UL, UR})
  {
    U[0] = 1.0 + 0.3 * u(rng);
    double m2 = 0.0;
    for (int d = 0; d < D; d++)
    {
      U[d + 1] = (near0 ? 0.02 : 0.6) * u(rng);
      m2 += U[d + 1] * U[d + 1];
    }
    U[V - 1] = 2.5 + 0.5 * m2 / U[0] + 0.2 * u(rng);
  }
  for (int v = 0; v < V; v++) w[v] = u(rng);
  Phys<double> ph = phys(false);
  ph.fconv = fconv;
  ph.rus_k = 0.0;
  const Phys<DD> pd = dual_phys(ph);
  double bL[V] = {0}, bR[V] = {0};
  if (fconv == 2)
    roe_vjp<D>(UL, UR, n, w, ph, bL, bR);
  else
    rusanov_vjp<D>(UL, UR, n, w, ph, bL, bR);
  for (int k = 0; k < 2 * V; k++)
  {
    DD L[V], R[V], F[V], nd[D];
    for (int d = 0; d < D; d++) nd[d] = DD(n[d]);
    for (int v = 0; v < V; v++)
    {
      L[v] = DD(UL[v], k == v ? 1.0 : 0.0);
      R[v] = DD(UR[v], k == V + v ? 1.0 : 0.0);
    }
    if (fconv == 2)
      roe<DD, D>(L, R, nd, F, pd);
    else
      rusanov<DD, D>(L, R, nd, F, pd);
    double s = 0.0;
    for (int v = 0; v < V; v++) s += w[v] * F[v].d;
    record(fconv == 2 ? "roe" : "rusanov", k < V ? bL[k] : bR[k - V], s);
  }
}

int main()
{
  std::mt19937_64 rng(20261203);
  for (int i = 0; i < 200; i++)
  {
    check_point<2>(rng, false);
    check_point<2>(rng, true);
    check_point<3>(rng, false);
    check_point<3>(rng, true);
    for (int fc : {0, 2})
      for (bool z : {false, true})
      {
        check_riemann<2>(rng, fc, z);
        check_riemann<3>(rng, fc, z);
      }
  }
  std::printf("worst relative error %.3e\n", g_worst);
  return g_worst > 1e-12 ? 1 : 0;
}
