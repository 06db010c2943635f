// Forward-mode dual numbers for pointwise Jacobian-transpose products.
//
// The residual's pointwise functions (fluxes, Riemann solvers, boundary ghost
// states, viscous normal flux) are templated on their arithmetic type; running
// them on Dual<double> with one input seeded gives one column of the local
// Jacobian exactly.  vjp_local() sums lambda . column over all seeded inputs,
// i.e. J^T lambda.  Comparisons and branches act on the value part, so a
// max() or a boundary-state switch contributes the derivative of the branch
// taken (the subgradient of the reference's max(|VnL|+aL, |VnR|+aR)).
#pragma once

#include <cuda_runtime.h>

#include "physics.cuh"

namespace zb {
namespace dev {

template <typename T>
struct Dual
{
  T v, d;
  __host__ __device__ constexpr Dual() : v(0), d(0) {}
  __host__ __device__ constexpr Dual(T x) : v(x), d(0) {}
  __host__ __device__ constexpr Dual(T x, T dx) : v(x), d(dx) {}
};

template <typename T> ZB_HD Dual<T> operator+(Dual<T> a, Dual<T> b) { return {a.v + b.v, a.d + b.d}; }
template <typename T> ZB_HD Dual<T> operator-(Dual<T> a, Dual<T> b) { return {a.v - b.v, a.d - b.d}; }
template <typename T> ZB_HD Dual<T> operator-(Dual<T> a) { return {-a.v, -a.d}; }
template <typename T> ZB_HD Dual<T> operator*(Dual<T> a, Dual<T> b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
template <typename T> ZB_HD Dual<T> operator/(Dual<T> a, Dual<T> b)
{
  const T q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
template <typename T> ZB_HD Dual<T> &operator+=(Dual<T> &a, Dual<T> b) { a = a + b; return a; }
template <typename T> ZB_HD Dual<T> &operator-=(Dual<T> &a, Dual<T> b) { a = a - b; return a; }
template <typename T> ZB_HD Dual<T> &operator*=(Dual<T> &a, Dual<T> b) { a = a * b; return a; }
template <typename T> ZB_HD Dual<T> &operator/=(Dual<T> &a, Dual<T> b) { a = a / b; return a; }
template <typename T> ZB_HD bool operator<(Dual<T> a, Dual<T> b) { return a.v < b.v; }
template <typename T> ZB_HD bool operator>(Dual<T> a, Dual<T> b) { return a.v > b.v; }
template <typename T> ZB_HD bool operator<=(Dual<T> a, Dual<T> b) { return a.v <= b.v; }
template <typename T> ZB_HD bool operator>=(Dual<T> a, Dual<T> b) { return a.v >= b.v; }
template <typename T> ZB_HD bool operator==(Dual<T> a, Dual<T> b) { return a.v == b.v; }

template <> ZB_HD Dual<double> dsqrt<Dual<double>>(Dual<double> x)
{
  const double s = sqrt(x.v);
  return {s, x.d / (2.0 * s)};
}
template <> ZB_HD Dual<double> dpow<Dual<double>>(Dual<double> x, Dual<double> y)
{
  // y is a constant exponent in every use (1.5, gamma, 1/(gamma-1))
  const double p = pow(x.v, y.v);
  return {p, y.v * pow(x.v, y.v - 1.0) * x.d};
}

template <typename T>
ZB_HD Phys<Dual<T>> dual_phys(const Phys<T> &p)
{
  Phys<Dual<T>> q;
  q.gamma = p.gamma;
  q.prandtl = p.prandtl;
  q.mu = p.mu;
  q.rt = p.rt;
  q.c_sth = p.c_sth;
  q.rus_k = p.rus_k;
  q.ldg_b = p.ldg_b;
  q.ldg_tau = p.ldg_tau;
  q.rho_fs = p.rho_fs;
  q.P_fs = p.P_fs;
  q.T_wall = p.T_wall;
  q.R_ref = p.R_ref;
  for (int d = 0; d < 3; d++)
  {
    q.V_fs[d] = p.V_fs[d];
    q.V_wall[d] = p.V_wall[d];
  }
  for (int v = 0; v < 5; v++) q.Ur[v] = p.Ur[v];
  q.Pr = p.Pr;
  q.er = p.er;
  q.inv_rr = p.inv_rr;
  q.mr2 = p.mr2;
  q.fix_vis = p.fix_vis;
  q.fconv = p.fconv;
  q.dev = p.dev;
  return q;
}

// g = J^T lam for y = f(x), x in R^NI, y in R^NO; f(const Dual* x, Dual* y).
template <int NI, int NO, typename F>
ZB_HD void vjp_local(F &&f, const double x[NI], const double lam[NO], double g[NI])
{
#pragma unroll 1
  for (int k = 0; k < NI; k++)
  {
    Dual<double> xd[NI], yd[NO];
#pragma unroll
    for (int i = 0; i < NI; i++) xd[i] = Dual<double>(x[i], i == k ? 1.0 : 0.0);
    f(xd, yd);
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < NO; i++) acc += lam[i] * yd[i].d;
    g[k] = acc;
  }
}

}  // namespace dev
}  // namespace zb
