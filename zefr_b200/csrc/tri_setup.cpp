// Host-side set-up of flux reconstruction on triangles: Williams-Shunn
// solution points, the orthonormal (Dubiner) basis, the dense FR operators
// with the 'M3' correction, flux-point tables and linear / quadratic shape
// functions.
//
// Reference sources followed (paths inside the reference project):
//   points, weights     src/points.cpp:226-636 (WS_Tri_pts, WS_Tri_weights)
//   point tables        src/tris.cpp:46-148 (set_locs, set_normals)
//   basis               src/polynomials.cpp:28-190 (Jacobi, Dubiner2D, dDubiner2D)
//   operators           src/elements.cpp:555-744 (setup_FR, triangle branch)
//   shape functions     src/tris.cpp:495-590
#include <cmath>
#include <cstring>

#include "zb_internal.hpp"

namespace zb {

// ---------------------------------------------------------------------------
// Williams-Shunn points (Williams, Shunn & Jameson, J. Comput. Appl. Math. 266
// (2014) 18-38) on the reference triangle {xi, eta >= -1, xi + eta <= 0}, in the
// reference's order.  The table is stored as symmetry orbits: a 3-orbit (a, b)
// lists (a,b), (b,a), (a,a); a 6-orbit (c, d, e) lists (c,d), (e,d), (d,e),
// (c,e), (e,c), (d,c); a 1-orbit is the centroid.  The numbers are the
// reference's own decimals, so the points (and with them every operator and
// the state layout) coincide.
// ---------------------------------------------------------------------------
struct WsOrbit
{
  int n;  // 1, 3 or 6
  double v[3];
  double w;
};

static std::vector<WsOrbit> ws_orbits(int P)
{
  switch (P)
  {
    case 1:
      return {{3, {-0.6666666666666660, 0.3333333333333320, 0}, 0.6666666666666660}};
    case 2:
      return {{3, {-0.8168475729804400, 0.6336951459608799, 0}, 0.2199034873106660},
              {3, {-0.1081030181680720, -0.7837939636638560, 0}, 0.4467631793560000}};
    case 3:
      return {{1, {-0.3333333333333330, 0, 0}, 0.4030859771694600},
              {3, {-0.8888718946604141, 0.7777437893208280, 0}, 0.0839110259932980},
              {6, {0.2684214954914460, -0.4089325765282140, -0.8594889189632320}, 0.2241968241417740}};
    case 4:
      return {{3, {-0.9282582446085320, 0.8565164892170640, 0}, 0.0358309100246060},
              {3, {-0.5165412084640660, 0.0330824169281320, 0}, 0.2554243917625300},
              {3, {-0.0513824244458420, -0.8972351511083160, 0}, 0.1524121247710700},
              {6, {0.5023672622129680, -0.5969922362364000, -0.9053750259765680}, 0.1114996200542300}};
    case 5:
      return {{3, {-0.9437740956346720, 0.8875481912693440, 0}, 0.0207187493930760},
              {3, {-0.6457218030613660, 0.2914436061227320, 0}, 0.1507897686534760},
              {3, {-0.1889828082651340, -0.6220343834697321, 0}, 0.1950956047464840},
              {6, {0.6358019600569980, -0.7028683754582260, -0.9329335845987720}, 0.0579385387449460},
              {6, {0.2099578235502660, -0.2856074027686380, -0.9243504207816280}, 0.0920927331918700}};
    case 6:
      return {{1, {-0.3333333333333330, 0, 0}, 0.1672164244312740},
              {3, {-0.9600456257556140, 0.9200912515112279, 0}, 0.0105443405609900},
              {3, {-0.7365564649400040, 0.4731129298800080, 0}, 0.0891058733590080},
              {3, {-0.0297293064130780, -0.9405413871738439, 0}, 0.0676314256083960},
              {6, {0.7358224202359001, -0.7840960363079780, -0.9517263839279220}, 0.0314209226803660},
              {6, {0.4017451407614460, -0.4583184541568660, -0.9434266866045800}, 0.0564102725612320},
              {6, {0.0733093684122760, -0.3669008023107660, -0.7064085661015100}, 0.1339919142556600}};
    case 7:
      return {{3, {-0.9576571544410700, 0.9153143088821400, 0}, 0.0112782475738200},
              {3, {-0.7988312052082240, 0.5976624104164480, 0}, 0.0542979363845560},
              {3, {-0.4579233845761360, -0.0841532308477280, 0}, 0.1262018250667180},
              {3, {-0.1196174831923360, -0.7607650336153280, 0}, 0.1035055913597980},
              {6, {0.7599592828544620, -0.9634866418505040, -0.7964726410039580}, 0.0197335071492920},
              {6, {0.1651240457273440, -0.2119334566600260, -0.9531905890673180}, 0.0440164096002940},
              {6, {0.5030612290855641, -0.5475089381815420, -0.9555522909040221}, 0.0332891401534720},
              {6, {0.2714743665262100, -0.5018415447573360, -0.7696328217688740}, 0.0886524762378280}};
    case 8:
      return {{3, {-0.8958458673313620, 0.7916917346627240, 0}, 0.0264519521410120},
              {3, {-0.7725869427780080, 0.5451738855560160, 0}, 0.0347516292773620},
              {3, {-0.5656623084521640, 0.1313246169043280, 0}, 0.0945461565676520},
              {3, {-0.2278544512773540, -0.5442910974452920, 0}, 0.1060044409420360},
              {3, {-0.0201481341734600, -0.9597037316530800, 0}, 0.0378851639278180},
              {6, {0.6693761812315560, -0.7035037567771640, -0.9658724244543920}, 0.0238755661869220},
              {6, {0.4144959853084960, -0.5795767423228601, -0.8349192429856360}, 0.0493958430852700},
              {6, {0.9258038332858580, -0.9258815152162200, -0.9999223180696380}, 0.0043857672678220},
              {6, {0.3480122228257960, -0.3820797590136400, -0.9659324638121560}, 0.0308750382999060},
              {6, {0.0838979176456600, -0.2793516463213580, -0.8045462713243020}, 0.0749814470654740}};
    default:
      ZB_THROW(ZB_ERR_UNSUPPORTED, "triangle solution points built for P = 1..8, not P = " + std::to_string(P));
  }
}

static void ws_points(int P, std::vector<double> &loc, std::vector<double> &w)
{
  loc.clear();
  w.clear();
  for (const WsOrbit &o : ws_orbits(P))
  {
    auto put = [&](double x, double y) {
      loc.push_back(x);
      loc.push_back(y);
      w.push_back(o.w);
    };
    if (o.n == 1)
      put(o.v[0], o.v[0]);
    else if (o.n == 3)
    {
      put(o.v[0], o.v[1]);
      put(o.v[1], o.v[0]);
      put(o.v[0], o.v[0]);
    }
    else
    {
      const double c = o.v[0], d = o.v[1], e = o.v[2];
      put(c, d);
      put(e, d);
      put(d, e);
      put(c, e);
      put(e, c);
      put(d, c);
    }
  }
}

// ---------------------------------------------------------------------------
// Orthonormal basis on the reference triangle (Dubiner / Koornwinder in the
// collapsed coordinates a = 2(1+xi)/(1-eta) - 1, b = eta; Hesthaven &
// Warburton, "Nodal Discontinuous Galerkin Methods", sec. 6.1):
//   psi_(i,j) = sqrt(2) P_i^(0,0)(a) P_j^(2i+1,0)(b) (1-b)^i
// with P^(alpha,beta) the Jacobi polynomials normalised to unit L2 norm on
// [-1,1] with weight (1-x)^alpha (1+x)^beta.  Modes are ordered by total
// degree k, then j = 0..k with i = k - j (the reference's mode order).
// ---------------------------------------------------------------------------
static double jacobi_n(double x, double al, double be, int n)
{
  // orthonormal Jacobi polynomials by their three-term recurrence, evaluated
  // upward with the same expressions per degree as the reference's recursive
  // HiFiLES form (src/polynomials.cpp:28-83), so the values agree bitwise
  const double c0 = std::pow(2.0, (-al - be - 1)) *
                    (std::tgamma(al + be + 2) / (std::tgamma(al + 1) * std::tgamma(be + 1)));
  double pm2 = std::sqrt(c0);
  if (n == 0) return pm2;
  double pm1 = 0.5 * std::sqrt(c0) * std::sqrt((al + be + 3) / ((al + 1) * (be + 1))) * (x * (al + be + 2) + (al - be));
  if (n == 1) return pm1;
  double p = pm1;
  for (int m = 2; m <= n; m++)
  {
    const double d0 = m * (m + al + be) * (m + al) * (m + be);
    const double d1 = ((2 * m) + al + be - 1) * ((2 * m) + al + be + 1);
    const double d3 = (2 * m) + al + be;
    const double d4 = (m - 1) * ((m - 1) + al + be) * ((m - 1) + al) * ((m - 1) + be);
    const double d5 = ((2 * (m - 1)) + al + be - 1) * ((2 * (m - 1)) + al + be + 1);
    const double d6 = (2 * (m - 1)) + al + be;
    const double d7 = -((al * al) - (be * be));
    const double d8 = ((2 * (m - 1)) + al + be) * ((2 * (m - 1)) + al + be + 2);
    const double d9 = (2.0 / d3) * std::sqrt(d0 / d1);
    const double d10 = (2.0 / d6) * std::sqrt(d4 / d5);
    const double d11 = d7 / d8;
    p = (1.0 / d9) * (x * pm1 - d10 * pm2 - d11 * pm1);
    pm2 = pm1;
    pm1 = p;
  }
  return p;
}

static double djacobi_n(double x, double al, double be, int n)
{
  if (n == 0) return 0.0;
  return std::sqrt(n * (n + al + be + 1)) * jacobi_n(x, al + 1, be + 1, n - 1);
}

static void mode_ij(int mode, int &i, int &j)
{
  int m = 0;
  for (int k = 0;; k++)
    for (int jj = 0; jj <= k; jj++, m++)
      if (m == mode)
      {
        j = jj;
        i = k - jj;
        return;
      }
}

static void collapse(double xi, double eta, double &a, double &b)
{
  a = (eta == 1.0) ? -1.0 : 2.0 * (1.0 + xi) / (1.0 - eta) - 1.0;
  b = eta;
}

double dubiner(int mode, double xi, double eta)
{
  int i, j;
  mode_ij(mode, i, j);
  double a, b;
  collapse(xi, eta, a, b);
  return std::sqrt(2.0) * jacobi_n(a, 0, 0, i) * jacobi_n(b, 2 * i + 1, 0, j) * std::pow(1.0 - b, i);
}

// d psi / d xi (dim 0) or d psi / d eta (dim 1), by the chain rule through
// (a, b): da/dxi = 2/(1-b), da/deta = (1+a)/(1-b)
double dubiner_d(int mode, double xi, double eta, int dim)
{
  int i, j;
  mode_ij(mode, i, j);
  double a, b;
  collapse(xi, eta, a, b);
  const double fa = jacobi_n(a, 0, 0, i), dfa = djacobi_n(a, 0, 0, i);
  const double gb = jacobi_n(b, 2 * i + 1, 0, j), dgb = djacobi_n(b, 2 * i + 1, 0, j);
  const double s2 = std::sqrt(2.0);
  if (dim == 0) return (i == 0) ? 0.0 : 2.0 * s2 * dfa * gb * std::pow(1.0 - b, i - 1);
  // eta derivative, grouped as the reference's dDubiner2D groups it
  const double j3 = dgb * std::pow(1.0 - b, i);
  if (i == 0) return s2 * fa * j3;
  const double j4 = gb * i * std::pow(1.0 - b, i - 1);
  return s2 * (dfa * gb * std::pow(1.0 - b, i - 1) * (1.0 + a) + fa * (j3 - j4));
}

// Gauss-Jordan inverse with partial pivoting of an n x n row-major matrix.
static std::vector<double> invert(std::vector<double> A, int n)
{
  std::vector<double> I((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) I[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; c++)
  {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
    if (A[(size_t)piv * n + c] == 0.0) ZB_THROW(ZB_ERR_INTERNAL, "singular Vandermonde matrix");
    if (piv != c)
      for (int k = 0; k < n; k++)
      {
        std::swap(A[(size_t)piv * n + k], A[(size_t)c * n + k]);
        std::swap(I[(size_t)piv * n + k], I[(size_t)c * n + k]);
      }
    const double d = A[(size_t)c * n + c];
    for (int k = 0; k < n; k++)
    {
      A[(size_t)c * n + k] /= d;
      I[(size_t)c * n + k] /= d;
    }
    for (int r = 0; r < n; r++)
    {
      if (r == c) continue;
      const double f = A[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++)
      {
        A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
        I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
      }
    }
  }
  return I;
}

// ---------------------------------------------------------------------------
// Point tables and dense FR operators of a triangle of order P
// ---------------------------------------------------------------------------
void tri_tables(Plan &p)
{
  const int P = p.order, N = p.N, S = p.nspts, Fp = p.nfpts, D = 2;
  ws_points(P, p.loc_spts, p.weights_spts);
  if ((int)p.weights_spts.size() != S) ZB_THROW(ZB_ERR_INTERNAL, "triangle point count");
  const std::vector<double> x = gauss_legendre_points(N), w1 = gauss_legendre_weights(N);
  p.ops.x = x;
  p.ops.w = w1;
  // flux points: bottom (x_j, -1), hypotenuse (x_{N-1-j}, x_j), left (-1, x_{N-1-j})
  p.loc_fpts.assign((size_t)Fp * 2, 0.0);
  p.tnorm.assign((size_t)Fp * 2, 0.0);
  const double h = std::sqrt(2.0) / 2;
  for (int face = 0; face < 3; face++)
    for (int j = 0; j < N; j++)
    {
      const int f = face * N + j;
      double lx, ly, nx, ny;
      if (face == 0) { lx = x[j]; ly = -1.0; nx = 0.0; ny = -1.0; }
      else if (face == 1) { lx = x[N - j - 1]; ly = x[j]; nx = h; ny = h; }
      else { lx = -1.0; ly = x[N - j - 1]; nx = -1.0; ny = 0.0; }
      p.loc_fpts[f * 2] = lx;
      p.loc_fpts[f * 2 + 1] = ly;
      p.tnorm[f * 2] = nx;
      p.tnorm[f * 2 + 1] = ny;
    }
  // Vandermonde of the orthonormal basis at the solution points
  std::vector<double> vand((size_t)S * S);
  for (int i = 0; i < S; i++)
    for (int j = 0; j < S; j++) vand[(size_t)i * S + j] = dubiner(j, p.loc_spts[i * 2], p.loc_spts[i * 2 + 1]);
  const std::vector<double> iv = invert(vand, S);
  // M0: nodal basis at flux points; M4: its derivative at solution points
  std::vector<double> &E = p.tri_oppE, &Dd = p.tri_oppD, &Df = p.tri_oppD_fpts, &Dv = p.tri_oppDiv,
                      &Dvf = p.tri_oppDiv_fpts;
  E.assign((size_t)Fp * S, 0.0);
  Dd.assign((size_t)D * S * S, 0.0);
  Df.assign((size_t)D * S * Fp, 0.0);
  Dv.assign((size_t)S * D * S, 0.0);
  Dvf.assign((size_t)S * Fp, 0.0);
  for (int s = 0; s < S; s++)
    for (int f = 0; f < Fp; f++)
    {
      double v = 0.0;
      for (int i = 0; i < S; i++) v += iv[(size_t)i * S + s] * dubiner(i, p.loc_fpts[f * 2], p.loc_fpts[f * 2 + 1]);
      E[(size_t)f * S + s] = v;
    }
  for (int d = 0; d < D; d++)
    for (int js = 0; js < S; js++)
      for (int is = 0; is < S; is++)
      {
        double v = 0.0;
        for (int i = 0; i < S; i++)
          v += iv[(size_t)i * S + js] * dubiner_d(i, p.loc_spts[is * 2], p.loc_spts[is * 2 + 1], d);
        Dd[((size_t)d * S + is) * S + js] = v;
      }
  // M1: the divergence of the flux at solution points is built for quads and
  // hexes only in the reference (src/elements.cpp:609-623 sits inside the
  // quad/hex branch), so its triangle oppDiv holds -M3 M2 alone.  The
  // reference form reproduces that; tri_volume_div = 1 adds M1 (textbook FR).
  if (p.params.tri_volume_div)
    for (int s = 0; s < S; s++)
      for (int d = 0; d < D; d++)
        for (int t = 0; t < S; t++) Dv[((size_t)s * D + d) * S + t] = Dd[((size_t)d * S + s) * S + t];
  // gbasis(mode, face pt) = w_k psi_mode(face point k): Gauss-Legendre
  // quadrature of the face Lagrange basis at its own nodes
  std::vector<double> gb((size_t)S * Fp, 0.0);
  for (int face = 0; face < 3; face++)
    for (int k = 0; k < N; k++)
    {
      const double q = x[k];
      double px, py;
      if (face == 0) { px = q; py = -1.0; }
      else if (face == 1) { px = -q; py = q; }
      else { px = -1.0; py = -q; }
      for (int m = 0; m < S; m++) gb[(size_t)m * Fp + face * N + k] = w1[k] * dubiner(m, px, py);
    }
  // M3 = vand gbasis (PyFR's correction operator)
  for (int i = 0; i < S; i++)
    for (int f = 0; f < Fp; f++)
    {
      double v = 0.0;
      for (int m = 0; m < S; m++) v += vand[(size_t)i * S + m] * gb[(size_t)m * Fp + f];
      Dvf[(size_t)i * Fp + f] = v;
    }
  // oppDiv -= M3 M2 with M2(f, d, t) = tnorm(f, d) oppE(f, t)
  for (int s = 0; s < S; s++)
    for (int dt = 0; dt < D * S; dt++)
    {
      const int d = dt / S, t = dt % S;
      double v = 0.0;
      for (int f = 0; f < Fp; f++) v += Dvf[(size_t)s * Fp + f] * (p.tnorm[f * 2 + d] * E[(size_t)f * S + t]);
      Dv[(size_t)s * D * S + dt] = -1.0 * v + Dv[(size_t)s * D * S + dt];
    }
  // gradient correction M6 = M3 tnorm, and oppD = M4 - M6 M0
  for (int d = 0; d < D; d++)
    for (int f = 0; f < Fp; f++)
      for (int s = 0; s < S; s++) Df[((size_t)d * S + s) * Fp + f] = Dvf[(size_t)s * Fp + f] * p.tnorm[f * 2 + d];
  for (int ds = 0; ds < D * S; ds++)
    for (int t = 0; t < S; t++)
    {
      double v = 0.0;
      for (int f = 0; f < Fp; f++) v += Df[(size_t)ds * Fp + f] * E[(size_t)f * S + t];
      Dd[(size_t)ds * S + t] = -1.0 * v + Dd[(size_t)ds * S + t];
    }
}

// Nodal shape functions of the linear (3-node) and quadratic (6-node)
// triangle at a reference point, in gmsh node order (src/tris.cpp:495-590):
// the Lagrange basis through the equispaced nodes, listed row by row
// (j fastest), mapped to gmsh order {0,1,2} / {0,3,1,5,4,2}.
void tri_shape(int nn, const double *loc, double *val, double *dval /* [2][nn] */)
{
  int order;
  std::vector<int> g;
  if (nn == 3) { order = 1; g = {0, 1, 2}; }
  else if (nn == 6) { order = 2; g = {0, 3, 1, 5, 4, 2}; }
  else ZB_THROW(ZB_ERR_UNSUPPORTED, "triangle with " + std::to_string(nn) + " nodes");
  std::vector<double> pts;
  for (int i = 0; i <= order; i++)
    for (int j = 0; j <= order - i; j++)
    {
      pts.push_back(-1.0 + 2.0 * j / order);
      pts.push_back(-1.0 + 2.0 * i / order);
    }
  std::vector<double> V((size_t)nn * nn);
  for (int i = 0; i < nn; i++)
    for (int j = 0; j < nn; j++) V[(size_t)i * nn + j] = dubiner(j, pts[i * 2], pts[i * 2 + 1]);
  const std::vector<double> iv = invert(V, nn);
  for (int nd = 0; nd < nn; nd++)
  {
    double v = 0.0, d0 = 0.0, d1 = 0.0;
    for (int i = 0; i < nn; i++)
    {
      v += iv[(size_t)i * nn + nd] * dubiner(i, loc[0], loc[1]);
      d0 += iv[(size_t)i * nn + nd] * dubiner_d(i, loc[0], loc[1], 0);
      d1 += iv[(size_t)i * nn + nd] * dubiner_d(i, loc[0], loc[1], 1);
    }
    val[g[nd]] = v;
    dval[g[nd]] = d0;
    dval[nn + g[nd]] = d1;
  }
}

}  // namespace zb
