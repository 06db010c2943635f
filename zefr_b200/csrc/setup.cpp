// Host-side set-up of the DFR residual: line operators, point tables, element
// metrics and face connectivity, reproducing the reference's orderings.
//
// Reference sources followed (paths inside the reference project):
//   polynomials        include/polynomials.hpp:16-76
//   DFR operators      src/elements.cpp:555-655, src/quads.cpp:239-361, src/hexas.cpp:385-475
//   point orderings    src/quads.cpp:47-158, src/hexas.cpp:52-240
//   shape functions    src/quads.cpp:500-560, src/hexas.cpp:749-834, src/funcs.cpp:1007-1200
//   metrics / normals  src/elements.cpp:325-407, 845-996
//   connectivity       src/geometry.cpp:202-300 (face node lists), 1159-1255 (periodic
//                      pairing), 1257-1744 (global flux points), src/solver.cpp:312-437
//                      (flux point orientation)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>

#include "zb_internal.hpp"

namespace zb {

// ---------------------------------------------------------------------------
// Polynomials
// ---------------------------------------------------------------------------

double lagrange(const std::vector<double> &g, int mode, double x)
{
  double val = 1.0;
  const int n = (int)g.size();
  for (int i = 0; i < mode; i++) val *= (x - g[i]) / (g[mode] - g[i]);
  for (int i = mode + 1; i < n; i++) val *= (x - g[i]) / (g[mode] - g[i]);
  return val;
}

double lagrange_d1(const std::vector<double> &g, int mode, double x)
{
  const int n = (int)g.size();
  double den = 1.0;
  for (int i = 0; i < mode; i++) den *= (g[mode] - g[i]);
  for (int i = mode + 1; i < n; i++) den *= (g[mode] - g[i]);
  double val = 0.0;
  for (int j = 0; j < n; j++)
  {
    if (j == mode) continue;
    double term = 1.0;
    for (int i = 0; i < n; i++)
      if (i != mode && i != j) term *= (x - g[i]);
    val += term;
  }
  return val / den;
}

// Gauss-Legendre nodes by Newton iteration on P_n (three-term recurrence),
// symmetrised so x[n-1-i] == -x[i] and the middle node of odd n is 0.
static void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w)
{
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; i++)
  {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 200; it++)
    {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++)
      {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = (n == 1) ? 1.0 : n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-17) break;
    }
    {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++)
      {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = (n == 1) ? 1.0 : n * (z * p1 - p0) / (z * z - 1.0);
    }
    const double wi = 2.0 / ((1.0 - z * z) * dp * dp);
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = wi;
    w[n - 1 - i] = wi;
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
  // Closed forms of the nodes for n <= 5 (the textbook expressions; the
  // reference evaluates the same ones, src/points.cpp:9-60), so the operators
  // built from them agree with the reference bit for bit.
  if (n == 2)
  {
    x[0] = -std::sqrt(1. / 3.);
    x[1] = std::sqrt(1. / 3.);
  }
  else if (n == 3)
  {
    x[0] = -std::sqrt(3. / 5.);
    x[2] = std::sqrt(3. / 5.);
  }
  else if (n == 4)
  {
    x[0] = -std::sqrt((3. + 2. * std::sqrt(6. / 5.)) / 7.);
    x[1] = -std::sqrt((3. - 2. * std::sqrt(6. / 5.)) / 7.);
    x[2] = std::sqrt((3. - 2. * std::sqrt(6. / 5.)) / 7.);
    x[3] = std::sqrt((3. + 2. * std::sqrt(6. / 5.)) / 7.);
  }
  else if (n == 5)
  {
    x[0] = -(1. / 3.) * std::sqrt(5. + 2. * std::sqrt(10. / 7.));
    x[1] = -(1. / 3.) * std::sqrt(5. - 2. * std::sqrt(10. / 7.));
    x[3] = (1. / 3.) * std::sqrt(5. - 2. * std::sqrt(10. / 7.));
    x[4] = (1. / 3.) * std::sqrt(5. + 2. * std::sqrt(10. / 7.));
  }
}

std::vector<double> gauss_legendre_points(int n)
{
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  return x;
}

std::vector<double> gauss_legendre_weights(int n)
{
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  return w;
}

LineOps make_line_ops(int N)
{
  LineOps o;
  o.N = N;
  gauss_legendre(N, o.x, o.w);
  std::vector<double> ext;
  ext.push_back(-1.0);
  for (double v : o.x) ext.push_back(v);
  ext.push_back(1.0);
  o.Em.resize(N);
  o.Ep.resize(N);
  o.D.resize(N * N);
  o.Dbm.resize(N);
  o.Dbp.resize(N);
  for (int m = 0; m < N; m++)
  {
    o.Em[m] = lagrange(o.x, m, -1.0);
    o.Ep[m] = lagrange(o.x, m, 1.0);
  }
  for (int i = 0; i < N; i++)
  {
    for (int m = 0; m < N; m++) o.D[i * N + m] = lagrange_d1(ext, m + 1, o.x[i]);
    o.Dbm[i] = lagrange_d1(ext, 0, o.x[i]);
    o.Dbp[i] = lagrange_d1(ext, N + 1, o.x[i]);
  }
  return o;
}

// ---------------------------------------------------------------------------
// Point tables
// ---------------------------------------------------------------------------

static void quad_tables(Plan &p)
{
  const int N = p.N;
  const auto &x = p.ops.x;
  p.loc_spts.assign(p.nspts * 2, 0.0);
  p.spt_idx.assign(p.nspts * 2, 0);
  p.weights_spts.assign(p.nspts, 0.0);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++)
    {
      int s = j + N * i;
      p.loc_spts[s * 2 + 0] = x[j];
      p.loc_spts[s * 2 + 1] = x[i];
      p.spt_idx[s * 2 + 0] = j;
      p.spt_idx[s * 2 + 1] = i;
      p.weights_spts[s] = p.ops.w[i] * p.ops.w[j];
    }
  p.loc_fpts.assign(p.nfpts * 2, 0.0);
  p.tnorm.assign(p.nfpts * 2, 0.0);
  p.fpt_dim.assign(p.nfpts, 0);
  p.fpt_side.assign(p.nfpts, 0);
  p.fpt_base.assign(p.nfpts, 0);
  p.fpt_stride.assign(p.nfpts, 0);
  for (int face = 0; face < 4; face++)
    for (int j = 0; j < N; j++)
    {
      int f = face * N + j;
      double lx = 0, ly = 0;
      int dim = 0, side = 0, base = 0, stride = 0;
      switch (face)
      {
        case 0: lx = x[j]; ly = -1.0; dim = 1; side = -1; base = j; stride = N; break;
        case 1: lx = 1.0; ly = x[j]; dim = 0; side = 1; base = N * j; stride = 1; break;
        case 2: lx = x[N - 1 - j]; ly = 1.0; dim = 1; side = 1; base = N - 1 - j; stride = N; break;
        default: lx = -1.0; ly = x[N - 1 - j]; dim = 0; side = -1; base = N * (N - 1 - j); stride = 1; break;
      }
      p.loc_fpts[f * 2 + 0] = lx;
      p.loc_fpts[f * 2 + 1] = ly;
      p.tnorm[f * 2 + dim] = (double)side;
      p.fpt_dim[f] = dim;
      p.fpt_side[f] = side;
      p.fpt_base[f] = base;
      p.fpt_stride[f] = stride;
    }
  p.spt_fm.assign(2 * p.nspts, 0);
  p.spt_fp.assign(2 * p.nspts, 0);
  for (int s = 0; s < p.nspts; s++)
  {
    int ix = p.spt_idx[s * 2], iy = p.spt_idx[s * 2 + 1];
    p.spt_fm[0 * p.nspts + s] = 3 * N + (N - 1 - iy);
    p.spt_fp[0 * p.nspts + s] = 1 * N + iy;
    p.spt_fm[1 * p.nspts + s] = ix;
    p.spt_fp[1 * p.nspts + s] = 2 * N + (N - 1 - ix);
  }
}

static void hex_tables(Plan &p)
{
  const int N = p.N, N2 = N * N;
  const auto &x = p.ops.x;
  p.loc_spts.assign(p.nspts * 3, 0.0);
  p.spt_idx.assign(p.nspts * 3, 0);
  p.weights_spts.assign(p.nspts, 0.0);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++)
      for (int k = 0; k < N; k++)
      {
        int s = k + N * (j + N * i);
        p.loc_spts[s * 3 + 0] = x[k];
        p.loc_spts[s * 3 + 1] = x[j];
        p.loc_spts[s * 3 + 2] = x[i];
        p.spt_idx[s * 3 + 0] = k;
        p.spt_idx[s * 3 + 1] = j;
        p.spt_idx[s * 3 + 2] = i;
        p.weights_spts[s] = p.ops.w[i] * p.ops.w[j] * p.ops.w[k];
      }
  p.loc_fpts.assign(p.nfpts * 3, 0.0);
  p.tnorm.assign(p.nfpts * 3, 0.0);
  p.fpt_dim.assign(p.nfpts, 0);
  p.fpt_side.assign(p.nfpts, 0);
  p.fpt_base.assign(p.nfpts, 0);
  p.fpt_stride.assign(p.nfpts, 0);
  for (int face = 0; face < 6; face++)
    for (int j = 0; j < N; j++)
      for (int k = 0; k < N; k++)
      {
        int f = face * N2 + j * N + k;
        int ix = 0, iy = 0, iz = 0;  // line coordinates (the normal one unused)
        double l[3] = {0, 0, 0};
        int dim = 0, side = 0;
        switch (face)
        {
          case 0: ix = k; iy = j; dim = 2; side = -1; l[0] = x[k]; l[1] = x[j]; l[2] = -1; break;
          case 1: ix = N - 1 - k; iy = j; dim = 2; side = 1; l[0] = x[N - 1 - k]; l[1] = x[j]; l[2] = 1; break;
          case 2: iy = k; iz = j; dim = 0; side = -1; l[0] = -1; l[1] = x[k]; l[2] = x[j]; break;
          case 3: iy = N - 1 - k; iz = j; dim = 0; side = 1; l[0] = 1; l[1] = x[N - 1 - k]; l[2] = x[j]; break;
          case 4: ix = N - 1 - k; iz = j; dim = 1; side = -1; l[0] = x[N - 1 - k]; l[1] = -1; l[2] = x[j]; break;
          default: ix = k; iz = j; dim = 1; side = 1; l[0] = x[k]; l[1] = 1; l[2] = x[j]; break;
        }
        for (int d = 0; d < 3; d++) p.loc_fpts[f * 3 + d] = l[d];
        p.tnorm[f * 3 + dim] = (double)side;
        p.fpt_dim[f] = dim;
        p.fpt_side[f] = side;
        const int strides[3] = {1, N, N2};
        int c[3] = {ix, iy, iz};
        c[dim] = 0;
        p.fpt_base[f] = c[0] + N * c[1] + N2 * c[2];
        p.fpt_stride[f] = strides[dim];
      }
  p.spt_fm.assign(3 * p.nspts, 0);
  p.spt_fp.assign(3 * p.nspts, 0);
  for (int s = 0; s < p.nspts; s++)
  {
    int ix = p.spt_idx[s * 3], iy = p.spt_idx[s * 3 + 1], iz = p.spt_idx[s * 3 + 2];
    p.spt_fm[0 * p.nspts + s] = 2 * N2 + iz * N + iy;
    p.spt_fp[0 * p.nspts + s] = 3 * N2 + iz * N + (N - 1 - iy);
    p.spt_fm[1 * p.nspts + s] = 4 * N2 + iz * N + (N - 1 - ix);
    p.spt_fp[1 * p.nspts + s] = 5 * N2 + iz * N + ix;
    p.spt_fm[2 * p.nspts + s] = iy * N + ix;
    p.spt_fp[2 * p.nspts + s] = N2 + iy * N + (N - 1 - ix);
  }
}

// ---------------------------------------------------------------------------
// Shape functions: Lagrange on equispaced nodes in gmsh node order
// ---------------------------------------------------------------------------

// gmsh node -> structured (i + nSide*j [+ nSide^2*k]) index
static std::vector<int> gmsh_to_structured(int gmsh_type)
{
  switch (gmsh_type)
  {
    case 3: return {0, 1, 3, 2};
    case 10: return {0, 2, 8, 6, 1, 5, 7, 3, 4};
    case 5: return {0, 1, 3, 2, 4, 5, 7, 6};
    default: ZB_THROW(ZB_ERR_UNSUPPORTED, "shape functions not built for gmsh type " + std::to_string(gmsh_type));
  }
}

struct Shape
{
  int nn = 0, D = 0;
  std::vector<double> val;   // [pts][nn]
  std::vector<double> dval;  // [D][pts][nn]
};

static Shape tensor_shape(int gmsh_type, int D, const std::vector<double> &loc, int npts)
{
  auto g2s = gmsh_to_structured(gmsh_type);
  const int nn = (int)g2s.size();
  const int nSide = (D == 2) ? (int)std::lround(std::sqrt((double)nn)) : (int)std::lround(std::cbrt((double)nn));
  std::vector<double> xl(nSide);
  const double dxi = 2.0 / (nSide - 1);
  for (int i = 0; i < nSide; i++) xl[i] = -1.0 + i * dxi;
  Shape s;
  s.nn = nn;
  s.D = D;
  s.val.assign((size_t)npts * nn, 0.0);
  s.dval.assign((size_t)D * npts * nn, 0.0);
  for (int pt = 0; pt < npts; pt++)
  {
    const double *l = &loc[(size_t)pt * D];
    for (int g = 0; g < nn; g++)
    {
      int st = g2s[g];
      int i = st % nSide, j = (st / nSide) % nSide, k = st / (nSide * nSide);
      if (D == 2)
      {
        s.val[(size_t)pt * nn + g] = lagrange(xl, i, l[0]) * lagrange(xl, j, l[1]);
        s.dval[((size_t)0 * npts + pt) * nn + g] = lagrange_d1(xl, i, l[0]) * lagrange(xl, j, l[1]);
        s.dval[((size_t)1 * npts + pt) * nn + g] = lagrange(xl, i, l[0]) * lagrange_d1(xl, j, l[1]);
      }
      else
      {
        double li = lagrange(xl, i, l[0]), lj = lagrange(xl, j, l[1]), lk = lagrange(xl, k, l[2]);
        double di = lagrange_d1(xl, i, l[0]), dj = lagrange_d1(xl, j, l[1]), dk = lagrange_d1(xl, k, l[2]);
        s.val[(size_t)pt * nn + g] = li * lj * lk;
        s.dval[((size_t)0 * npts + pt) * nn + g] = di * lj * lk;
        s.dval[((size_t)1 * npts + pt) * nn + g] = li * dj * lk;
        s.dval[((size_t)2 * npts + pt) * nn + g] = li * lj * dk;
      }
    }
  }
  return s;
}

// triangle shape functions at npts reference points (tri_setup.cpp)
static Shape simplex_shape(int nn, const std::vector<double> &loc, int npts)
{
  Shape s;
  s.nn = nn;
  s.D = 2;
  s.val.assign((size_t)npts * nn, 0.0);
  s.dval.assign((size_t)2 * npts * nn, 0.0);
  std::vector<double> v(nn), dv(2 * nn);
  for (int pt = 0; pt < npts; pt++)
  {
    tri_shape(nn, &loc[(size_t)pt * 2], v.data(), dv.data());
    for (int g = 0; g < nn; g++)
    {
      s.val[(size_t)pt * nn + g] = v[g];
      s.dval[((size_t)0 * npts + pt) * nn + g] = dv[g];
      s.dval[((size_t)1 * npts + pt) * nn + g] = dv[nn + g];
    }
  }
  return s;
}

// ---------------------------------------------------------------------------
// Metrics
// ---------------------------------------------------------------------------

// jaco[d1][d2] at one point of one element; returns adjugate (reference
// inv_jaco layout inv[d1][d2]) and determinant (src/elements.cpp:964-996).
static void adjugate(int D, const double J[3][3], double inv[3][3], double &det)
{
  if (D == 2)
  {
    det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    inv[0][0] = J[1][1];
    inv[0][1] = -J[1][0];
    inv[1][0] = -J[0][1];
    inv[1][1] = J[0][0];
  }
  else
  {
    const double xr = J[0][0], xs = J[1][0], xt = J[2][0];
    const double yr = J[0][1], ys = J[1][1], yt = J[2][1];
    const double zr = J[0][2], zs = J[1][2], zt = J[2][2];
    det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
    inv[0][0] = ys * zt - yt * zs; inv[0][1] = xt * zs - xs * zt; inv[0][2] = xs * yt - xt * ys;
    inv[1][0] = yt * zr - yr * zt; inv[1][1] = xr * zt - xt * zr; inv[1][2] = xt * yr - xr * yt;
    inv[2][0] = yr * zs - ys * zr; inv[2][1] = xs * zr - xr * zs; inv[2][2] = xr * ys - xs * yr;
  }
}

// ---------------------------------------------------------------------------
// Connectivity
// ---------------------------------------------------------------------------

// Corner-node lists of each element face (reference src/geometry.cpp:218-268).
static std::vector<std::vector<int>> face_corner_nodes(int etype)
{
  if (etype == ET_QUAD) return {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  if (etype == ET_TRI) return {{0, 1}, {1, 2}, {2, 0}};
  return {{0, 1, 2, 3}, {5, 4, 7, 6}, {0, 3, 7, 4}, {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};
}

typedef std::vector<int64_t> FaceKey;

struct FaceKeyHash
{
  size_t operator()(const FaceKey &k) const
  {
    uint64_t h = 1469598103934665603ull;
    for (int64_t v : k)
    {
      h ^= (uint64_t)v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    }
    return (size_t)h;
  }
};

void build_plan(const zb_mesh &mesh, const zb_params &params, Plan &p)
{
  if (mesh.ndims != 2 && mesh.ndims != 3) ZB_THROW(ZB_ERR_ARG, "ndims must be 2 or 3");
  if (params.order < 0 || params.order > 9) ZB_THROW(ZB_ERR_UNSUPPORTED, "order must be 0..9");
  if (mesh.n_eles <= 0 || mesh.coords == nullptr || mesh.ele2nodes == nullptr)
    ZB_THROW(ZB_ERR_ARG, "empty mesh");
  p.params = params;
  p.ndims = mesh.ndims;
  p.gmsh_type = mesh.gmsh_type;
  p.nnodes_ele = mesh.nodes_per_ele;
  if ((mesh.gmsh_type == 3 && mesh.nodes_per_ele == 4) || (mesh.gmsh_type == 10 && mesh.nodes_per_ele == 9))
    p.etype = ET_QUAD;
  else if (mesh.gmsh_type == 5 && mesh.nodes_per_ele == 8)
    p.etype = ET_HEX;
  else if ((mesh.gmsh_type == 2 && mesh.nodes_per_ele == 3) || (mesh.gmsh_type == 9 && mesh.nodes_per_ele == 6))
    p.etype = ET_TRI;
  else
    ZB_THROW(ZB_ERR_UNSUPPORTED, "element type not built: gmsh type " + std::to_string(mesh.gmsh_type));
  if ((p.etype != ET_HEX && p.ndims != 2) || (p.etype == ET_HEX && p.ndims != 3))
    ZB_THROW(ZB_ERR_MESH, "element type does not match ndims");

  const int D = p.ndims;
  p.order = params.order;
  p.N = params.order + 1;
  p.nvars = D + 2;
  p.neles = mesh.n_eles;
  p.tile = 8;
  p.ntiles = (p.neles + p.tile - 1) / p.tile;
  p.neles_pad = p.ntiles * p.tile;
  if (p.etype == ET_TRI)
  {
    // flux reconstruction on triangles (src/tris.cpp:24-43)
    p.nfaces = 3;
    p.nfpts_face = p.N;
    p.nspts = p.N * (p.N + 1) / 2;
    p.nfpts = 3 * p.N;
    p.ops.N = p.N;
    tri_tables(p);
  }
  else
  {
    p.nfaces = (D == 2) ? 4 : 6;
    p.nfpts_face = (D == 2) ? p.N : p.N * p.N;
    p.nspts = (D == 2) ? p.N * p.N : p.N * p.N * p.N;
    p.nfpts = p.nfaces * p.nfpts_face;
    p.ops = make_line_ops(p.N);
    if (D == 2)
      quad_tables(p);
    else
      hex_tables(p);
  }

  const int64_t E = p.neles;
  const int S = p.nspts, Fp = p.nfpts, nn = p.nnodes_ele;
  for (int64_t e = 0; e < E; e++)
    for (int n = 0; n < nn; n++)
    {
      int64_t g = mesh.ele2nodes[e * nn + n];
      if (g < 0 || g >= mesh.n_nodes) ZB_THROW(ZB_ERR_MESH, "element node id out of range");
    }

  // nodes(node, dim, ele)
  p.nodes.assign((size_t)nn * D * E, 0.0);
  for (int64_t e = 0; e < E; e++)
    for (int n = 0; n < nn; n++)
      for (int d = 0; d < D; d++)
        p.nodes[((size_t)n * D + d) * E + e] = mesh.coords[mesh.ele2nodes[e * nn + n] * 3 + d];

  Shape shs = (p.etype == ET_TRI) ? simplex_shape(nn, p.loc_spts, S) : tensor_shape(mesh.gmsh_type, D, p.loc_spts, S);
  Shape shf = (p.etype == ET_TRI) ? simplex_shape(nn, p.loc_fpts, Fp) : tensor_shape(mesh.gmsh_type, D, p.loc_fpts, Fp);

  p.dshape_spts = shs.dval;
  p.dshape_fpts = shf.dval;
  p.shape_fpts = shf.val;
  p.shape_spts = shs.val;
  p.coord_spts.assign((size_t)S * D * E, 0.0);
  p.coord_fpts.assign((size_t)Fp * D * E, 0.0);
  p.jaco_det_spts.assign((size_t)S * E, 0.0);
  p.inv_jaco_spts.assign((size_t)D * S * D * E, 0.0);
  std::vector<double> dA_own((size_t)Fp * E, 0.0);
  std::vector<double> unorm_own((size_t)Fp * D * E, 0.0);

  for (int64_t e = 0; e < E; e++)
  {
    for (int s = 0; s < S; s++)
    {
      for (int d = 0; d < D; d++)
      {
        double acc = 0.0;
        for (int n = 0; n < nn; n++) acc += shs.val[(size_t)s * nn + n] * p.nodes[((size_t)n * D + d) * E + e];
        p.coord_spts[((size_t)s * D + d) * E + e] = acc;
      }
      double J[3][3] = {{0}}, inv[3][3] = {{0}}, det = 0;
      for (int d1 = 0; d1 < D; d1++)
        for (int d2 = 0; d2 < D; d2++)
        {
          double acc = 0.0;
          for (int n = 0; n < nn; n++)
            acc += shs.dval[((size_t)d1 * S + s) * nn + n] * p.nodes[((size_t)n * D + d2) * E + e];
          J[d1][d2] = acc;
        }
      adjugate(D, J, inv, det);
      if (det < 0) ZB_THROW(ZB_ERR_MESH, "negative Jacobian at solution point of element " + std::to_string(e));
      p.jaco_det_spts[(size_t)s * E + e] = det;
      for (int d1 = 0; d1 < D; d1++)
        for (int d2 = 0; d2 < D; d2++) p.inv_jaco_spts[(((size_t)d1 * S + s) * D + d2) * E + e] = inv[d1][d2];
    }
    for (int f = 0; f < Fp; f++)
    {
      for (int d = 0; d < D; d++)
      {
        double acc = 0.0;
        for (int n = 0; n < nn; n++) acc += shf.val[(size_t)f * nn + n] * p.nodes[((size_t)n * D + d) * E + e];
        p.coord_fpts[((size_t)f * D + d) * E + e] = acc;
      }
      double J[3][3] = {{0}}, inv[3][3] = {{0}}, det = 0;
      for (int d1 = 0; d1 < D; d1++)
        for (int d2 = 0; d2 < D; d2++)
        {
          double acc = 0.0;
          for (int n = 0; n < nn; n++)
            acc += shf.dval[((size_t)d1 * Fp + f) * nn + n] * p.nodes[((size_t)n * D + d2) * E + e];
          J[d1][d2] = acc;
        }
      adjugate(D, J, inv, det);
      double nrm[3] = {0, 0, 0};
      for (int d1 = 0; d1 < D; d1++)
        for (int d2 = 0; d2 < D; d2++) nrm[d1] += inv[d2][d1] * p.tnorm[f * D + d2];
      double a = 0.0;
      for (int d = 0; d < D; d++) a += nrm[d] * nrm[d];
      a = std::sqrt(a);
      dA_own[(size_t)f * E + e] = a;
      for (int d = 0; d < D; d++) unorm_own[((size_t)f * D + d) * E + e] = nrm[d] / a;
    }
  }

  // ---- boundary faces ----
  const auto fcn = face_corner_nodes(p.etype);
  const int ncorner = (int)fcn[0].size();
  std::unordered_map<FaceKey, int, FaceKeyHash> bnd_bc;  // sorted corner nodes -> bc
  std::vector<FaceKey> bnd_keys;
  for (int64_t b = 0; b < mesh.n_bnd_faces; b++)
  {
    if (mesh.nodes_per_face < ncorner) ZB_THROW(ZB_ERR_MESH, "boundary face has too few nodes");
    FaceKey k(ncorner);
    for (int i = 0; i < ncorner; i++) k[i] = mesh.face_nodes[b * mesh.nodes_per_face + i];
    std::sort(k.begin(), k.end());
    int bc = mesh.face_bc[b];
    if (bc == ZB_BC_NONE) continue;
    if (!bnd_bc.count(k)) bnd_keys.push_back(k);
    bnd_bc[k] = bc;
  }

  // ---- periodic pairing: faces whose centroids agree in every dimension in
  // which the face is not planar (reference src/geometry.cpp:1159-1255) ----
  std::unordered_map<FaceKey, FaceKey, FaceKeyHash> per_pair;
  {
    const double tol = 1e-6;
    struct PF { FaceKey key; double c[3]; int planar_dim; };
    std::vector<PF> pfs;
    for (auto &k : bnd_keys)
    {
      if (bnd_bc[k] != ZB_BC_PERIODIC) continue;
      PF f;
      f.key = k;
      f.planar_dim = -1;
      for (int d = 0; d < D; d++)
      {
        double c = 0.0;
        for (int64_t n : k) c += mesh.coords[n * 3 + d];
        f.c[d] = c / (double)k.size();
        bool on_plane = true;
        for (int64_t n : k)
          if (std::fabs(mesh.coords[n * 3 + d] - mesh.coords[k[0] * 3 + d]) > tol) on_plane = false;
        if (on_plane && f.planar_dim < 0) f.planar_dim = d;
      }
      if (f.planar_dim < 0) ZB_THROW(ZB_ERR_MESH, "periodic face is not axis-aligned");
      pfs.push_back(f);
    }
    // bucket by (planar dim, quantised in-plane centroid)
    std::map<std::vector<int64_t>, std::vector<int>> buckets;
    auto qkey = [&](const PF &f, const int *shift) {
      std::vector<int64_t> q;
      q.push_back(f.planar_dim);
      int si = 0;
      for (int d = 0; d < D; d++)
        if (d != f.planar_dim) q.push_back((int64_t)std::floor(f.c[d] / (4 * tol)) + shift[si++]);
      return q;
    };
    const int zero[3] = {0, 0, 0};
    for (int i = 0; i < (int)pfs.size(); i++) buckets[qkey(pfs[i], zero)].push_back(i);
    for (int i = 0; i < (int)pfs.size(); i++)
    {
      const PF &f1 = pfs[i];
      const FaceKey *best = nullptr;
      int nsh = D - 1;
      int combos = 1;
      for (int q = 0; q < nsh; q++) combos *= 3;
      for (int c = 0; c < combos; c++)
      {
        int sh[3] = {0, 0, 0};
        int cc = c;
        for (int q = 0; q < nsh; q++) { sh[q] = cc % 3 - 1; cc /= 3; }
        auto it = buckets.find(qkey(f1, sh));
        if (it == buckets.end()) continue;
        for (int j : it->second)
        {
          if (j == i) continue;
          const PF &f2 = pfs[j];
          if (f2.key.size() != f1.key.size()) continue;
          bool match = true;
          for (int d = 0; d < D; d++)
            if (d != f1.planar_dim && std::fabs(f1.c[d] - f2.c[d]) >= tol) match = false;
          if (!match) continue;
          if (std::fabs(f1.c[f1.planar_dim] - f2.c[f1.planar_dim]) < tol) continue;  // same plane
          if (best == nullptr || f2.key < *best) best = &f2.key;
        }
      }
      if (best == nullptr) ZB_THROW(ZB_ERR_MESH, "Unpaired periodic face detected");
      per_pair[f1.key] = *best;
    }
  }

  // ---- faces in element order: first visitor is the left side
  // (reference src/geometry.cpp:1433-1640) ----
  p.partner.assign((size_t)Fp * E, 0);
  p.slot.assign((size_t)Fp * E, 0);
  p.fnorm.assign((size_t)Fp * D * E, 0.0);
  p.fdA.assign((size_t)Fp * E, 0.0);
  struct FaceRec { int64_t eL; int nL; int64_t eR; int nR; int bc; };
  std::unordered_map<FaceKey, int64_t, FaceKeyHash> face_id;
  std::vector<FaceRec> faces;
  faces.reserve((size_t)E * p.nfaces / 2 + 16);
  for (int64_t e = 0; e < E; e++)
    for (int n = 0; n < p.nfaces; n++)
    {
      FaceKey k(ncorner);
      for (int i = 0; i < ncorner; i++) k[i] = mesh.ele2nodes[e * nn + fcn[n][i]];
      std::sort(k.begin(), k.end());
      auto bit = bnd_bc.find(k);
      if (bit != bnd_bc.end() && bit->second == ZB_BC_PERIODIC)
      {
        auto pit = per_pair.find(k);
        if (pit != per_pair.end() && face_id.count(pit->second)) k = pit->second;
      }
      auto fit = face_id.find(k);
      if (fit == face_id.end())
      {
        FaceRec r{e, n, -1, -1, 0};
        auto b2 = bnd_bc.find(k);
        if (b2 != bnd_bc.end() && b2->second != ZB_BC_PERIODIC) r.bc = b2->second;
        face_id[k] = (int64_t)faces.size();
        faces.push_back(r);
      }
      else
      {
        FaceRec &r = faces[fit->second];
        if (r.eR >= 0 || r.bc != 0) ZB_THROW(ZB_ERR_MESH, "face shared by more than two elements");
        r.eR = e;
        r.nR = n;
      }
    }

  const int nf = p.nfpts_face;
  p.n_gfpts_int = 0;
  p.n_gfpts_bnd = 0;
  for (const FaceRec &r : faces)
  {
    if (r.eR < 0)
    {
      if (r.bc == 0) ZB_THROW(ZB_ERR_MESH, "unmatched interior face (missing boundary tag?)");
      p.n_gfpts_bnd += nf;
      for (int q = 0; q < nf; q++)
      {
        int f = r.nL * nf + q;
        size_t i = (size_t)f * E + r.eL;
        p.partner[i] = -1 - r.bc;
        p.slot[i] = 0;
        p.fdA[i] = dA_own[i];
        for (int d = 0; d < D; d++) p.fnorm[((size_t)f * D + d) * E + r.eL] = unorm_own[((size_t)f * D + d) * E + r.eL];
      }
      continue;
    }
    p.n_gfpts_int += nf;
    // pair flux points by position relative to each side's centroid (handles
    // the periodic translation); equivalent to the reference's fuzzy sort
    double cL[3] = {0, 0, 0}, cR[3] = {0, 0, 0};
    for (int q = 0; q < nf; q++)
      for (int d = 0; d < D; d++)
      {
        cL[d] += p.coord_fpts[((size_t)(r.nL * nf + q) * D + d) * E + r.eL] / nf;
        cR[d] += p.coord_fpts[((size_t)(r.nR * nf + q) * D + d) * E + r.eR] / nf;
      }
    double scale = 0.0;
    for (int q = 0; q < nf; q++)
      for (int d = 0; d < D; d++)
        scale = std::max(scale, std::fabs(p.coord_fpts[((size_t)(r.nL * nf + q) * D + d) * E + r.eL] - cL[d]));
    const double tol = std::max(1e-6, 1e-6 * scale);
    for (int q = 0; q < nf; q++)
    {
      int fL = r.nL * nf + q;
      int best = -1;
      double bestd = 1e300;
      for (int q2 = 0; q2 < nf; q2++)
      {
        int fR = r.nR * nf + q2;
        double dist = 0.0;
        for (int d = 0; d < D; d++)
        {
          double a = p.coord_fpts[((size_t)fL * D + d) * E + r.eL] - cL[d];
          double b = p.coord_fpts[((size_t)fR * D + d) * E + r.eR] - cR[d];
          dist = std::max(dist, std::fabs(a - b));
        }
        if (dist < bestd) { bestd = dist; best = fR; }
      }
      if (best < 0 || bestd > tol) ZB_THROW(ZB_ERR_MESH, "flux points of a face do not coincide");
      const int fR = best;
      size_t iL = (size_t)fL * E + r.eL, iR = (size_t)fR * E + r.eR;
      p.partner[iL] = r.eR * Fp + fR;
      p.partner[iR] = r.eL * Fp + fL;
      p.slot[iL] = 0;
      p.slot[iR] = 1;
      p.fdA[iL] = dA_own[iL];
      p.fdA[iR] = dA_own[iR];
      for (int d = 0; d < D; d++)
      {
        double nv = unorm_own[((size_t)fL * D + d) * E + r.eL];
        p.fnorm[((size_t)fL * D + d) * E + r.eL] = nv;
        p.fnorm[((size_t)fR * D + d) * E + r.eR] = nv;
      }
    }
  }
  for (int64_t e = 0; e < E; e++)
    for (int f = 0; f < Fp; f++)
    {
      int64_t pr = p.partner[(size_t)f * E + e];
      if (pr >= 0)
      {
        int64_t e2 = pr / Fp;
        int f2 = (int)(pr % Fp);
        if (p.partner[(size_t)f2 * E + e2] != e * Fp + f) ZB_THROW(ZB_ERR_INTERNAL, "asymmetric face pairing");
      }
    }
}

void Plan::dense_operators(std::vector<double> &oppE, std::vector<double> &oppD,
                           std::vector<double> &oppD_fpts, std::vector<double> &oppDiv,
                           std::vector<double> &oppDiv_fpts) const
{
  const int S = nspts, Fp = nfpts, D = ndims, Nn = N;
  if (etype == ET_TRI)
  {
    oppE = tri_oppE;
    oppD = tri_oppD;
    oppD_fpts = tri_oppD_fpts;
    oppDiv = tri_oppDiv;
    oppDiv_fpts = tri_oppDiv_fpts;
    return;
  }
  oppE.assign((size_t)Fp * S, 0.0);
  oppD.assign((size_t)D * S * S, 0.0);
  oppD_fpts.assign((size_t)D * S * Fp, 0.0);
  oppDiv.assign((size_t)S * D * S, 0.0);
  oppDiv_fpts.assign((size_t)S * Fp, 0.0);
  for (int f = 0; f < Fp; f++)
    for (int m = 0; m < Nn; m++)
    {
      int s = fpt_base[f] + m * fpt_stride[f];
      oppE[(size_t)f * S + s] = (fpt_side[f] < 0) ? ops.Em[m] : ops.Ep[m];
    }
  const int strides[3] = {1, Nn, Nn * Nn};
  for (int d = 0; d < D; d++)
    for (int s = 0; s < S; s++)
    {
      int i = spt_idx[s * D + d];
      int base = s - i * strides[d];
      for (int m = 0; m < Nn; m++)
      {
        int s2 = base + m * strides[d];
        oppD[((size_t)d * S + s) * S + s2] = ops.D[i * Nn + m];
        oppDiv[((size_t)s * D + d) * S + s2] = ops.D[i * Nn + m];
      }
      int fm = spt_fm[d * S + s], fp = spt_fp[d * S + s];
      oppD_fpts[((size_t)d * S + s) * Fp + fm] = ops.Dbm[i];
      oppD_fpts[((size_t)d * S + s) * Fp + fp] = ops.Dbp[i];
      oppDiv_fpts[(size_t)s * Fp + fm] += -ops.Dbm[i];
      oppDiv_fpts[(size_t)s * Fp + fp] += ops.Dbp[i];
    }
}

// ---------------------------------------------------------------------------
// Deck parameters (reference src/input.cpp:440-539)
// ---------------------------------------------------------------------------

void params_from_deck(const zb_deck &in, zb_params &out)
{
  std::memset(&out, 0, sizeof(out));
  out.order = in.order;
  out.viscous = in.viscous;
  out.fconv = in.fconv;
  out.precision = in.precision;
  out.gamma = in.gamma;
  out.prandtl = in.prandtl;
  out.rus_k = in.rus_k;
  out.ldg_b = in.ldg_b;
  out.ldg_tau = in.ldg_tau;
  out.dt = in.dt;
  out.fix_vis = in.fix_vis;
  double rho_fs = in.rho_fs, P_fs = in.P_fs, T_fs = in.T_fs, T_wall = in.T_wall, R = in.R;
  double v_mag_fs = in.mach_fs * std::sqrt(in.gamma * in.P_fs / in.rho_fs);
  double nfs[3] = {in.nx_fs, in.ny_fs, in.nz_fs};
  double mag = std::sqrt(nfs[0] * nfs[0] + nfs[1] * nfs[1] + nfs[2] * nfs[2]);
  for (int i = 0; i < 3; i++) nfs[i] /= mag;
  double nw[3] = {in.nx_wall, in.ny_wall, in.nz_wall};
  const int D = in.ndims;
  if (!in.viscous)
  {
    for (int i = 0; i < 3; i++) out.V_fs[i] = nfs[i] * v_mag_fs;
    out.rho_fs = rho_fs;
    out.P_fs = P_fs;
    out.T_wall = T_wall;
    return;
  }
  if (in.disable_nondim)
  {
    T_fs = P_fs / (rho_fs * R);
    out.mu = rho_fs * v_mag_fs * in.L_fs / in.Re_fs;
    out.R_ref = R;
    for (int d = 0; d < D; d++) out.V_fs[d] = v_mag_fs * nfs[d];
    double vw = in.mach_wall * std::sqrt(in.gamma * R * T_wall);
    for (int d = 0; d < D; d++) out.V_wall[d] = vw * nw[d] / v_mag_fs;
    out.fix_vis = 1;
    out.rho_fs = rho_fs;
    out.P_fs = P_fs;
    out.T_wall = T_wall;
    return;
  }
  double V_fs_mag = in.mach_fs * std::sqrt(in.gamma * R * T_fs);
  double V[3] = {0, 0, 0};
  for (int d = 0; d < D; d++) V[d] = V_fs_mag * nfs[d];
  double mu = (rho_fs * V_fs_mag * in.L_fs) / in.Re_fs;
  if (!in.fix_vis) mu = mu * std::pow(T_fs / in.T_gas, 1.5) * ((in.T_gas + in.S) / (T_fs + in.S));
  rho_fs = mu * in.Re_fs / (V_fs_mag * in.L_fs);
  P_fs = rho_fs * R * T_fs;
  out.rt = in.T_gas * R / (V_fs_mag * V_fs_mag);
  out.c_sth = in.S / in.T_gas;
  double rho_ref = rho_fs, P_ref = rho_fs * V_fs_mag * V_fs_mag, mu_ref = rho_fs * V_fs_mag;
  out.R_ref = R * T_fs / (V_fs_mag * V_fs_mag);
  out.mu = mu / mu_ref;
  out.rho_fs = rho_fs / rho_ref;
  for (int d = 0; d < D; d++) out.V_fs[d] = V[d] / V_fs_mag;
  out.P_fs = P_fs / P_ref;
  double vw = in.mach_wall * std::sqrt(in.gamma * R * T_wall);
  for (int d = 0; d < D; d++) out.V_wall[d] = vw * nw[d] / V_fs_mag;
  out.T_wall = T_wall / T_fs;
}

}  // namespace zb
