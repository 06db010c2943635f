// Element geometry as device functions of the element nodes.
//
// The set-up metrics the residual is built on -- adjugate and |J| at the
// solution points, unit normal and area factor at the flux points -- from
// node coordinates in the reference's nodes(node, dim, ele) layout: the
// set-up's calc_transforms and calc_normals (reference src/elements.cpp:
// 845-996; its GPU forms src/elements_kernels.cu:1649-1737 with
// inverse_transform_2d/3d and 1896-1950 with calc_normals).  Every product
// and sum is rounded once, in the set-up's order (build_plan, setup.cpp), so
// the device metrics equal the host set-up's bit for bit.
//
// The adjoint maps the metric adjoint that zb_vjp_geometry returns back to
// the element nodes (shape and wall-displacement gradients), and
// ctx_set_nodes moves a context's mesh in place: new metrics in both
// precision forms without a new plan.
//
// Threads run one per (point, element) with the element index fastest, so
// the node, metric and table reads of a warp are coalesced or broadcast; the
// node adjoint is gathered per (node, dim, element) in a fixed order
// (deterministic, no atomics).
#include "context.hpp"
#include "ctx_impl.cuh"

namespace zb {
namespace geo {

__device__ __forceinline__ double m_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double a_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double s_(double a, double b) { return __dsub_rn(a, b); }

// M[a][d] = sum_n dshape[a][p][n] * nodes[n][d][e] (reference direction a,
// physical direction d), summed in node order from zero
template <int D>
__device__ __forceinline__ void jacobian(const double *__restrict__ dsh, const double *__restrict__ nodes, int npts,
                                         int p, int nn, int64_t E, int64_t e, double M[D][D])
{
  for (int a = 0; a < D; a++)
    for (int d = 0; d < D; d++)
    {
      double acc = 0.0;
      for (int n = 0; n < nn; n++)
        acc = a_(acc, m_(__ldg(dsh + ((size_t)a * npts + p) * nn + n), nodes[((size_t)n * D + d) * E + e]));
      M[a][d] = acc;
    }
}

// Adjugate in the reference inv_jaco orientation (C[a][d] is the cofactor of
// M[a][d]) and the determinant, with the set-up's expressions
__device__ __forceinline__ void adjugate(const double M[2][2], double C[2][2], double &det)
{
  det = s_(m_(M[0][0], M[1][1]), m_(M[0][1], M[1][0]));
  C[0][0] = M[1][1];
  C[0][1] = -M[1][0];
  C[1][0] = -M[0][1];
  C[1][1] = M[0][0];
}

__device__ __forceinline__ void adjugate(const double M[3][3], double C[3][3], double &det)
{
  const double xr = M[0][0], xs = M[1][0], xt = M[2][0];
  const double yr = M[0][1], ys = M[1][1], yt = M[2][1];
  const double zr = M[0][2], zs = M[1][2], zt = M[2][2];
  det = a_(s_(m_(xr, s_(m_(ys, zt), m_(yt, zs))), m_(xs, s_(m_(yr, zt), m_(yt, zr)))),
           m_(xt, s_(m_(yr, zs), m_(ys, zr))));
  C[0][0] = s_(m_(ys, zt), m_(yt, zs));
  C[0][1] = s_(m_(xt, zs), m_(xs, zt));
  C[0][2] = s_(m_(xs, yt), m_(xt, ys));
  C[1][0] = s_(m_(yt, zr), m_(yr, zt));
  C[1][1] = s_(m_(xr, zt), m_(xt, zr));
  C[1][2] = s_(m_(xt, yr), m_(xr, yt));
  C[2][0] = s_(m_(yr, zs), m_(ys, zr));
  C[2][1] = s_(m_(xs, zr), m_(xr, zs));
  C[2][2] = s_(m_(xr, ys), m_(xs, yr));
}

// Reverse of the adjugate: Mb += (dC/dM)^T Cb.  Each 3D cofactor is
// C[i][k] = M[i1][k1] M[i2][k2] - M[i2][k1] M[i1][k2] (i1 = i+1, i2 = i+2,
// k1 = k+1, k2 = k+2 mod 3).
__device__ __forceinline__ void adjugate_vjp(const double M[2][2], const double Cb[2][2], double Mb[2][2])
{
  Mb[1][1] += Cb[0][0];
  Mb[1][0] -= Cb[0][1];
  Mb[0][1] -= Cb[1][0];
  Mb[0][0] += Cb[1][1];
}

__device__ __forceinline__ void adjugate_vjp(const double M[3][3], const double Cb[3][3], double Mb[3][3])
{
#pragma unroll
  for (int i = 0; i < 3; i++)
  {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
      const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
      const double g = Cb[i][k];
      Mb[i1][k1] += g * M[i2][k2];
      Mb[i2][k2] += g * M[i1][k1];
      Mb[i2][k1] -= g * M[i1][k2];
      Mb[i1][k2] -= g * M[i2][k1];
    }
  }
}

// Unnormalised outward normal nrm[d1] = sum_d2 C[d2][d1] tnorm[d2] and its length
template <int D>
__device__ __forceinline__ double face_normal(const double C[D][D], const double *__restrict__ tn, double nrm[D])
{
  for (int d1 = 0; d1 < D; d1++)
  {
    double acc = 0.0;
    for (int d2 = 0; d2 < D; d2++) acc = a_(acc, m_(C[d2][d1], __ldg(tn + d2)));
    nrm[d1] = acc;
  }
  double q = 0.0;
  for (int d = 0; d < D; d++) q = a_(q, m_(nrm[d], nrm[d]));
  return __dsqrt_rn(q);
}

struct Tabs
{
  const double *dss, *dsf, *ss, *sf, *tn;  // dshape_spts, dshape_fpts, shape_spts, shape_fpts, tnorm
};

// Forward metrics at every (point, element): solution points give inv_jaco
// [D][S][D][E] and jaco_det [S][E]; flux points the own unit normal
// [Fp][D][E] and dA [Fp][E].  Optional: coordinates of both point sets and a
// flag raised on a negative |J| at a solution point.
template <int D>
__global__ void k_geo_eval(const double *__restrict__ nodes, Tabs t, int S, int Fp, int nn, int64_t E,
                           double *__restrict__ inv, double *__restrict__ det, double *__restrict__ unorm,
                           double *__restrict__ dA, double *__restrict__ cspts, double *__restrict__ cfpts,
                           int *__restrict__ bad)
{
  const int64_t total = (int64_t)(S + Fp) * E;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int p = (int)(i / E);
    const int64_t e = i - (int64_t)p * E;
    double M[D][D], C[D][D], dt;
    if (p < S)
    {
      jacobian<D>(t.dss, nodes, S, p, nn, E, e, M);
      adjugate(M, C, dt);
      det[(size_t)p * E + e] = dt;
      if (bad && dt < 0.0) *bad = 1;
      for (int a = 0; a < D; a++)
        for (int d = 0; d < D; d++) inv[(((size_t)a * S + p) * D + d) * E + e] = C[a][d];
      if (cspts)
        for (int d = 0; d < D; d++)
        {
          double acc = 0.0;
          for (int n = 0; n < nn; n++) acc = a_(acc, m_(__ldg(t.ss + (size_t)p * nn + n), nodes[((size_t)n * D + d) * E + e]));
          cspts[((size_t)p * D + d) * E + e] = acc;
        }
    }
    else
    {
      const int f = p - S;
      jacobian<D>(t.dsf, nodes, Fp, f, nn, E, e, M);
      adjugate(M, C, dt);
      double nrm[D];
      const double a = face_normal<D>(C, t.tn + (size_t)f * D, nrm);
      dA[(size_t)f * E + e] = a;
      for (int d = 0; d < D; d++) unorm[((size_t)f * D + d) * E + e] = __ddiv_rn(nrm[d], a);
      if (cfpts)
        for (int d = 0; d < D; d++)
        {
          double acc = 0.0;
          for (int n = 0; n < nn; n++) acc = a_(acc, m_(__ldg(t.sf + (size_t)f * nn + n), nodes[((size_t)n * D + d) * E + e]));
          cfpts[((size_t)f * D + d) * E + e] = acc;
        }
    }
  }
}

// The face normal of both sides of an interior face is the left element's;
// boundary points keep their own.  right[f*E+e] is the left partner's
// (f', e') as f'*E+e' at a right-side point, else -1.
__global__ void k_geo_face_normals(const double *__restrict__ unorm, const int64_t *__restrict__ right,
                                   double *__restrict__ norm, int D, int Fp, int64_t E)
{
  const int64_t total = (int64_t)Fp * E;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int f = (int)(i / E);
    const int64_t e = i - (int64_t)f * E;
    const int64_t r = right[i];
    const int fs = r < 0 ? f : (int)(r / E);
    const int64_t es = r < 0 ? e : r - (int64_t)fs * E;
    for (int d = 0; d < D; d++) norm[((size_t)f * D + d) * E + e] = unorm[((size_t)fs * D + d) * E + es];
  }
}

// Reverse of k_geo_face_normals: the own normal's adjoint is the point's own
// weight (boundary and left-side points) plus, at a left-side point, its
// right partner's.  left[f*E+e] is the right partner as f'*E+e' at a
// left-side point, else -1.
__global__ void k_geo_face_normals_vjp(const double *__restrict__ norm_bar, const int64_t *__restrict__ right,
                                       const int64_t *__restrict__ left, double *__restrict__ unorm_bar, int D,
                                       int Fp, int64_t E)
{
  const int64_t total = (int64_t)Fp * E;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int f = (int)(i / E);
    const int64_t e = i - (int64_t)f * E;
    const bool own = right[i] < 0;
    const int64_t l = left[i];
    const int fr = l < 0 ? 0 : (int)(l / E);
    const int64_t er = l < 0 ? 0 : l - (int64_t)fr * E;
    for (int d = 0; d < D; d++)
    {
      double g = (own && norm_bar) ? norm_bar[((size_t)f * D + d) * E + e] : 0.0;
      if (l >= 0 && norm_bar) g += norm_bar[((size_t)fr * D + d) * E + er];
      unorm_bar[((size_t)f * D + d) * E + e] = g;
    }
  }
}

// Jacobian adjoint Jb [D][S+Fp][D][E] (solution points, then flux points)
// from the metric adjoints; null adjoints count as zero
template <int D>
__global__ void k_geo_points_vjp(const double *__restrict__ nodes, Tabs t, int S, int Fp, int nn, int64_t E,
                                 const double *__restrict__ inv_bar, const double *__restrict__ det_bar,
                                 const double *__restrict__ unorm_bar, const double *__restrict__ dA_bar,
                                 double *__restrict__ Jb)
{
  const int P = S + Fp;
  const int64_t total = (int64_t)P * E;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int p = (int)(i / E);
    const int64_t e = i - (int64_t)p * E;
    double M[D][D], C[D][D], Cb[D][D], Mb[D][D], dt;
    for (int a = 0; a < D; a++)
      for (int d = 0; d < D; d++) Mb[a][d] = 0.0;
    if (p < S)
    {
      jacobian<D>(t.dss, nodes, S, p, nn, E, e, M);
      adjugate(M, C, dt);
      const double db = det_bar ? det_bar[(size_t)p * E + e] : 0.0;
      for (int a = 0; a < D; a++)
        for (int d = 0; d < D; d++)
        {
          Cb[a][d] = inv_bar ? inv_bar[(((size_t)a * S + p) * D + d) * E + e] : 0.0;
          Mb[a][d] = db * C[a][d];  // d det / d M = cofactor
        }
    }
    else
    {
      const int f = p - S;
      jacobian<D>(t.dsf, nodes, Fp, f, nn, E, e, M);
      adjugate(M, C, dt);
      double nrm[D], u[D], ub[D];
      const double a = face_normal<D>(C, t.tn + (size_t)f * D, nrm);
      const double ab = dA_bar ? dA_bar[(size_t)f * E + e] : 0.0;
      double udot = 0.0;
      for (int d = 0; d < D; d++)
      {
        u[d] = nrm[d] / a;
        ub[d] = unorm_bar[((size_t)f * D + d) * E + e];
        udot += ub[d] * u[d];
      }
      // u = nrm/|nrm|, dA = |nrm|: nrm_bar = (ub - (ub.u) u)/|nrm| + dA_bar u
      double nb[D];
      for (int d = 0; d < D; d++) nb[d] = (ub[d] - udot * u[d]) / a + ab * u[d];
      for (int d2 = 0; d2 < D; d2++)
        for (int d1 = 0; d1 < D; d1++) Cb[d2][d1] = nb[d1] * __ldg(t.tn + (size_t)f * D + d2);
    }
    adjugate_vjp(M, Cb, Mb);
    for (int a = 0; a < D; a++)
      for (int d = 0; d < D; d++) Jb[(((size_t)a * P + p) * D + d) * E + e] = Mb[a][d];
  }
}

// Node adjoint nodes_bar[n][d][e] = sum_a sum_p dshape[a][p][n] Jb[a][p][d][e]
// over the solution points, then the flux points, in a fixed order
template <int D>
__global__ void k_geo_nodes_vjp(const double *__restrict__ Jb, Tabs t, int S, int Fp, int nn, int64_t E,
                                double *__restrict__ nodes_bar)
{
  const int P = S + Fp;
  const int64_t total = (int64_t)nn * D * E;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int nd = (int)(i / E);
    const int64_t e = i - (int64_t)nd * E;
    const int n = nd / D, d = nd % D;
    double acc = 0.0;
    for (int a = 0; a < D; a++)
    {
      for (int p = 0; p < S; p++)
        acc += __ldg(t.dss + ((size_t)a * S + p) * nn + n) * Jb[(((size_t)a * P + p) * D + d) * E + e];
      for (int f = 0; f < Fp; f++)
        acc += __ldg(t.dsf + ((size_t)a * Fp + f) * nn + n) * Jb[(((size_t)a * P + S + f) * D + d) * E + e];
    }
    nodes_bar[i] = acc;
  }
}

// Reference-layout metrics to the context's tile layout (as upload_static:
// padded lanes repeat element 0)
template <typename T>
__global__ void k_geo_tiles(const double *__restrict__ inv, const double *__restrict__ det,
                            const double *__restrict__ norm, const double *__restrict__ dA, T *__restrict__ mets,
                            T *__restrict__ fgeo, int64_t ntiles, int64_t E, int S, int Fp, int D)
{
  const int NM = D * D + 1;
  const int64_t nm = ntiles * S * NM * TW, nf = ntiles * Fp * (D + 1) * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nm + nf; i += (int64_t)gridDim.x * blockDim.x)
  {
    if (i < nm)
    {
      const int l = (int)(i % TW);
      const int k = (int)((i / TW) % NM);
      const int64_t ts = i / ((int64_t)TW * NM);  // tile * S + s
      const int s = (int)(ts % S);
      const int64_t e = (ts / S) * TW + l;
      const int64_t es = e < E ? e : 0;
      double v;
      if (k < D * D)
        v = inv[(((size_t)(k / D) * S + s) * D + (k % D)) * E + es];
      else
        v = det[(size_t)s * E + es];
      mets[i] = (T)v;
    }
    else
    {
      const int64_t j = i - nm;
      const int l = (int)(j % TW);
      const int k = (int)((j / TW) % (D + 1));
      const int64_t tf = j / ((int64_t)TW * (D + 1));  // tile * Fp + f
      const int f = (int)(tf % Fp);
      const int64_t e = (tf / Fp) * TW + l;
      const int64_t es = e < E ? e : 0;
      const double v = k < D ? norm[((size_t)f * D + k) * E + es] : dA[(size_t)f * E + es];
      fgeo[j] = (T)v;
    }
  }
}

}  // namespace geo

namespace {

unsigned blocks_for(int64_t work)
{
  int64_t b = (work + 255) / 256;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 64 ? 148 * 64 : b));
}

void *galloc(size_t bytes)
{
  void *p = nullptr;
  const cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    ZB_THROW(ZB_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  return p;
}

// sizes of the reference-layout arrays
struct GeoSizes
{
  size_t nodes, inv, det, norm, dA, cs, cf, Jb;
  explicit GeoSizes(const Plan &p)
  {
    const size_t D = p.ndims, S = p.nspts, Fp = p.nfpts, E = p.neles, nn = p.nnodes_ele;
    nodes = nn * D * E;
    inv = D * S * D * E;
    det = S * E;
    norm = Fp * D * E;
    dA = Fp * E;
    cs = S * D * E;
    cf = Fp * D * E;
    Jb = D * (S + Fp) * D * E;
  }
};

// tables and face pairing on the device, allocated on first use
void ensure_tables(Ctx *c)
{
  if (c->geo_tab) return;
  const Plan &p = c->plan;
  if (p.dshape_spts.empty() || p.shape_spts.empty()) ZB_THROW(ZB_ERR_INTERNAL, "plan has no shape tables");
  std::vector<double> tab;
  tab.insert(tab.end(), p.dshape_spts.begin(), p.dshape_spts.end());
  tab.insert(tab.end(), p.dshape_fpts.begin(), p.dshape_fpts.end());
  tab.insert(tab.end(), p.shape_spts.begin(), p.shape_spts.end());
  tab.insert(tab.end(), p.shape_fpts.begin(), p.shape_fpts.end());
  tab.insert(tab.end(), p.tnorm.begin(), p.tnorm.end());
  const int64_t E = p.neles, Fp = p.nfpts;
  std::vector<int64_t> pair((size_t)2 * Fp * E, -1);
  for (int64_t f = 0; f < Fp; f++)
    for (int64_t e = 0; e < E; e++)
    {
      const size_t i = (size_t)f * E + e;
      const int64_t pr = p.partner[i];
      if (pr < 0) continue;
      const int64_t q = (pr % Fp) * E + pr / Fp;  // partner as f'*E+e'
      if (p.slot[i] == 1)
        pair[i] = q;  // right side: normal from the left partner
      else
        pair[(size_t)Fp * E + i] = q;  // left side: the right partner's normal weight comes here
    }
  double *t = (double *)galloc(tab.size() * sizeof(double));
  int64_t *pp = (int64_t *)galloc(pair.size() * sizeof(int64_t));
  CK(cudaMemcpyAsync(t, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(pp, pair.data(), pair.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->geo_tab = t;
  c->geo_pair = pp;
}

geo::Tabs tables(const Ctx *c)
{
  const Plan &p = c->plan;
  const size_t D = p.ndims, S = p.nspts, Fp = p.nfpts, nn = p.nnodes_ele;
  geo::Tabs t;
  t.dss = c->geo_tab;
  t.dsf = t.dss + D * S * nn;
  t.ss = t.dsf + D * Fp * nn;
  t.sf = t.ss + S * nn;
  t.tn = t.sf + Fp * nn;
  return t;
}

double *scratch(Ctx *c, size_t doubles)
{
  const size_t bytes = doubles * sizeof(double);
  if (bytes > c->geo_work_bytes)
  {
    // earlier geometry work queued on the stream may still read the old buffer
    CK(cudaStreamSynchronize(c->stream));
    if (c->geo_work) cudaFree(c->geo_work);
    c->geo_work = nullptr;
    c->geo_work_bytes = 0;
    c->geo_work = (double *)galloc(bytes);
    c->geo_work_bytes = bytes;
  }
  return c->geo_work;
}

// forward metrics into device arrays (reference layouts); unorm is scratch
void eval_device(Ctx *c, const double *nodes, double *inv, double *det, double *norm, double *dA, double *unorm,
                 double *cs, double *cf, int *bad)
{
  const Plan &p = c->plan;
  const int S = p.nspts, Fp = p.nfpts, nn = p.nnodes_ele, D = p.ndims;
  const int64_t E = p.neles;
  const geo::Tabs t = tables(c);
  const unsigned g1 = blocks_for((int64_t)(S + Fp) * E), g2 = blocks_for((int64_t)Fp * E);
  if (D == 2)
    geo::k_geo_eval<2><<<g1, 256, 0, c->stream>>>(nodes, t, S, Fp, nn, E, inv, det, unorm, dA, cs, cf, bad);
  else
    geo::k_geo_eval<3><<<g1, 256, 0, c->stream>>>(nodes, t, S, Fp, nn, E, inv, det, unorm, dA, cs, cf, bad);
  geo::k_geo_face_normals<<<g2, 256, 0, c->stream>>>(unorm, c->geo_pair, norm, D, Fp, E);
  c->launches += 2;
  CK(cudaGetLastError());
}

}  // namespace

void ctx_geometry_eval(Ctx *c, const double *nodes, double *inv_jaco, double *jaco_det, double *norm, double *dA,
                       int where)
{
  if (!nodes || !inv_jaco || !jaco_det || !norm || !dA) ZB_THROW(ZB_ERR_ARG, "null geometry array");
  if (where != ZB_HOST && where != ZB_DEVICE) ZB_THROW(ZB_ERR_ARG, "where must be ZB_HOST or ZB_DEVICE");
  ensure_tables(c);
  const GeoSizes z(c->plan);
  const bool host = where == ZB_HOST;
  // scratch: unorm, then (host calls) the staged node and output arrays
  double *w = scratch(c, z.norm + (host ? z.nodes + z.inv + z.det + z.norm + z.dA : 0));
  double *unorm = w, *q = w + z.norm;
  const double *dn = nodes;
  double *di = inv_jaco, *dd = jaco_det, *dnm = norm, *da = dA;
  if (host)
  {
    double *sn = q;
    di = sn + z.nodes;
    dd = di + z.inv;
    dnm = dd + z.det;
    da = dnm + z.norm;
    CK(cudaMemcpyAsync(sn, nodes, z.nodes * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    dn = sn;
  }
  eval_device(c, dn, di, dd, dnm, da, unorm, nullptr, nullptr, nullptr);
  if (host)
  {
    CK(cudaMemcpyAsync(inv_jaco, di, z.inv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(jaco_det, dd, z.det * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(norm, dnm, z.norm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(dA, da, z.dA * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
}

void ctx_geometry_eval_vjp(Ctx *c, const double *nodes, const double *inv_jaco_bar, const double *jaco_det_bar,
                           const double *norm_bar, const double *dA_bar, double *nodes_bar, int where)
{
  if (!nodes || !nodes_bar) ZB_THROW(ZB_ERR_ARG, "null node array");
  if (where != ZB_HOST && where != ZB_DEVICE) ZB_THROW(ZB_ERR_ARG, "where must be ZB_HOST or ZB_DEVICE");
  ensure_tables(c);
  const Plan &p = c->plan;
  const GeoSizes z(p);
  const int S = p.nspts, Fp = p.nfpts, nn = p.nnodes_ele, D = p.ndims;
  const int64_t E = p.neles;
  const bool host = where == ZB_HOST;
  // scratch: Jb, unorm_bar, then (host calls) the staged inputs and output
  double *w = scratch(c, z.Jb + z.norm + (host ? 2 * z.nodes + z.inv + z.det + z.norm + z.dA : 0));
  double *Jb = w, *ub = w + z.Jb;
  const double *dn = nodes, *ib = inv_jaco_bar, *db = jaco_det_bar, *nb = norm_bar, *ab = dA_bar;
  double *out = nodes_bar;
  if (host)
  {
    double *q = ub + z.norm;
    auto put = [&](const double *src, size_t n) -> const double * {
      if (!src) return nullptr;
      CK(cudaMemcpyAsync(q, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      const double *r = q;
      q += n;
      return r;
    };
    dn = put(nodes, z.nodes);
    ib = put(inv_jaco_bar, z.inv);
    db = put(jaco_det_bar, z.det);
    nb = put(norm_bar, z.norm);
    ab = put(dA_bar, z.dA);
    out = q;
  }
  const geo::Tabs t = tables(c);
  const unsigned g1 = blocks_for((int64_t)(S + Fp) * E), g2 = blocks_for((int64_t)Fp * E),
                 g3 = blocks_for((int64_t)nn * D * E);
  geo::k_geo_face_normals_vjp<<<g2, 256, 0, c->stream>>>(nb, c->geo_pair, c->geo_pair + (size_t)Fp * E, ub, D, Fp,
                                                         E);
  if (D == 2)
  {
    geo::k_geo_points_vjp<2><<<g1, 256, 0, c->stream>>>(dn, t, S, Fp, nn, E, ib, db, ub, ab, Jb);
    geo::k_geo_nodes_vjp<2><<<g3, 256, 0, c->stream>>>(Jb, t, S, Fp, nn, E, out);
  }
  else
  {
    geo::k_geo_points_vjp<3><<<g1, 256, 0, c->stream>>>(dn, t, S, Fp, nn, E, ib, db, ub, ab, Jb);
    geo::k_geo_nodes_vjp<3><<<g3, 256, 0, c->stream>>>(Jb, t, S, Fp, nn, E, out);
  }
  c->launches += 3;
  CK(cudaGetLastError());
  if (host)
  {
    CK(cudaMemcpyAsync(nodes_bar, out, z.nodes * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
}

void ctx_set_nodes(Ctx *c, const double *nodes, int where)
{
  if (!nodes) ZB_THROW(ZB_ERR_ARG, "null node array");
  if (where != ZB_HOST && where != ZB_DEVICE) ZB_THROW(ZB_ERR_ARG, "where must be ZB_HOST or ZB_DEVICE");
  ensure_tables(c);
  Plan &p = c->plan;
  const GeoSizes z(p);
  double *w = scratch(c, z.nodes + z.inv + z.det + z.norm + z.dA + z.norm + z.cs + z.cf + 1);
  double *dn = w, *di = dn + z.nodes, *dd = di + z.inv, *dnm = dd + z.det, *da = dnm + z.norm, *un = da + z.dA,
         *cs = un + z.norm, *cf = cs + z.cs;
  int *bad = (int *)(cf + z.cf);
  CK(cudaMemcpyAsync(dn, nodes, z.nodes * sizeof(double),
                     where == ZB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  eval_device(c, dn, di, dd, dnm, da, un, cs, cf, bad);
  int hbad = 0;
  CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (hbad) ZB_THROW(ZB_ERR_MESH, "negative Jacobian at a solution point of the moved mesh");
  // the context's metrics in its own precision form
  const int64_t work = c->ntiles * (c->S * (c->D * c->D + 1) + c->Fp * (c->D + 1)) * TW;
  if (c->prec == ZB_FP64)
    geo::k_geo_tiles<double><<<blocks_for(work), 256, 0, c->stream>>>(di, dd, dnm, da, (double *)c->mets,
                                                                      (double *)c->fgeo, c->ntiles, p.neles, c->S,
                                                                      c->Fp, c->D);
  else
    geo::k_geo_tiles<float><<<blocks_for(work), 256, 0, c->stream>>>(di, dd, dnm, da, (float *)c->mets,
                                                                     (float *)c->fgeo, c->ntiles, p.neles, c->S,
                                                                     c->Fp, c->D);
  c->launches++;
  CK(cudaGetLastError());
  // host copy of the geometry (coordinates for the wall-force moments and the
  // CFL line lengths, volumes for the CFL step)
  CK(cudaMemcpyAsync(p.nodes.data(), dn, z.nodes * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p.inv_jaco_spts.data(), di, z.inv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p.jaco_det_spts.data(), dd, z.det * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p.fnorm.data(), dnm, z.norm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p.fdA.data(), da, z.dA * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p.coord_spts.data(), cs, z.cs * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(p.coord_fpts.data(), cf, z.cf * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (c->dwall)
  {
    cudaFree(c->dwall);
    c->dwall = nullptr;
  }
  ctx_refresh_cfl_geometry(c);
}

}  // namespace zb
