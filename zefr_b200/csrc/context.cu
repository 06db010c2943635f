// Device context: buffers in the tile-major layout, layout conversion, kernel
// dispatch over (dimension, order, precision) and explicit RK44 stepping.
#include "ctx_impl.cuh"
#include "hex_kernels.cuh"
#include "tri_kernels.cuh"
#include "tri_tc_kernels.cuh"
#include "time_kernels.cuh"

namespace zb {

using dev::Args;
using dev::LineOpsT;
using dev::Shape;
using dev::TW;


// ---------------------------------------------------------------------------
// layout conversion kernels
// ---------------------------------------------------------------------------

// reference-strided FP64 -> tile-major T, minus the reference state ref[v]
// (nullptr: none); padded elements copy element 0
template <typename T>
__global__ void k_to_tiles(const double *__restrict__ src, T *__restrict__ dst, T *__restrict__ comp,
                           const double *__restrict__ ref, int64_t neles, int64_t ntiles, int npts, int nv, int64_t ss,
                           int64_t vs, int64_t es)
{
  const int64_t total = ntiles * npts * nv * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int v = (int)((i / TW) % nv);
    const int p = (int)((i / ((int64_t)TW * nv)) % npts);
    const int64_t t = i / ((int64_t)TW * nv * npts);
    int64_t e = t * TW + l;
    if (e >= neles) e = 0;
    const double x = src[p * ss + v * vs + e * es];
    dst[i] = (T)(ref ? x - ref[v] : x);
    if (comp) comp[i] = T(0);
  }
}

template <typename T>
__global__ void k_from_tiles(const T *__restrict__ srcT, const T *__restrict__ comp, const double *__restrict__ ref,
                             double *__restrict__ dst, int64_t neles, int npts, int nv, int64_t ss, int64_t vs,
                             int64_t es)
{
  const int64_t total = neles * npts * nv;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int64_t e = i % neles;
    const int v = (int)((i / neles) % nv);
    const int p = (int)(i / (neles * nv));
    const int64_t t = e / TW;
    const int l = (int)(e % TW);
    const int64_t j = ((t * npts + p) * nv + v) * TW + l;
    double val = (double)srcT[j];
    if (comp) val -= (double)comp[j];
    if (ref) val += ref[v];
    dst[p * ss + v * vs + e * es] = val;
  }
}

// per-variable sum over all points and elements of a reference-strided array
__global__ void k_var_sums(const double *__restrict__ src, int64_t neles, int npts, int nv, int64_t ss, int64_t vs,
                           int64_t es, double *out)
{
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int64_t n = neles * npts;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int64_t e = i % neles;
    const int p = (int)(i / neles);
    for (int v = 0; v < nv; v++) acc[v] += src[p * ss + v * vs + e * es];
  }
  for (int v = 0; v < nv; v++)
  {
    double x = acc[v];
    for (int o = 16; o > 0; o /= 2) x += __shfl_down_sync(0xffffffff, x, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[v], x);
  }
}

// FP64 residual norms of report_residuals: max, sum |r|, sum r^2 with r = divF/|J|
template <typename T>
__global__ void k_norms(const T *__restrict__ divF, const T *__restrict__ mets, int64_t neles, int S, int V, int NM,
                        int DD, double *out)
{
  __shared__ double red[3][8][32];
  double mx[8], l1[8], l2[8];
  for (int v = 0; v < 8; v++) mx[v] = l1[v] = l2[v] = 0.0;
  const int64_t npts = neles * S;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npts; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int64_t e = i % neles;
    const int s = (int)(i / neles);
    const int64_t t = e / TW;
    const int l = (int)(e % TW);
    const double det = (double)mets[((t * S + s) * NM + DD) * TW + l];
    for (int v = 0; v < V; v++)
    {
      const double r = (double)divF[((t * S + s) * V + v) * TW + l] / det;
      const double a = fabs(r);
      mx[v] = (a > mx[v] || a != a) ? a : mx[v];
      l1[v] += a;
      l2[v] += r * r;
    }
  }
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  for (int v = 0; v < V; v++)
  {
    for (int o = 16; o > 0; o /= 2)
    {
      const double m2 = __shfl_down_sync(0xffffffff, mx[v], o);
      mx[v] = (m2 > mx[v] || m2 != m2) ? m2 : mx[v];
      l1[v] += __shfl_down_sync(0xffffffff, l1[v], o);
      l2[v] += __shfl_down_sync(0xffffffff, l2[v], o);
    }
    if (lane == 0)
    {
      red[0][v][warp] = mx[v];
      red[1][v][warp] = l1[v];
      red[2][v][warp] = l2[v];
    }
  }
  __syncthreads();
  if (threadIdx.x < V)
  {
    const int v = threadIdx.x;
    double m = 0, s1 = 0, s2 = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++)
    {
      m = (red[0][v][w] > m || red[0][v][w] != red[0][v][w]) ? red[0][v][w] : m;
      s1 += red[1][v][w];
      s2 += red[2][v][w];
    }
    // non-negative doubles order like their bit patterns; NaN (0x7ff8...) wins
    atomicMax(reinterpret_cast<unsigned long long *>(&out[v]), (unsigned long long)__double_as_longlong(m));
    atomicAdd(&out[V + v], s1);
    atomicAdd(&out[2 * V + v], s2);
  }
}

// FP64 volume integrals of report_turbulent_stats (src/solver.cpp:7813-7917):
// out[0] = sum |J| w 1/2 rho |u|^2, out[1] = sum |J| w 1/2 rho |curl u|^2 (when
// the physical gradient is given), out[2] = sum |J| w (volume)
template <typename T>
__global__ void k_functionals(const T *__restrict__ U, const T *__restrict__ dU, const T *__restrict__ mets,
                              const double *__restrict__ w, const double *__restrict__ ref, int64_t neles, int S,
                              int D, double *out)
{
  const int V = D + 2, NM = D * D + 1;
  double ke = 0.0, en = 0.0, vol = 0.0;
  const int64_t n = neles * S;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int64_t e = i % neles;
    const int s = (int)(i / neles);
    const int64_t t = e / TW;
    const int l = (int)(e % TW);
    double u[5];
    for (int v = 0; v < V; v++)
      u[v] = (double)U[((t * S + s) * V + v) * TW + l] + (ref ? ref[v] : 0.0);
    const double jw = (double)mets[((t * S + s) * NM + D * D) * TW + l] * w[s];
    const double rho = u[0];
    double vel[3] = {0, 0, 0}, q2 = 0.0;
    for (int d = 0; d < D; d++)
    {
      vel[d] = u[d + 1] / rho;
      q2 += vel[d] * vel[d];
    }
    ke += jw * 0.5 * rho * q2;
    vol += jw;
    if (dU)
    {
      double g[3][3] = {{0}};  // g[i][j] = d u_i / d x_j
      for (int i2 = 0; i2 < D; i2++)
        for (int j = 0; j < D; j++)
        {
          const double dm = (double)dU[(((t * D + j) * S + s) * V + i2 + 1) * TW + l];
          const double dr = (double)dU[(((t * D + j) * S + s) * V + 0) * TW + l];
          g[i2][j] = (dm - dr * vel[i2]) / rho;
        }
      double w2;
      if (D == 3)
      {
        const double wx = g[2][1] - g[1][2], wy = g[0][2] - g[2][0], wz = g[1][0] - g[0][1];
        w2 = wx * wx + wy * wy + wz * wz;
      }
      else
      {
        const double wz = g[1][0] - g[0][1];
        w2 = wz * wz;
      }
      en += jw * 0.5 * rho * w2;
    }
  }
  for (int o = 16; o > 0; o /= 2)
  {
    ke += __shfl_down_sync(0xffffffff, ke, o);
    en += __shfl_down_sync(0xffffffff, en, o);
    vol += __shfl_down_sync(0xffffffff, vol, o);
  }
  if ((threadIdx.x & 31) == 0)
  {
    atomicAdd(&out[0], ke);
    atomicAdd(&out[1], en);
    atomicAdd(&out[2], vol);
  }
}

// FP64 force and moment (about the origin) on wall boundaries of
// FRSolver::compute_moments (src/solver.cpp:7600-7811): per wall flux point
// w (P n - tau n) dA from the element's own trace and its extrapolated
// corrected gradient.  The reference's 3D branch reads flux point 0's state
// for the stress (src/solver.cpp:7716-7720); this uses each point's own.
struct WallArgs
{
  double gamma, mu, rt, c_sth;
  int fix_vis, viscous, D, S, Fp;
  int64_t ntiles, neles;
};

template <typename T>
__global__ void k_wall_force(const T *__restrict__ Ufp, const T *__restrict__ dU, const T *__restrict__ fgeo,
                             const int *__restrict__ nbr, const double *__restrict__ dE, const double *__restrict__ fw,
                             const double *__restrict__ cfp, const double *__restrict__ ref, const WallArgs w,
                             double *out)
{
  const int D = w.D, V = D + 2, S = w.S, Fp = w.Fp;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int64_t total = w.ntiles * Fp * TW;
  for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(gid % TW);
    const int f = (int)((gid / TW) % Fp);
    const int64_t t = gid / ((int64_t)TW * Fp);
    const int64_t e = t * TW + l;
    if (e >= w.neles) continue;
    const int code = nbr[(t * Fp + f) * TW + l];
    if (code >= 0) continue;
    const int bc = -code - 1;
    if (bc != 5 && bc != 6 && bc != 7 && bc != 8 && bc != 9) continue;
    double u[5], n[3] = {0, 0, 0};
    for (int v = 0; v < V; v++) u[v] = (double)Ufp[((t * Fp + f) * V + v) * TW + l] + (ref ? ref[v] : 0.0);
    for (int d = 0; d < D; d++) n[d] = (double)fgeo[((t * Fp + f) * (D + 1) + d) * TW + l];
    const double dA = (double)fgeo[((t * Fp + f) * (D + 1) + D) * TW + l];
    const double rho = u[0];
    double vel[3] = {0, 0, 0}, q2 = 0.0;
    for (int d = 0; d < D; d++)
    {
      vel[d] = u[d + 1] / rho;
      q2 += vel[d] * vel[d];
    }
    const double P = (w.gamma - 1.0) * (u[V - 1] - 0.5 * rho * q2);
    const double wt = fw[f] * dA;
    double F[3] = {0, 0, 0};
    for (int d = 0; d < D; d++) F[d] = wt * P * n[d];
    if (w.viscous)
    {
      double g[3][3];  // g[i][j] = d u_i / d x_j at the flux point
      for (int j = 0; j < D; j++)
      {
        double dr = 0.0, dm[3] = {0, 0, 0};
        for (int sp = 0; sp < S; sp++)
        {
          const double c = dE[(size_t)f * S + sp];
          dr += c * (double)dU[(((t * D + j) * S + sp) * V + 0) * TW + l];
          for (int i = 0; i < D; i++) dm[i] += c * (double)dU[(((t * D + j) * S + sp) * V + i + 1) * TW + l];
        }
        for (int i = 0; i < D; i++) g[i][j] = (dm[i] - dr * vel[i]) / rho;
      }
      double mu = w.mu;
      if (!w.fix_vis)
      {
        const double e_int = u[V - 1] / rho - 0.5 * q2;
        const double rr = (w.gamma - 1.0) * e_int / w.rt;
        mu = w.mu * pow(rr, 1.5) * (1.0 + w.c_sth) / (rr + w.c_sth);
      }
      double diag = 0.0;
      for (int d = 0; d < D; d++) diag += g[d][d];
      diag /= 3.0;
      for (int i = 0; i < D; i++)
      {
        double taun = 0.0;
        for (int j = 0; j < D; j++)
          taun += ((i == j) ? 2.0 * mu * (g[i][i] - diag) : mu * (g[i][j] + g[j][i])) * n[j];
        F[i] -= wt * taun;
      }
    }
    double x[3] = {0, 0, 0};
    for (int d = 0; d < D; d++) x[d] = cfp[((size_t)f * D + d) * w.neles + e];
    for (int d = 0; d < D; d++) acc[d] += F[d];
    if (D == 3)
    {
      acc[3] += x[1] * F[2] - x[2] * F[1];
      acc[4] += x[2] * F[0] - x[0] * F[2];
    }
    acc[5] += x[0] * F[1] - x[1] * F[0];
  }
  for (int k = 0; k < 6; k++)
  {
    double a = acc[k];
    for (int o = 16; o > 0; o /= 2) a += __shfl_down_sync(0xffffffff, a, o);
    if ((threadIdx.x & 31) == 0 && a != 0.0) atomicAdd(&out[k], a);
  }
}

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------


template <typename T, typename A, int D, int N>
static void launch_extrap_impl(Ctx &c)
{
  using G = Shape<D, N>;
  const int64_t work = c.ntiles * G::Fp * TW;
  ProfScope ps(c, ZB_K_EXTRAP);
  if constexpr (D == 3)
    dev::k_hex_extrap<T, A, N><<<(unsigned)c.ntiles, TW * N * N, 0, c.stream>>>((const T *)c.U, (T *)c.Ufp[c.cur],
                                                                                c.ntiles, line_ops<A, N>(c.plan));
  else
    dev::k_extrap<T, A, D, N><<<grid_for(work, 256), 256, 0, c.stream>>>((const T *)c.U, (T *)c.Ufp[c.cur],
                                                                           c.ntiles, line_ops<A, N>(c.plan));
  c.launches++;
  CK(cudaGetLastError());
}


template <typename T, typename A, int D, int N>
static void launch_stage_impl(Ctx &c, const StageCfg &sc)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, NT = G::NT;
  const Args<T, A> a = make_args<T, A>(c, sc);
  const LineOpsT<A, N> ops = line_ops<A, N>(c.plan);
  const size_t ops_bytes = sizeof(LineOpsT<A, N>);
  if constexpr (D == 3)
  {
    // hexahedra: column-mapped kernels, TW x N^2 threads per tile
    constexpr int HT = TW * N * N;
    if (!c.plan.params.viscous)
    {
      const size_t smem = (size_t)(S * V + 3 * S * V + Fp * V) * TW * sizeof(A);
      set_smem(dev::k_hex_euler<T, A, N>, smem);
      ProfScope ps(c, ZB_K_EULER);
      dev::k_hex_euler<T, A, N><<<(unsigned)c.ntiles, HT, smem, c.stream>>>(a, ops);
      c.launches++;
      CK(cudaGetLastError());
    }
    else
    {
      constexpr int ZG = dev::HexNsShape<A, N>::grad_zs, ZF = dev::HexNsShape<A, N>::face_zs;
      const size_t smem1 = (size_t)((S * V + Fp * V + 3 * S * V) * TW + 3 * N * TW) * sizeof(A);  // + sX padding
      set_smem(dev::k_hex_ns_grad<T, A, N>, smem1);
      if (!sc.face_only)
      {
        ProfScope ps(c, ZB_K_NS_GRAD);
        dev::k_hex_ns_grad<T, A, N><<<(unsigned)c.ntiles, HT * ZG, smem1, c.stream>>>(a, ops);
        c.launches++;
        CK(cudaGetLastError());
      }
      if (sc.grad_only) return;
      const size_t smem2 = (size_t)(Fp * V + S * V) * TW * sizeof(A);
      set_smem(dev::k_hex_ns_face<T, A, N>, smem2);
      ProfScope ps(c, ZB_K_NS_FACE);
      dev::k_hex_ns_face<T, A, N><<<(unsigned)c.ntiles, HT * ZF, smem2, c.stream>>>(a, ops);
      c.launches++;
      CK(cudaGetLastError());
    }
    if (sc.extrap_next)
    {
      if (a.Fcom)
        c.ufp_valid = false;  // the state changed and no traces were stored
      else
        c.cur ^= 1;
    }
    return;
  }
  if (!c.plan.params.viscous)
  {
    const size_t smem = (size_t)(S * V + D * S * V + Fp * V) * TW * sizeof(A) + ops_bytes;
    set_smem(dev::k_euler<T, A, D, N>, smem);
    ProfScope ps(c, ZB_K_EULER);
    dev::k_euler<T, A, D, N><<<(unsigned)c.ntiles, NT, smem, c.stream>>>(a, ops);
    c.launches++;
    CK(cudaGetLastError());
  }
  else
  {
    const size_t smem1 = (size_t)(S * V + Fp * V + D * S * V) * TW * sizeof(A) + ops_bytes;
    set_smem(dev::k_ns_grad<T, A, D, N>, smem1);
    if (!sc.face_only)
    {
      ProfScope ps(c, ZB_K_NS_GRAD);
      dev::k_ns_grad<T, A, D, N><<<(unsigned)c.ntiles, NT, smem1, c.stream>>>(a, ops);
      c.launches++;
      CK(cudaGetLastError());
    }
    if (sc.grad_only) return;
    const size_t smem2 = (size_t)(Fp * V + S * V) * TW * sizeof(A) + ops_bytes;
    set_smem(dev::k_ns_face<T, A, D, N>, smem2);
    ProfScope ps(c, ZB_K_NS_FACE);
    dev::k_ns_face<T, A, D, N><<<(unsigned)c.ntiles, NT, smem2, c.stream>>>(a, ops);
    c.launches++;
    CK(cudaGetLastError());
  }
  if (sc.extrap_next) c.cur ^= 1;
}


// Triangles: dense-operator kernels (tri_kernels.cuh)
template <typename T, typename A, int N>
static void launch_extrap_tri(Ctx &c)
{
  using G = dev::TriShape<N>;
  ProfScope ps(c, ZB_K_EXTRAP);
  dev::k_tri_extrap<T, A, N><<<grid_for(c.ntiles * G::Fp * TW, 128), 128, 0, c.stream>>>(
      (const T *)c.U, (T *)c.Ufp[c.cur], c.ntiles, (const A *)c.dops);
  c.launches++;
  CK(cudaGetLastError());
}

template <typename T, typename A, int N>
static void launch_stage_tri(Ctx &c, const StageCfg &sc)
{
  using G = dev::TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, D = 2;
  const Args<T, A> a = make_args<T, A>(c, sc);
  if (c.tc_err_host && *c.tc_err_host)
  {
    *c.tc_err_host = 0;
    ZB_THROW(ZB_ERR_CUDA, "a tensor-core completion wait of an earlier launch timed out");
  }
  const size_t ops = (size_t)G::OPS_PAD;
  if (!c.plan.params.viscous)
  {
    const size_t smem = (ops + (size_t)(S * V + D * S * V + Fp * V) * TW) * sizeof(A);
    set_smem(dev::k_tri_euler<T, A, N>, smem);
    ProfScope ps(c, ZB_K_EULER);
    dev::k_tri_euler<T, A, N><<<(unsigned)c.ntiles, 128, smem, c.stream>>>(a);
    c.launches++;
    CK(cudaGetLastError());
  }
  else
  {
    const size_t smem1 = (ops + (size_t)(S * V + Fp * V + D * S * V) * TW) * sizeof(A);
    if (!sc.face_only)
    {
      ProfScope ps(c, ZB_K_NS_GRAD);
      bool launched = false;
      if constexpr (std::is_same<A, float>::value && N <= 5)
      {
        if (c.plan.params.tensor_ops)
        {
          using C = dev::TriTc<N>;
          set_smem(dev::k_tri_ns_grad_tc<N>, C::SMEM);
          const int64_t groups = (c.ntiles + C::TILES - 1) / C::TILES;
          dev::k_tri_ns_grad_tc<N><<<(unsigned)groups, C::NT, C::SMEM, c.stream>>>(a);
          launched = true;
        }
      }
      if (!launched)
      {
        set_smem(dev::k_tri_ns_grad<T, A, N>, smem1);
        dev::k_tri_ns_grad<T, A, N><<<(unsigned)c.ntiles, 128, smem1, c.stream>>>(a);
      }
      c.launches++;
      CK(cudaGetLastError());
    }
    if (sc.grad_only) return;
    const size_t smem2 = (ops + (size_t)(Fp * V + S * V) * TW) * sizeof(A);
    set_smem(dev::k_tri_ns_face<T, A, N>, smem2);
    ProfScope ps(c, ZB_K_NS_FACE);
    dev::k_tri_ns_face<T, A, N><<<(unsigned)c.ntiles, 128, smem2, c.stream>>>(a);
    c.launches++;
    CK(cudaGetLastError());
  }
  if (sc.extrap_next) c.cur ^= 1;
}

template <typename T, typename A, int D, int N>
static void bind(Ctx &c)
{
  c.launch_extrap = &launch_extrap_impl<T, A, D, N>;
  c.launch_stage = &launch_stage_impl<T, A, D, N>;
  c.launch_dt = &launch_dt_impl<T, A, D, N>;
}

template <typename T, typename A>
static void bind_t(Ctx &c)
{
  const int D = c.D, N = c.N;
  if (c.plan.etype == ET_TRI)
  {
#define ZB_BIND_TRI(NN)                                   \
  if (N == NN)                                            \
  {                                                       \
    c.launch_extrap = &launch_extrap_tri<T, A, NN>;       \
    c.launch_stage = &launch_stage_tri<T, A, NN>;         \
    return;                                               \
  }
    ZB_BIND_TRI(2) ZB_BIND_TRI(3) ZB_BIND_TRI(4) ZB_BIND_TRI(5) ZB_BIND_TRI(6) ZB_BIND_TRI(7) ZB_BIND_TRI(8)
    ZB_BIND_TRI(9)
#undef ZB_BIND_TRI
    ZB_THROW(ZB_ERR_UNSUPPORTED, "no triangle kernels for P=" + std::to_string(N - 1));
  }
#define ZB_BIND(DD, NN) \
  if (D == DD && N == NN) { bind<T, A, DD, NN>(c); return; }
  ZB_BIND(2, 2) ZB_BIND(2, 3) ZB_BIND(2, 4) ZB_BIND(2, 5) ZB_BIND(2, 6)
  ZB_BIND(3, 2) ZB_BIND(3, 3) ZB_BIND(3, 4) ZB_BIND(3, 5)
#undef ZB_BIND
  ZB_THROW(ZB_ERR_UNSUPPORTED, "no kernels built for ndims=" + std::to_string(D) + " P=" + std::to_string(N - 1));
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

static void *dalloc(size_t bytes)
{
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    ZB_THROW(ZB_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  return p;
}

static void free_all(Ctx *c)
{
  void *bufs[] = {c->U, c->U_ini, c->divF[0], c->divF[1], c->divF[2], c->divF[3], c->divF_vol, c->Ufp[0],
                  c->Ufp[1], c->Fvn, c->Fcom, c->mets, c->fgeo, c->Ucomp, c->nbr, c->dtmp, c->dred, c->dref,
                  c->dU, c->dweights, c->dfun, c->lam, c->Lfp, c->Ubfp, c->dUbfp, c->UCb, c->Ubx, c->Ubar, c->pbar, c->dops, c->dwall,
                  c->mbar, c->gbar, c->nbx, c->mbar_acc, c->gbar_acc, c->d_dt, c->dt_ele, c->h_ref, c->evol,
                  c->dfw, c->U_til, c->rk_err, c->rkv, c->rkfvn, c->geo_tab, c->geo_pair, c->geo_work};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (c->tc_err_host) cudaFreeHost(const_cast<int *>(c->tc_err_host));
  for (int b = 0; b < 2; b++)
  {
    if (c->pipe_in[b]) cudaFree(c->pipe_in[b]);
    if (c->pipe_out[b]) cudaFree(c->pipe_out[b]);
  }
  if (c->pipe_h2d) cudaStreamDestroy(c->pipe_h2d);
  if (c->pipe_d2h) cudaStreamDestroy(c->pipe_d2h);
  for (auto e : c->pipe_ev)
    if (e) cudaEventDestroy(e);
  for (auto &r : c->recs)
  {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : c->pool) cudaEventDestroy(e);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
}

template <typename T>
static void upload_static(Ctx &c)
{
  const Plan &p = c.plan;
  const int64_t E = p.neles, nt = c.ntiles;
  const int S = c.S, Fp = c.Fp, D = c.D, NM = D * D + 1;
  std::vector<T> mets((size_t)nt * S * NM * TW);
  std::vector<T> fgeo((size_t)nt * Fp * (D + 1) * TW);
  std::vector<int> nbr((size_t)nt * Fp * TW);
  for (int64_t t = 0; t < nt; t++)
    for (int l = 0; l < TW; l++)
    {
      int64_t e = t * TW + l;
      const bool pad = (e >= E);
      const int64_t es = pad ? 0 : e;
      for (int s = 0; s < S; s++)
      {
        for (int d1 = 0; d1 < D; d1++)
          for (int d2 = 0; d2 < D; d2++)
            mets[((t * S + s) * NM + d1 * D + d2) * TW + l] =
                (T)p.inv_jaco_spts[(((size_t)d1 * S + s) * D + d2) * E + es];
        mets[((t * S + s) * NM + D * D) * TW + l] = (T)p.jaco_det_spts[(size_t)s * E + es];
      }
      for (int f = 0; f < Fp; f++)
      {
        for (int d = 0; d < D; d++)
          fgeo[((t * Fp + f) * (D + 1) + d) * TW + l] = (T)p.fnorm[((size_t)f * D + d) * E + es];
        fgeo[((t * Fp + f) * (D + 1) + D) * TW + l] = (T)p.fdA[(size_t)f * E + es];
        int code;
        if (pad)
        {
          code = 2 * (int)((t * Fp + f) * TW + l);  // pair with itself
        }
        else
        {
          const int64_t pr = p.partner[(size_t)f * E + e];
          if (pr < 0)
            code = (int)pr;
          else
          {
            const int64_t e2 = pr / Fp;
            const int f2 = (int)(pr % Fp);
            const int64_t pidx = ((e2 / TW) * Fp + f2) * TW + (e2 % TW);
            if (pidx >= (int64_t(1) << 30)) ZB_THROW(ZB_ERR_UNSUPPORTED, "mesh too large for 32-bit face index");
            code = (int)(2 * pidx + p.slot[(size_t)f * E + e]);
          }
        }
        nbr[(t * Fp + f) * TW + l] = code;
      }
    }
  CK(cudaMemcpyAsync(c.mets, mets.data(), mets.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(c.fgeo, fgeo.data(), fgeo.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
  CK(cudaMemcpyAsync(c.nbr, nbr.data(), nbr.size() * sizeof(int), cudaMemcpyHostToDevice, c.stream));
  CK(cudaStreamSynchronize(c.stream));
}

Ctx *ctx_create(const Plan &plan)
{
  std::unique_ptr<Ctx> c(new Ctx());
  c->plan = plan;
  CK(cudaGetDevice(&c->dev));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->own_stream = true;
  c->prec = plan.params.precision;
  if (c->prec != ZB_FP64 && c->prec != ZB_MIXED) ZB_THROW(ZB_ERR_ARG, "unknown precision");
  c->tsz = (c->prec == ZB_FP64) ? sizeof(double) : sizeof(float);
  c->asz = c->tsz;
  c->D = plan.ndims;
  c->N = plan.N;
  c->S = plan.nspts;
  c->Fp = plan.nfpts;
  c->V = plan.nvars;
  c->ntiles = plan.ntiles;
  c->dt = plan.params.dt;
  if (plan.tile != TW) ZB_THROW(ZB_ERR_INTERNAL, "plan tile width does not match kernels");
  if (plan.params.tensor_ops && !(c->prec == ZB_MIXED && plan.etype == ET_TRI && plan.params.viscous && plan.order <= 4))
    ZB_THROW(ZB_ERR_UNSUPPORTED, "tensor-core operator products are built for the mixed form on triangles "
                                 "(Navier-Stokes, P <= 4)");
  if (c->prec == ZB_FP64)
  {
    bind_t<double, double>(*c);
    bind_vjp(*c);
  }
  else
    bind_t<float, float>(*c);
  try
  {
    const size_t nU = (size_t)c->ntiles * c->S * c->V * TW;
    const size_t nF = (size_t)c->ntiles * c->Fp * c->V * TW;
    c->U = dalloc(nU * c->tsz);
    c->U_ini = dalloc(nU * c->tsz);
    for (int s = 0; s < c->nstages; s++) c->divF[s] = dalloc(nU * c->tsz);
    c->Ufp[0] = dalloc(nF * c->tsz);
    c->Ufp[1] = dalloc(nF * c->tsz);
    if (plan.params.viscous)
    {
      c->divF_vol = dalloc(nU * c->asz);
      c->Fvn = dalloc(nF * c->tsz);
      if (c->D == 3) c->Fcom = dalloc(nF * c->tsz);  // hexahedra: one-sided common flux
      c->fused_traces = c->Fcom && (plan.params.ldg_b == 0.5 || plan.params.ldg_b == -0.5);
    }
    if (c->prec != ZB_FP64) c->Ucomp = dalloc(nU * c->tsz);
    c->mets = dalloc((size_t)c->ntiles * c->S * (c->D * c->D + 1) * TW * c->tsz);
    c->fgeo = dalloc((size_t)c->ntiles * c->Fp * (c->D + 1) * TW * c->tsz);
    c->nbr = (int *)dalloc((size_t)c->ntiles * c->Fp * TW * sizeof(int));
    c->dred = (double *)dalloc(3 * 8 * sizeof(double));
    c->dref = (double *)dalloc(8 * sizeof(double));
    if (plan.params.tensor_ops)
    {
      void *h = nullptr, *dp = nullptr;
      CK(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped));
      c->tc_err_host = static_cast<volatile int *>(h);
      *c->tc_err_host = 0;
      CK(cudaHostGetDevicePointer(&dp, h, 0));
      c->tc_err_dev = static_cast<int *>(dp);
    }
    CK(cudaMemsetAsync(c->dref, 0, 8 * sizeof(double), c->stream));
    if (c->prec == ZB_FP64)
      upload_static<double>(*c);
    else
      upload_static<float>(*c);
    if (plan.etype == ET_TRI)
    {
      // oppE, oppD, oppD_fpts, oppDiv, oppDiv_fpts back to back (TriShape)
      std::vector<double> ops;
      for (const auto *v : {&plan.tri_oppE, &plan.tri_oppD, &plan.tri_oppD_fpts, &plan.tri_oppDiv,
                            &plan.tri_oppDiv_fpts})
        ops.insert(ops.end(), v->begin(), v->end());
      c->dops = dalloc(ops.size() * c->asz);
      if (c->asz == sizeof(double))
        CK(cudaMemcpy(c->dops, ops.data(), ops.size() * sizeof(double), cudaMemcpyHostToDevice));
      else
      {
        std::vector<float> f(ops.begin(), ops.end());
        CK(cudaMemcpy(c->dops, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
      }
    }
    // zero the state so a residual before set_state is well defined (all zeros)
    CK(cudaMemsetAsync(c->U, 0, nU * c->tsz, c->stream));
    if (c->Ucomp) CK(cudaMemsetAsync(c->Ucomp, 0, nU * c->tsz, c->stream));
    for (int s = 0; s < c->nstages; s++) CK(cudaMemsetAsync(c->divF[s], 0, nU * c->tsz, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  catch (...)
  {
    free_all(c.get());
    throw;
  }
  return c.release();
}

void ctx_destroy(Ctx *c)
{
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  delete c;
}

void ctx_info(const Ctx *c, zb_info *out)
{
  const Plan &p = c->plan;
  out->ndims = p.ndims;
  out->nvars = p.nvars;
  out->nspts = p.nspts;
  out->nfpts = p.nfpts;
  out->order = p.order;
  out->etype = p.etype;
  out->n_eles = p.neles;
  out->n_eles_pad = p.neles_pad;
  out->n_gfpts = p.n_gfpts_int + p.n_gfpts_bnd;
  out->n_gfpts_int = p.n_gfpts_int;
  out->n_gfpts_bnd = p.n_gfpts_bnd;
  out->nstages = c->nstages;
  out->tile = TW;
  out->precision = c->prec;
}

void ctx_set_stream(Ctx *c, void *stream)
{
  CK(cudaStreamSynchronize(c->stream));
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
}

void ctx_set_dt(Ctx *c, double dt) { c->dt = dt; }

void ctx_set_freestream(Ctx *c, double rho_fs, const double *V_fs, double P_fs)
{
  // launches read the parameters by value, so queued work keeps the old ones
  c->plan.params.rho_fs = rho_fs;
  for (int d = 0; d < 3; d++) c->plan.params.V_fs[d] = V_fs[d];
  c->plan.params.P_fs = P_fs;
}

static const double *stage_in(Ctx *c, const double *src, size_t extent_elems, int where)
{
  if (where == ZB_DEVICE) return src;
  const size_t bytes = extent_elems * sizeof(double);
  if (bytes > c->dtmp_bytes)
  {
    if (c->dtmp) cudaFree(c->dtmp);
    c->dtmp = nullptr;
    c->dtmp = (double *)dalloc(bytes);
    c->dtmp_bytes = bytes;
  }
  CK(cudaMemcpyAsync(c->dtmp, src, bytes, cudaMemcpyHostToDevice, c->stream));
  return c->dtmp;
}

static size_t extent(const Ctx *c, int64_t ss, int64_t vs, int64_t es, int npts)
{
  if (ss < 0 || vs < 0 || es < 0) ZB_THROW(ZB_ERR_ARG, "negative strides are not supported");
  return (size_t)((npts - 1) * ss + (c->V - 1) * vs + (c->plan.neles - 1) * es + 1);
}

void ctx_set_state(Ctx *c, const double *U, int64_t ss, int64_t vs, int64_t es, int where)
{
  c->split_phase = 0;
  if (!U) ZB_THROW(ZB_ERR_ARG, "null state");
  const size_t ext = extent(c, ss, vs, es, c->S);
  const double *src = stage_in(c, U, ext, where);
  const int64_t work = c->ntiles * c->S * c->V * TW;
  if (c->prec != ZB_FP64)
  {
    // reference state of the perturbation form: the state's mean per variable
    // (FP64 reduction), rounded to FP32 so U = Ur + U' holds exactly in FP32
    CK(cudaMemsetAsync(c->dred, 0, 8 * sizeof(double), c->stream));
    const int64_t n = c->plan.neles * c->S;
    k_var_sums<<<grid_for(n, 256), 256, 0, c->stream>>>(src, c->plan.neles, c->S, c->V, ss, vs, es, c->dred);
    c->launches++;
    CK(cudaGetLastError());
    double h[8];
    CK(cudaMemcpyAsync(h, c->dred, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int v = 0; v < c->V; v++)
    {
      const double mean = h[v] / (double)n;
      c->uref[v] = std::isfinite(mean) ? (double)(float)mean : 0.0;
    }
    CK(cudaMemcpyAsync(c->dref, c->uref, sizeof(c->uref), cudaMemcpyHostToDevice, c->stream));
  }
  {
    ProfScope ps(*c, ZB_K_TO_TILES);
    if (c->prec == ZB_FP64)
      k_to_tiles<double><<<grid_for(work, 256), 256, 0, c->stream>>>(src, (double *)c->U, nullptr, nullptr,
                                                                       c->plan.neles, c->ntiles, c->S, c->V, ss, vs, es);
    else
      k_to_tiles<float><<<grid_for(work, 256), 256, 0, c->stream>>>(src, (float *)c->U, (float *)c->Ucomp, c->dref,
                                                                      c->plan.neles, c->ntiles, c->S, c->V, ss, vs, es);
    c->launches++;
    CK(cudaGetLastError());
  }
  if (where == ZB_HOST) CK(cudaStreamSynchronize(c->stream));
  c->ufp_valid = false;
}

static void from_tiles(Ctx *c, const void *srcT, const void *comp, const double *ref, double *out, int64_t ss,
                       int64_t vs, int64_t es, int where)
{
  const size_t ext = extent(c, ss, vs, es, c->S);
  double *dst = out;
  if (where == ZB_HOST)
  {
    const size_t bytes = ext * sizeof(double);
    if (bytes > c->dtmp_bytes)
    {
      if (c->dtmp) cudaFree(c->dtmp);
      c->dtmp = nullptr;
      c->dtmp = (double *)dalloc(bytes);
      c->dtmp_bytes = bytes;
    }
    dst = c->dtmp;
    // a strided caller buffer has holes the export must leave intact: start
    // from its contents (a dense buffer is overwritten entirely)
    if (ext != (size_t)c->S * c->V * c->plan.neles)
      CK(cudaMemcpyAsync(dst, out, bytes, cudaMemcpyHostToDevice, c->stream));
  }
  const int64_t work = c->plan.neles * c->S * c->V;
  {
  ProfScope ps(*c, ZB_K_FROM_TILES);
  if (c->prec == ZB_FP64)
    k_from_tiles<double><<<grid_for(work, 256), 256, 0, c->stream>>>((const double *)srcT, (const double *)comp, ref,
                                                                       dst, c->plan.neles, c->S, c->V, ss, vs, es);
  else
    k_from_tiles<float><<<grid_for(work, 256), 256, 0, c->stream>>>((const float *)srcT, (const float *)comp, ref,
                                                                      dst, c->plan.neles, c->S, c->V, ss, vs, es);
  c->launches++;
  CK(cudaGetLastError());
  }
  if (where == ZB_HOST)
  {
    CK(cudaMemcpyAsync(out, dst, ext * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
}

void ctx_get_state(Ctx *c, double *U, int64_t ss, int64_t vs, int64_t es, int where)
{
  if (!U) ZB_THROW(ZB_ERR_ARG, "null state");
  from_tiles(c, c->U, c->Ucomp, c->prec != ZB_FP64 ? c->dref : nullptr, U, ss, vs, es, where);
}

static void ensure_ufp(Ctx *c)
{
  if (!c->ufp_valid)
  {
    c->launch_extrap(*c);
    c->ufp_valid = true;
  }
}

// traces for a residual or RK stage: none when the gradient kernel forms them
// from the state (hexahedral Navier-Stokes with one-sided LDG)
static void ensure_stage_ufp(Ctx *c)
{
  if (!c->fused_traces) ensure_ufp(c);
}

void ctx_compute_residual(Ctx *c, unsigned stage)
{
  if (stage >= (unsigned)c->nstages) ZB_THROW(ZB_ERR_ARG, "stage out of range");
  c->split_phase = 0;
  // extrapolate_U is step 1 of the reference residual (src/solver.cpp:1516-1518)
  c->ufp_valid = false;
  ensure_stage_ufp(c);
  StageCfg sc{stage, 0, 0, 0};
  c->launch_stage(*c, sc);
}

void ctx_get_residual(Ctx *c, unsigned stage, double *out, int64_t ss, int64_t vs, int64_t es, int where)
{
  if (stage >= (unsigned)c->nstages) ZB_THROW(ZB_ERR_ARG, "stage out of range");
  if (!out) ZB_THROW(ZB_ERR_ARG, "null output");
  from_tiles(c, c->divF[stage], nullptr, nullptr, out, ss, vs, es, where);
}

// divF_spts(stage) of n states held in host memory, dense in the reference
// layout [nspts][nvars][n_eles].  A software pipeline over two input and two
// output staging buffers: the host-to-device copy of state i+1 (its own
// stream and copy engine) and the device-to-host copy of residual i-1 (the
// other copy engine) run while residual i is computed on the context's
// stream; events hand each buffer from one stream to the next.
void ctx_residuals_host(Ctx *c, unsigned stage, int n, const double *const *U, double *const *R)
{
  if (stage >= (unsigned)c->nstages) ZB_THROW(ZB_ERR_ARG, "stage out of range");
  if (n < 0) ZB_THROW(ZB_ERR_ARG, "negative state count");
  if (n == 0) return;
  if (!U || !R) ZB_THROW(ZB_ERR_ARG, "null state or residual list");
  for (int i = 0; i < n; i++)
    if (!U[i] || !R[i]) ZB_THROW(ZB_ERR_ARG, "null state or residual pointer at index " + std::to_string(i));
  const int64_t E = c->plan.neles;
  const size_t ext = (size_t)c->S * c->V * E, bytes = ext * sizeof(double);
  if (!c->pipe_h2d)
  {
    for (int b = 0; b < 2; b++)
    {
      c->pipe_in[b] = (double *)dalloc(bytes);
      c->pipe_out[b] = (double *)dalloc(bytes);
    }
    CK(cudaStreamCreateWithFlags(&c->pipe_h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->pipe_d2h, cudaStreamNonBlocking));
    for (auto &e : c->pipe_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  // events per buffer b: in_ready, in_free, out_ready, out_free
  cudaEvent_t *in_ready = c->pipe_ev, *in_free = c->pipe_ev + 2, *out_ready = c->pipe_ev + 4,
              *out_free = c->pipe_ev + 6;
  const int64_t ss = (int64_t)c->V * E, vs = E, es = 1;
  // nothing queued earlier on the context's stream may still use the buffers
  CK(cudaEventRecord(in_free[0], c->stream));
  CK(cudaEventRecord(in_free[1], c->stream));
  CK(cudaEventRecord(out_free[0], c->stream));
  CK(cudaEventRecord(out_free[1], c->stream));
  for (int i = 0; i < n; i++)
  {
    const int b = i & 1;
    CK(cudaStreamWaitEvent(c->pipe_h2d, in_free[b], 0));
    CK(cudaMemcpyAsync(c->pipe_in[b], U[i], bytes, cudaMemcpyHostToDevice, c->pipe_h2d));
    CK(cudaEventRecord(in_ready[b], c->pipe_h2d));
    CK(cudaStreamWaitEvent(c->stream, in_ready[b], 0));
    ctx_set_state(c, c->pipe_in[b], ss, vs, es, ZB_DEVICE);
    CK(cudaEventRecord(in_free[b], c->stream));
    ctx_compute_residual(c, stage);
    CK(cudaStreamWaitEvent(c->stream, out_free[b], 0));
    from_tiles(c, c->divF[stage], nullptr, nullptr, c->pipe_out[b], ss, vs, es, ZB_DEVICE);
    CK(cudaEventRecord(out_ready[b], c->stream));
    CK(cudaStreamWaitEvent(c->pipe_d2h, out_ready[b], 0));
    CK(cudaMemcpyAsync(R[i], c->pipe_out[b], bytes, cudaMemcpyDeviceToHost, c->pipe_d2h));
    CK(cudaEventRecord(out_free[b], c->pipe_d2h));
  }
  CK(cudaStreamSynchronize(c->pipe_d2h));
  CK(cudaStreamSynchronize(c->pipe_h2d));
}

static StageCfg rk_stage_cfg(const Ctx *c, unsigned stage)
{
  StageCfg sc;
  sc.stage = stage;
  sc.rk_mode = (stage + 1 < (unsigned)c->nstages) ? 1 : 2;
  sc.save_ini = (stage == 0);
  sc.extrap_next = 1;
  return sc;
}

void ctx_rk_stage(Ctx *c, unsigned stage)
{
  if (stage >= (unsigned)c->nstages) ZB_THROW(ZB_ERR_ARG, "stage out of range");
  if (c->ts.scheme != ZB_RK44) ZB_THROW(ZB_ERR_UNSUPPORTED, "stage-wise stepping is built for RK44");
  c->split_phase = 0;
  ensure_stage_ufp(c);
  c->launch_stage(*c, rk_stage_cfg(c, stage));
}

// Split residual and RK stage (compute_residual_start/mid/finish,
// src/solver.cpp:1647-1829; step_RK_stage_start/mid/finish, 3696-3760).
// start: the state's flux-point traces (extrapolate_U; nothing for
// hexahedral Navier-Stokes with one-sided LDG, whose gradient kernel forms
// the traces from the state); mid: for
// Navier-Stokes the gradient kernel (common solution, corrected gradient,
// fluxes, volume divergence); finish: the common fluxes and surface
// correction (the whole Euler kernel), with the RK update for a stage.
// The three calls in order equal zb_compute_residual / zb_rk_stage.
static void split_expect(Ctx *c, unsigned stage, int phase, int rk, const char *call)
{
  if (stage >= (unsigned)c->nstages) ZB_THROW(ZB_ERR_ARG, "stage out of range");
  if (rk && c->ts.scheme != ZB_RK44) ZB_THROW(ZB_ERR_UNSUPPORTED, "stage-wise stepping is built for RK44");
  if (c->split_phase != phase || (phase != 0 && (c->split_stage != stage || c->split_rk != rk)))
  {
    c->split_phase = 0;
    ZB_THROW(ZB_ERR_ARG, std::string(call) + " out of order: call _start, _mid and _finish of one stage in turn");
  }
}

void ctx_residual_split(Ctx *c, unsigned stage, int part, int rk)
{
  static const char *names[2][3] = {{"compute_residual_start", "compute_residual_mid", "compute_residual_finish"},
                                    {"rk_stage_start", "rk_stage_mid", "rk_stage_finish"}};
  if (part < 0 || part > 2) ZB_THROW(ZB_ERR_ARG, "split part out of range");
  split_expect(c, stage, part, rk ? 1 : 0, names[rk ? 1 : 0][part]);
  const bool visc = c->plan.params.viscous != 0;
  if (part == 0)
  {
    if (!rk) c->ufp_valid = false;
    ensure_stage_ufp(c);
    c->split_stage = stage;
    c->split_rk = rk ? 1 : 0;
    c->split_phase = 1;
    return;
  }
  StageCfg sc = rk ? rk_stage_cfg(c, stage) : StageCfg{stage, 0, 0, 0};
  if (part == 1)
  {
    if (visc)
    {
      sc.grad_only = 1;
      c->launch_stage(*c, sc);
    }
    c->split_phase = 2;
    return;
  }
  sc.face_only = visc ? 1 : 0;
  c->split_phase = 0;
  c->launch_stage(*c, sc);
}

void ctx_step(Ctx *c, int n) { ctx_step_scheme(c, n); }

void ctx_norms(Ctx *c, double *out)
{
  const int V = c->V;
  CK(cudaMemsetAsync(c->dred, 0, 3 * 8 * sizeof(double), c->stream));
  const int64_t work = c->plan.neles * c->S;
  const int blocks = grid_for(work, 256);
  {
  ProfScope ps(*c, ZB_K_NORMS);
  if (c->prec == ZB_FP64)
    k_norms<double><<<blocks, 256, 0, c->stream>>>((const double *)c->divF[0], (const double *)c->mets, c->plan.neles,
                                                   c->S, V, c->D * c->D + 1, c->D * c->D, c->dred);
  else
    k_norms<float><<<blocks, 256, 0, c->stream>>>((const float *)c->divF[0], (const float *)c->mets, c->plan.neles,
                                                  c->S, V, c->D * c->D + 1, c->D * c->D, c->dred);
  c->launches++;
  CK(cudaGetLastError());
  }
  double h[24];
  CK(cudaMemcpyAsync(h, c->dred, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const double ndof = (double)c->plan.neles * c->S;
  bool bad = false;
  for (int v = 0; v < V; v++)
  {
    out[v] = h[v] / ndof;
    out[V + v] = h[V + v] / ndof;
    out[2 * V + v] = std::sqrt(h[2 * V + v]) / ndof;
    if (!std::isfinite(h[v]) || !std::isfinite(h[V + v]) || !std::isfinite(h[2 * V + v])) bad = true;
  }
  if (bad) ZB_THROW(ZB_ERR_NONFINITE, "NaN in residual");
}

void ctx_sync(Ctx *c) { CK(cudaStreamSynchronize(c->stream)); }

int64_t ctx_launches(const Ctx *c) { return c->launches; }

void ctx_functionals(Ctx *c, double *out)
{
  const size_t nU = (size_t)c->ntiles * c->S * c->V * TW;
  if (!c->dweights)
  {
    c->dweights = (double *)dalloc(c->S * sizeof(double));
    if (!c->dfun) c->dfun = (double *)dalloc(8 * sizeof(double));
    CK(cudaMemcpyAsync(c->dweights, c->plan.weights_spts.data(), c->S * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
  }
  const bool grad = c->plan.params.viscous != 0;
  if (grad)
  {
    if (!c->dU) c->dU = dalloc(nU * c->D * c->tsz);
    // gradient of the current state: extrapolation + the gradient kernel only
    c->ufp_valid = false;
    ensure_ufp(c);
    StageCfg sc{0, 0, 0, 0};
    sc.want_dU = 1;
    sc.grad_only = 1;
    c->launch_stage(*c, sc);
  }
  CK(cudaMemsetAsync(c->dfun, 0, 4 * sizeof(double), c->stream));
  const int64_t n = c->plan.neles * c->S;
  const double *ref = c->prec == ZB_FP64 ? nullptr : c->dref;
  if (c->prec == ZB_FP64)
    k_functionals<double><<<grid_for(n, 256), 256, 0, c->stream>>>(
        (const double *)c->U, grad ? (const double *)c->dU : nullptr, (const double *)c->mets, c->dweights, ref,
        c->plan.neles, c->S, c->D, c->dfun);
  else
    k_functionals<float><<<grid_for(n, 256), 256, 0, c->stream>>>(
        (const float *)c->U, grad ? (const float *)c->dU : nullptr, (const float *)c->mets, c->dweights, ref,
        c->plan.neles, c->S, c->D, c->dfun);
  c->launches++;
  CK(cudaGetLastError());
  double h[4];
  CK(cudaMemcpyAsync(h, c->dfun, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  out[0] = h[0];
  out[1] = grad ? h[1] : 0.0;
  out[2] = h[2];
}

// acc[i] += x[i]
__global__ void k_accumulate(double *__restrict__ acc, const double *__restrict__ x, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    acc[i] += x[i];
}

// tile-layout geometry adjoint -> the reference layouts of zb_plan_get
static void geo_to_reference(Ctx *c, const double *dm, const double *dg, double *inv_jaco_bar, double *jaco_det_bar,
                             double *norm_bar, double *dA_bar)
{
  const int S = c->S, Fp = c->Fp, D = c->D, NM = D * D + 1;
  const int64_t E = c->plan.neles;
  std::vector<double> hm((size_t)c->ntiles * S * NM * TW), hg((size_t)c->ntiles * Fp * (D + 1) * TW);
  CK(cudaMemcpyAsync(hm.data(), dm, hm.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(hg.data(), dg, hg.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int64_t e = 0; e < E; e++)
  {
    const int64_t t = e / TW;
    const int l = (int)(e % TW);
    for (int sp = 0; sp < S; sp++)
    {
      for (int d1 = 0; d1 < D; d1++)
        for (int d2 = 0; d2 < D; d2++)
          inv_jaco_bar[(((size_t)d1 * S + sp) * D + d2) * E + e] = hm[(((size_t)t * S + sp) * NM + d1 * D + d2) * TW + l];
      jaco_det_bar[(size_t)sp * E + e] = hm[(((size_t)t * S + sp) * NM + D * D) * TW + l];
    }
    for (int f = 0; f < Fp; f++)
    {
      for (int d = 0; d < D; d++)
        norm_bar[((size_t)f * D + d) * E + e] = hg[(((size_t)t * Fp + f) * (D + 1) + d) * TW + l];
      dA_bar[(size_t)f * E + e] = hg[(((size_t)t * Fp + f) * (D + 1) + D) * TW + l];
    }
  }
}

void ctx_geometry_adjoint_get(Ctx *c, double *inv_jaco_bar, double *jaco_det_bar, double *norm_bar, double *dA_bar,
                              int reset)
{
  if (!c->mbar_acc) ZB_THROW(ZB_ERR_ARG, "no geometry adjoint has been accumulated");
  geo_to_reference(c, c->mbar_acc, c->gbar_acc, inv_jaco_bar, jaco_det_bar, norm_bar, dA_bar);
  if (reset)
  {
    const int NM = c->D * c->D + 1;
    CK(cudaMemsetAsync(c->mbar_acc, 0, (size_t)c->ntiles * c->S * NM * TW * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->gbar_acc, 0, (size_t)c->ntiles * c->Fp * (c->D + 1) * TW * sizeof(double), c->stream));
  }
}

static void ensure_adjoint_buffers(Ctx *c)
{
  if (c->prec != ZB_FP64) ZB_THROW(ZB_ERR_UNSUPPORTED, "the adjoint is built for the plain FP64 form only");
  if (!c->launch_vjp)
    ZB_THROW(ZB_ERR_UNSUPPORTED, "no adjoint kernels for ndims=" + std::to_string(c->D) + " P=" + std::to_string(c->N - 1));
  const size_t nU = (size_t)c->ntiles * c->S * c->V * TW;
  const size_t nF = (size_t)c->ntiles * c->Fp * c->V * TW;
  if (!c->lam)
  {
    c->lam = (double *)dalloc(nU * sizeof(double));
    c->Ubar = (double *)dalloc(nU * sizeof(double));
    c->Lfp = (double *)dalloc(nF * sizeof(double));
    c->Ubfp = (double *)dalloc(nF * sizeof(double));
    c->pbar = (double *)dalloc((size_t)c->ntiles * 5 * sizeof(double));
    if (c->plan.params.viscous)
    {
      c->dUbfp = (double *)dalloc(nF * c->D * sizeof(double));
      c->UCb = (double *)dalloc(nF * sizeof(double));
      c->Ubx = (double *)dalloc(nF * sizeof(double));
    }
  }
}

// The adjoint of the residual at the context's current state for the weight
// already in c->lam (tile layout), into c->Ubar; optionally the free-stream
// adjoint (`params`: per tile in c->pbar, and with param_bar also summed over
// tiles on the host) and the geometry adjoint (c->mbar / c->gbar, added to
// the device sums with `accumulate`).  The geometry adjoint of the viscous
// form reads this state's forward viscous normal flux from c->Fvn: computed
// here unless `fvn_ready` says the caller has put it there.
static void vjp_tiles(Ctx *c, bool params, double *param_bar, bool geo, bool accumulate, bool fvn_ready = false)
{
  // linearisation point: the current state and its traces
  c->ufp_valid = false;
  ensure_ufp(c);
  const int NM = c->D * c->D + 1;
  if (geo)
  {
    if (!c->mbar)
    {
      c->mbar = (double *)dalloc((size_t)c->ntiles * c->S * NM * TW * sizeof(double));
      c->gbar = (double *)dalloc((size_t)c->ntiles * c->Fp * (c->D + 1) * TW * sizeof(double));
      c->nbx = (double *)dalloc((size_t)c->ntiles * c->Fp * c->D * TW * sizeof(double));
    }
    // the face values need the forward viscous normal fluxes of this state
    // (residual register 0 is overwritten with this state's residual)
    if (c->plan.params.viscous && !fvn_ready)
    {
      StageCfg sc{0, 0, 0, 0};
      c->need_fvn = true;
      c->launch_stage(*c, sc);
      c->need_fvn = false;
    }
  }
  c->launch_vjp(*c, params || param_bar, geo);
  if (accumulate)
  {
    const size_t nm = (size_t)c->ntiles * c->S * NM * TW, ng = (size_t)c->ntiles * c->Fp * (c->D + 1) * TW;
    if (!c->mbar_acc)
    {
      c->mbar_acc = (double *)dalloc(nm * sizeof(double));
      c->gbar_acc = (double *)dalloc(ng * sizeof(double));
      CK(cudaMemsetAsync(c->mbar_acc, 0, nm * sizeof(double), c->stream));
      CK(cudaMemsetAsync(c->gbar_acc, 0, ng * sizeof(double), c->stream));
    }
    k_accumulate<<<grid_for((int64_t)nm, 256), 256, 0, c->stream>>>(c->mbar_acc, c->mbar, (int64_t)nm);
    k_accumulate<<<grid_for((int64_t)ng, 256), 256, 0, c->stream>>>(c->gbar_acc, c->gbar, (int64_t)ng);
    c->launches += 2;
    CK(cudaGetLastError());
  }
  if (param_bar)
  {
    std::vector<double> h((size_t)c->ntiles * 5);
    CK(cudaMemcpyAsync(h.data(), c->pbar, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // fixed-order sum over tiles of the real elements (padded lanes repeat element 0)
    for (int k = 0; k < 5; k++) param_bar[k] = 0.0;
    for (int64_t t = 0; t < c->ntiles; t++)
      for (int k = 0; k < 5; k++) param_bar[k] += h[(size_t)t * 5 + k];
  }
}

void ctx_vjp(Ctx *c, const double *lam, double *Ubar, int64_t ss, int64_t vs, int64_t es, int where,
             double *param_bar, double *inv_jaco_bar, double *jaco_det_bar, double *norm_bar, double *dA_bar,
             bool accumulate)
{
  const bool geo_out = inv_jaco_bar || jaco_det_bar || norm_bar || dA_bar;
  if (geo_out && !(inv_jaco_bar && jaco_det_bar && norm_bar && dA_bar))
    ZB_THROW(ZB_ERR_ARG, "the geometry adjoint needs all four output arrays");
  const bool geo = geo_out || accumulate;
  ensure_adjoint_buffers(c);
  if (!lam || !Ubar) ZB_THROW(ZB_ERR_ARG, "null adjoint buffer");
  const size_t ext = extent(c, ss, vs, es, c->S);
  const double *src = stage_in(c, lam, ext, where);
  {
    const int64_t work = c->ntiles * c->S * c->V * TW;
    ProfScope ps(*c, ZB_K_TO_TILES);
    k_to_tiles<double><<<grid_for(work, 256), 256, 0, c->stream>>>(src, c->lam, nullptr, nullptr, c->plan.neles,
                                                                     c->ntiles, c->S, c->V, ss, vs, es);
    c->launches++;
    CK(cudaGetLastError());
  }
  vjp_tiles(c, param_bar != nullptr, param_bar, geo, accumulate);
  from_tiles(c, c->Ubar, nullptr, nullptr, Ubar, ss, vs, es, where);
  if (geo_out) geo_to_reference(c, c->mbar, c->gbar, inv_jaco_bar, jaco_det_bar, norm_bar, dA_bar);
}

// ---------------------------------------------------------------------------
// reverse of one RK44 step (tile layout, FP64)
// ---------------------------------------------------------------------------

// out = a - (c * (1/|J|)) * r per point (the RK stage update)
__global__ void k_stage_state(double *__restrict__ out, const double *__restrict__ a, const double *__restrict__ r,
                              const double *__restrict__ mets, double c, int64_t ntiles, int S, int V, int NM, int DD)
{
  const int64_t total = ntiles * S * V * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int64_t ps = i / ((int64_t)TW * V);
    const double inv = 1.0 / mets[(ps * NM + DD) * TW + l];
    out[i] = a[i] - c * inv * r[i];
  }
}

// lam = cb * (1/|J|) * ubar1 [+ ca * (1/|J|) * ubs]: the stage residual's
// adjoint weight (cb = -b_s dt, ca = -a_s dt)
__global__ void k_stage_weight(double *__restrict__ lam, const double *__restrict__ ubar1,
                               const double *__restrict__ ubs, const double *__restrict__ mets, double cb, double ca,
                               int64_t ntiles, int S, int V, int NM, int DD)
{
  const int64_t total = ntiles * S * V * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int64_t ps = i / ((int64_t)TW * V);
    const double inv = 1.0 / mets[(ps * NM + DD) * TW + l];
    double w = cb * inv * ubar1[i];
    if (ubs) w = w + ca * inv * ubs[i];
    lam[i] = w;
  }
}

// |J| part of the geometry adjoint from the update's 1/|J|:
// acc(|J|) += c * sum_v x_v y_v / |J|^2, and acc(U) += u (state adjoint sum)
__global__ void k_det_adjoint(double *__restrict__ mbar_acc, const double *__restrict__ x,
                              const double *__restrict__ y, const double *__restrict__ mets, double c, int64_t ntiles,
                              int S, int V, int NM, int DD)
{
  const int64_t total = ntiles * S * TW;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(i % TW);
    const int64_t ps = i / TW;  // tile * S + s
    const double det = mets[(ps * NM + DD) * TW + l];
    const double inv = 1.0 / det;
    double acc = 0.0;
    for (int v = 0; v < V; v++) acc += x[(ps * V + v) * TW + l] * y[(ps * V + v) * TW + l];
    mbar_acc[(ps * NM + DD) * TW + l] += c * acc * (inv * inv);
  }
}

__global__ void k_add(double *__restrict__ a, const double *__restrict__ b, int64_t n)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] += b[i];
}

void ctx_rk_step_vjp(Ctx *c, const double *U0, const double *Ubar1, double *Ubar0, int64_t ss, int64_t vs,
                     int64_t es, int where, double *param_bar, bool geometry)
{
  if (!U0 || !Ubar1 || !Ubar0) ZB_THROW(ZB_ERR_ARG, "null state or adjoint buffer");
  if (c->nstages != 4) ZB_THROW(ZB_ERR_UNSUPPORTED, "the step adjoint is built for RK44");
  if (c->use_dt_dev || c->use_dt_ele)
    ZB_THROW(ZB_ERR_UNSUPPORTED, "the step adjoint takes the fixed step of set_dt (dt_type 0)");
  ensure_adjoint_buffers(c);
  const int64_t nU = c->ntiles * c->S * c->V * TW;
  const int S = c->S, V = c->V, NM = c->D * c->D + 1, DD = c->D * c->D;
  const unsigned grid = grid_for(nU, 256);
  if (!c->rkv)
  {
    // stage states 0..3, stage residuals 0..3, the end state's adjoint, one
    // stage adjoint and the running result, in the tile layout; the
    // free-stream adjoint per tile summed over the stages
    c->rkv = (double *)dalloc(((size_t)11 * nU + (size_t)c->ntiles * 5) * sizeof(double));
  }
  double *pb_acc = c->rkv + (size_t)11 * nU;
  // the geometry adjoint of the viscous form needs each stage's forward
  // viscous normal flux: kept from the forward sweep
  const bool keep_fvn = geometry && c->plan.params.viscous;
  const size_t nF = (size_t)c->ntiles * c->Fp * V * TW;
  if (keep_fvn && !c->rkfvn) c->rkfvn = (double *)dalloc(4 * nF * sizeof(double));
  double *Us[4], *Rs[4];
  for (int s = 0; s < 4; s++)
  {
    Us[s] = c->rkv + (size_t)s * nU;
    Rs[s] = c->rkv + (size_t)(4 + s) * nU;
  }
  double *ub1 = c->rkv + (size_t)8 * nU, *ubs = c->rkv + (size_t)9 * nU, *ub0 = c->rkv + (size_t)10 * nU;
  const double dt = c->dt;
  // inputs to the tile layout
  {
    const size_t ext = extent(c, ss, vs, es, c->S);
    const double *src = stage_in(c, U0, ext, where);
    k_to_tiles<double><<<grid, 256, 0, c->stream>>>(src, Us[0], nullptr, nullptr, c->plan.neles, c->ntiles, S, V, ss,
                                                    vs, es);
    src = stage_in(c, Ubar1, ext, where);
    k_to_tiles<double><<<grid, 256, 0, c->stream>>>(src, ub1, nullptr, nullptr, c->plan.neles, c->ntiles, S, V, ss,
                                                    vs, es);
    c->launches += 2;
    CK(cudaGetLastError());
  }
  // forward: the stage states and residuals (FRSolver::step_RK's stages)
  for (int s = 0; s < 4; s++)
  {
    CK(cudaMemcpyAsync(c->U, Us[s], (size_t)nU * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    c->ufp_valid = false;
    ensure_ufp(c);
    StageCfg sc{0, 0, 0, 0};
    c->need_fvn = keep_fvn;
    c->launch_stage(*c, sc);
    c->need_fvn = false;
    CK(cudaMemcpyAsync(Rs[s], c->divF[0], (size_t)nU * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (keep_fvn)
      CK(cudaMemcpyAsync(c->rkfvn + s * nF, c->Fvn, nF * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (s < 3)
    {
      k_stage_state<<<grid, 256, 0, c->stream>>>(Us[s + 1], Us[0], Rs[s], (const double *)c->mets, kRkAlpha[s] * dt,
                                                 c->ntiles, S, V, NM, DD);
      c->launches++;
      CK(cudaGetLastError());
    }
  }
  // reverse: Ubar0 = Ubar1 + sum_s (dR_s/dU_s)^T lam_s with the stage weights
  // lam_s = -b_s dt/|J| Ubar1 - a_s dt/|J| Ubar_{s+1}
  CK(cudaMemcpyAsync(ub0, ub1, (size_t)nU * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (param_bar) CK(cudaMemsetAsync(pb_acc, 0, (size_t)c->ntiles * 5 * sizeof(double), c->stream));
  for (int s = 3; s >= 0; s--)
  {
    k_stage_weight<<<grid, 256, 0, c->stream>>>(c->lam, ub1, s < 3 ? ubs : nullptr, (const double *)c->mets,
                                                -kRkBeta[s] * dt, s < 3 ? -kRkAlpha[s] * dt : 0.0, c->ntiles, S, V,
                                                NM, DD);
    c->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->U, Us[s], (size_t)nU * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (keep_fvn)
      CK(cudaMemcpyAsync(c->Fvn, c->rkfvn + s * nF, nF * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    vjp_tiles(c, param_bar != nullptr, nullptr, geometry, geometry, keep_fvn);
    if (param_bar)
    {
      k_accumulate<<<grid_for(c->ntiles * 5, 256), 256, 0, c->stream>>>(pb_acc, c->pbar, c->ntiles * 5);
      c->launches++;
      CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(ubs, c->Ubar, (size_t)nU * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    k_add<<<grid, 256, 0, c->stream>>>(ub0, ubs, nU);
    c->launches++;
    CK(cudaGetLastError());
    if (geometry && s > 0)
    {
      // U_s = U_0 - a_{s-1} dt R_{s-1} / |J|
      k_det_adjoint<<<grid_for(c->ntiles * S * TW, 256), 256, 0, c->stream>>>(
          c->mbar_acc, ubs, Rs[s - 1], (const double *)c->mets, kRkAlpha[s - 1] * dt, c->ntiles, S, V, NM, DD);
      c->launches++;
      CK(cudaGetLastError());
    }
  }
  if (geometry)
  {
    // U_1 = U_0 - dt sum_s b_s R_s / |J|
    for (int s = 0; s < 4; s++)
    {
      k_det_adjoint<<<grid_for(c->ntiles * S * TW, 256), 256, 0, c->stream>>>(
          c->mbar_acc, ub1, Rs[s], (const double *)c->mets, kRkBeta[s] * dt, c->ntiles, S, V, NM, DD);
      c->launches++;
      CK(cudaGetLastError());
    }
  }
  if (param_bar)
  {
    // one read of the stage-summed tiles, summed over tiles in a fixed order
    std::vector<double> h((size_t)c->ntiles * 5);
    CK(cudaMemcpyAsync(h.data(), pb_acc, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double pacc[5] = {0, 0, 0, 0, 0};
    for (int64_t t = 0; t < c->ntiles; t++)
      for (int k = 0; k < 5; k++) pacc[k] += h[(size_t)t * 5 + k];
    for (int k = 0; k < 5; k++) param_bar[k] += pacc[k];
  }
  from_tiles(c, ub0, nullptr, nullptr, Ubar0, ss, vs, es, where);
  c->ufp_valid = false;
}

void ctx_wall_force(Ctx *c, double *out)
{
  const Plan &p = c->plan;
  const int S = c->S, Fp = c->Fp, D = c->D;
  if (!c->dwall)
  {
    // dense extrapolation (FP64), face quadrature weights, flux point coordinates
    std::vector<double> oppE, oD, oDf, oDv, oDvf;
    p.dense_operators(oppE, oD, oDf, oDv, oDvf);
    std::vector<double> fw((size_t)Fp);
    const std::vector<double> w1 = gauss_legendre_weights(c->N);
    for (int f = 0; f < Fp; f++)
    {
      if (p.etype == ET_HEX)
      {
        const int r = f % (c->N * c->N);
        fw[f] = w1[r / c->N] * w1[r % c->N];
      }
      else
        fw[f] = w1[f % c->N];
    }
    const size_t nE = oppE.size(), nC = p.coord_fpts.size();
    c->dwall = (double *)dalloc((nE + Fp + nC + 8) * sizeof(double));
    CK(cudaMemcpy(c->dwall, oppE.data(), nE * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->dwall + nE, fw.data(), Fp * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->dwall + nE + Fp, p.coord_fpts.data(), nC * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (!c->dfun) c->dfun = (double *)dalloc(8 * sizeof(double));
  const bool visc = p.params.viscous != 0;
  const size_t nU = (size_t)c->ntiles * S * c->V * TW;
  if (visc)
  {
    if (!c->dU) c->dU = dalloc(nU * D * c->tsz);
    c->ufp_valid = false;
    ensure_ufp(c);
    StageCfg sc{0, 0, 0, 0};
    sc.want_dU = 1;
    sc.grad_only = 1;
    c->launch_stage(*c, sc);
  }
  else
    ensure_ufp(c);
  CK(cudaMemsetAsync(c->dfun, 0, 8 * sizeof(double), c->stream));
  WallArgs w;
  w.gamma = p.params.gamma;
  w.mu = p.params.mu;
  w.rt = p.params.rt;
  w.c_sth = p.params.c_sth;
  w.fix_vis = p.params.fix_vis;
  w.viscous = visc ? 1 : 0;
  w.D = D;
  w.S = S;
  w.Fp = Fp;
  w.ntiles = c->ntiles;
  w.neles = p.neles;
  const double *dE = c->dwall, *fw = c->dwall + (size_t)Fp * S, *cfp = fw + Fp;
  const double *ref = c->prec == ZB_FP64 ? nullptr : c->dref;
  const int blocks = grid_for(c->ntiles * Fp * TW, 256);
  {
    ProfScope ps(*c, ZB_K_FUNCTIONALS);
    if (c->prec == ZB_FP64)
      k_wall_force<double><<<blocks, 256, 0, c->stream>>>((const double *)c->Ufp[c->cur], (const double *)c->dU,
                                                          (const double *)c->fgeo, c->nbr, dE, fw, cfp, ref, w, c->dfun);
    else
      k_wall_force<float><<<blocks, 256, 0, c->stream>>>((const float *)c->Ufp[c->cur], (const float *)c->dU,
                                                         (const float *)c->fgeo, c->nbr, dE, fw, cfp, ref, w, c->dfun);
    c->launches++;
    CK(cudaGetLastError());
  }
  double h[8];
  CK(cudaMemcpyAsync(h, c->dfun, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 6; k++) out[k] = h[k];
}

void ctx_profile_enable(Ctx *c, int on)
{
  CK(cudaStreamSynchronize(c->stream));
  c->profiling = (on != 0);
}

void ctx_profile_read(Ctx *c, double *ms, int64_t *count)
{
  CK(cudaStreamSynchronize(c->stream));
  for (auto &r : c->recs)
  {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, r.a, r.b));
    c->prof_ms[r.kid] += t;
    c->prof_n[r.kid] += 1;
    c->pool.push_back(r.a);
    c->pool.push_back(r.b);
  }
  c->recs.clear();
  for (int k = 0; k < ZB_NKERNELS; k++)
  {
    if (ms) ms[k] = c->prof_ms[k];
    if (count) count[k] = c->prof_n[k];
    c->prof_ms[k] = 0.0;
    c->prof_n[k] = 0;
  }
}

}  // namespace zb
