// Flux-reconstruction residual kernels for triangles of order P = N - 1 with
// dense operators (S = N(N+1)/2 solution points, Fp = 3N flux points).
//
// Same tile-major layout, face codes and pointwise physics as the tensor-
// product kernels (dfr_kernels.cuh); the operators are the reference's dense
// oppE, oppD, oppD_fpts, oppDiv, oppDiv_fpts (src/elements.cpp:656-744),
// applied as the reference's products apply them (src/elements.cpp:
// 1337-1501): one sum over the whole row in ascending column order, the
// flux-point (correction) sum added after the solution-point sum.
#pragma once

#include "dfr_kernels.cuh"

namespace zb {
namespace dev {

template <int N>
struct TriShape
{
  static constexpr int D = 2, V = 4, NM = 5;
  static constexpr int S = N * (N + 1) / 2;
  static constexpr int Fp = 3 * N;
  static constexpr int NT = 128;
  // dense operator block: oppE [Fp][S], oppD [D][S][S], oppD_fpts [D][S][Fp],
  // oppDiv [S][D*S], oppDiv_fpts [S][Fp]
  static constexpr int OE = 0, OD = OE + Fp * S, ODF = OD + D * S * S, ODV = ODF + D * S * Fp,
                       ODVF = ODV + S * D * S, NOPS = ODVF + S * Fp;
  // the tile arrays that follow the operator block in shared memory start on
  // a 16-byte boundary
  static constexpr int OPS_PAD = ((NOPS + 3) / 4) * 4;
  static_assert(V == 4, "the shared tile arrays hold four variables per point");
};

// Shared-memory tile arrays of these kernels (states, common solutions,
// gradients, fluxes) keep the variables of one (point, element) in 16-byte
// groups, [P][4/W][TW][W] with W = 16 / sizeof(A): FP32 holds all four
// variables in one group, FP64 two groups of two.  One 16-byte load per group
// fetches a point's variables where the global [P][V][TW] order takes four
// loads, and the eight elements of a warp's point read 128 contiguous bytes
// per group (no bank conflicts).
template <typename A>
struct TVec
{
  static constexpr int W = 16 / (int)sizeof(A), G = 4 / W;
};

// offset of (point p, element l, variable v)
template <typename A>
__device__ __forceinline__ int tix(int p, int l, int v)
{
  return ((p * TVec<A>::G + v / TVec<A>::W) * TW + l) * TVec<A>::W + v % TVec<A>::W;
}

// offset of (point p, element l)'s first group
template <typename A>
__device__ __forceinline__ int tvl(int p, int l)
{
  return tix<A>(p, l, 0);
}

__device__ __forceinline__ void ld4(const float *p, float x[4])
{
  const float4 q = *reinterpret_cast<const float4 *>(p);
  x[0] = q.x;
  x[1] = q.y;
  x[2] = q.z;
  x[3] = q.w;
}

// the second group of two doubles sits TW groups further on
__device__ __forceinline__ void ld4(const double *p, double x[4])
{
  const double2 a = *reinterpret_cast<const double2 *>(p);
  const double2 b = *reinterpret_cast<const double2 *>(p + 2 * TW);
  x[0] = a.x;
  x[1] = a.y;
  x[2] = b.x;
  x[3] = b.y;
}

__device__ __forceinline__ void st4(float *p, const float x[4])
{
  *reinterpret_cast<float4 *>(p) = make_float4(x[0], x[1], x[2], x[3]);
}

__device__ __forceinline__ void st4(double *p, const double x[4])
{
  *reinterpret_cast<double2 *>(p) = make_double2(x[0], x[1]);
  *reinterpret_cast<double2 *>(p + 2 * TW) = make_double2(x[2], x[3]);
}

// global [S][V][TW] tile -> the shared layout above
template <typename T, typename A, int S>
__device__ __forceinline__ void load_tile_vl(const T *__restrict__ src, A *dst)
{
  for (int i = threadIdx.x; i < S * 4 * TW; i += blockDim.x)
  {
    const int l = i % TW, v = (i / TW) % 4, p = i / (4 * TW);
    dst[tix<A>(p, l, v)] = src[i];
  }
}

// X_v(f) = sum_s E[f][s] Y_v(s) for the four variables of a shared tile array
template <typename A, int N>
__device__ __forceinline__ void tri_extrap4(const A *sY, const A *E, int f, int l, A out[4])
{
  constexpr int S = TriShape<N>::S;
#pragma unroll
  for (int v = 0; v < 4; v++) out[v] = A(0);
#pragma unroll
  for (int t = 0; t < S; t++)
  {
    A x[4];
    ld4(sY + tvl<A>(t, l), x);
    const A e = E[f * S + t];
#pragma unroll
    for (int v = 0; v < 4; v++) out[v] += e * x[v];
  }
}

template <typename A, int N>
__device__ __forceinline__ void load_tri_ops(A *sops, const A *g)
{
  for (int i = threadIdx.x; i < TriShape<N>::NOPS; i += blockDim.x) sops[i] = g[i];
}

// X(f) = sum_s E[f][s] Y(s) for component v of a tile array in smem [S][nv][TW]
// (the RK-updated state, as store_rk leaves it)
template <typename A, int N>
__device__ __forceinline__ A tri_extrap(const A *sY, const A *E, int f, int v, int l, int nv)
{
  constexpr int S = TriShape<N>::S;
  A acc = A(0);
#pragma unroll
  for (int t = 0; t < S; t++) acc += E[f * S + t] * sY[(t * nv + v) * TW + l];
  return acc;
}

template <typename T, typename A, int N>
__global__ void __launch_bounds__(128) k_tri_extrap(const T *__restrict__ U, T *__restrict__ Ufp, int64_t ntiles,
                                                    const A *__restrict__ dops)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V;
  __shared__ A sE[Fp * S];
  for (int i = threadIdx.x; i < Fp * S; i += blockDim.x) sE[i] = dops[G::OE + i];
  __syncthreads();
  const int64_t total = ntiles * Fp * TW;
  for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(gid % TW);
    const int f = (int)((gid / TW) % Fp);
    const int64_t tile = gid / ((int64_t)TW * Fp);
    const T *Ut = U + tile * (int64_t)S * V * TW;
    T *out = Ufp + (tile * Fp + f) * (int64_t)V * TW;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = A(0);
#pragma unroll
      for (int t = 0; t < S; t++) acc += sE[f * S + t] * (A)Ut[(t * V + v) * TW + l];
      out[v * TW + l] = (T)acc;
    }
  }
}

template <typename T, typename A, int N>
__device__ __forceinline__ void tri_extrap_next(const Args<T, A> &a, int64_t tile, const A *sUnew, const A *E)
{
  using G = TriShape<N>;
  constexpr int Fp = G::Fp, V = G::V;
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    T *out = a.Ufp_next + (tile * Fp + f) * (int64_t)V * TW;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW + l] = (T)tri_extrap<A, N>(sUnew, E, f, v, l, V);
  }
}

// transformed flux F~_d = adj[d][.] . F at solution point s into sF [D*S] points
template <typename T, typename A>
__device__ __forceinline__ void tri_transform(const Args<T, A> &a, int64_t tile, int s, int l, const A F[4][2],
                                              A *sF, int S)
{
  const T *m = a.mets + (tile * S + s) * (int64_t)5 * TW + l;
  A adj[2][2];
#pragma unroll
  for (int d1 = 0; d1 < 2; d1++)
#pragma unroll
    for (int d2 = 0; d2 < 2; d2++) adj[d1][d2] = m[(d1 * 2 + d2) * TW];
#pragma unroll
  for (int d1 = 0; d1 < 2; d1++)
  {
    A Ft[4];
#pragma unroll
    for (int v = 0; v < 4; v++) Ft[v] = F[v][0] * adj[d1][0] + F[v][1] * adj[d1][1];
    st4(sF + tvl<A>(d1 * S + s, l), Ft);
  }
}

// divF(s) = sum_k oppDiv[s][k] F~(k) + sum_f oppDiv_fpts[s][f] Fc(f), then store / RK
template <typename T, typename A, int N>
__device__ __forceinline__ void tri_finish(const Args<T, A> &a, int64_t tile, int s, int l, const A *sF,
                                           const A *sFc, const A *ops, A *sUnew, const A *vol_in)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, D = 2;
  A vol[V], surf[V];
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    surf[v] = A(0);
    vol[v] = A(0);
  }
  if (vol_in)
  {
#pragma unroll
    for (int v = 0; v < V; v++) vol[v] = vol_in[v];
  }
  else
  {
    const A *Dv = ops + G::ODV + s * D * S;
#pragma unroll
    for (int k = 0; k < D * S; k++)
    {
      A x[4];
      ld4(sF + tvl<A>(k, l), x);
#pragma unroll
      for (int v = 0; v < V; v++) vol[v] += Dv[k] * x[v];
    }
  }
  const A *Dvf = ops + G::ODVF + s * Fp;
#pragma unroll
  for (int f = 0; f < Fp; f++)
  {
    A x[4];
    ld4(sFc + tvl<A>(f, l), x);
#pragma unroll
    for (int v = 0; v < V; v++) surf[v] += Dvf[f] * x[v];
  }
  A res[V];
#pragma unroll
  for (int v = 0; v < V; v++) res[v] = vol[v] + surf[v];
  store_rk<T, A, S, V, 5>(a, tile, s, l, res, sUnew);
}

// ---------------------------------------------------------------------------
// Euler: volume flux, common flux and divergence of one tile.
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(128) k_tri_euler(const __grid_constant__ Args<T, A> a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, D = 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sops = reinterpret_cast<A *>(smem_raw);
  A *sU = sops + G::OPS_PAD;  // [S] points; then the RK-updated state as store_rk writes it
  A *sF = sU + S * V * TW;
  A *sFc = sF + D * S * V * TW;
  load_tri_ops<A, N>(sops, a.dops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  load_tile_vl<T, A, S>(a.U + tile * (int64_t)S * V * TW, sU);
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A U[V], F[V][D], P, Pp;
    ld4(sU + tvl<A>(s, l), U);
    flux_conv_stored<A, D>(U, F, P, Pp, a.ph);
    tri_transform<T, A>(a, tile, s, l, F, sF, S);
  }
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    A n[D];
    const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    const A dA = g[D * TW];
    A Uo[V], Un[V], UL[V], UR[V], UB[V], Fc[V];
    const T *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0) gather_fpt<T, A, V>(a.Ufp, code >> 1, Un);
    conv_common<T, A, D>(a, Uo, Un, code, n, UL, UR, UB, Fc);
    const bool right = (code >= 0) && (code & 1);
    A out[V];
#pragma unroll
    for (int v = 0; v < V; v++) out[v] = right ? -Fc[v] * dA : Fc[v] * dA;
    st4(sFc + tvl<A>(f, l), out);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    tri_finish<T, A, N>(a, tile, s, l, sF, sFc, sops, a.extrap_next ? sU : nullptr, nullptr);
  }
  if (a.extrap_next)
  {
    __syncthreads();
    tri_extrap_next<T, A, N>(a, tile, sU, sops + G::OE);
  }
}

// ---------------------------------------------------------------------------
// Navier-Stokes kernel 1: LDG common solution, corrected gradient, own viscous
// normal flux, volume flux and its divergence.
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(128) k_tri_ns_grad(const __grid_constant__ Args<T, A> a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, D = 2, NM = 5;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sops = reinterpret_cast<A *>(smem_raw);
  A *sU = sops + G::OPS_PAD;    // [S] points
  A *sUC = sU + S * V * TW;      // [Fp] points
  A *sdU = sUC + Fp * V * TW;    // [D*S] points: physical gradient, then F~
  load_tri_ops<A, N>(sops, a.dops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  load_tile_vl<T, A, S>(a.U + tile * (int64_t)S * V * TW, sU);
  const A beta = a.ph.ldg_b;
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    A Uo[V], UC[V];
    const T *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0)
    {
      A Un[V];
      gather_fpt<T, A, V>(a.Ufp, code >> 1, Un);
      const int slot = code & 1;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        const A ul = slot ? Un[v] : Uo[v];
        const A ur = slot ? Uo[v] : Un[v];
        if (beta == A(0.5))
          UC[v] = ur;
        else if (beta == A(-0.5))
          UC[v] = ul;
        else
          UC[v] = A(0.5) * (ul + ur) - beta * (ul - ur);
      }
    }
    else
    {
      A n[D], Ua[V], URa[V], UBa[V];
      const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
      for (int d = 0; d < D; d++) n[d] = g[d * TW];
      to_abs<A, D>(Uo, Ua, a.ph);
      ghost_state<A, D>(-code - 1, Ua, n, URa, UBa, a.ph);
      to_stored<A, D>(UBa, UC, a.ph);
    }
    st4(sUC + tvl<A>(f, l), UC);
  }
  __syncthreads();
  // gradient: oppD U + oppD_fpts Ucomm, then physical
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A tdU[V][D];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      const A *Dd = sops + G::OD + (d * S + s) * S;
      const A *Df = sops + G::ODF + (d * S + s) * Fp;
      A acc[V], cor[V];
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        acc[v] = A(0);
        cor[v] = A(0);
      }
#pragma unroll
      for (int t = 0; t < S; t++)
      {
        A x[4];
        ld4(sU + tvl<A>(t, l), x);
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] += Dd[t] * x[v];
      }
#pragma unroll
      for (int f = 0; f < Fp; f++)
      {
        A x[4];
        ld4(sUC + tvl<A>(f, l), x);
#pragma unroll
        for (int v = 0; v < V; v++) cor[v] += Df[f] * x[v];
      }
#pragma unroll
      for (int v = 0; v < V; v++) tdU[v][d] = acc[v] + cor[v];
    }
    const T *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    A adj[D][D];
#pragma unroll
    for (int d1 = 0; d1 < D; d1++)
#pragma unroll
      for (int d2 = 0; d2 < D; d2++) adj[d1][d2] = m[(d1 * D + d2) * TW];
    const A inv_det = A(1) / m[D * D * TW];
#pragma unroll
    for (int d1 = 0; d1 < D; d1++)
    {
      A g[V];
#pragma unroll
      for (int v = 0; v < V; v++) g[v] = (tdU[v][0] * adj[0][d1] + tdU[v][1] * adj[1][d1]) * inv_det;
      st4(sdU + tvl<A>(d1 * S + s, l), g);
    }
  }
  __syncthreads();
  if (a.dU_out)
  {
    // back to the global [D][S][V][TW] order
    T *g = a.dU_out + tile * (int64_t)D * S * V * TW;
    for (int i = threadIdx.x; i < D * S * V * TW; i += blockDim.x)
    {
      const int l = i % TW, v = (i / TW) % V, p = i / (V * TW);
      g[i] = (T)sdU[tix<A>(p, l, v)];
    }
  }
  // own viscous normal flux at flux points
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    if (code >= 0 && ((beta == A(0.5) && (code & 1)) || (beta == A(-0.5) && !(code & 1)))) continue;
    A n[D];
    const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    A Uf[V], dUf[V][D], Fn[V];
    const T *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uf[v] = uo[v * TW];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      A x[V];
      tri_extrap4<A, N>(sdU + d * S * V * TW, sops + G::OE, f, l, x);
#pragma unroll
      for (int v = 0; v < V; v++) dUf[v][d] = x[v];
    }
    A Ua[V];
    to_abs<A, D>(Uf, Ua, a.ph);
    if (code >= 0)
      visc_normal<A, D>(Ua, dUf, n, Fn, a.ph);
    else
    {
      A UR[V], UB[V], dUB[V][D];
      ghost_state<A, D>(-code - 1, Ua, n, UR, UB, a.ph);
      ghost_grad<A, D>(-code - 1, Ua, dUf, n, dUB);
      visc_normal<A, D>(UB, dUB, n, Fn, a.ph);
    }
    T *out = a.Fvn + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = Fn[v];
  }
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A U[V], dU[V][D], F[V][D], P, Pp, Ua[V];
    ld4(sU + tvl<A>(s, l), U);
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      A x[V];
      ld4(sdU + tvl<A>(d * S + s, l), x);
#pragma unroll
      for (int v = 0; v < V; v++) dU[v][d] = x[v];
    }
    flux_conv_stored<A, D>(U, F, P, Pp, a.ph);
    to_abs<A, D>(U, Ua, a.ph);
    flux_visc_add<A, D>(Ua, dU, F, a.ph);
    // each thread rewrites only its own point of sdU
    tri_transform<T, A>(a, tile, s, l, F, sdU, S);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A vol[V];
#pragma unroll
    for (int v = 0; v < V; v++) vol[v] = A(0);
    const A *Dv = sops + G::ODV + s * D * S;
#pragma unroll
    for (int k = 0; k < D * S; k++)
    {
      A x[V];
      ld4(sdU + tvl<A>(k, l), x);
#pragma unroll
      for (int v = 0; v < V; v++) vol[v] += Dv[k] * x[v];
    }
    A *out = a.divF_vol + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = vol[v];
  }
}

// ---------------------------------------------------------------------------
// Navier-Stokes kernel 2: convective + LDG common flux, correction, RK.
// ---------------------------------------------------------------------------
template <typename T, typename A, int N>
__global__ void __launch_bounds__(128) k_tri_ns_face(const __grid_constant__ Args<T, A> a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, D = 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sops = reinterpret_cast<A *>(smem_raw);
  A *sFc = sops + G::OPS_PAD;   // [Fp] points
  A *sUnew = sFc + Fp * V * TW;  // RK-updated state as store_rk writes it, [S][V][TW]
  load_tri_ops<A, N>(sops, a.dops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  const A beta = a.ph.ldg_b, tau = a.ph.ldg_tau;
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    A n[D];
    const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    const A dA = g[D * TW];
    A Uo[V], Un[V], UL[V], UR[V], UB[V], Fc[V], Fv[V];
    const T *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0) gather_fpt<T, A, V>(a.Ufp, code >> 1, Un);
    conv_common<T, A, D>(a, Uo, Un, code, n, UL, UR, UB, Fc);
    const T *fvo = a.Fvn + (tile * Fp + f) * (int64_t)V * TW + l;
    if (code >= 0)
    {
      const int slot = code & 1;
      A FnL[V], FnR[V];
      if (beta == A(0.5))
      {
        if (slot == 0)
        {
#pragma unroll
          for (int v = 0; v < V; v++) FnL[v] = fvo[v * TW];
        }
        else
          gather_fpt<T, A, V>(a.Fvn, code >> 1, FnL);
#pragma unroll
        for (int v = 0; v < V; v++) FnR[v] = A(0);
      }
      else if (beta == A(-0.5))
      {
        if (slot == 1)
        {
#pragma unroll
          for (int v = 0; v < V; v++) FnR[v] = fvo[v * TW];
        }
        else
          gather_fpt<T, A, V>(a.Fvn, code >> 1, FnR);
#pragma unroll
        for (int v = 0; v < V; v++) FnL[v] = A(0);
      }
      else
      {
        A Fo[V], Fx[V];
#pragma unroll
        for (int v = 0; v < V; v++) Fo[v] = fvo[v * TW];
        gather_fpt<T, A, V>(a.Fvn, code >> 1, Fx);
#pragma unroll
        for (int v = 0; v < V; v++)
        {
          FnL[v] = slot ? Fx[v] : Fo[v];
          FnR[v] = slot ? Fo[v] : Fx[v];
        }
      }
#pragma unroll
      for (int v = 0; v < V; v++)
        Fv[v] = A(0.5) * (FnL[v] + FnR[v]) + tau * (UL[v] - UR[v]) + beta * (FnL[v] - FnR[v]);
    }
    else
    {
#pragma unroll
      for (int v = 0; v < V; v++) Fv[v] = fvo[v * TW] + tau * (UL[v] - UB[v]);
    }
    const bool right = (code >= 0) && (code & 1);
    A out[V];
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = right ? -Fc[v] * dA : Fc[v] * dA;
      if (right)
        acc -= Fv[v] * dA;
      else
        acc += Fv[v] * dA;
      out[v] = acc;
    }
    st4(sFc + tvl<A>(f, l), out);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A vol[V];
    const A *dv = a.divF_vol + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) vol[v] = dv[v * TW];
    tri_finish<T, A, N>(a, tile, s, l, nullptr, sFc, sops, a.extrap_next ? sUnew : nullptr, vol);
  }
  if (a.extrap_next)
  {
    __syncthreads();
    tri_extrap_next<T, A, N>(a, tile, sUnew, sops + G::OE);
  }
}

}  // namespace dev
}  // namespace zb
