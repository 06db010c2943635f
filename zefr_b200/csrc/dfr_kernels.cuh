// Tensor-product DFR residual kernels for quadrilaterals (D = 2) and
// hexahedra (D = 3) of order P = N - 1, templated on the arithmetic type.
//
// Data layout in HBM is tile-major structure-of-arrays: TW consecutive
// elements form a tile and every per-element array is stored as
//   [tile][point][component][TW]
// so one CTA reads its whole tile as one contiguous chunk and, inside it, the
// TW elements of a (point, component) pair sit in one 32- or 64-byte run.
//
// Reference: the residual is FRSolver::compute_residual (src/solver.cpp:1494-
// 1645).  Its dense operator products (src/elements.cpp:1337-1501) are applied
// here as line operators: every nonzero of oppE, oppD, oppD_fpts, oppDiv and
// oppDiv_fpts for quads and hexes lies on the line of points through a
// solution point (src/elements.cpp:592-655), and the nonzeros are summed in the
// same order as the reference's row-major products.
#pragma once

#include <cstdint>

#include "physics.cuh"

namespace zb {
namespace dev {

constexpr int TW = 8;  // elements per tile

template <int D, int N>
struct Shape
{
  static constexpr int S = (D == 2) ? N * N : N * N * N;
  static constexpr int NF = (D == 2) ? N : N * N;  // flux points per face
  static constexpr int Fp = 2 * D * NF;
  static constexpr int V = D + 2;
  static constexpr int NM = D * D + 1;  // adjugate entries + |J|
  static constexpr int NT = (D == 2) ? ((S * TW <= 128) ? 128 : 256) : 256;
};

// Prefetch `bytes` (a multiple of 16, 16-byte aligned) from global memory
// into L2 without waiting: one bulk request, no registers held
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <typename T, int N>
struct LineOpsT
{
  T Dm[N * N];  // Dm[i*N+m] = l'_{m+1}(x_i) on [-1, x, 1]
  T Em[N], Ep[N], Dbm[N], Dbp[N];
};

// T: storage type of state, traces and metrics; A: arithmetic type.
template <typename T, typename A>
struct Args
{
  const T *U;        // [tile][S][V][TW]
  const T *Ufp;      // [tile][Fp][V][TW] extrapolated state (this stage)
  T *Ufp_next;       // extrapolation of the updated state (next stage)
  const T *mets;     // [tile][S][NM][TW]: adj[d1][d2] (reference inv_jaco), |J|
  const T *fgeo;     // [tile][Fp][D+1][TW]: face unit normal (left side), own dA
  const int *nbr;    // [tile][Fp][TW]: 2*partner+slot, or -1-bc
  T *divF;           // [tile][S][V][TW] residual of this stage
  A *divF_vol;       // NS: volume part of the residual (arithmetic type: it cancels
                     // against the surface part)
  T *Fvn;            // NS: viscous normal flux at own flux points
  const double *dt_dev;  // optional: the step as computed on the device (CFL, global)
  const double *dt_ele;  // optional: per-element step [tile * TW + lane] (CFL, local)
  T *Fcom;           // NS hexahedra, LDG beta = +-1/2, optional: common flux (convective
                     // + viscous, not dA-scaled) at the flux points whose side supplies
                     // the LDG normal flux; the partner reads it from there
  T *dU_out;         // NS, optional: physical gradient [tile][D][S][V][TW] (the
                     // reference keeps it in dU_spts for diagnostics)
  // RK update fused into the last kernel of a stage
  int rk_mode;       // 0: none; 1: U = U_ini - a dt/|J| divF; 2: final combination
  int save_ini;      // stage 0: write U_ini = U before updating
  int extrap_next;   // write Ufp_next from the updated state
  int nprev;         // final stage: number of earlier divF registers
  T *Uout;           // updated state (may alias U)
  T *U_ini;          // RK start state
  T *Ucomp;          // compensated-summation remainder (final stage, nullptr = off)
  const T *divF_prev[6];
  A rk_coef[6];      // a_s (mode 1: [0]) or b_s (mode 2)
  A dt;
  int64_t ntiles;
  const A *dops;     // triangles: dense operators (TriOps layout), nullptr otherwise
  int *err;          // tensor-core kernels: set when a completion wait gave up
  Phys<A> ph;
};

// Flux point f -> normal dimension, side (-1/+1), first spt of its line and
// stride along the line (orderings of src/quads.cpp:108-148, src/hexas.cpp:148-205).
template <int D, int N>
__device__ __forceinline__ void fpt_line(int f, int &dim, int &side, int &base, int &stride)
{
  if (D == 2)
  {
    const int face = f / N, j = f % N;
    switch (face)
    {
      case 0: dim = 1; side = -1; base = j; stride = N; break;
      case 1: dim = 0; side = 1; base = N * j; stride = 1; break;
      case 2: dim = 1; side = 1; base = N - 1 - j; stride = N; break;
      default: dim = 0; side = -1; base = N * (N - 1 - j); stride = 1; break;
    }
  }
  else
  {
    constexpr int N2 = N * N;
    const int face = f / N2, r = f % N2, j = r / N, k = r % N;
    switch (face)
    {
      case 0: dim = 2; side = -1; base = k + N * j; stride = N2; break;
      case 1: dim = 2; side = 1; base = (N - 1 - k) + N * j; stride = N2; break;
      case 2: dim = 0; side = -1; base = N * k + N2 * j; stride = 1; break;
      case 3: dim = 0; side = 1; base = N * (N - 1 - k) + N2 * j; stride = 1; break;
      case 4: dim = 1; side = -1; base = (N - 1 - k) + N2 * j; stride = N; break;
      default: dim = 1; side = 1; base = k + N2 * j; stride = N; break;
    }
  }
}

// Solution point s: line coordinate along dimension d and the flux points at
// the -/+ ends of that line.
template <int D, int N>
__device__ __forceinline__ void spt_ends(int s, int d, int &i, int &fm, int &fp)
{
  if (D == 2)
  {
    const int ix = s % N, iy = s / N;
    if (d == 0) { i = ix; fm = 3 * N + (N - 1 - iy); fp = N + iy; }
    else { i = iy; fm = ix; fp = 2 * N + (N - 1 - ix); }
  }
  else
  {
    constexpr int N2 = N * N;
    const int ix = s % N, iy = (s / N) % N, iz = s / N2;
    if (d == 0) { i = ix; fm = 2 * N2 + iz * N + iy; fp = 3 * N2 + iz * N + (N - 1 - iy); }
    else if (d == 1) { i = iy; fm = 4 * N2 + iz * N + (N - 1 - ix); fp = 5 * N2 + iz * N + ix; }
    else { i = iz; fm = iy * N + ix; fp = N2 + iy * N + (N - 1 - ix); }
  }
}

template <int N>
__device__ __forceinline__ constexpr int pow_n(int d)
{
  return d == 0 ? 1 : (d == 1 ? N : N * N);
}

// Face id -> (dimension, side) for summing surface terms in flux point order.
template <int D>
__device__ __forceinline__ void face_dim_side(int face, int &dim, int &side)
{
  if (D == 2)
  {
    dim = (face == 0 || face == 2) ? 1 : 0;
    side = (face == 1 || face == 2) ? 1 : -1;
  }
  else
  {
    dim = (face < 2) ? 2 : (face < 4 ? 0 : 1);
    side = (face % 2 == 0) ? -1 : 1;
  }
}

template <typename A, int N>
__device__ __forceinline__ void load_ops(A *sops, const LineOpsT<A, N> &ops, int tid, int nth)
{
  const A *src = reinterpret_cast<const A *>(&ops);
  constexpr int n = N * N + 4 * N;
  for (int i = tid; i < n; i += nth) sops[i] = src[i];
}

template <typename A, int N>
__device__ __forceinline__ void load_ops(A *sops, const LineOpsT<A, N> &ops)
{
  load_ops<A, N>(sops, ops, threadIdx.x, blockDim.x);
}

// Barrier of the threads running one tile: the whole block (bar == 0) or a
// warp-aligned group of nth threads on named barrier `bar` (batched stages).
__device__ __forceinline__ void group_sync(int bar, int nth)
{
  if (bar == 0)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nth) : "memory");
}

// Shared-memory views of the line operators
template <typename A, int N>
struct SOps
{
  const A *Dm, *Em, *Ep, *Dbm, *Dbp;
  __device__ SOps(const A *p) : Dm(p), Em(p + N * N), Ep(p + N * N + N), Dbm(p + N * N + 2 * N), Dbp(p + N * N + 3 * N) {}
};

// extrapolate component v of the tile state in smem (layout [S][V][TW]) to flux point f
template <typename A, int D, int N>
__device__ __forceinline__ A extrap_smem(const A *sX, const SOps<A, N> &o, int f, int v, int l, int nv)
{
  int dim, side, base, stride;
  fpt_line<D, N>(f, dim, side, base, stride);
  const A *E = side < 0 ? o.Em : o.Ep;
  A acc = E[0] * sX[((base)*nv + v) * TW + l];
#pragma unroll
  for (int m = 1; m < N; m++) acc += E[m] * sX[((base + m * stride) * nv + v) * TW + l];
  return acc;
}

// read the neighbour's copy of a [tile][Fp][V][TW] array
template <typename T, typename A, int V>
__device__ __forceinline__ void gather_fpt(const T *src, int pidx, A out[V])
{
  const int64_t row = (int64_t)(pidx / TW) * V;
  const int lane = pidx % TW;
#pragma unroll
  for (int v = 0; v < V; v++) out[v] = (A)src[(row + v) * TW + lane];
}

// ---------------------------------------------------------------------------
// Extrapolate the state to flux points: U_fpts = oppE U_spts (src/elements.cpp:1337-1360)
// ---------------------------------------------------------------------------
template <typename T, typename A, int D, int N>
__global__ void __launch_bounds__(256) k_extrap(const T *__restrict__ U, T *__restrict__ Ufp, int64_t ntiles,
                                                const __grid_constant__ LineOpsT<A, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V;
  const int64_t total = ntiles * Fp * TW;
  for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(gid % TW);
    const int f = (int)((gid / TW) % Fp);
    const int64_t tile = gid / ((int64_t)TW * Fp);
    int dim, side, base, stride;
    fpt_line<D, N>(f, dim, side, base, stride);
    const T *Ut = U + tile * (int64_t)S * V * TW;
    T *out = Ufp + (tile * Fp + f) * (int64_t)V * TW;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = (side < 0 ? ops.Em[0] : ops.Ep[0]) * (A)Ut[((base)*V + v) * TW + l];
#pragma unroll
      for (int m = 1; m < N; m++)
        acc += (side < 0 ? ops.Em[m] : ops.Ep[m]) * (A)Ut[((base + m * stride) * V + v) * TW + l];
      out[v * TW + l] = (T)acc;
    }
  }
}

// ---------------------------------------------------------------------------
// Common convective flux at one own flux point (Rusanov or Roe) plus ghost
// states on boundaries; returns the outward, dA-scaled own-side value in Fc
// (src/faces.cpp:1243-1364, 1616-1640).  For viscous runs the LDG part is
// added by the caller.
// ---------------------------------------------------------------------------
template <typename T, typename A, int D>
__device__ __forceinline__ void conv_common(const Args<T, A> &a, const A Uo[D + 2], const A Un[D + 2], int code,
                                            const A n[D], A UL[D + 2], A UR[D + 2], A UB[D + 2], A F[D + 2])
{
  if (code >= 0)
  {
    const int slot = code & 1;
#pragma unroll
    for (int v = 0; v < D + 2; v++)
    {
      UL[v] = slot ? Un[v] : Uo[v];
      UR[v] = slot ? Uo[v] : Un[v];
      UB[v] = UR[v];
    }
  }
  else
  {
    A Ua[D + 2], URa[D + 2], UBa[D + 2];
#pragma unroll
    for (int v = 0; v < D + 2; v++) UL[v] = Uo[v];
    to_abs<A, D>(Uo, Ua, a.ph);
    ghost_state<A, D>(-code - 1, Ua, n, URa, UBa, a.ph);
    to_stored<A, D>(URa, UR, a.ph);
    to_stored<A, D>(UBa, UB, a.ph);
  }
  if (a.ph.fconv == 2)
    roe<A, D>(UL, UR, n, F, a.ph);
  else
    rusanov<A, D>(UL, UR, n, F, a.ph);
}

// time step of element (tile, lane): per element, device-computed or fixed
template <typename T, typename A>
__device__ __forceinline__ A step_dt(const Args<T, A> &a, int64_t tile, int l)
{
  if (a.dt_ele) return (A)a.dt_ele[tile * TW + l];
  if (a.dt_dev) return (A)a.dt_dev[0];
  return a.dt;
}

// ---------------------------------------------------------------------------
// Store the residual of one point and apply the optional RK update
// (src/solver.cpp:2916-2937, 3040-3094).
// ---------------------------------------------------------------------------
template <typename T, typename A, int S, int V, int NM>
__device__ __forceinline__ void store_rk(const Args<T, A> &a, int64_t tile, int s, int l, const A res[V], A *sUnew)
{
  constexpr int D = NM == 5 ? 2 : 3, MAXPREV = 3;
  const int64_t base = (tile * S + s) * (int64_t)V * TW;
  if (a.rk_mode == 0)
  {
#pragma unroll
    for (int v = 0; v < V; v++) a.divF[base + v * TW + l] = res[v];
    return;
  }
  // every load of the point before the first store: a load cannot move above
  // a store that may alias it, so interleaving them serialises the accesses
  const A detJ = a.mets[((tile * S + s) * NM + D * D) * TW + l];
  const A dtv = step_dt(a, tile, l);
  const bool fast = a.rk_mode == 1 || a.nprev <= MAXPREV;
  A u_ini[V], prev[MAXPREV][V], comp[V];
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    const int64_t idx = base + v * TW + l;
    u_ini[v] = a.save_ini ? (A)a.U[idx] : (A)a.U_ini[idx];
    comp[v] = (a.rk_mode == 2 && a.Ucomp) ? (A)a.Ucomp[idx] : A(0);
  }
  if (a.rk_mode == 2 && fast)
  {
#pragma unroll
    for (int st = 0; st < MAXPREV; st++)
      if (st < a.nprev)
      {
#pragma unroll
        for (int v = 0; v < V; v++) prev[st][v] = (A)a.divF_prev[st][base + v * TW + l];
      }
  }
#pragma unroll
  for (int v = 0; v < V; v++) a.divF[base + v * TW + l] = res[v];
#pragma unroll
  for (int v = 0; v < V; v++)
  {
    const int64_t idx = base + v * TW + l;
    if (a.save_ini) a.U_ini[idx] = u_ini[v];
    A unew;
    if (a.rk_mode == 1)
      unew = u_ini[v] - a.rk_coef[0] * dtv / detJ * res[v];
    else if (a.Ucomp)
    {
      // Kahan-compensated accumulation of the step increment; the
      // remainder includes the rounding of the stored state
      A delta = A(0);
      if (fast)
      {
#pragma unroll
        for (int st = 0; st < MAXPREV; st++)
          if (st < a.nprev) delta -= a.rk_coef[st] * dtv / detJ * prev[st][v];
      }
      else
        for (int st = 0; st < a.nprev; st++) delta -= a.rk_coef[st] * dtv / detJ * (A)a.divF_prev[st][idx];
      delta -= a.rk_coef[a.nprev] * dtv / detJ * res[v];
      const A y = delta - comp[v];
      unew = (A)(T)(u_ini[v] + y);
      a.Ucomp[idx] = (T)((unew - u_ini[v]) - y);
    }
    else
    {
      // reference order: U = U_ini; U -= b_s dt/|J| divF_s for s = 0..
      unew = u_ini[v];
      if (fast)
      {
#pragma unroll
        for (int st = 0; st < MAXPREV; st++)
          if (st < a.nprev) unew -= a.rk_coef[st] * dtv / detJ * prev[st][v];
      }
      else
        for (int st = 0; st < a.nprev; st++) unew -= a.rk_coef[st] * dtv / detJ * a.divF_prev[st][idx];
      unew -= a.rk_coef[a.nprev] * dtv / detJ * res[v];
    }
    a.Uout[idx] = unew;
    if (sUnew) sUnew[(s * V + v) * TW + l] = (A)(T)unew;  // the state as stored
  }
}

// ---------------------------------------------------------------------------
// Final per-point residual: volume part + surface correction, then optional
// RK update (src/solver.cpp:2916-2937, 3040-3094).
// ---------------------------------------------------------------------------
template <typename T, typename A, int D, int N>
__device__ __forceinline__ void finish_point(const Args<T, A> &a, int64_t tile, int s, int l, const A vol[D + 2],
                                             const A *sFc, const SOps<A, N> &o, A *sUnew)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, V = G::V, NM = G::NM;
  A surf[V];
#pragma unroll
  for (int v = 0; v < V; v++) surf[v] = A(0);
  // surface terms in ascending flux point order = ascending face order
#pragma unroll
  for (int face = 0; face < 2 * D; face++)
  {
    int dim, side;
    face_dim_side<D>(face, dim, side);
    int i, fm, fp;
    spt_ends<D, N>(s, dim, i, fm, fp);
    const int f = side < 0 ? fm : fp;
    const A c = side < 0 ? -o.Dbm[i] : o.Dbp[i];
#pragma unroll
    for (int v = 0; v < V; v++) surf[v] += c * sFc[(f * V + v) * TW + l];
  }
  A res[V];
#pragma unroll
  for (int v = 0; v < V; v++) res[v] = vol[v] + surf[v];
  store_rk<T, A, S, V, NM>(a, tile, s, l, res, sUnew);
}

template <typename T, typename A, int D, int N>
__device__ __forceinline__ void extrap_next_tile(const Args<T, A> &a, int64_t tile, const A *sUnew, const SOps<A, N> &o,
                                                 int tid, int nth)
{
  using G = Shape<D, N>;
  constexpr int Fp = G::Fp, V = G::V;
  for (int it = tid; it < Fp * TW; it += nth)
  {
    const int f = it / TW, l = it % TW;
    T *out = a.Ufp_next + (tile * Fp + f) * (int64_t)V * TW;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW + l] = extrap_smem<A, D, N>(sUnew, o, f, v, l, V);
  }
}

template <typename T, typename A, int D, int N>
__device__ __forceinline__ void extrap_next_tile(const Args<T, A> &a, int64_t tile, const A *sUnew, const SOps<A, N> &o)
{
  extrap_next_tile<T, A, D, N>(a, tile, sUnew, o, threadIdx.x, blockDim.x);
}

// ---------------------------------------------------------------------------
// Euler: volume flux, common flux and divergence of one tile in one kernel.
// ---------------------------------------------------------------------------
template <typename T, typename A, int D, int N>
__device__ __forceinline__ void euler_tile(const Args<T, A> &a, const LineOpsT<A, N> &ops, int64_t tile,
                                           unsigned char *smem_raw, int tid, int nth, int bar)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, NM = G::NM;
  A *sU = reinterpret_cast<A *>(smem_raw);
  A *sF = sU + S * V * TW;
  A *sFc = sF + D * S * V * TW;
  A *sops = sFc + Fp * V * TW;
  load_ops<A, N>(sops, ops, tid, nth);
  {
    const T *src = a.U + tile * (int64_t)S * V * TW;
    for (int i = tid; i < S * V * TW; i += nth) sU[i] = src[i];
  }
  group_sync(bar, nth);
  SOps<A, N> o(sops);
  // transformed volume flux F~ = adj F (src/elements.cpp:1588-1699)
  for (int it = tid; it < S * TW; it += nth)
  {
    const int s = it / TW, l = it % TW;
    A U[V], F[V][D], P, Pp;
#pragma unroll
    for (int v = 0; v < V; v++) U[v] = sU[(s * V + v) * TW + l];
    flux_conv_stored<A, D>(U, F, P, Pp, a.ph);
    const T *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    A adj[D][D];
#pragma unroll
    for (int d1 = 0; d1 < D; d1++)
#pragma unroll
      for (int d2 = 0; d2 < D; d2++) adj[d1][d2] = m[(d1 * D + d2) * TW];
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d1 = 0; d1 < D; d1++)
      {
        A t = F[v][0] * adj[d1][0];
#pragma unroll
        for (int d2 = 1; d2 < D; d2++) t += F[v][d2] * adj[d1][d2];
        sF[((d1 * S + s) * V + v) * TW + l] = t;
      }
  }
  // common flux at the tile's flux points
  for (int it = tid; it < Fp * TW; it += nth)
  {
    const int f = it / TW, l = it % TW;
    const int64_t fi = (tile * Fp + f) * (int64_t)TW + l;
    const int code = a.nbr[fi];
    A n[D], dA;
    const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    dA = g[D * TW];
    A Uo[V], Un[V], UL[V], UR[V], UB[V], Fc[V];
    const T *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0) gather_fpt<T, A, V>(a.Ufp, code >> 1, Un);
    conv_common<T, A, D>(a, Uo, Un, code, n, UL, UR, UB, Fc);
    const bool right = (code >= 0) && (code & 1);
#pragma unroll
    for (int v = 0; v < V; v++) sFc[(f * V + v) * TW + l] = right ? -Fc[v] * dA : Fc[v] * dA;
  }
  group_sync(bar, nth);
  for (int it = tid; it < S * TW; it += nth)
  {
    const int s = it / TW, l = it % TW;
    A vol[V];
#pragma unroll
    for (int v = 0; v < V; v++) vol[v] = A(0);
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
        const A c = o.Dm[i * N + m];
#pragma unroll
        for (int v = 0; v < V; v++) vol[v] += c * sF[((d * S + b + m * st) * V + v) * TW + l];
      }
    }
    finish_point<T, A, D, N>(a, tile, s, l, vol, sFc, o, a.extrap_next ? sU : nullptr);
  }
  if (a.extrap_next)
  {
    group_sync(bar, nth);
    extrap_next_tile<T, A, D, N>(a, tile, sU, o, tid, nth);
  }
}


// Shared memory of euler_tile (elements of the arithmetic type)
template <int D, int N>
constexpr int euler_smem_elems()
{
  return (Shape<D, N>::S * Shape<D, N>::V * (1 + D) + Shape<D, N>::Fp * Shape<D, N>::V) * TW + N * N + 4 * N;
}

template <typename T, typename A, int D, int N>
__global__ void __launch_bounds__(Shape<D, N>::NT) k_euler(const __grid_constant__ Args<T, A> a,
                                                                   const __grid_constant__ LineOpsT<A, N> ops)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  euler_tile<T, A, D, N>(a, ops, tile, smem_raw, threadIdx.x, blockDim.x, 0);
}

// ---------------------------------------------------------------------------
// Navier-Stokes kernel 1: common solution, corrected gradient, viscous normal
// flux at own flux points, volume flux and its divergence
// (src/solver.cpp:1540-1600; src/elements.cpp:1393-1447, 1588-1699;
//  src/faces.cpp:1366-1474, 508-710).
// ---------------------------------------------------------------------------
template <typename T, typename A, int D, int N>
__global__ void __launch_bounds__(Shape<D, N>::NT, (D == 3) ? 2 : 1) k_ns_grad(const __grid_constant__ Args<T, A> a,
                                                                                       const __grid_constant__ LineOpsT<A, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V, NM = G::NM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sU = reinterpret_cast<A *>(smem_raw);
  A *sUC = sU + S * V * TW;
  A *sdU = sUC + Fp * V * TW;  // [D][S][V][TW]: physical gradient, then F~
  A *sops = sdU + D * S * V * TW;
  load_ops<A, N>(sops, ops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  {
    const T *src = a.U + tile * (int64_t)S * V * TW;
    for (int i = threadIdx.x; i < S * V * TW; i += blockDim.x) sU[i] = src[i];
  }
  __syncthreads();
  SOps<A, N> o(sops);
  const A beta = a.ph.ldg_b;
  // common solution at own flux points (LDG, flip_beta = 1)
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int64_t fi = (tile * Fp + f) * (int64_t)TW + l;
    const int code = a.nbr[fi];
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
#pragma unroll
    for (int v = 0; v < V; v++) sUC[(f * V + v) * TW + l] = UC[v];
  }
  __syncthreads();
  // corrected reference gradient, transformed to physical space
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A tdU[V][D];
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
        A acc = A(0);
#pragma unroll
        for (int m = 0; m < N; m++) acc += o.Dm[i * N + m] * sU[((b + m * st) * V + v) * TW + l];
        const A cm = o.Dbm[i] * sUC[(fm * V + v) * TW + l];
        const A cp = o.Dbp[i] * sUC[(fp * V + v) * TW + l];
        tdU[v][d] = acc + ((fm < fp) ? (cm + cp) : (cp + cm));
      }
    }
    const T *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    A adj[D][D];
#pragma unroll
    for (int d1 = 0; d1 < D; d1++)
#pragma unroll
      for (int d2 = 0; d2 < D; d2++) adj[d1][d2] = m[(d1 * D + d2) * TW];
    const A inv_det = A(1) / m[D * D * TW];
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d1 = 0; d1 < D; d1++)
      {
        A g = tdU[v][0] * adj[0][d1];
#pragma unroll
        for (int d2 = 1; d2 < D; d2++) g += tdU[v][d2] * adj[d2][d1];
        sdU[((d1 * S + s) * V + v) * TW + l] = g * inv_det;
      }
  }
  __syncthreads();
  if (a.dU_out)
  {
    T *g = a.dU_out + tile * (int64_t)D * S * V * TW;
    for (int i = threadIdx.x; i < D * S * V * TW; i += blockDim.x) g[i] = (T)sdU[i];
  }
  // viscous normal flux at own flux points (own side; boundaries: prescribed side)
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int64_t fi = (tile * Fp + f) * (int64_t)TW + l;
    const int code = a.nbr[fi];
    if (code >= 0 && ((beta == A(0.5) && (code & 1)) || (beta == A(-0.5) && !(code & 1)))) continue;
    A n[D];
    const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    A Uf[V], dUf[V][D], Fn[V];
    const T *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      Uf[v] = uo[v * TW];
#pragma unroll
      for (int d = 0; d < D; d++) dUf[v][d] = extrap_smem<A, D, N>(sdU + d * S * V * TW, o, f, v, l, V);
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
  // flux at solution points, transformed: F~ = adj (F_conv + F_visc)
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A U[V], dU[V][D], F[V][D];
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      U[v] = sU[(s * V + v) * TW + l];
#pragma unroll
      for (int d = 0; d < D; d++) dU[v][d] = sdU[((d * S + s) * V + v) * TW + l];
    }
    A P, Pp, Ua[V];
    flux_conv_stored<A, D>(U, F, P, Pp, a.ph);
    to_abs<A, D>(U, Ua, a.ph);
    flux_visc_add<A, D>(Ua, dU, F, a.ph);
    const T *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    A adj[D][D];
#pragma unroll
    for (int d1 = 0; d1 < D; d1++)
#pragma unroll
      for (int d2 = 0; d2 < D; d2++) adj[d1][d2] = m[(d1 * D + d2) * TW];
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d1 = 0; d1 < D; d1++)
      {
        A t = F[v][0] * adj[d1][0];
#pragma unroll
        for (int d2 = 1; d2 < D; d2++) t += F[v][d2] * adj[d1][d2];
        sdU[((d1 * S + s) * V + v) * TW + l] = t;
      }
  }
  __syncthreads();
  // volume divergence
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A vol[V];
#pragma unroll
    for (int v = 0; v < V; v++) vol[v] = A(0);
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
        const A c = o.Dm[i * N + m];
#pragma unroll
        for (int v = 0; v < V; v++) vol[v] += c * sdU[((d * S + b + m * st) * V + v) * TW + l];
      }
    }
    A *out = a.divF_vol + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = vol[v];
  }
}

// ---------------------------------------------------------------------------
// Navier-Stokes kernel 2: convective + LDG common flux, surface correction,
// optional RK update (src/faces.cpp:1476-1614; src/elements.cpp:1476-1501).
// ---------------------------------------------------------------------------
template <typename T, typename A, int D, int N>
__global__ void __launch_bounds__(Shape<D, N>::NT) k_ns_face(const __grid_constant__ Args<T, A> a,
                                                                     const __grid_constant__ LineOpsT<A, N> ops)
{
  using G = Shape<D, N>;
  constexpr int S = G::S, Fp = G::Fp, V = G::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A *sFc = reinterpret_cast<A *>(smem_raw);
  A *sUnew = sFc + Fp * V * TW;
  A *sops = sUnew + S * V * TW;
  load_ops<A, N>(sops, ops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  __syncthreads();
  SOps<A, N> o(sops);
  const A beta = a.ph.ldg_b, tau = a.ph.ldg_tau;
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int64_t fi = (tile * Fp + f) * (int64_t)TW + l;
    const int code = a.nbr[fi];
    A n[D], dA;
    const T *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    dA = g[D * TW];
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
      // own side is left when slot == 0
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
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      A acc = right ? -Fc[v] * dA : Fc[v] * dA;
      if (right)
        acc -= Fv[v] * dA;
      else
        acc += Fv[v] * dA;
      sFc[(f * V + v) * TW + l] = acc;
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    A vol[V];
    const A *dv = a.divF_vol + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) vol[v] = dv[v * TW];
    finish_point<T, A, D, N>(a, tile, s, l, vol, sFc, o, a.extrap_next ? sUnew : nullptr);
  }
  if (a.extrap_next)
  {
    __syncthreads();
    extrap_next_tile<T, A, D, N>(a, tile, sUnew, o);
  }
}

}  // namespace dev
}  // namespace zb
