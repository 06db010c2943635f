// Adjoint (vector-Jacobian product) of the triangle residual, plain FP64:
// Ubar = (d divF / d U)^T lam and the free-stream adjoint, for the dense
// flux-reconstruction operators of tri_kernels.cuh (the reference's oppE,
// oppD, oppD_fpts, oppDiv, oppDiv_fpts, src/elements.cpp:656-744, applied
// as in src/elements.cpp:1337-1501).  The reference has no adjoint.
//
// The passes are those of the tensor-product adjoint (adjoint.cuh) with every
// line operator replaced by the transpose of a dense one:
//   lift        Lfp(f)       = sum_s oppDiv_fpts[s][f] lam(s)
//   volume      F~bar_d(t)   = sum_s oppDiv[s][d S + t] lam(s)
//   traces      Ubar(s)     += sum_f oppE[f][s] Ubfp(f)
//   gradient    gbar(s)     += sum_f oppE[f][s] dUbfp(f);  Ubar(s) += sum_d,s' oppD[d][s'][s] tdUbar_d(s')
//   common sol. UCbar(f)     = sum_d,s' oppD_fpts[d][s'][f] tdUbar_d(s')
// with the pointwise reverse-mode functions (flux, Riemann, LDG, boundary
// states) shared with the tensor-product adjoint.  The operators sit in shared
// memory; the tile arrays are [P][V][TW].
#pragma once

#include "adjoint.cuh"
#include "tri_kernels.cuh"

namespace zb {
namespace dev {

// summed weight on the common flux of own flux point f (tensor-product form:
// face_weight) for the triangle flux-point count
template <int N>
__device__ __forceinline__ void tri_face_weight(const AdjArgs &a, int64_t tile, int f, int l, int code, double n[2],
                                                double w[4])
{
  constexpr int Fp = TriShape<N>::Fp, V = 4, D = 2;
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

// Lfp = oppDiv_fpts^T lam, one thread per (flux point, element)
template <int N>
__global__ void __launch_bounds__(128) k_tri_adj_lift(const __grid_constant__ AdjArgs a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = 4;
  __shared__ double sDvf[S * Fp];
  for (int i = threadIdx.x; i < S * Fp; i += blockDim.x) sDvf[i] = a.dops[G::ODVF + i];
  __syncthreads();
  const int64_t total = a.ntiles * Fp * TW;
  for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (int64_t)gridDim.x * blockDim.x)
  {
    const int l = (int)(gid % TW);
    const int f = (int)((gid / TW) % Fp);
    const int64_t tile = gid / ((int64_t)TW * Fp);
    const double *Lt = a.lam + tile * (int64_t)S * V * TW;
    double *out = a.Lfp + (tile * Fp + f) * (int64_t)V * TW;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double acc = 0.0;
#pragma unroll
      for (int s = 0; s < S; s++) acc += sDvf[s * Fp + f] * Lt[(s * V + v) * TW + l];
      out[v * TW + l] = acc;
    }
  }
}

// weight on the physical flux at solution point t (volume term): F~bar_d(t)
// from oppDiv^T lam, then Fb[v][k] = sum_d adj[d][k] F~bar_d[v]
template <int N>
__device__ __forceinline__ void tri_vol_weight(const AdjArgs &a, const double *ops, int64_t tile, int t, int l,
                                               double Fb[4][2])
{
  using G = TriShape<N>;
  constexpr int S = G::S, V = 4, D = 2, NM = 5;
  const double *Lt = a.lam + tile * (int64_t)S * V * TW;
  double Ft[D][V];
#pragma unroll
  for (int d = 0; d < D; d++)
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double acc = 0.0;
#pragma unroll
      for (int s = 0; s < S; s++) acc += ops[G::ODV + s * D * S + d * S + t] * Lt[(s * V + v) * TW + l];
      Ft[d][v] = acc;
    }
  const double *mt = a.mets + (tile * S + t) * (int64_t)NM * TW + l;
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

// Euler: volume flux, face fluxes, transposed extrapolation
template <int N>
__global__ void __launch_bounds__(128) k_tri_adj_euler(const __grid_constant__ AdjArgs a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = 4, D = 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sops = reinterpret_cast<double *>(smem_raw);
  double *sUb = sops + G::OPS_PAD;  // [S][V][TW]
  double *sUbfp = sUb + S * V * TW;  // [Fp][V][TW]
  load_tri_ops<double, N>(sops, a.dops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  __syncthreads();
  double pb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double Fb[V][D], U[V], Ub[V];
    tri_vol_weight<N>(a, sops, tile, s, l, Fb);
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
  }
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    double n[D], w[V], Uo[V], Ub[V];
    tri_face_weight<N>(a, tile, f, l, code, n, w);
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
    for (int f = 0; f < Fp; f++)
    {
      const double e = sops[G::OE + f * S + s];
#pragma unroll
      for (int v = 0; v < V; v++) acc[v] += e * sUbfp[(f * V + v) * TW + l];
    }
    double *out = a.Ubar + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = acc[v];
  }
}

// Navier-Stokes pass 1: recompute the common solution and the gradient, the
// adjoint of the volume flux, of the face fluxes and of the gradient; writes
// the solution-point part of Ubar, the trace adjoint (Ubfp, and the partner's
// Riemann part in Ubx) and the common-solution adjoint (UCb)
template <int N>
__global__ void __launch_bounds__(128) k_tri_adj_ns1(const __grid_constant__ AdjArgs a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = 4, D = 2, NM = 5;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sops = reinterpret_cast<double *>(smem_raw);
  double *sU = sops + G::OPS_PAD;   // [S][V][TW]
  double *sUC = sU + S * V * TW;     // [Fp][V][TW] common solution
  double *sdU = sUC + Fp * V * TW;   // [D][S][V][TW] physical gradient
  double *sUb = sdU + D * S * V * TW;  // [S][V][TW] volume-flux U adjoint
  double *sG = sUb + S * V * TW;     // [D][S][V][TW] gradient adjoint
  load_tri_ops<double, N>(sops, a.dops);
  const int64_t tile = blockIdx.x;
  if (tile >= a.ntiles) return;
  const double beta = a.ph.ldg_b, tau = a.ph.ldg_tau;
  double pb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  {
    const double *src = a.U + tile * (int64_t)S * V * TW;
    for (int i = threadIdx.x; i < S * V * TW; i += blockDim.x) sU[i] = src[i];
  }
  // common solution (as k_tri_ns_grad)
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    double Uo[V], UC[V];
    const double *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0)
    {
      double Un[V];
      gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
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
  // physical gradient (as k_tri_ns_grad: solution-point sum, then the
  // flux-point sum, added)
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double tdU[V][D];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      const double *Dd = sops + G::OD + (d * S + s) * S;
      const double *Df = sops + G::ODF + (d * S + s) * Fp;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        double acc = 0.0, cor = 0.0;
#pragma unroll
        for (int t = 0; t < S; t++) acc += Dd[t] * sU[(t * V + v) * TW + l];
#pragma unroll
        for (int f = 0; f < Fp; f++) cor += Df[f] * sUC[(f * V + v) * TW + l];
        tdU[v][d] = acc + cor;
      }
    }
    const double *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    const double inv_det = 1.0 / m[D * D * TW];
#pragma unroll
    for (int d1 = 0; d1 < D; d1++)
#pragma unroll
      for (int v = 0; v < V; v++)
        sdU[((d1 * S + s) * V + v) * TW + l] =
            (tdU[v][0] * m[(0 * D + d1) * TW] + tdU[v][1] * m[(1 * D + d1) * TW]) * inv_det;
  }
  __syncthreads();
  // adjoint of the face fluxes at own flux points
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    double n[D], w[V], Uo[V], dUo[V][D], Ub[V], dUb[V][D];
    tri_face_weight<N>(a, tile, f, l, code, n, w);
    const double *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      Uo[v] = uo[v * TW];
      Ub[v] = 0.0;
#pragma unroll
      for (int d = 0; d < D; d++)
      {
        double acc = 0.0;
#pragma unroll
        for (int t = 0; t < S; t++) acc += sops[G::OE + f * S + t] * sdU[((d * S + t) * V + v) * TW + l];
        dUo[v][d] = acc;
        dUb[v][d] = 0.0;
      }
    }
    if (code >= 0)
    {
      const bool own_left = !(code & 1);
      if (own_left)
      {
        // one reverse sweep of the shared Riemann flux gives both sides'
        // adjoints: keep the left's, leave the right's at the partner
        double Un[V], bL[V], bR[V];
        gather_fpt<double, double, V>(a.Ufp, code >> 1, Un);
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
    double *ub = a.Ubfp + (tile * Fp + f) * (int64_t)V * TW + l;
    double *dub = a.dUbfp + (tile * Fp + f) * (int64_t)V * D * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      ub[v * TW] = Ub[v];
#pragma unroll
      for (int d = 0; d < D; d++) dub[(v * D + d) * TW] = dUb[v][d];
    }
  }
  // adjoint of the volume flux: U and gradient parts (sUb, sG are distinct
  // from sdU, which the face pass above reads)
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double Fb[V][D], U[V], dU[V][D], Ub[V], dUb[V][D];
    tri_vol_weight<N>(a, sops, tile, s, l, Fb);
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
  }
  __syncthreads();
  // gradient adjoint: the transposed extrapolation of the gradient-trace
  // adjoint, then to the reference gradient: tdUb[v][d2] = sum_d1 adj[d2][d1]
  // gb[v][d1] / |J| (written over sG in place, own point only)
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double g[V][D];
#pragma unroll
    for (int v = 0; v < V; v++)
#pragma unroll
      for (int d = 0; d < D; d++) g[v][d] = sG[((d * S + s) * V + v) * TW + l];
#pragma unroll
    for (int f = 0; f < Fp; f++)
    {
      const double e = sops[G::OE + f * S + s];
      const double *dub = a.dUbfp + (tile * Fp + f) * (int64_t)V * D * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++)
#pragma unroll
        for (int d = 0; d < D; d++) g[v][d] += e * dub[(v * D + d) * TW];
    }
    const double *m = a.mets + (tile * S + s) * (int64_t)NM * TW + l;
    const double inv_det = 1.0 / m[D * D * TW];
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
  // U part of the reference gradient: Ub(s) += sum_d,s' oppD[d][s'][s] tdUb_d(s')
  for (int it = threadIdx.x; it < S * TW; it += blockDim.x)
  {
    const int s = it / TW, l = it % TW;
    double acc[V];
#pragma unroll
    for (int v = 0; v < V; v++) acc[v] = sUb[(s * V + v) * TW + l];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int sp = 0; sp < S; sp++)
      {
        const double c = sops[G::OD + (d * S + sp) * S + s];
#pragma unroll
        for (int v = 0; v < V; v++) acc[v] += c * sG[((d * S + sp) * V + v) * TW + l];
      }
    double *out = a.Ubar + (tile * S + s) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = acc[v];
  }
  // common-solution part: UCb(f) = sum_d,s' oppD_fpts[d][s'][f] tdUb_d(s')
  for (int it = threadIdx.x; it < Fp * TW; it += blockDim.x)
  {
    const int f = it / TW, l = it % TW;
    double ucb[V];
#pragma unroll
    for (int v = 0; v < V; v++)
    {
      double acc = 0.0;
#pragma unroll
      for (int d = 0; d < D; d++)
#pragma unroll
        for (int sp = 0; sp < S; sp++)
          acc += sops[G::ODF + (d * S + sp) * Fp + f] * sG[((d * S + sp) * V + v) * TW + l];
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
#pragma unroll
      for (int v = 0; v < V; v++) ub[v * TW] += Ub[v];
    }
  }
  if (a.pbar) block_sum5(pb, a.pbar + tile * 5);
}

// Navier-Stokes pass 2: both sides' common-solution adjoints and the
// partner's Riemann part reach the own trace; transposed extrapolation
template <int N>
__global__ void __launch_bounds__(128) k_tri_adj_ns2(const __grid_constant__ AdjArgs a)
{
  using G = TriShape<N>;
  constexpr int S = G::S, Fp = G::Fp, V = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *sE = reinterpret_cast<double *>(smem_raw);  // oppE [Fp][S]
  double *sUbfp = sE + ((Fp * S + 1) / 2) * 2;          // [Fp][V][TW]
  for (int i = threadIdx.x; i < Fp * S; i += blockDim.x) sE[i] = a.dops[G::OE + i];
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
      const double *ux = a.Ubx + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
      for (int v = 0; v < V; v++) Ub[v] += ux[v * TW];
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
    for (int f = 0; f < Fp; f++)
    {
      const double e = sE[f * S + s];
#pragma unroll
      for (int v = 0; v < V; v++) acc[v] += e * sUbfp[(f * V + v) * TW + l];
    }
#pragma unroll
    for (int v = 0; v < V; v++) out[v * TW] = acc[v];
  }
}

template <int N>
constexpr size_t tri_adj_ns1_smem()
{
  using G = TriShape<N>;
  return ((size_t)G::OPS_PAD + (size_t)(G::S * 4 + G::Fp * 4 + 2 * G::S * 4 + G::S * 4 + 2 * G::S * 4) * TW) *
         sizeof(double);
}

template <int N>
constexpr size_t tri_adj_euler_smem()
{
  using G = TriShape<N>;
  return ((size_t)G::OPS_PAD + (size_t)(G::S * 4 + G::Fp * 4) * TW) * sizeof(double);
}

template <int N>
constexpr size_t tri_adj_ns2_smem()
{
  using G = TriShape<N>;
  return ((size_t)((G::Fp * G::S + 1) / 2) * 2 + (size_t)G::Fp * 4 * TW) * sizeof(double);
}

}  // namespace dev
}  // namespace zb
