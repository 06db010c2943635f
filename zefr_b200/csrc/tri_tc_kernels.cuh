// Triangle Navier-Stokes gradient kernel of the mixed form with its dense
// operator products on the tensor pipe (tcgen05, TF32x3 split products, FP32
// accumulation in tensor memory).  Same results as k_tri_ns_grad<float>
// (tri_kernels.cuh) up to FP32 rounding: the products are the reference's
// oppD U + oppD_fpts Ucomm (src/elements.cpp:1393-1447), oppE dU
// (1362-1391) and oppDiv F (1449-1474).
//
// One CTA takes four tiles (32 elements).  The 128 (element, variable) pairs
// are the M = 128 rows of each MMA, row r = 32 q + 4 l + v for tile q,
// element l, variable v, so the TMEM lane a thread of warp q reads holds one
// (element, variable) and its values at every output point.  The pointwise
// physics (LDG common solution, viscous normal flux, volume flux) keeps the
// one-thread-per-(point, element) mapping of the CUDA-core kernel and meets
// the products through the shared tile arrays, whose [P][TW][4] order puts
// the 32 rows of a warp's lane quarter at 32 consecutive words.
//
// Products (K-major operands, no swizzle, tc_ops.cuh):
//   1. reference gradient   D1[r][d S + s] = sum_k A1[r][k] B1[d S + s][k],
//      A1 = [U | Ucomm] (K = S + Fp), B1 = [oppD_d | oppD_fpts_d]
//   2. gradient at flux points, per dimension d:  D2_d[r][f] = sum_s
//      dU_d[r][s] oppE[f][s]
//   3. volume divergence    D3[r][s] = sum_k F~[r][k] oppDiv[s][k], K = D S
#pragma once

#include "tc_ops.cuh"
#include "tri_kernels.cuh"

namespace zb {
namespace dev {

template <int N>
struct TriTc
{
  using G = TriShape<N>;
  static constexpr int S = G::S, Fp = G::Fp, V = 4, D = 2;
  static constexpr int TILES = 4, ROWS = TILES * TW * V;  // 128
  static constexpr int NT = 256;                          // threads per CTA
  static constexpr int r8(int x) { return (x + 7) / 8 * 8; }
  static constexpr int r16(int x) { return (x + 15) / 16 * 16; }
  static constexpr int K1 = r8(S + Fp), N1 = r16(D * S);
  static constexpr int K2 = r8(S), N2 = r16(Fp);
  static constexpr int K3 = r8(D * S), N3 = r16(S);
  // tensor-memory columns: D1 | D2_0 | D2_1 | D3
  static constexpr int C1 = 0, C2 = N1, C3 = N1 + 2 * N2, NCOLS_USED = N1 + 2 * N2 + N3;
  static constexpr int TMEM_COLS = NCOLS_USED <= 32 ? 32 : NCOLS_USED <= 64 ? 64 : NCOLS_USED <= 128 ? 128 : 256;
  // shared memory (bytes): operands hi/lo, A stage hi/lo, tile arrays
  static constexpr int B1_BYTES = N1 * K1 * 4, B2_BYTES = N2 * K2 * 4, B3_BYTES = N3 * K3 * 4;
  static constexpr int KMAX = K1 > 2 * K2 ? (K1 > K3 ? K1 : K3) : (2 * K2 > K3 ? 2 * K2 : K3);
  static constexpr int A_BYTES = ROWS * KMAX * 4;
  static constexpr int TILE_U = S * V * TW, TILE_UC = Fp * V * TW, TILE_DU = D * S * V * TW, TILE_DUF = D * Fp * V * TW;
  static constexpr int OFF_B1 = 0, OFF_B2 = OFF_B1 + 2 * B1_BYTES, OFF_B3 = OFF_B2 + 2 * B2_BYTES,
                       OFF_A = OFF_B3 + 2 * B3_BYTES, OFF_U = OFF_A + 2 * A_BYTES,
                       OFF_UC = OFF_U + TILES * TILE_U * 4, OFF_DU = OFF_UC + TILES * TILE_UC * 4,
                       OFF_DUF = OFF_DU + TILES * TILE_DU * 4, OFF_BAR = OFF_DUF + TILES * TILE_DUF * 4,
                       SMEM = OFF_BAR + 16;
  static_assert(ROWS == 128, "four tiles of eight elements and four variables");
  static_assert(NCOLS_USED <= 256, "tensor-memory columns");
  static_assert(NT >= ROWS && NT % 32 == 0, "the first four warps read the 128 TMEM lanes");
};

// stores x (this row's value at K index k) into a K-major operand of KP
// columns, split into hi and lo parts
__device__ __forceinline__ void tc_put(unsigned char *hi, unsigned char *lo, int r, int k, int KP, float x)
{
  float h, l;
  tc::split_tf32(x, h, l);
  const uint32_t off = tc::kmajor_offset(r, k, KP);
  *reinterpret_cast<float *>(hi + off) = h;
  *reinterpret_cast<float *>(lo + off) = l;
}

// all products of one GEMM, issued by one thread: D (+)= A B^T over KP
__device__ __forceinline__ void tc_gemm(uint32_t d_tmem, const unsigned char *ah, const unsigned char *al,
                                        const unsigned char *bh, const unsigned char *bl, int KP, int NP)
{
  const uint32_t idesc = tc::tf32_idesc(128, NP);
  const uint32_t sbo = (uint32_t)(KP / 4) * 128;
  const uint32_t a_h = tc::smem_addr(ah), a_l = tc::smem_addr(al), b_h = tc::smem_addr(bh), b_l = tc::smem_addr(bl);
  for (int j = 0; j < KP / tc::kTf32K; j++)
  {
    const uint32_t ko = (uint32_t)j * 256;
    const uint64_t dAh = tc::kmajor_desc(a_h + ko, 128, sbo), dAl = tc::kmajor_desc(a_l + ko, 128, sbo);
    const uint64_t dBh = tc::kmajor_desc(b_h + ko, 128, sbo), dBl = tc::kmajor_desc(b_l + ko, 128, sbo);
    tc::mma_tf32(d_tmem, dAh, dBh, idesc, j > 0);
    tc::mma_tf32(d_tmem, dAh, dBl, idesc, true);
    tc::mma_tf32(d_tmem, dAl, dBh, idesc, true);
  }
}

template <int N>
__global__ void __launch_bounds__(TriTc<N>::NT) k_tri_ns_grad_tc(const __grid_constant__ Args<float, float> a)
{
  using G = TriShape<N>;
  using C = TriTc<N>;
  constexpr int S = G::S, Fp = G::Fp, V = 4, D = 2, NM = 5, TILES = C::TILES;
  constexpr uint32_t kPolls = 1u << 24;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *sB1h = smem + C::OFF_B1, *sB1l = sB1h + C::B1_BYTES;
  unsigned char *sB2h = smem + C::OFF_B2, *sB2l = sB2h + C::B2_BYTES;
  unsigned char *sB3h = smem + C::OFF_B3, *sB3l = sB3h + C::B3_BYTES;
  unsigned char *sAh = smem + C::OFF_A, *sAl = sAh + C::A_BYTES;
  float *sU = reinterpret_cast<float *>(smem + C::OFF_U);
  float *sUC = reinterpret_cast<float *>(smem + C::OFF_UC);
  float *sdU = reinterpret_cast<float *>(smem + C::OFF_DU);
  float *sdUf = reinterpret_cast<float *>(smem + C::OFF_DUF);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + C::OFF_BAR);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t tile0 = (int64_t)blockIdx.x * TILES;
  const int ntl = (int)((a.ntiles - tile0) < TILES ? (a.ntiles - tile0) : TILES);
  const float beta = a.ph.ldg_b;
  const float *ops = a.dops;

  // operators into K-major hi/lo images (zero padding)
  for (int i = tid; i < C::N1 * C::K1; i += C::NT)
  {
    const int n = i / C::K1, k = i % C::K1;
    float x = 0.f;
    if (n < D * S)
    {
      const int d = n / S, s = n % S;
      if (k < S)
        x = ops[G::OD + (d * S + s) * S + k];
      else if (k < S + Fp)
        x = ops[G::ODF + (d * S + s) * Fp + (k - S)];
    }
    tc_put(sB1h, sB1l, n, k, C::K1, x);
  }
  for (int i = tid; i < C::N2 * C::K2; i += C::NT)
  {
    const int f = i / C::K2, k = i % C::K2;
    tc_put(sB2h, sB2l, f, k, C::K2, (f < Fp && k < S) ? ops[G::OE + f * S + k] : 0.f);
  }
  for (int i = tid; i < C::N3 * C::K3; i += C::NT)
  {
    const int s = i / C::K3, k = i % C::K3;
    tc_put(sB3h, sB3l, s, k, C::K3, (s < S && k < D * S) ? ops[G::ODV + s * D * S + k] : 0.f);
  }
  if (warp == 0) tc::tmem_alloc(tslot, C::TMEM_COLS);
  if (tid == 0)
  {
    tc::mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // state tiles
  for (int q = 0; q < ntl; q++)
  {
    const float *src = a.U + (tile0 + q) * (int64_t)S * V * TW;
    float *dst = sU + q * C::TILE_U;
    for (int i = tid; i < S * 4 * TW; i += C::NT)
    {
      const int l = i % TW, v = (i / TW) % 4, p = i / (4 * TW);
      dst[tix<float>(p, l, v)] = src[i];
    }
  }
  // LDG common solution at the flux points (as k_tri_ns_grad)
  for (int it = tid; it < ntl * Fp * TW; it += C::NT)
  {
    const int q = it / (Fp * TW), f = (it / TW) % Fp, l = it % TW;
    const int64_t tile = tile0 + q;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + l];
    float Uo[V], UC[V];
    const float *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + l;
#pragma unroll
    for (int v = 0; v < V; v++) Uo[v] = uo[v * TW];
    if (code >= 0)
    {
      float Un[V];
      gather_fpt<float, float, V>(a.Ufp, code >> 1, Un);
      const int slot = code & 1;
#pragma unroll
      for (int v = 0; v < V; v++)
      {
        const float ul = slot ? Un[v] : Uo[v];
        const float ur = slot ? Uo[v] : Un[v];
        if (beta == 0.5f)
          UC[v] = ur;
        else if (beta == -0.5f)
          UC[v] = ul;
        else
          UC[v] = 0.5f * (ul + ur) - beta * (ul - ur);
      }
    }
    else
    {
      float n[D], Ua[V], URa[V], UBa[V];
      const float *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + l;
#pragma unroll
      for (int d = 0; d < D; d++) n[d] = g[d * TW];
      to_abs<float, D>(Uo, Ua, a.ph);
      ghost_state<float, D>(-code - 1, Ua, n, URa, UBa, a.ph);
      to_stored<float, D>(UBa, UC, a.ph);
    }
    st4(sUC + q * C::TILE_UC + tvl<float>(f, l), UC);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  // row of this thread in the products (warps 0-3: the 128 TMEM lanes)
  const int r = tid, q = r >> 5, l = (r >> 2) & (TW - 1), v = r & 3;
  const bool row_thread = tid < C::ROWS;
  const bool row_live = row_thread && q < ntl;
  const int64_t tile_r = tile0 + q;
  const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;

  // ---- product 1: [U | Ucomm] against [oppD | oppD_fpts] ------------------
  if (row_thread)
  {
    for (int k = 0; k < C::K1; k++)
    {
      float x = 0.f;
      if (row_live)
      {
        if (k < S)
          x = sU[q * C::TILE_U + tix<float>(k, l, v)];
        else if (k < S + Fp)
          x = sUC[q * C::TILE_UC + tix<float>(k - S, l, v)];
      }
      tc_put(sAh, sAl, r, k, C::K1, x);
    }
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0)
  {
    tc::fence_after_sync();
    tc_gemm(tmem + C::C1, sAh, sAl, sB1h, sB1l, C::K1, C::N1);
    tc::mma_commit(mbar);
  }
  ok = __syncthreads_and(tc::mbar_wait(mbar, phase, kPolls) ? 1 : 0) != 0;
  phase ^= 1;
  tc::fence_after_sync();
  // physical gradient: thread r holds this (element, variable)'s reference
  // gradient at every solution point
  if (row_thread && ok)
  {
    float td[C::N1];
#pragma unroll
    for (int c0 = 0; c0 < C::N1; c0 += 16) tc::tmem_ld16(lane_base + C::C1 + c0, td + c0);
    constexpr int HALF = C::ROWS * C::K2 * 4;
    if (row_live)
    {
#pragma unroll
      for (int s = 0; s < S; s++)
      {
        const float *m = a.mets + (tile_r * S + s) * (int64_t)NM * TW + l;
        const float a00 = m[0], a01 = m[TW], a10 = m[2 * TW], a11 = m[3 * TW];
        const float inv_det = 1.f / m[4 * TW];
        const float g0 = (td[s] * a00 + td[S + s] * a10) * inv_det;
        const float g1 = (td[s] * a01 + td[S + s] * a11) * inv_det;
        sdU[q * C::TILE_DU + tix<float>(s, l, v)] = g0;
        sdU[q * C::TILE_DU + tix<float>(S + s, l, v)] = g1;
        if (a.dU_out)
        {
          a.dU_out[(((tile_r * D + 0) * S + s) * V + v) * TW + l] = g0;
          a.dU_out[(((tile_r * D + 1) * S + s) * V + v) * TW + l] = g1;
        }
        // operands of product 2: the two dimensions side by side
        tc_put(sAh, sAl, r, s, C::K2, g0);
        tc_put(sAh + HALF, sAl + HALF, r, s, C::K2, g1);
      }
    }
    for (int s = row_live ? S : 0; s < C::K2; s++)
    {
      tc_put(sAh, sAl, r, s, C::K2, 0.f);
      tc_put(sAh + HALF, sAl + HALF, r, s, C::K2, 0.f);
    }
  }
  // ---- product 2: gradient at the flux points ------------------------------
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0 && ok)
  {
    tc::fence_after_sync();
    constexpr int HALF = C::ROWS * C::K2 * 4;
    tc_gemm(tmem + C::C2, sAh, sAl, sB2h, sB2l, C::K2, C::N2);
    tc_gemm(tmem + C::C2 + C::N2, sAh + HALF, sAl + HALF, sB2h, sB2l, C::K2, C::N2);
    tc::mma_commit(mbar);
  }
  if (ok)
  {
    ok = __syncthreads_and(tc::mbar_wait(mbar, phase, kPolls) ? 1 : 0) != 0;
    phase ^= 1;
  }
  tc::fence_after_sync();
  if (row_thread && ok)
  {
    float x[16];
#pragma unroll
    for (int d = 0; d < D; d++)
#pragma unroll
      for (int c0 = 0; c0 < C::N2; c0 += 16)
      {
        tc::tmem_ld16(lane_base + C::C2 + d * C::N2 + c0, x);
        if (row_live)
        {
#pragma unroll
          for (int i = 0; i < 16; i++)
            if (c0 + i < Fp) sdUf[q * C::TILE_DUF + tix<float>(d * Fp + c0 + i, l, v)] = x[i];
        }
      }
  }
  tc::fence_before_sync();
  __syncthreads();
  // own viscous normal flux at flux points (as k_tri_ns_grad)
  for (int it = tid; it < ntl * Fp * TW && ok; it += C::NT)
  {
    const int qq = it / (Fp * TW), f = (it / TW) % Fp, ll = it % TW;
    const int64_t tile = tile0 + qq;
    const int code = a.nbr[(tile * Fp + f) * (int64_t)TW + ll];
    if (code >= 0 && ((beta == 0.5f && (code & 1)) || (beta == -0.5f && !(code & 1)))) continue;
    float n[D];
    const float *g = a.fgeo + (tile * Fp + f) * (int64_t)(D + 1) * TW + ll;
#pragma unroll
    for (int d = 0; d < D; d++) n[d] = g[d * TW];
    float Uf[V], dUf[V][D], Fn[V];
    const float *uo = a.Ufp + (tile * Fp + f) * (int64_t)V * TW + ll;
#pragma unroll
    for (int vv = 0; vv < V; vv++) Uf[vv] = uo[vv * TW];
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      float x[V];
      ld4(sdUf + qq * C::TILE_DUF + tvl<float>(d * Fp + f, ll), x);
#pragma unroll
      for (int vv = 0; vv < V; vv++) dUf[vv][d] = x[vv];
    }
    float Ua[V];
    to_abs<float, D>(Uf, Ua, a.ph);
    if (code >= 0)
      visc_normal<float, D>(Ua, dUf, n, Fn, a.ph);
    else
    {
      float UR[V], UB[V], dUB[V][D];
      ghost_state<float, D>(-code - 1, Ua, n, UR, UB, a.ph);
      ghost_grad<float, D>(-code - 1, Ua, dUf, n, dUB);
      visc_normal<float, D>(UB, dUB, n, Fn, a.ph);
    }
    float *out = a.Fvn + (tile * Fp + f) * (int64_t)V * TW + ll;
#pragma unroll
    for (int vv = 0; vv < V; vv++) out[vv * TW] = Fn[vv];
  }
  // volume flux, transformed, into sdU (each thread rewrites its own point;
  // the flux-point loop above reads sdUf only)
  for (int it = tid; it < ntl * S * TW && ok; it += C::NT)
  {
    const int qq = it / (S * TW), s = (it / TW) % S, ll = it % TW;
    const int64_t tile = tile0 + qq;
    float U[V], dU[V][D], F[V][D], P, Pp, Ua[V];
    ld4(sU + qq * C::TILE_U + tvl<float>(s, ll), U);
#pragma unroll
    for (int d = 0; d < D; d++)
    {
      float x[V];
      ld4(sdU + qq * C::TILE_DU + tvl<float>(d * S + s, ll), x);
#pragma unroll
      for (int vv = 0; vv < V; vv++) dU[vv][d] = x[vv];
    }
    flux_conv_stored<float, D>(U, F, P, Pp, a.ph);
    to_abs<float, D>(U, Ua, a.ph);
    flux_visc_add<float, D>(Ua, dU, F, a.ph);
    tri_transform<float, float>(a, tile, s, ll, F, sdU + qq * C::TILE_DU, S);
  }
  __syncthreads();
  // ---- product 3: volume divergence ----------------------------------------
  if (row_thread && ok)
  {
    for (int k = 0; k < C::K3; k++)
      tc_put(sAh, sAl, r, k, C::K3, (row_live && k < D * S) ? sdU[q * C::TILE_DU + tix<float>(k, l, v)] : 0.f);
  }
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0 && ok)
  {
    tc::fence_after_sync();
    tc_gemm(tmem + C::C3, sAh, sAl, sB3h, sB3l, C::K3, C::N3);
    tc::mma_commit(mbar);
  }
  if (ok)
  {
    ok = __syncthreads_and(tc::mbar_wait(mbar, phase, kPolls) ? 1 : 0) != 0;
    phase ^= 1;
  }
  tc::fence_after_sync();
  if (row_thread && ok)
  {
    float x[16];
#pragma unroll
    for (int c0 = 0; c0 < C::N3; c0 += 16)
    {
      tc::tmem_ld16(lane_base + C::C3 + c0, x);
      if (row_live)
      {
#pragma unroll
        for (int i = 0; i < 16; i++)
          if (c0 + i < S) a.divF_vol[(tile_r * S + c0 + i) * (int64_t)V * TW + v * TW + l] = x[i];
      }
    }
  }
  if (!ok)
  {
    if (tid == 0 && a.err) *reinterpret_cast<volatile int *>(a.err) = 1;
    // the MMAs of the unfinished product may still be running: wait once
    // more (bounded) before the tensor memory is released
    tc::mbar_wait(mbar, phase ^ 1, kPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, C::TMEM_COLS);
}

}  // namespace dev
}  // namespace zb
