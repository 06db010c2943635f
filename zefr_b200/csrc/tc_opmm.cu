// Operator products on the tensor pipe: C = alpha A B + beta C for a small
// constant operator A [m][k] applied to every column of B [k][n] (n = element
// count x variables, the reference's layout [point][var][element]), the
// product the reference hands to GiMMiK or cuBLAS (gimmik_mm_gpu,
// include/gimmik.h:5-22, src/gimmik_gpu.cu:31183-31577; its calls in
// src/elements.cpp:1337-1501).
//
// FP32 in and out.  Each product is split into TF32 parts (x = hi + lo) and
// formed as A_hi B_hi + A_hi B_lo + A_lo B_hi with FP32 accumulation in
// tensor memory ("TF32x3"), which keeps about 21 bits of each operand, near
// FP32 arithmetic; plain TF32 (10 bits) would not.
//
// Mapping: one CTA of 128 threads (a warpgroup) takes 128 columns of B at a
// time as the M = 128 rows of one tcgen05 MMA: D[col][row of A] =
// sum_k B^T[col][k] A[row][k], so thread t owns column t and reads its
// results from TMEM lane t.  The operator's hi and lo parts sit in shared
// memory for the CTA's life; the columns are staged K block by K block (32
// values of K, four MMA steps of 8).
#include <cstdint>
#include <string>

#include "context.hpp"
#include "tc_ops.cuh"

namespace zb {
namespace {

constexpr int kCols = 128;       // columns per CTA pass = MMA M
constexpr int kKB = 32;          // K values staged per block
constexpr uint32_t kPolls = 1u << 24;

__host__ __device__ constexpr int round_up(int x, int m) { return (x + m - 1) / m * m; }

__host__ __device__ constexpr uint32_t tmem_cols_for(int np)
{
  return np <= 32 ? 32u : np <= 64 ? 64u : np <= 128 ? 128u : 256u;
}

// dynamic shared memory: [op hi][op lo][B^T hi][B^T lo], then the mbarrier
// and the TMEM address slot
__global__ void __launch_bounds__(kCols) k_opmm_tf32x3(int m, int n, int k, float alpha, const float *__restrict__ a,
                                                       int lda, const float *__restrict__ b, int ldb, float beta,
                                                       float *__restrict__ c, int ldc, int *err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  const int NP = round_up(m, 16), KP = round_up(k, kKB);
  const uint32_t op_bytes = (uint32_t)NP * KP * 4, bt_bytes = (uint32_t)kCols * kKB * 4;
  unsigned char *sAh = smem, *sAl = smem + op_bytes;
  unsigned char *sBh = smem + 2 * op_bytes, *sBl = sBh + bt_bytes;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sBl + bt_bytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = tmem_cols_for(NP);

  // operator, split once, K-major image of NP rows x KP
  for (int i = tid; i < NP * KP; i += kCols)
  {
    const int r = i / KP, kk = i % KP;
    const float x = (r < m && kk < k) ? a[(int64_t)r * lda + kk] : 0.f;
    float hi, lo;
    tc::split_tf32(x, hi, lo);
    const uint32_t off = tc::kmajor_offset(r, kk, KP);
    *reinterpret_cast<float *>(sAh + off) = hi;
    *reinterpret_cast<float *>(sAl + off) = lo;
  }
  if (warp == 0) tc::tmem_alloc(tslot, ncols);
  if (tid == 0)
  {
    tc::mbar_init(mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = tc::tf32_idesc(kCols, NP);
  const uint32_t sbo_op = (uint32_t)(KP / 4) * 128, sbo_bt = (uint32_t)(kKB / 4) * 128;
  uint32_t phase = 0;
  bool ok = true;
  const int64_t nchunks = ((int64_t)n + kCols - 1) / kCols;
  for (int64_t ch = blockIdx.x; ch < nchunks && ok; ch += gridDim.x)
  {
    const int64_t col = ch * kCols + tid;
    const bool live = col < n;
    for (int kb = 0; kb < KP / kKB && ok; kb++)
    {
      // this column's K block: hi and lo, 16 bytes per store
#pragma unroll
      for (int q = 0; q < kKB / 4; q++)
      {
        float4 h, l;
        float *hp = &h.x, *lp = &l.x;
#pragma unroll
        for (int j = 0; j < 4; j++)
        {
          const int kk = kb * kKB + q * 4 + j;
          const float x = (live && kk < k) ? b[(int64_t)kk * ldb + col] : 0.f;
          tc::split_tf32(x, hp[j], lp[j]);
        }
        const uint32_t off = tc::kmajor_offset(tid, q * 4, kKB);
        *reinterpret_cast<float4 *>(sBh + off) = h;
        *reinterpret_cast<float4 *>(sBl + off) = l;
      }
      tc::fence_smem_to_async();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0)
      {
        tc::fence_after_sync();
        const uint32_t ah = tc::smem_addr(sAh), al = tc::smem_addr(sAl);
        const uint32_t bh = tc::smem_addr(sBh), bl = tc::smem_addr(sBl);
#pragma unroll
        for (int j = 0; j < kKB / tc::kTf32K; j++)
        {
          // K step: 8 values = two 16-byte chunks, 256 bytes further along K
          const uint32_t kop = (uint32_t)(kb * kKB + j * tc::kTf32K) / 4 * 128, kbt = (uint32_t)j * 256;
          const uint64_t dBh = tc::kmajor_desc(bh + kbt, 128, sbo_bt), dBl = tc::kmajor_desc(bl + kbt, 128, sbo_bt);
          const uint64_t dAh = tc::kmajor_desc(ah + kop, 128, sbo_op), dAl = tc::kmajor_desc(al + kop, 128, sbo_op);
          tc::mma_tf32(tmem, dBh, dAh, idesc, kb > 0 || j > 0);
          tc::mma_tf32(tmem, dBh, dAl, idesc, true);
          tc::mma_tf32(tmem, dBl, dAh, idesc, true);
        }
        tc::mma_commit(mbar);
      }
      // every thread waits; the CTA agrees on the outcome so that all its
      // threads leave the loops together
      ok = __syncthreads_and(tc::mbar_wait(mbar, phase, kPolls) ? 1 : 0) != 0;
      phase ^= 1;
      tc::fence_after_sync();
    }
    if (!ok) break;
    // results: lane = column, TMEM columns = rows of A
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < NP; c0 += 16)
    {
      float v[16];
      tc::tmem_ld16(lane_base + (uint32_t)c0, v);
      if (live)
      {
#pragma unroll
        for (int i = 0; i < 16; i++)
        {
          const int r = c0 + i;
          if (r < m)
          {
            float *dst = c + (int64_t)r * ldc + col;
            *dst = beta == 0.f ? alpha * v[i] : alpha * v[i] + beta * *dst;
          }
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  if (!ok)
  {
    if (tid == 0) *reinterpret_cast<volatile int *>(err) = 1;
    // the MMAs of the unfinished step may still be running: wait once more
    // (bounded) before the tensor memory is released
    tc::mbar_wait(mbar, phase ^ 1, kPolls);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, ncols);
}

}  // namespace

size_t opmm_tc_smem_bytes(int m, int k)
{
  const int NP = round_up(m, 16), KP = round_up(k, kKB);
  return (size_t)2 * NP * KP * 4 + (size_t)2 * kCols * kKB * 4 + 16;
}

// Launches the product on `st` without waiting for it.  err_host / err_dev:
// one int of mapped pinned host memory (host and device addresses) that a
// kernel whose tensor-core wait timed out sets; it is checked, and cleared,
// when the next product is launched.
void opmm_tc(int m, int n, int k, float alpha, const float *a, int lda, const float *b, int ldb, float beta, float *c,
             int ldc, cudaStream_t st, volatile int *err_host, int *err_dev, int max_ctas)
{
  if (*err_host)
  {
    *err_host = 0;
    ZB_THROW(ZB_ERR_CUDA, "operator product: a tensor-core completion wait of an earlier product timed out");
  }
  if (m < 1 || n < 0 || k < 1) ZB_THROW(ZB_ERR_ARG, "operator product: m and k must be positive, n non-negative");
  if (m > 256) ZB_THROW(ZB_ERR_UNSUPPORTED, "operator product on the tensor pipe: m <= 256");
  if (lda < k || ldb < n || ldc < n) ZB_THROW(ZB_ERR_ARG, "operator product: leading dimension too small");
  const size_t smem = opmm_tc_smem_bytes(m, k);
  if (smem > 220 * 1024)
    ZB_THROW(ZB_ERR_UNSUPPORTED, "operator product on the tensor pipe: operator of " + std::to_string(m) + " x " +
                                     std::to_string(k) + " does not fit in shared memory");
  if (n == 0) return;
  cudaError_t e = cudaFuncSetAttribute(k_opmm_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string("operator product set-up: ") + cudaGetErrorString(e));
  const int64_t chunks = ((int64_t)n + kCols - 1) / kCols;
  // resident CTAs: shared memory and tensor-memory columns (512 per SM)
  const int by_smem = (int)((227 * 1024) / (smem + 1024));
  const int by_tmem = (int)(512 / tmem_cols_for(round_up(m, 16)));
  int per_sm = by_smem < by_tmem ? by_smem : by_tmem;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)148 * per_sm;
  if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
  if (grid > chunks) grid = chunks;
  k_opmm_tf32x3<<<(unsigned)grid, kCols, smem, st>>>(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, err_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) ZB_THROW(ZB_ERR_CUDA, std::string("operator product launch: ") + cudaGetErrorString(e));
}

}  // namespace zb
