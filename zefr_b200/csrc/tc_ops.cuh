// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a:
// shared-memory matrix descriptors, the instruction descriptor of a
// kind::tf32 MMA with FP32 accumulation in tensor memory (TMEM), TMEM
// allocation, MMA issue and completion through an mbarrier, TMEM loads, and
// the split of an FP32 value into two TF32 parts for split-precision
// ("TF32x3") products.
//
// Operand layout used throughout: K-major, no swizzle.  An operand of R rows
// and KP columns (K) is stored as core matrices of 8 rows x 16 bytes (four
// FP32/TF32 values of K); within a group of 8 rows the KP/4 core matrices are
// adjacent (leading byte offset 128 B), and groups of 8 rows are SBO bytes
// apart:  byte(r, k) = (r / 8) * SBO + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4.
#pragma once
#include <cstdint>

namespace zb {
namespace tc {

// K extent of one kind::tf32 MMA (32 bytes of K)
constexpr int kTf32K = 8;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// version 1 (sm_100): start address, leading byte offset (between the two
// 16-byte K chunks one MMA reads) and stride byte offset (between groups of 8
// rows), all in 16-byte units.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, no swizzle
}

// Instruction descriptor: D = F32 (bits 4-5 = 1), A = B = TF32 (bits 7-9 and
// 10-12 = 2), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// TMEM allocation by one whole warp; the base address is written to *slot
// (shared memory).  ncols: a power of two, 32..512.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[desc] * B[desc]^T, issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate));
}

// arrive on the mbarrier once every MMA this thread issued has completed
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
}

// Wait for the phase with the given parity to complete; gives up after
// max_polls polls and returns false (the caller records the failure).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t max_polls)
{
  const uint32_t a = smem_addr(mbar);
  for (uint32_t i = 0; i < max_polls; i++)
  {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (the warp reads
// its own 32-lane quarter: lanes 32 (warp % 4) .. + 31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// x = hi + lo + O(2^-22 |x|) with hi and lo TF32 (round to nearest, ties away)
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo)
{
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  hi = __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hi));
  lo = __uint_as_float(l);
}

// byte offset of (row r, k) in a K-major no-swizzle operand with KP columns
__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k, int KP)
{
  return (uint32_t)((r >> 3) * (KP / 4) * 128 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

}  // namespace tc
}  // namespace zb
