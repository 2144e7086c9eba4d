// tcgen05.cuh -- the 5th-generation tensor-core primitives the descriptor
// kernel's mixed-precision ANN uses (sm_100a, inline PTX).
//
// Operands are 16-bit (FP16 or BF16) tiles in shared memory in the K-major,
// no-swizzle canonical layout: 8-row x 16-byte core matrices, the two
// K-adjacent core matrices of one MMA (K = 16) 128 bytes apart (leading byte
// offset), consecutive 8-row groups K/8 x 128 bytes apart (stride byte
// offset).  Accumulators live in tensor memory (TMEM); one thread issues the
// MMAs and commits them to an mbarrier, and every wait on it is bounded.
#pragma once

#include <cstdint>

namespace nepx {
namespace tc {

constexpr long long kWaitCycles = 4000000000ll;   // ~2 s at the B200 clock

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) of a 16-bit K-major no-swizzle tile with K columns
__host__ __device__ __forceinline__ uint32_t off16(int r, int k, int K)
{
  return static_cast<uint32_t>(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 +
                               (k & 7) * 2);
}

// Shared-memory matrix descriptor of a tile with K columns: start address,
// leading byte offset 128, stride byte offset K/8 x 128, descriptor version 1,
// no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, int K)
{
  const uint64_t lbo = 128u >> 4;
  const uint64_t sbo = static_cast<uint64_t>((K >> 3) * 128) >> 4;
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, A and B both FP16
// (bf16 = false) or both BF16, K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool bf16)
{
  return (1u << 4) | ((bf16 ? 1u : 0u) << 7) | ((bf16 ? 1u : 0u) << 10) |
         (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
    "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                 mbar)
               : "memory");
}

// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void before_sync()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void after_sync()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase of the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
    if (ok) return true;
    if (clock64() - t0 > kWaitCycles) return false;
  }
}

// Allocates `cols` TMEM columns (a power of two >= 32) for the CTA: the whole
// warp calls it; the base address lands in *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, int cols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                 smem_u32(slot)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int cols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
               : "memory");
}

// 16 consecutive TMEM columns of this thread's lane; the wait is part of the
// same statement so no register is read before the load lands.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
    "%12, %13, %14, %15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;\n"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15])
    : "r"(taddr)
    : "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

}  // namespace tc
}  // namespace nepx
