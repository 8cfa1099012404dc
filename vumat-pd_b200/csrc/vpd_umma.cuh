// sm_100a tensor-core primitives for the surrogate network: tcgen05 MMA (BF16 in, FP32
// accumulate in tensor memory), TMEM allocation and loads, and bounded mbarrier waits.
//
// Shared-memory operands use the K-major, no-swizzle canonical layout: the matrix is cut into
// core matrices of 8 rows x 16 bytes (8 bf16) stored as 128 contiguous bytes; along K the
// core matrices are 128 bytes apart (leading byte offset), along rows 8-row groups are
// (K / 8) * 128 bytes apart (stride byte offset). One MMA consumes a K = 16 slice (two core
// matrices along K); the next slice starts 256 bytes later.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vpd {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with ktotal columns.
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, int ktotal) {
  return (uint32_t)((row >> 3) * (ktotal / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100 layout: version 1 in bits 46-47, no swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor, kind::f16 with BF16 A/B, FP32 accumulator, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4)                       // c_format F32
         | (1u << 7)                     // a_format BF16
         | (1u << 10)                    // b_format BF16
         | ((uint32_t)(n >> 3) << 17)    // N / 8
         | ((uint32_t)(m >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrives on the mbarrier once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the mbarrier phase with the given parity; gives up after `limit` polls and
// returns false (the caller reports the timeout instead of spinning forever).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit) {
  const uint32_t addr = smem_u32(mbar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done)
      return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes generic-proxy shared-memory writes visible to the tensor cores (async proxy).
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Warp-collective: allocates ncols TMEM columns, writes the base address to *dst (smem).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// Warp-collective: each thread reads 16 consecutive FP32 columns of its TMEM lane
// (lane = 32 * warp-in-quadrant + lane id; taddr carries the warp's lane base in bits 16+).
// The load and its wait are one asm statement: tcgen05.ld writes its registers
// asynchronously, and with a separate wait the compiler may move uses of the registers above
// the wait (nothing ties them to it).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *out) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int c = 0; c < 16; ++c)
    out[c] = __uint_as_float(r[c]);
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (one row per thread), waited for in
// the same asm statement so the compiler cannot read the registers early.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *out) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int c = 0; c < 32; ++c)
    out[c] = __uint_as_float(r[c]);
}

// D[128 x N] (TMEM, FP32) = A[128 x K] * B[N x K]^T with both operands K-major in shared
// memory; issued by one thread. accumulate = 0 overwrites D.
__device__ __forceinline__ void gemm_issue(uint32_t tmem_d, uint32_t a_addr, uint32_t b_addr, int K, int N,
                                           bool accumulate) {
  const uint32_t idesc = idesc_bf16(128, N);
  const uint32_t sbo_a = (uint32_t)(K / 8) * 128u, sbo_b = sbo_a;
  for (int kk = 0; kk < K / 16; ++kk) {
    const uint64_t ad = smem_desc(a_addr + kk * 256u, 128u, sbo_a);
    const uint64_t bd = smem_desc(b_addr + kk * 256u, 128u, sbo_b);
    mma_bf16(tmem_d, ad, bd, idesc, (accumulate || kk > 0) ? 1u : 0u);
  }
}

}  // namespace umma
}  // namespace vpd
