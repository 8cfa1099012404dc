// Device building blocks of the surrogate network on the tensor cores, shared by the training
// kernels (vpd_mlp.cu) and the fused surrogate material kernel (vpd_surrogate.cu): BF16
// operand staging in the K-major no-swizzle layout, one 128-row GEMM issued by one thread and
// awaited by the block through an mbarrier, and the per-row hidden-layer epilogue.
#pragma once

#include "vpd_mlp.cuh"
#include "vpd_umma.cuh"

namespace vpd {

using umma::kmajor_offset;
using umma::smem_u32;

constexpr uint32_t kWaitLimit = 1u << 24;  // mbarrier polls before a wait is declared failed

// tanh on the special-function unit (tanh.approx.f32, relative error about 2^-11, below the
// BF16 rounding of the stored activations).
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// SiLU z sigmoid(z) with sigmoid(z) = (1 + tanh(z / 2)) / 2: silu = h + h tanh(h), h = z / 2.
__device__ __forceinline__ float silu(float z) {
  const float h = 0.5f * z;
  return fmaf(h, tanh_approx(h), h);
}
__device__ __forceinline__ float silu_grad(float z) {
  const float s = fmaf(0.5f, tanh_approx(0.5f * z), 0.5f);
  return s * fmaf(z, 1.0f - s, 1.0f);
}

// Shared-memory store of one bf16 element at (row, k) of a K-major tile.
__device__ __forceinline__ void st_bf16(unsigned char *tile, int row, int k, int ktotal, float v) {
  *reinterpret_cast<__nv_bfloat16 *>(tile + kmajor_offset(row, k, ktotal)) = __float2bfloat16(v);
}

// Copies a row-major bf16 matrix [rows][cols] (16-byte aligned) into a K-major tile (K = cols),
// 16 bytes at a time with cp.async: every copy of the thread is in flight at once. The copies
// complete at stage_wait(), which every thread calls before the barrier that publishes them.
__device__ __forceinline__ void stage_rowmajor(unsigned char *tile, const __nv_bfloat16 *src, int rows, int cols) {
  const int chunks = rows * cols / 8;
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int row = c / (cols / 8), k = (c % (cols / 8)) * 8;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(tile + kmajor_offset(row, k, cols))),
                 "l"(src + (size_t)row * cols + k)
                 : "memory");
  }
}
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct Sync {
  uint64_t *mbar;
  uint32_t phase;
  unsigned *err;   // ORed with `bit` when a wait times out
  unsigned bit;
  bool ok;
  // Every thread of the block calls this; the outcome is made uniform so a timeout cannot
  // split the block's control flow around later barriers.
  __device__ void wait() {
    const bool got = ok && umma::mbar_wait(mbar, phase, kWaitLimit);
    ok = __syncthreads_and(got) != 0;
    if (!ok && threadIdx.x == 0)
      atomicOr(err, bit);
    phase ^= 1u;
    umma::fence_after_sync();
  }
};

// Issues D = A * B^T on one thread and waits for it on all threads.
__device__ __forceinline__ void gemm(Sync &sy, uint32_t tmem_d, const unsigned char *a, const unsigned char *b,
                                     int K, int N) {
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (threadIdx.x == 0) {
    umma::gemm_issue(tmem_d, smem_u32(a), smem_u32(b), K, N, false);
    umma::commit(sy.mbar);
  }
  sy.wait();
}

// The network's biases (b1, b2, b3: 128 each; b4: 16) copied into shared memory once per block:
// the epilogues read them as broadcast 16-byte loads.
constexpr int kBiasFloats = 3 * kMlpHidden + kMlpOut;
__device__ __forceinline__ void stage_biases(float *dst, const MlpWeights &w) {
  for (int c = threadIdx.x; c < kBiasFloats; c += blockDim.x)
    dst[c] = c < kMlpHidden ? w.b1[c]
                            : (c < 2 * kMlpHidden ? w.b2[c - kMlpHidden]
                                                  : (c < 3 * kMlpHidden ? w.b3[c - 2 * kMlpHidden]
                                                                        : w.b4[c - 3 * kMlpHidden]));
}

// Hidden-layer epilogue for the calling thread's row, 32 columns per TMEM load: bias, SiLU,
// next operand (bf16) in A; optionally the pre-activation and activation to global memory.
// `bias` points at the layer's 128 biases (shared or global memory, 16-byte aligned).
__device__ __forceinline__ void hidden_epilogue(uint32_t trow, const float *bias, unsigned char *A, float *z_out,
                                                __nv_bfloat16 *y_out) {
  const int t = threadIdx.x;
#pragma unroll 1
  for (int c0 = 0; c0 < kMlpHidden; c0 += 32) {
    float v[32];
    umma::tmem_ld32(trow + c0, v);
    __align__(16) __nv_bfloat16 yb[32];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 bb = *reinterpret_cast<const float4 *>(bias + c0 + 4 * q);
      const float z[4] = {v[4 * q] + bb.x, v[4 * q + 1] + bb.y, v[4 * q + 2] + bb.z, v[4 * q + 3] + bb.w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        yb[4 * q + c] = __float2bfloat16(silu(z[c]));
        if (z_out)
          z_out[c0 + 4 * q + c] = z[c];
      }
    }
    // four 16-byte rows of core matrices
#pragma unroll
    for (int k = 0; k < 4; ++k)
      *reinterpret_cast<uint4 *>(A + kmajor_offset(t, c0 + 8 * k, kMlpHidden)) =
          *reinterpret_cast<const uint4 *>(yb + 8 * k);
    if (y_out)
#pragma unroll
      for (int k = 0; k < 4; ++k)
        *reinterpret_cast<uint4 *>(y_out + c0 + 8 * k) = *reinterpret_cast<const uint4 *>(yb + 8 * k);
  }
}

}  // namespace vpd
