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

// Copies a row-major bf16 matrix [rows][cols] into a K-major tile (K = cols), 16 bytes at a time.
__device__ __forceinline__ void stage_rowmajor(unsigned char *tile, const __nv_bfloat16 *src, int rows, int cols) {
  const int chunks = rows * cols / 8;
  for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
    const int row = c / (cols / 8), k = (c % (cols / 8)) * 8;
    *reinterpret_cast<uint4 *>(tile + kmajor_offset(row, k, cols)) =
        *reinterpret_cast<const uint4 *>(src + (size_t)row * cols + k);
  }
}

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

// Hidden-layer epilogue for the calling thread's row: bias, SiLU, next operand (bf16) in A;
// optionally the pre-activation and activation to global memory.
__device__ __forceinline__ void hidden_epilogue(uint32_t trow, const float *bias, unsigned char *A, float *z_out,
                                                __nv_bfloat16 *y_out) {
  const int t = threadIdx.x;
  for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
    float v[16];
    umma::tmem_ld16(trow + c0, v);
    __align__(16) float bb[16];
#pragma unroll
    for (int q = 0; q < 4; ++q)  // the bias row, four 16-byte loads (same for every thread)
      *reinterpret_cast<float4 *>(bb + 4 * q) = __ldg(reinterpret_cast<const float4 *>(bias + c0) + q);
    __align__(16) __nv_bfloat16 yb[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const float z = v[c] + bb[c];
      yb[c] = __float2bfloat16(silu(z));
      if (z_out)
        z_out[c0 + c] = z;
    }
    // two 16-byte rows of core matrices
    *reinterpret_cast<uint4 *>(A + kmajor_offset(t, c0, kMlpHidden)) = *reinterpret_cast<const uint4 *>(yb);
    *reinterpret_cast<uint4 *>(A + kmajor_offset(t, c0 + 8, kMlpHidden)) =
        *reinterpret_cast<const uint4 *>(yb + 8);
    if (y_out) {
      *reinterpret_cast<uint4 *>(y_out + c0) = *reinterpret_cast<const uint4 *>(yb);
      *reinterpret_cast<uint4 *>(y_out + c0 + 8) = *reinterpret_cast<const uint4 *>(yb + 8);
    }
  }
}

}  // namespace vpd
