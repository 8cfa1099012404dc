// The surrogate network's forward and backward passes on the tensor cores.
//
// Network: 10 -> 128 -> 128 -> 128 -> 7 with SiLU activations, BF16 weights and activations,
// FP32 accumulation. Inputs and outputs are padded to 16 columns (zero weights outside).
// Each CTA takes a tile of 128 batch rows with 128 threads, thread t owning row t: its row of
// every accumulator sits in TMEM lane t, so the epilogue (bias, SiLU, BF16 conversion, writing
// the next layer's operand into shared memory) is row-local. The MMAs are tcgen05.mma
// kind::f16 (BF16 x BF16 -> FP32 in TMEM), issued by one thread, completion signalled through
// an mbarrier (tcgen05.commit); every wait is bounded and reports a timeout in *err.
//
// Backward (same tiling): dZ = dY * SiLU'(Z); dW = dZ^T Y_prev is a 128 x 128 (or 128 x 16)
// product over the tile's rows, accumulated into FP32 gradient buffers with atomics; dY_prev =
// dZ W. Operands that the products need transposed are staged transposed into shared memory.
#include "vpd_mlp_tile.cuh"

#include <algorithm>
#include <vector>

namespace vpd {

// ------------------------------------------------------------------ forward
// smem: W1 (128x16) | W2 (128x128) | W3 | W4 (16x128) | A (128x128) | X0 (128x16) | barrier |
//       biases
constexpr size_t kFwdSmem = 4096 + 32768 + 32768 + 4096 + 32768 + 4096 + 64 + 4 * kBiasFloats;

__device__ __forceinline__ void stage_weights_fwd(unsigned char *s, const MlpWeights &w) {
  stage_rowmajor(s, w.w1, kMlpHidden, kMlpIn);
  stage_rowmajor(s + 4096, w.w2, kMlpHidden, kMlpHidden);
  stage_rowmajor(s + 4096 + 32768, w.w3, kMlpHidden, kMlpHidden);
  stage_rowmajor(s + 4096 + 65536, w.w4, kMlpOut, kMlpHidden);
}

__global__ void __launch_bounds__(128, 1) k_mlp_forward(MlpWeights w, const float *x, int64_t B, float *out,
                                                        MlpActs acts, unsigned *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sW1 = smem, *sW2 = smem + 4096, *sW3 = sW2 + 32768, *sW4 = sW3 + 32768;
  unsigned char *sA = sW4 + 4096, *sX = sA + 32768;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sX + 4096);
  float *sBias = reinterpret_cast<float *>(sX + 4096 + 64);
  __shared__ uint32_t s_tmem;
  const int t = threadIdx.x;
  const int64_t row = (int64_t)blockIdx.x * 128 + t;
  if (t < 32)
    umma::tmem_alloc(&s_tmem, 128);
  if (t == 0)
    umma::mbar_init(mbar, 1);
  stage_weights_fwd(smem, w);
  stage_biases(sBias, w);
  float xin[kMlpIn];
#pragma unroll
  for (int c = 0; c < kMlpIn; ++c)
    xin[c] = row < B ? x[row * kMlpIn + c] : 0.0f;
#pragma unroll
  for (int c = 0; c < kMlpIn; ++c)
    st_bf16(sX, t, c, kMlpIn, xin[c]);
  if (acts.y0 && row < B)
#pragma unroll
    for (int c = 0; c < kMlpIn; ++c)
      acts.y0[row * kMlpIn + c] = __float2bfloat16(xin[c]);
  stage_wait();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = s_tmem;
  const uint32_t trow = tmem + ((uint32_t)(t & ~31) << 16);  // this warp's TMEM lanes
  Sync sy{mbar, 0u, err, 1u, true};
  const bool keep = row < B;
  gemm(sy, tmem, sX, sW1, kMlpIn, kMlpHidden);
  hidden_epilogue(trow, sBias, sA, keep && acts.z1 ? acts.z1 + row * kMlpHidden : nullptr,
                  keep && acts.y1 ? acts.y1 + row * kMlpHidden : nullptr);
  gemm(sy, tmem, sA, sW2, kMlpHidden, kMlpHidden);
  hidden_epilogue(trow, sBias + kMlpHidden, sA, keep && acts.z2 ? acts.z2 + row * kMlpHidden : nullptr,
                  keep && acts.y2 ? acts.y2 + row * kMlpHidden : nullptr);
  gemm(sy, tmem, sA, sW3, kMlpHidden, kMlpHidden);
  hidden_epilogue(trow, sBias + 2 * kMlpHidden, sA, keep && acts.z3 ? acts.z3 + row * kMlpHidden : nullptr,
                  keep && acts.y3 ? acts.y3 + row * kMlpHidden : nullptr);
  gemm(sy, tmem, sA, sW4, kMlpHidden, kMlpOut);
  float v[16];
  if (sy.ok)
    umma::tmem_ld16(trow, v);
  if (keep)
#pragma unroll
    for (int c = 0; c < kMlpOut; ++c)
      out[row * kMlpOut + c] = sy.ok ? v[c] + w.b4[c] : 0.0f;
  umma::fence_before_sync();
  __syncthreads();
  if (t < 32)
    umma::tmem_dealloc(tmem, 128);
}

// ------------------------------------------------------------------ backward
// smem: Wt2 (128x128) | Wt3 | Wt4 (128x16) | A (dZ, 128x128) | At (dZ^T, 128x128) |
//       Bt (Y_prev^T, 128x128) | small (dZ4^T 16x128) | barrier
constexpr size_t kBwdSmem = 32768 * 2 + 4096 + 32768 * 3 + 4096 + 64;

// Column sums of a 16-column slab over the 32 lanes of a warp, by halving: each step a lane
// keeps half of its columns and adds the partner's copy of them (16 shuffles in all). Lane l
// returns the sum of column col = 8 b4 + 4 b3 + 2 b2 + b1 (b_k: bit k of l); lanes l and l ^ 1
// hold the same column.
__device__ __forceinline__ float warp_column_sums16(const float (&v)[16], int lane, int &col) {
  const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4, h1 = lane & 2;
  float a[8], b[4], d[2];
#pragma unroll
  for (int c = 0; c < 8; ++c)
    a[c] = (h4 ? v[c + 8] : v[c]) + __shfl_xor_sync(0xffffffffu, h4 ? v[c] : v[c + 8], 16);
#pragma unroll
  for (int c = 0; c < 4; ++c)
    b[c] = (h3 ? a[c + 4] : a[c]) + __shfl_xor_sync(0xffffffffu, h3 ? a[c] : a[c + 4], 8);
#pragma unroll
  for (int c = 0; c < 2; ++c)
    d[c] = (h2 ? b[c + 2] : b[c]) + __shfl_xor_sync(0xffffffffu, h2 ? b[c] : b[c + 2], 4);
  float e = (h1 ? d[1] : d[0]) + __shfl_xor_sync(0xffffffffu, h1 ? d[0] : d[1], 2);
  e += __shfl_xor_sync(0xffffffffu, e, 1);
  col = (h4 ? 8 : 0) + (h3 ? 4 : 0) + (h2 ? 2 : 0) + (h1 ? 1 : 0);
  return e;
}

// Thread t copies its batch row of a row-major bf16 matrix [rows][kin] into column t of a
// K-major tile whose rows are the kin inputs (K = the 128 batch rows): 16-byte row loads,
// and the 2-byte stores of a warp fall in four 16-byte runs.
__device__ __forceinline__ void stage_row_as_column(unsigned char *tile, const __nv_bfloat16 *src, int64_t row,
                                                    int64_t rows, int kin) {
  const int t = threadIdx.x;
  for (int c8 = 0; c8 < kin; c8 += 8) {
    uint4 q = make_uint4(0u, 0u, 0u, 0u);
    if (row < rows)
      q = *reinterpret_cast<const uint4 *>(src + row * kin + c8);
    const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&q);
#pragma unroll
    for (int j = 0; j < 8; ++j)
      *reinterpret_cast<__nv_bfloat16 *>(tile + kmajor_offset(c8 + j, t, 128)) = e[j];
  }
}

// One 128-row batch tile per block. The weight gradients of the tile (tensor-core products in
// TMEM) and its bias gradients (warp column sums) are written to the block's slice of
// `partials` [gridDim.x][kMlpParams]; k_sum_partials adds the slices in block order, so the
// result does not depend on the order the blocks run in. wt holds W2^T, W3^T and W4^T
// (row-major [in][out]), made once per pass by k_transpose_weights.
__global__ void __launch_bounds__(128, 1) k_mlp_backward(MlpWeights w, const __nv_bfloat16 *wt, MlpActs acts,
                                                         const float *gout, int64_t B, float *partials,
                                                         unsigned *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sWt2 = smem, *sWt3 = smem + 32768, *sWt4 = smem + 65536;
  unsigned char *sA = sWt4 + 4096, *sAt = sA + 32768, *sBt = sAt + 32768, *sSm = sBt + 32768;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sSm + 4096);
  __shared__ uint32_t s_tmem;
  __shared__ float s_db[4][kMlpHidden];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t row0 = (int64_t)blockIdx.x * 128, row = row0 + t;
  const bool keep = row < B;
  const MlpGrads g = mlp_grads(partials + (size_t)blockIdx.x * kMlpParams);
  if (t < 32)
    umma::tmem_alloc(&s_tmem, 256);
  if (t == 0)
    umma::mbar_init(mbar, 1);
  // transposed weights: B operand rows = layer inputs, K = layer outputs
  stage_rowmajor(sWt2, wt, kMlpHidden, kMlpHidden);
  stage_rowmajor(sWt3, wt + 16384, kMlpHidden, kMlpHidden);
  stage_rowmajor(sWt4, wt + 32768, kMlpHidden, kMlpOut);
  stage_wait();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = s_tmem;
  const uint32_t lane_base = (uint32_t)(t & ~31) << 16;
  const uint32_t tdy = tmem + lane_base, tdw = tmem + 128 + lane_base;
  Sync sy{mbar, 0u, err, 1u, true};

  // ---- output layer: dZ4 = gout
  float dz4[kMlpOut];
#pragma unroll
  for (int c = 0; c < kMlpOut; ++c)
    dz4[c] = keep ? gout[row * kMlpOut + c] : 0.0f;
#pragma unroll
  for (int c = 0; c < kMlpOut; ++c) {
    st_bf16(sA, t, c, kMlpOut, dz4[c]);          // A for dY3: rows x K=16
    st_bf16(sSm, c, t, 128, dz4[c]);             // B for dW4^T: N=16 rows x K=128 rows
  }
  {
    int col;
    const float sum = warp_column_sums16(dz4, lane, col);
    if (!(lane & 1))
      s_db[warp][col] = sum;
  }
  stage_row_as_column(sBt, acts.y3, row, B, kMlpHidden);  // Y3^T (rows = 128 inputs, K = batch rows)
  // dW4^T [in][out] = Y3^T dZ4 ; dY3 = dZ4 W4
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (t < kMlpOut)
    g.b4[t] = s_db[0][t] + s_db[1][t] + s_db[2][t] + s_db[3][t];
  if (t == 0) {
    umma::gemm_issue(tmem + 128, smem_u32(sBt), smem_u32(sSm), 128, kMlpOut, false);
    umma::gemm_issue(tmem, smem_u32(sA), smem_u32(sWt4), kMlpOut, kMlpHidden, false);
    umma::commit(mbar);
  }
  sy.wait();
  if (sy.ok) {
    // thread t holds dW4^T row t (input t): grad_w4[out][t]
    float v[16];
    umma::tmem_ld16(tdw, v);
#pragma unroll
    for (int c = 0; c < kMlpOut; ++c)
      g.w4[(size_t)c * kMlpHidden + t] = v[c];
  }

  // ---- hidden layers 3, 2, 1
  for (int layer = 3; layer >= 1 && sy.ok; --layer) {
    const float *z = layer == 3 ? acts.z3 : (layer == 2 ? acts.z2 : acts.z1);
    const __nv_bfloat16 *yprev = layer == 3 ? acts.y2 : (layer == 2 ? acts.y1 : acts.y0);
    const int kin = layer == 1 ? kMlpIn : kMlpHidden;
    float *gw = layer == 3 ? g.w3 : (layer == 2 ? g.w2 : g.w1);
    float *gb = layer == 3 ? g.b3 : (layer == 2 ? g.b2 : g.b1);
    // dZ = dY * SiLU'(Z): this thread's row of dY from TMEM
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tdy + c0, v);
      __align__(16) __nv_bfloat16 zb[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        v[c] = keep ? v[c] * silu_grad(z[row * kMlpHidden + c0 + c]) : 0.0f;
        zb[c] = __float2bfloat16(v[c]);
        *reinterpret_cast<__nv_bfloat16 *>(sAt + kmajor_offset(c0 + c, t, 128)) = zb[c];  // dW's A
      }
      // A for dY_prev: rows x K=128 outputs, two 16-byte rows of core matrices
      *reinterpret_cast<uint4 *>(sA + kmajor_offset(t, c0, kMlpHidden)) = *reinterpret_cast<const uint4 *>(zb);
      *reinterpret_cast<uint4 *>(sA + kmajor_offset(t, c0 + 8, kMlpHidden)) =
          *reinterpret_cast<const uint4 *>(zb + 8);
      int col;
      const float sum = warp_column_sums16(v, lane, col);
      if (!(lane & 1))
        s_db[warp][c0 + col] = sum;
    }
    stage_row_as_column(sBt, yprev, row, B, kin);  // Y_prev^T (rows = inputs, K = batch rows)
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    gb[t] = s_db[0][t] + s_db[1][t] + s_db[2][t] + s_db[3][t];
    if (t == 0) {
      umma::gemm_issue(tmem + 128, smem_u32(sAt), smem_u32(sBt), 128, kin, false);  // dW [out][in]
      if (layer > 1)
        umma::gemm_issue(tmem, smem_u32(sA), smem_u32(layer == 3 ? sWt3 : sWt2), kMlpHidden, kMlpHidden,
                         false);  // dY_prev
      umma::commit(mbar);
    }
    sy.wait();
    if (sy.ok)
      for (int c0 = 0; c0 < kin; c0 += 16) {  // this thread's row of dW [out][in]
        float v[16];
        umma::tmem_ld16(tdw + c0, v);
        float4 *dst = reinterpret_cast<float4 *>(gw + (size_t)t * kin + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (t < 32)
    umma::tmem_dealloc(tmem, 256);
}

// W2^T, W3^T and W4^T (row-major [in][out]) for the backward pass's B operands.
__global__ void k_transpose_weights(MlpWeights w, __nv_bfloat16 *wt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < 2 * 16384) {
    const int l = e >> 14, r = (e >> 7) & 127, c = e & 127;  // wt[l][r = in][c = out]
    wt[e] = (l ? w.w3 : w.w2)[c * 128 + r];
  } else if (e < 2 * 16384 + 2048) {
    const int f = e - 2 * 16384, r = f >> 4, c = f & 15;  // [in 128][out 16]
    wt[e] = w.w4[c * 128 + r];
  }
}

// grad[i] = sum over blocks b (in order) of partials[b][i].
__global__ void k_sum_partials(const float *partials, int nblocks, float *grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams)
    return;
  float s = 0.0f;
  for (int b = 0; b < nblocks; ++b)
    s += partials[(size_t)b * kMlpParams + i];
  grad[i] = s;
}

// ------------------------------------------------------------------ Adam and helpers
__global__ void k_adam(float *p, float *m, float *v, float *grad, __nv_bfloat16 *pb, int64_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi, v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (pb)
    pb[i] = __float2bfloat16(pi);
  grad[i] = 0.0f;
}

// MSE gradient and loss over the first `cols` outputs: gout = 2 (out - target) / (B cols).
__global__ void k_mse_grad(const float *out, const float *target, int64_t B, int cols, float *gout,
                           float *loss) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (i < B)
    for (int c = 0; c < kMlpOut; ++c) {
      const float d = c < cols ? out[i * kMlpOut + c] - target[i * kMlpOut + c] : 0.0f;
      gout[i * kMlpOut + c] = 2.0f * d / (float)(B * cols);
      l += d * d;
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0)
    atomicAdd(loss, l / (float)(B * cols));
}

int mlp_forward(const MlpWeights &w, const float *x, int64_t B, float *out, const MlpActs &acts, unsigned *err,
                cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    VPD_CUDA(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem));
    VPD_CUDA(cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmem));
    configured = true;
  }
  k_mlp_forward<<<(unsigned)((B + 127) / 128), 128, kFwdSmem, s>>>(w, x, B, out, acts, err);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int64_t mlp_backward_blocks(int64_t B) { return (B + 127) / 128; }

int mlp_backward(const MlpWeights &w, const MlpActs &acts, const float *gout, int64_t B, float *grad,
                 const MlpBackwardScratch &scr, unsigned *err, cudaStream_t s) {
  const int64_t nb = mlp_backward_blocks(B);
  k_transpose_weights<<<(2 * 16384 + 2048 + 255) / 256, 256, 0, s>>>(w, scr.wt);
  VPD_CUDA(cudaGetLastError());
  k_mlp_backward<<<(unsigned)nb, 128, kBwdSmem, s>>>(w, scr.wt, acts, gout, B, scr.partials, err);
  VPD_CUDA(cudaGetLastError());
  k_sum_partials<<<(unsigned)((kMlpParams + 255) / 256), 256, 0, s>>>(scr.partials, (int)nb, grad);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int mlp_adam(float *p, float *m, float *v, float *grad, __nv_bfloat16 *pb, int64_t n, float lr, int step,
             cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, m, v, grad, pb, n, lr, b1, b2, 1e-8f, c1, c2);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int mlp_mse_grad(const float *out, const float *target, int64_t B, int cols, float *gout, float *loss,
                 cudaStream_t s) {
  k_mse_grad<<<(unsigned)((B + 255) / 256), 256, 0, s>>>(out, target, B, cols, gout, loss);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd

// ------------------------------------------------------------------ C ABI (device pointers)
namespace {
int check_err(unsigned *derr, cudaStream_t s) {
  unsigned e = 0;
  VPD_CUDA(cudaMemcpyAsync(&e, derr, sizeof e, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (e)
    return vpd::set_error(VPD_ERR_CUDA, "surrogate network: tensor-core wait timed out");
  return VPD_OK;
}
}  // namespace

using namespace vpd;

extern "C" int vpd_mlp_forward(const uint16_t *weights, const float *biases, const float *x, int64_t batch,
                               float *out, void *stream) {
  if (!weights || !biases || !x || !out || batch < 1)
    return set_error(VPD_ERR_INVALID, "vpd_mlp_forward: invalid argument");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned *derr = nullptr;
  VPD_CUDA(cudaMalloc(&derr, sizeof(unsigned)));
  VPD_CUDA(cudaMemsetAsync(derr, 0, sizeof(unsigned), s));
  const MlpWeights w = mlp_weights(reinterpret_cast<const __nv_bfloat16 *>(weights), biases);
  int rc = mlp_forward(w, x, batch, out, MlpActs{}, derr, s);
  if (rc == VPD_OK)
    rc = check_err(derr, s);
  cudaFree(derr);
  return rc;
}

extern "C" int vpd_mlp_gradients(const uint16_t *weights, const float *biases, const float *x,
                                 const float *gout, int64_t batch, float *grad, void *stream) {
  if (!weights || !biases || !x || !gout || !grad || batch < 1)
    return set_error(VPD_ERR_INVALID, "vpd_mlp_gradients: invalid argument");
  cudaStream_t s = (cudaStream_t)stream;
  const MlpWeights w = mlp_weights(reinterpret_cast<const __nv_bfloat16 *>(weights), biases);
  unsigned char *buf = nullptr;
  const size_t nb = (size_t)batch;
  const size_t blocks = (size_t)mlp_backward_blocks(batch);
  const size_t bytes = nb * kMlpIn * 2 + nb * kMlpHidden * (4 * 3 + 2 * 3) + nb * kMlpOut * 4 + 256 +
                       sizeof(float) * blocks * kMlpParams + sizeof(uint16_t) * kMlpWeights;
  VPD_CUDA(cudaMalloc(&buf, bytes));
  MlpActs a;
  unsigned char *q = buf;
  a.y0 = reinterpret_cast<__nv_bfloat16 *>(q), q += nb * kMlpIn * 2;
  a.z1 = reinterpret_cast<float *>(q), q += nb * kMlpHidden * 4;
  a.z2 = reinterpret_cast<float *>(q), q += nb * kMlpHidden * 4;
  a.z3 = reinterpret_cast<float *>(q), q += nb * kMlpHidden * 4;
  a.y1 = reinterpret_cast<__nv_bfloat16 *>(q), q += nb * kMlpHidden * 2;
  a.y2 = reinterpret_cast<__nv_bfloat16 *>(q), q += nb * kMlpHidden * 2;
  a.y3 = reinterpret_cast<__nv_bfloat16 *>(q), q += nb * kMlpHidden * 2;
  float *out = reinterpret_cast<float *>(q), *derrf = out + nb * kMlpOut;
  unsigned *derr = reinterpret_cast<unsigned *>(derrf);
  q = reinterpret_cast<unsigned char *>(derrf) + 256;
  MlpBackwardScratch scr;
  scr.partials = reinterpret_cast<float *>(q), q += sizeof(float) * blocks * kMlpParams;
  scr.wt = reinterpret_cast<__nv_bfloat16 *>(q);
  int rc = VPD_OK;
  cudaError_t e = cudaMemsetAsync(derr, 0, sizeof(unsigned), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(grad, 0, sizeof(float) * kMlpParams, s);
  if (e != cudaSuccess)
    rc = cuda_error(e, "vpd_mlp_gradients");
  if (rc == VPD_OK)
    rc = mlp_forward(w, x, batch, out, a, derr, s);
  if (rc == VPD_OK)
    rc = mlp_backward(w, a, gout, batch, grad, scr, derr, s);
  if (rc == VPD_OK)
    rc = check_err(derr, s);
  cudaFree(buf);
  return rc;
}
