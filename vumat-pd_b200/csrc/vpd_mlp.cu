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
// smem: W1 (128x16) | W2 (128x128) | W3 | W4 (16x128) | A (128x128) | X0 (128x16) | barrier
constexpr size_t kFwdSmem = 4096 + 32768 + 32768 + 4096 + 32768 + 4096 + 64;

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
  __shared__ uint32_t s_tmem;
  const int t = threadIdx.x;
  const int64_t row = (int64_t)blockIdx.x * 128 + t;
  if (t < 32)
    umma::tmem_alloc(&s_tmem, 128);
  if (t == 0)
    umma::mbar_init(mbar, 1);
  stage_weights_fwd(smem, w);
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
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = s_tmem;
  const uint32_t trow = tmem + ((uint32_t)(t & ~31) << 16);  // this warp's TMEM lanes
  Sync sy{mbar, 0u, err, 1u, true};
  const bool keep = row < B;
  gemm(sy, tmem, sX, sW1, kMlpIn, kMlpHidden);
  hidden_epilogue(trow, w.b1, sA, keep && acts.z1 ? acts.z1 + row * kMlpHidden : nullptr,
                  keep && acts.y1 ? acts.y1 + row * kMlpHidden : nullptr);
  gemm(sy, tmem, sA, sW2, kMlpHidden, kMlpHidden);
  hidden_epilogue(trow, w.b2, sA, keep && acts.z2 ? acts.z2 + row * kMlpHidden : nullptr,
                  keep && acts.y2 ? acts.y2 + row * kMlpHidden : nullptr);
  gemm(sy, tmem, sA, sW3, kMlpHidden, kMlpHidden);
  hidden_epilogue(trow, w.b3, sA, keep && acts.z3 ? acts.z3 + row * kMlpHidden : nullptr,
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

// Accumulates the calling thread's TMEM row of a weight-gradient product into grad[row][*].
__device__ __forceinline__ void flush_grad(uint32_t trow, int ncols, float *grad_row, int stride) {
  for (int c0 = 0; c0 < ncols; c0 += 16) {
    float v[16];
    umma::tmem_ld16(trow + c0, v);
#pragma unroll
    for (int c = 0; c < 16; ++c)
      if (c0 + c < ncols)
        atomicAdd(grad_row + (size_t)(c0 + c) * stride, v[c]);
  }
}

__global__ void __launch_bounds__(128, 1) k_mlp_backward(MlpWeights w, MlpActs acts, const float *gout,
                                                         int64_t B, MlpGrads g, unsigned *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *sWt2 = smem, *sWt3 = smem + 32768, *sWt4 = smem + 65536;
  unsigned char *sA = sWt4 + 4096, *sAt = sA + 32768, *sBt = sAt + 32768, *sSm = sBt + 32768;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sSm + 4096);
  __shared__ uint32_t s_tmem;
  __shared__ float s_db[kMlpHidden];
  const int t = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * 128, row = row0 + t;
  const bool keep = row < B;
  if (t < 32)
    umma::tmem_alloc(&s_tmem, 256);
  if (t == 0)
    umma::mbar_init(mbar, 1);
  // transposed weights: B operand rows = layer inputs, K = layer outputs
  stage_transposed(sWt2, w.w2, kMlpHidden, kMlpHidden);
  stage_transposed(sWt3, w.w3, kMlpHidden, kMlpHidden);
  stage_transposed(sWt4, w.w4, kMlpOut, kMlpHidden);
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
    atomicAdd(g.b4 + c, dz4[c]);
  }
  // Y3^T into Bt (rows = 128 inputs, K = batch rows)
  for (int e = t; e < 128 * kMlpHidden; e += 128) {
    const int r = e / kMlpHidden, c = e % kMlpHidden;
    const __nv_bfloat16 y = row0 + r < B ? acts.y3[(row0 + r) * kMlpHidden + c] : __float2bfloat16(0.0f);
    *reinterpret_cast<__nv_bfloat16 *>(sBt + kmajor_offset(c, r, 128)) = y;
  }
  // dW4^T [in][out] = Y3^T dZ4 ; dY3 = dZ4 W4
  umma::fence_proxy_async();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
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
      atomicAdd(g.w4 + (size_t)c * kMlpHidden + t, v[c]);
  }

  // ---- hidden layers 3, 2, 1
  for (int layer = 3; layer >= 1 && sy.ok; --layer) {
    const float *z = layer == 3 ? acts.z3 : (layer == 2 ? acts.z2 : acts.z1);
    const __nv_bfloat16 *yprev = layer == 3 ? acts.y2 : (layer == 2 ? acts.y1 : acts.y0);
    const int kin = layer == 1 ? kMlpIn : kMlpHidden;
    float *gw = layer == 3 ? g.w3 : (layer == 2 ? g.w2 : g.w1);
    float *gb = layer == 3 ? g.b3 : (layer == 2 ? g.b2 : g.b1);
    // dZ = dY * SiLU'(Z): this thread's row of dY from TMEM
    if (t < kMlpHidden)
      s_db[t] = 0.0f;
    __syncthreads();
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tdy + c0, v);
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        const float dz = keep ? v[c] * silu_grad(z[row * kMlpHidden + c0 + c]) : 0.0f;
        st_bf16(sA, t, c0 + c, kMlpHidden, dz);   // A for dY_prev: rows x K=128 outputs
        st_bf16(sAt, c0 + c, t, 128, dz);         // A for dW: outputs x K=128 rows
        atomicAdd(&s_db[c0 + c], dz);
      }
    }
    // Y_prev^T into Bt (rows = inputs, K = batch rows)
    for (int e = t; e < 128 * kin; e += 128) {
      const int r = e / kin, c = e % kin;
      const __nv_bfloat16 y = row0 + r < B ? yprev[(row0 + r) * kin + c] : __float2bfloat16(0.0f);
      *reinterpret_cast<__nv_bfloat16 *>(sBt + kmajor_offset(c, r, 128)) = y;
    }
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (t < kMlpHidden)
      atomicAdd(gb + t, s_db[t]);
    if (t == 0) {
      umma::gemm_issue(tmem + 128, smem_u32(sAt), smem_u32(sBt), 128, kin, false);  // dW [out][in]
      if (layer > 1)
        umma::gemm_issue(tmem, smem_u32(sA), smem_u32(layer == 3 ? sWt3 : sWt2), kMlpHidden, kMlpHidden,
                         false);  // dY_prev
      umma::commit(mbar);
    }
    sy.wait();
    if (sy.ok)
      flush_grad(tdw, kin, gw + (size_t)t * kin, 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (t < 32)
    umma::tmem_dealloc(tmem, 256);
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

int mlp_backward(const MlpWeights &w, const MlpActs &acts, const float *gout, int64_t B, const MlpGrads &g,
                 unsigned *err, cudaStream_t s) {
  k_mlp_backward<<<(unsigned)((B + 127) / 128), 128, kBwdSmem, s>>>(w, acts, gout, B, g, err);
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
  const size_t bytes = nb * kMlpIn * 2 + nb * kMlpHidden * (4 * 3 + 2 * 3) + nb * kMlpOut * 4 + 256;
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
  int rc = VPD_OK;
  cudaError_t e = cudaMemsetAsync(derr, 0, sizeof(unsigned), s);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(grad, 0, sizeof(float) * kMlpParams, s);
  if (e != cudaSuccess)
    rc = cuda_error(e, "vpd_mlp_gradients");
  if (rc == VPD_OK)
    rc = mlp_forward(w, x, batch, out, a, derr, s);
  if (rc == VPD_OK)
    rc = mlp_backward(w, a, gout, batch, mlp_grads(grad), derr, s);
  if (rc == VPD_OK)
    rc = check_err(derr, s);
  cudaFree(buf);
  return rc;
}
