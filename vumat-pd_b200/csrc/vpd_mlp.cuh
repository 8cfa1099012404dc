// Surrogate network: sizes, parameter/activation/gradient views and launchers (vpd_mlp.cu).
#pragma once

#include "vpd_internal.h"

#include <cuda_bf16.h>

namespace vpd {

constexpr int kMlpIn = 16;      // 10 features, zero padded
constexpr int kMlpHidden = 128;
constexpr int kMlpOut = 16;     // 7 targets, zero padded
constexpr int kMlpFeatures = 10;
constexpr int kMlpTargets = 7;
// flat parameter order: w1 [128][16], w2 [128][128], w3 [128][128], w4 [16][128] (row-major
// [out][in]), then b1 [128], b2 [128], b3 [128], b4 [16]
constexpr int64_t kMlpWeights = 128 * 16 + 128 * 128 * 2 + 16 * 128;
constexpr int64_t kMlpParams = kMlpWeights + 128 * 3 + 16;

struct MlpWeights {
  const __nv_bfloat16 *w1, *w2, *w3, *w4;
  const float *b1, *b2, *b3, *b4;
};

// Activations kept for the backward pass (any pointer may be null in inference).
struct MlpActs {
  __nv_bfloat16 *y0;              // [B][16] inputs as fed
  float *z1, *z2, *z3;            // [B][128] pre-activations
  __nv_bfloat16 *y1, *y2, *y3;    // [B][128] activations
};

struct MlpGrads {  // FP32 accumulators, same shapes as the parameters
  float *w1, *w2, *w3, *w4, *b1, *b2, *b3, *b4;
};

__host__ __device__ inline MlpWeights mlp_weights(const __nv_bfloat16 *wb, const float *bias) {
  return MlpWeights{wb, wb + 2048, wb + 2048 + 16384, wb + 2048 + 32768,
                    bias, bias + 128, bias + 256, bias + 384};
}
__host__ __device__ inline MlpGrads mlp_grads(float *g) {
  return MlpGrads{g, g + 2048, g + 2048 + 16384, g + 2048 + 32768,
                  g + kMlpWeights, g + kMlpWeights + 128, g + kMlpWeights + 256, g + kMlpWeights + 384};
}

int mlp_forward(const MlpWeights &w, const float *x, int64_t B, float *out, const MlpActs &acts,
                unsigned *err, cudaStream_t s);
// Scratch of one backward pass: the transposed weights (VPD_MLP_WEIGHTS - 2048 bf16) and one
// partial gradient per 128-row block (mlp_backward_blocks(B) x kMlpParams floats).
struct MlpBackwardScratch {
  __nv_bfloat16 *wt;
  float *partials;
};
int64_t mlp_backward_blocks(int64_t B);
// grad [kMlpParams] = d/dparams of sum(out * gout) over the batch (overwritten, not accumulated).
int mlp_backward(const MlpWeights &w, const MlpActs &acts, const float *gout, int64_t B, float *grad,
                 const MlpBackwardScratch &scr, unsigned *err, cudaStream_t s);
int mlp_adam(float *p, float *m, float *v, float *grad, __nv_bfloat16 *pb, int64_t n, float lr,
             int step, cudaStream_t s);
int mlp_mse_grad(const float *out, const float *target, int64_t B, int cols, float *gout,
                 float *loss, cudaStream_t s);

}  // namespace vpd
