// The learned Johnson-Cook update (no counterpart in the reference):
//
//   k_surrogate_samples    training increments generated and solved by the device VUMAT
//                          (jc_trial + jc_bisection + jc_finish, the plain path's own code)
//   train_surrogate        Adam on the weighted MSE, with the tensor-core forward and backward
//                          kernels of vpd_mlp.cu
//   k_material_surrogate   the material stage with the learned return map, 128 points per
//                          tile: the kinematics and the elastic trial (vpd_material.cuh), the
//                          network's guess for the points that need it, then per point the
//                          Newton acceptance (vpd_surrogate.cuh) or the bisection fallback, the
//                          radial scaling, the force map and the diagnostics partials. With the
//                          network guess for every yielding point it is a persistent kernel
//                          with the weights staged once per CTA and the network as four
//                          tcgen05 products per tile (thread t = point t = TMEM lane t); with
//                          the hybrid guess the few points without plastic history are
//                          evaluated by the block on the CUDA cores (sparse_net_ratio).
#include "vpd_material.cuh"
#include "vpd_mlp_tile.cuh"
#include "vpd_surrogate.cuh"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace vpd {

// ------------------------------------------------------------------ training samples
__device__ __forceinline__ double sample_uniform(uint64_t seed, int64_t k, int d) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * ((uint64_t)k * 64u + (uint64_t)d + 1u);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ double sample_gauss(uint64_t seed, int64_t k, int d) {  // Box-Muller
  const double u1 = 1.0 - sample_uniform(seed, k, d), u2 = sample_uniform(seed, k, d + 1);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

// Unit deviatoric direction in the norm a:a = a0^2 + a1^2 + a2^2 + 2 (a3^2 + a4^2 + a5^2).
__device__ __forceinline__ void deviatoric_unit(double *a) {
  const double m = (a[0] + a[1] + a[2]) / 3.0;
  a[0] -= m, a[1] -= m, a[2] -= m;
  double nn = a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + 2.0 * (a[3] * a[3] + a[4] * a[4] + a[5] * a[5]);
  nn = nn > 1.0e-300 ? sqrt(nn) : 1.0;
#pragma unroll
  for (int c = 0; c < 6; ++c)
    a[c] /= nn;
}

// One sample is one increment from a sampled state (the synthetic training set of the
// surrogate): strain increment N(0, 1e-4) per component for even rows, log-uniform magnitude
// 1e-8..1e-3 in a random direction for odd rows (the small increments of an explicit step);
// eqps log-uniform [1e-6, 0.5]; total equivalent strain rate log-uniform [1e-3, 1e4] /s, which
// sets dt; T uniform [293, 1200] K; old deviatoric stress between the increment's direction
// and a random one, on the yield surface (yield stress at the sampled rate) for 70 % of rows
// and inside it otherwise; pressure N(0, (0.3 sigma_y)^2). The VUMAT's bisection (cold start)
// solves it; its plastic increment and stress increment are the targets.
__global__ void k_surrogate_samples(JcParams jc, uint64_t seed, int64_t count, float *X, float *Y, double *rec) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count)
    return;
  double inc[6];
  if ((k & 1) == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c)
      inc[c] = 1.0e-4 * sample_gauss(seed, k, 2 * c);
  } else {
    double nn = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c)
      inc[c] = sample_gauss(seed, k, 2 * c), nn += inc[c] * inc[c];
    const double mag = pow(10.0, -8.0 + 5.0 * sample_uniform(seed, k, 12)) / sqrt(nn > 0.0 ? nn : 1.0);
#pragma unroll
    for (int c = 0; c < 6; ++c)
      inc[c] *= mag;
  }
  const double lo = log10(1.0e-6), hi = log10(0.5);
  const double epOld = pow(10.0, lo + (hi - lo) * sample_uniform(seed, k, 13));
  const double rate = pow(10.0, -3.0 + 7.0 * sample_uniform(seed, k, 14)) * 1.0e-3;  // per ms
  const double temperature = 293.0 + 907.0 * sample_uniform(seed, k, 15);
  double deq = equivalent_increment(inc);
  deq = deq > 1.0e-300 ? deq : 1.0e-300;
  const double dt = deq / rate;
  const double oldYield = jc_yield(jc, epOld, rate, temperature);
  double dinc[6], rnd[6], dir[6];
#pragma unroll
  for (int c = 0; c < 6; ++c)
    dinc[c] = inc[c], rnd[c] = sample_gauss(seed, k, 16 + 2 * c);
  deviatoric_unit(dinc);
  deviatoric_unit(rnd);
  const double a = sample_uniform(seed, k, 28);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    dir[c] = a * dinc[c] + (1.0 - a) * rnd[c];
  deviatoric_unit(dir);
  const double qOld = oldYield * (sample_uniform(seed, k, 29) < 0.7 ? 1.0 : 0.5 + 0.5 * sample_uniform(seed, k, 30));
  const double pressure = 0.3 * oldYield * sample_gauss(seed, k, 31);
  const double s = sqrt(2.0 / 3.0) * qOld;
  JcPoint pt;
#pragma unroll
  for (int c = 0; c < 6; ++c)
    pt.stress[c] = s * dir[c] + (c < 3 ? pressure : 0.0);
  pt.state[0] = 1.0, pt.state[1] = epOld, pt.state[2] = temperature, pt.state[3] = oldYield;
  pt.state[4] = 0.0, pt.state[5] = 0.0;
  pt.eInternal = 0.0, pt.eInelastic = 0.0;
  double old[6];
#pragma unroll
  for (int c = 0; c < 6; ++c)
    old[c] = pt.stress[c];

  JcTrial t;
  jc_trial(jc, inc, pt, t);  // state[0] = 1: never the initialising call
  const double yield0 = jc_yield0(jc, t);
  const bool plastic = t.qTrial - yield0 >= jc.tolerance;
  float f[SURROGATE_FEATURES];
  surrogate_features(jc, dt, inc, t, f);
  double epInc, yield;
  const int it = jc_bisection(jc, dt, t, 0.0, epInc, yield);
  jc_finish(jc, inc, t, epInc, yield, (double)it, pt);

  float *x = X + 16 * k, *y = Y + 16 * k;
#pragma unroll
  for (int c = 0; c < 16; ++c)
    x[c] = c < SURROGATE_FEATURES ? f[c] : 0.0f, y[c] = 0.0f;
  y[0] = plastic ? (float)(epInc / floor_increment(jc, t)) : 0.0f;
#pragma unroll
  for (int c = 0; c < 6; ++c)
    y[1 + c] = (float)((pt.stress[c] - old[c]) / (2.0 * jc.mu * deq));
  y[15] = plastic ? 1.0f : 0.0f;
  if (rec) {
    double *r = rec + (size_t)VPD_SAMPLE_RECORD * k;
#pragma unroll
    for (int c = 0; c < 6; ++c)
      r[c] = inc[c], r[6 + c] = old[c], r[16 + c] = pt.stress[c];
    r[12] = epOld, r[13] = temperature, r[14] = oldYield, r[15] = dt;
    r[22] = epInc, r[23] = (double)it, r[24] = plastic ? 1.0 : 0.0, r[25] = yield0;
  }
}

int surrogate_samples_dev(const JcParams &jc, uint64_t seed, int64_t count, float *X, float *Y, double *rec,
                          cudaStream_t s) {
  k_surrogate_samples<<<(unsigned)((count + 127) / 128), 128, 0, s>>>(jc, seed, count, X, Y, rec);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

// ------------------------------------------------------------------ training
__global__ void k_gather_rows(const float *X, const float *Y, int64_t rows, uint64_t mul, uint64_t add,
                              int64_t first, int64_t B, float *Xb, float *Yb) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B * 16)
    return;
  const int64_t r = e >> 4, c = e & 15;
  const int64_t src = (int64_t)((mul * (uint64_t)(first + r) + add) % (uint64_t)rows);  // a permutation
  Xb[e] = X[src * 16 + c];
  Yb[e] = Y[src * 16 + c];
}

// Weighted MSE over the 7 targets (row weight in target column 15, target 0 weighted 4):
// gout = d loss / d out, loss += this batch's mean.
__global__ void k_weighted_mse(const float *out, const float *target, int64_t B, float *gout, float *loss) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (i < B) {
    const float w = target[i * 16 + 15];
    const float norm = 1.0f / (float)(B * SURROGATE_TARGETS);
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const float cw = c == 0 ? 4.0f : 1.0f;
      const float d = c < SURROGATE_TARGETS ? out[i * 16 + c] - target[i * 16 + c] : 0.0f;
      gout[i * 16 + c] = 2.0f * w * cw * d * norm;
      l += w * cw * d * d * norm;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0)
    atomicAdd(loss, l);
}

__global__ void k_to_bf16(const float *p, __nv_bfloat16 *q, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    q[i] = __float2bfloat16(p[i]);
}

namespace {

// Device buffers of one training run, freed on every exit path.
struct TrainBuffers {
  std::vector<void *> ptrs;
  ~TrainBuffers() {
    for (void *p : ptrs)
      cudaFree(p);
  }
  template <typename T> int alloc(T **p, size_t count) {
    void *q = nullptr;
    VPD_CUDA(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    ptrs.push_back(q);
    *p = static_cast<T *>(q);
    return VPD_OK;
  }
};

struct StreamGuard {
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~StreamGuard() {
    if (s)
      cudaStreamSynchronize(s), cudaStreamDestroy(s);
    if (e0)
      cudaEventDestroy(e0);
    if (e1)
      cudaEventDestroy(e1);
  }
};

uint64_t splitmix(uint64_t &state) {
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Multiplier of the affine row permutation of one epoch (coprime to the row count).
uint64_t epoch_multiplier(uint64_t rows, int epoch) {
  uint64_t a = (2654435761ull + 2ull * (uint64_t)epoch * 1013904223ull) % rows;
  a = a ? a : 1;
  while (std::gcd(a, rows) != 1)
    a = a + 1 < rows ? a + 1 : 1;
  return a;
}

int check_config(const vpd_surrogate_config *c) {
  if (!c)
    return set_error(VPD_ERR_INVALID, "vpd_train_surrogate: null config");
  for (int k = 0; k < 14; ++k)
    if (!std::isfinite(c->props[k]))
      return set_error(VPD_ERR_INVALID, "vpd_train_surrogate: non-finite material property");
  if (c->batch < 128 || c->epochs < 1 || c->epochs > VPD_SURROGATE_MAX_EPOCHS ||
      !(c->learning_rate > 0.0) || !(c->validation_fraction >= 0.0 && c->validation_fraction <= 0.5))
    return set_error(VPD_ERR_INVALID, "vpd_train_surrogate: batch >= 128, 1 <= epochs <= 64, "
                                      "learning_rate > 0, validation_fraction in [0, 0.5]");
  const int64_t val = (int64_t)((double)c->samples * c->validation_fraction);
  if (c->samples - val < c->batch)
    return set_error(VPD_ERR_INVALID, "vpd_train_surrogate: fewer training samples than one batch");
  return VPD_OK;
}

}  // namespace

int train_surrogate(const vpd_surrogate_config &cfg, uint16_t *w_out, float *b_out, vpd_surrogate_report *rep) {
  const JcParams jc = make_jc_params(cfg.props);
  const int64_t S = cfg.samples, V = (int64_t)((double)S * cfg.validation_fraction), T = S - V;
  const int64_t B = cfg.batch;
  StreamGuard g;
  VPD_CUDA(cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking));
  VPD_CUDA(cudaEventCreate(&g.e0));
  VPD_CUDA(cudaEventCreate(&g.e1));
  cudaStream_t s = g.s;
  TrainBuffers buf;
  float *X = nullptr, *Y = nullptr, *Xb = nullptr, *Yb = nullptr, *out = nullptr, *gout = nullptr;
  float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr, *P = nullptr, *M = nullptr, *Vm = nullptr, *G = nullptr;
  float *loss = nullptr, *vout = nullptr;
  __nv_bfloat16 *y0 = nullptr, *y1 = nullptr, *y2 = nullptr, *y3 = nullptr, *Wb = nullptr;
  unsigned *err = nullptr;
  int rc;
  const int64_t VB = std::max<int64_t>(V, 1);
  if ((rc = buf.alloc(&X, S * 16)) || (rc = buf.alloc(&Y, S * 16)) || (rc = buf.alloc(&Xb, B * 16)) ||
      (rc = buf.alloc(&Yb, B * 16)) || (rc = buf.alloc(&out, B * 16)) || (rc = buf.alloc(&gout, B * 16)) ||
      (rc = buf.alloc(&z1, B * 128)) || (rc = buf.alloc(&z2, B * 128)) || (rc = buf.alloc(&z3, B * 128)) ||
      (rc = buf.alloc(&y0, B * 16)) || (rc = buf.alloc(&y1, B * 128)) || (rc = buf.alloc(&y2, B * 128)) ||
      (rc = buf.alloc(&y3, B * 128)) || (rc = buf.alloc(&P, kMlpParams)) || (rc = buf.alloc(&M, kMlpParams)) ||
      (rc = buf.alloc(&Vm, kMlpParams)) || (rc = buf.alloc(&G, kMlpParams)) || (rc = buf.alloc(&Wb, kMlpWeights)) ||
      (rc = buf.alloc(&loss, VPD_SURROGATE_MAX_EPOCHS + 1)) || (rc = buf.alloc(&vout, VB * 16)) ||
      (rc = buf.alloc(&err, 1)))
    return rc;
  MlpBackwardScratch bscr{};
  if ((rc = buf.alloc(&bscr.wt, kMlpWeights)) ||
      (rc = buf.alloc(&bscr.partials, (size_t)mlp_backward_blocks(B) * kMlpParams)))
    return rc;
  if ((rc = surrogate_samples_dev(jc, cfg.seed, S, X, Y, nullptr, s)))
    return rc;

  // initial parameters: uniform with variance 1 / fan_in; the padded input columns and
  // output rows are zero and stay zero (their gradients vanish)
  std::vector<float> p0((size_t)kMlpParams, 0.0f);
  {
    uint64_t st = cfg.seed ^ 0x5DEECE66Dull;
    const int rows[4] = {128, 128, 128, 16}, cols[4] = {16, 128, 128, 128}, fan[4] = {10, 128, 128, 128};
    size_t off = 0;
    for (int l = 0; l < 4; ++l) {
      const double bound = std::sqrt(3.0 / fan[l]);
      for (int r = 0; r < rows[l]; ++r)
        for (int c = 0; c < cols[l]; ++c) {
          const double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
          const bool pad = (l == 0 && c >= SURROGATE_FEATURES) || (l == 3 && r >= SURROGATE_TARGETS);
          p0[off + (size_t)r * cols[l] + c] = pad ? 0.0f : (float)((2.0 * u - 1.0) * bound);
        }
      off += (size_t)rows[l] * cols[l];
    }
  }
  VPD_CUDA(cudaMemcpyAsync(P, p0.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemsetAsync(M, 0, sizeof(float) * kMlpParams, s));
  VPD_CUDA(cudaMemsetAsync(Vm, 0, sizeof(float) * kMlpParams, s));
  VPD_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * kMlpParams, s));
  VPD_CUDA(cudaMemsetAsync(loss, 0, sizeof(float) * (VPD_SURROGATE_MAX_EPOCHS + 1), s));
  VPD_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), s));
  k_to_bf16<<<(unsigned)((kMlpWeights + 255) / 256), 256, 0, s>>>(P, Wb, kMlpWeights);
  VPD_CUDA(cudaGetLastError());

  const MlpWeights w = mlp_weights(Wb, P + kMlpWeights);
  const MlpActs acts{y0, z1, z2, z3, y1, y2, y3};
  const int64_t steps = T / B;
  int adam_step = 0;
  VPD_CUDA(cudaEventRecord(g.e0, s));
  for (int e = 0; e < cfg.epochs; ++e) {
    const uint64_t mul = epoch_multiplier((uint64_t)T, e), add = (uint64_t)e * 7919u % (uint64_t)T;
    for (int64_t k = 0; k < steps; ++k) {
      k_gather_rows<<<(unsigned)((B * 16 + 255) / 256), 256, 0, s>>>(X, Y, T, mul, add, k * B, B, Xb, Yb);
      VPD_CUDA(cudaGetLastError());
      if ((rc = mlp_forward(w, Xb, B, out, acts, err, s)))
        return rc;
      k_weighted_mse<<<(unsigned)((B + 255) / 256), 256, 0, s>>>(out, Yb, B, gout, loss + e);
      VPD_CUDA(cudaGetLastError());
      if ((rc = mlp_backward(w, acts, gout, B, G, bscr, err, s)))
        return rc;
      ++adam_step;
      if ((rc = mlp_adam(P, M, Vm, G, Wb, kMlpWeights, (float)cfg.learning_rate, adam_step, s)) ||
          (rc = mlp_adam(P + kMlpWeights, M + kMlpWeights, Vm + kMlpWeights, G + kMlpWeights, nullptr,
                         kMlpParams - kMlpWeights, (float)cfg.learning_rate, adam_step, s)))
        return rc;
    }
  }
  VPD_CUDA(cudaEventRecord(g.e1, s));
  // held-out rows: forward pass and the weighted loss
  if (V > 0) {
    if ((rc = mlp_forward(w, X + T * 16, V, vout, MlpActs{}, err, s)))
      return rc;
  }
  std::vector<float> losses(VPD_SURROGATE_MAX_EPOCHS + 1), hv((size_t)V * 16), hy((size_t)V * 16);
  unsigned herr = 0;
  VPD_CUDA(cudaMemcpyAsync(losses.data(), loss, sizeof(float) * losses.size(), cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, s));
  if (V > 0) {
    VPD_CUDA(cudaMemcpyAsync(hv.data(), vout, sizeof(float) * hv.size(), cudaMemcpyDeviceToHost, s));
    VPD_CUDA(cudaMemcpyAsync(hy.data(), Y + T * 16, sizeof(float) * hy.size(), cudaMemcpyDeviceToHost, s));
  }
  std::vector<uint16_t> hw((size_t)kMlpWeights);
  VPD_CUDA(cudaMemcpyAsync(hw.data(), Wb, sizeof(uint16_t) * kMlpWeights, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaMemcpyAsync(b_out, P + kMlpWeights, sizeof(float) * (kMlpParams - kMlpWeights),
                           cudaMemcpyDeviceToHost, s));
  // plastic fraction over all samples (target column 15)
  std::vector<float> all_w((size_t)S);
  VPD_CUDA(cudaMemcpy2DAsync(all_w.data(), sizeof(float), Y + 15, 16 * sizeof(float), sizeof(float), (size_t)S,
                             cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (herr)
    return set_error(VPD_ERR_CUDA, "vpd_train_surrogate: tensor-core wait timed out");
  std::copy(hw.begin(), hw.end(), w_out);
  if (rep) {
    *rep = vpd_surrogate_report{};
    rep->epochs_run = cfg.epochs;
    for (int e = 0; e < cfg.epochs; ++e)
      rep->epoch_loss[e] = steps ? (double)losses[e] / (double)steps : 0.0;
    double vl = 0.0, r2 = 0.0, s2 = 0.0, np = 0.0;
    for (int64_t i = 0; i < V; ++i) {
      const float *o = &hv[(size_t)i * 16], *t = &hy[(size_t)i * 16];
      if (t[15] == 0.0f)
        continue;
      np += 1.0;
      const double d0 = o[0] - t[0];
      r2 += d0 * d0;
      vl += 4.0 * d0 * d0;
      for (int c = 1; c < SURROGATE_TARGETS; ++c) {
        const double d = o[c] - t[c];
        s2 += d * d;
        vl += d * d;
      }
    }
    rep->validation_loss = V ? vl / ((double)V * SURROGATE_TARGETS) : 0.0;
    rep->ratio_rmse = np ? std::sqrt(r2 / np) : 0.0;
    rep->stress_rmse = np ? std::sqrt(s2 / (np * 6.0)) : 0.0;
    double pf = 0.0;
    for (float x : all_w)
      pf += x;
    rep->plastic_fraction = S ? pf / (double)S : 0.0;
    float ms = 0.0f;
    VPD_CUDA(cudaEventElapsedTime(&ms, g.e0, g.e1));
    rep->train_ms = ms;
  }
  return VPD_OK;
}

// ------------------------------------------------------------------ fused material kernel
// smem: W1 | W2 | W3 | W4 | A (128 x 128; the layer-1 input X sits in its first 4 KB, dead
// once the first product has completed) | mbarrier | biases
constexpr size_t kSurrSmem = 4096 + 32768 + 32768 + 4096 + 32768 + 64 + 4 * kBiasFloats;

// ------------------------------------------------------------------ sparse network inference
// The network's plastic-ratio output for ONE point, evaluated by the whole block on the CUDA
// cores: thread t computes hidden unit t of each layer (the FP32 dot product of its BF16 weight
// row with the previous layer's BF16 activations, then the bias and SiLU, rounded to BF16 as
// the tensor-core kernels store it). This serves the hybrid guess, where only the points
// without plastic history need the network (about 60 of 228k yielding points per increment
// on the 250k-point bar in plastic flow, in 3 % of the tiles): the material kernel then keeps
// four blocks per SM, without the 108 KB of staged weights and the TMEM of the tensor-core
// path. Every thread of the 128-thread block calls it.
struct SparseNet {
  float x[16];  // the point's features, BF16-rounded, zero padded
  float h[2][kMlpHidden];
  float red[kMaterialThreads / 32];
};

__device__ __forceinline__ float bf16_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }
__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16(v)); }

// sum_k row[k] in[k] over 8 k8 groups of 8 (row: bf16, 16-byte aligned; in: shared memory)
__device__ __forceinline__ float dot_bf16_row(const __nv_bfloat16 *row, const float *in, int k8s) {
  const uint4 *r = reinterpret_cast<const uint4 *>(row);
  float z = 0.0f;
#pragma unroll 4
  for (int k8 = 0; k8 < k8s; ++k8) {
    const uint4 q = __ldg(r + k8);
    const float4 a = *reinterpret_cast<const float4 *>(in + 8 * k8);
    const float4 b = *reinterpret_cast<const float4 *>(in + 8 * k8 + 4);
    z = fmaf(bf16_lo(q.x), a.x, z), z = fmaf(bf16_hi(q.x), a.y, z);
    z = fmaf(bf16_lo(q.y), a.z, z), z = fmaf(bf16_hi(q.y), a.w, z);
    z = fmaf(bf16_lo(q.z), b.x, z), z = fmaf(bf16_hi(q.z), b.y, z);
    z = fmaf(bf16_lo(q.w), b.z, z), z = fmaf(bf16_hi(q.w), b.w, z);
  }
  return z;
}

__device__ float sparse_net_ratio(const MlpWeights &w, SparseNet &s) {
  const int t = threadIdx.x;
  s.h[0][t] = bf16_round(silu(dot_bf16_row(w.w1 + t * kMlpIn, s.x, kMlpIn / 8) + w.b1[t]));
  __syncthreads();
  s.h[1][t] = bf16_round(silu(dot_bf16_row(w.w2 + t * kMlpHidden, s.h[0], kMlpHidden / 8) + w.b2[t]));
  __syncthreads();
  s.h[0][t] = bf16_round(silu(dot_bf16_row(w.w3 + t * kMlpHidden, s.h[1], kMlpHidden / 8) + w.b3[t]));
  __syncthreads();
  float v = __bfloat162float(w.w4[t]) * s.h[0][t];  // output 0: row 0 of W4
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((t & 31) == 0)
    s.red[t >> 5] = v;
  __syncthreads();
  const float r = (s.red[0] + s.red[1]) + (s.red[2] + s.red[3]) + w.b4[0];
  __syncthreads();  // s is reused by the next point
  return r;
}

struct SurrogateInput {
  float f[SURROGATE_FEATURES];
};

struct StrainIncrement {
  double v[6];
};

// surrogate_features, out of line with its inputs by value (see sparse_network_guesses).
__device__ __noinline__ SurrogateInput features_out_of_line(JcParams jc, double dt, StrainIncrement inc,
                                                             JcTrial tr) {
  SurrogateInput in;
  surrogate_features(jc, dt, inc.v, tr, in.f);
  return in;
}

// The network guesses of the block's points that need one (pending), one point at a time;
// returns the calling thread's (0 where it needs none). Every thread of the block calls it. Kept
// out of line: it runs in few tiles, and inlined its registers would raise the whole kernel's.
__device__ __noinline__ float sparse_network_guesses(const uint16_t *sw, const float *sb, SurrogateInput in,
                                                     bool pending) {
  __shared__ SparseNet sn;
  __shared__ int s_who;
  const MlpWeights w = mlp_weights(reinterpret_cast<const __nv_bfloat16 *>(sw), sb);
  const int t = threadIdx.x;
  float ratio = 0.0f;
  while (__syncthreads_or(pending)) {
    if (t == 0)
      s_who = kMaterialThreads;
    __syncthreads();
    if (pending)
      atomicMin(&s_who, t);
    __syncthreads();
    const int who = s_who;
    if (t == who)
#pragma unroll
      for (int c = 0; c < 16; ++c)
        sn.x[c] = c < SURROGATE_FEATURES ? bf16_round(in.f[c]) : 0.0f;
    __syncthreads();
    const float r = sparse_net_ratio(w, sn);
    if (t == who)
      ratio = r, pending = false;
  }
  return ratio;
}

// MODE: SURR_WARM (no network), SURR_SPARSE (hybrid guess: sparse_net_ratio for the points
// without plastic history), SURR_TENSOR (network guess: the tensor-core network on every tile
// with a yielding point; persistent blocks with the weights staged once).
enum SurrogateMode { SURR_WARM = 0, SURR_SPARSE = 1, SURR_TENSOR = 2 };

// Blocks per SM: two for the tensor-core variant (its shared-memory weights), three for the
// hybrid guess (fewer spills of its larger body: 0.399 against 0.423 ms at four blocks on the
// 1M-point bar in plastic flow), four for the warm start.
template <int MODE, int MINB = (MODE == SURR_TENSOR ? 2 : 4)>
__global__ void __launch_bounds__(kMaterialThreads, MINB)
    k_material_surrogate(const __grid_constant__ StepParams p) {
  constexpr bool NET = MODE == SURR_TENSOR;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  const int t = threadIdx.x;
  const int64_t n = p.n, tiles = (n + 127) / 128;
  unsigned char *sW1 = smem, *sW2 = smem + 4096, *sW3 = sW2 + 32768, *sW4 = sW3 + 32768, *sA = sW4 + 4096;
  unsigned char *sX = sA;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sA + 32768);
  float *sBias = reinterpret_cast<float *>(sA + 32768 + 64);
  const MlpWeights w = mlp_weights(reinterpret_cast<const __nv_bfloat16 *>(p.sw), p.sb);
  Sync sy{mbar, 0u, p.status, STATUS_SURROGATE_WAIT, true};
  uint32_t tmem = 0, trow = 0;
  if (NET) {
    if (t < 32)
      umma::tmem_alloc(&s_tmem, 128);
    if (t == 0)
      umma::mbar_init(mbar, 1);
    stage_rowmajor(sW1, w.w1, kMlpHidden, kMlpIn);
    stage_rowmajor(sW2, w.w2, kMlpHidden, kMlpHidden);
    stage_rowmajor(sW3, w.w3, kMlpHidden, kMlpHidden);
    stage_rowmajor(sW4, w.w4, kMlpOut, kMlpHidden);
    stage_biases(sBias, w);
    stage_wait();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    tmem = s_tmem;
    trow = tmem + ((uint32_t)(t & ~31) << 16);
  }
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t i = tile * 128 + t;
    double part[PM_COUNT] = {};
    double maxEqps = 0.0;
    MaterialPoint m;
    JcTrial tr;
    bool active = false, plastic = false, use_net = false;
    double yield0 = 0.0;
    float f[SURROGATE_FEATURES] = {};
    if (i < n) {
      material_load(p, i, m);
      active = jc_trial(p.jc, m.inc, m.pt, tr);  // false: the initialising call completed m.pt
      if (active) {
        yield0 = jc_yield0(p.jc, tr);
        plastic = tr.qTrial - yield0 >= p.jc.tolerance;
        // hybrid: the previous plastic increment where there is one, else the network
        use_net = plastic && (p.surr_guess == VPD_GUESS_NETWORK ||
                              (p.surr_guess == VPD_GUESS_HYBRID && !(m.pt.state[4] > 0.0)));
        if (NET && use_net)
          surrogate_features(p.jc, p.dt, m.inc, tr, f);
      }
    }
    float ratio = 0.0f;
    if (MODE == SURR_SPARSE && __syncthreads_or(use_net)) {  // block-uniform, 3 % of the tiles
      SurrogateInput in{};
      if (use_net)
        in = features_out_of_line(p.jc, p.dt, StrainIncrement{{m.inc[0], m.inc[1], m.inc[2], m.inc[3], m.inc[4],
                                                                m.inc[5]}},
                                  tr);
      ratio = sparse_network_guesses(p.sw, p.sb, in, use_net);
    }
    if (NET) {
      // the tile's points that need the network (uniform branch: a block-wide vote)
      if (__syncthreads_or(use_net) && sy.ok) {
#pragma unroll
        for (int c = 0; c < kMlpIn; ++c)
          st_bf16(sX, t, c, kMlpIn, c < SURROGATE_FEATURES ? f[c] : 0.0f);
        gemm(sy, tmem, sX, sW1, kMlpIn, kMlpHidden);
        if (sy.ok)
          hidden_epilogue(trow, sBias, sA, nullptr, nullptr);
        gemm(sy, tmem, sA, sW2, kMlpHidden, kMlpHidden);
        if (sy.ok)
          hidden_epilogue(trow, sBias + kMlpHidden, sA, nullptr, nullptr);
        gemm(sy, tmem, sA, sW3, kMlpHidden, kMlpHidden);
        if (sy.ok)
          hidden_epilogue(trow, sBias + 2 * kMlpHidden, sA, nullptr, nullptr);
        gemm(sy, tmem, sA, sW4, kMlpHidden, kMlpOut);
        if (sy.ok) {
          float v[16];
          umma::tmem_ld16(trow, v);
          ratio = v[0] + sBias[3 * kMlpHidden];
        }
      }
    }
    if (active) {
      double epInc = 0.0, yield = yield0;
      int iterations = 1;  // an elastic trial ends the bisection at its first iteration
      if (plastic) {
        const double guess = use_net ? (double)ratio * floor_increment(p.jc, tr) : m.pt.state[4];
        if (!jc_newton(p.jc, p.dt, tr, guess, p.surr_steps, epInc, yield, iterations)) {
          iterations = jc_bisection(p.jc, p.dt, tr, m.pt.state[4], epInc, yield);
          part[PM_FALLBACK] = 1.0;
        }
      }
      jc_finish(p.jc, m.inc, tr, epInc, yield, (double)iterations, m.pt);
    }
    if (i < n) {
      const double fallback = part[PM_FALLBACK];
      material_store(p, i, m, part, maxEqps);
      part[PM_FALLBACK] = fallback;
    }
    material_reduce(p, part, maxEqps, tile);
  }
  if (NET) {
    umma::fence_before_sync();
    __syncthreads();
    if (t < 32)
      umma::tmem_dealloc(tmem, 128);
  }
}

static int g_surrogate_sms = 0;

int prepare_material_surrogate() {
  int dev = 0;
  VPD_CUDA(cudaGetDevice(&dev));
  VPD_CUDA(cudaDeviceGetAttribute(&g_surrogate_sms, cudaDevAttrMultiProcessorCount, dev));
  VPD_CUDA(cudaFuncSetAttribute(k_material_surrogate<SURR_TENSOR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSurrSmem));
  return VPD_OK;
}

int launch_material_surrogate(const StepParams &p, cudaStream_t s) {
  const int64_t tiles = (p.n + 127) / 128;
  if (p.surr_guess == VPD_GUESS_NETWORK) {
    if (!g_surrogate_sms)
      return set_error(VPD_ERR_INVALID, "surrogate kernel not prepared (vpd_set_surrogate)");
    // persistent: two CTAs per SM, each staging the weights once
    const int64_t grid = std::min<int64_t>(tiles, 2 * (int64_t)g_surrogate_sms);
    k_material_surrogate<SURR_TENSOR><<<(unsigned)grid, kMaterialThreads, kSurrSmem, s>>>(p);
  } else if (p.surr_guess == VPD_GUESS_HYBRID) {
    k_material_surrogate<SURR_SPARSE, 3><<<(unsigned)tiles, kMaterialThreads, 0, s>>>(p);
  } else {
    k_material_surrogate<SURR_WARM><<<(unsigned)tiles, kMaterialThreads, 0, s>>>(p);
  }
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd

// ------------------------------------------------------------------ C ABI
using namespace vpd;

extern "C" int vpd_surrogate_samples(const double *props, uint64_t seed, int64_t count, float *features,
                                     float *targets, double *records) {
  if (!props || !features || !targets || count < 1)
    return set_error(VPD_ERR_INVALID, "vpd_surrogate_samples: invalid argument");
  for (int k = 0; k < 14; ++k)
    if (!std::isfinite(props[k]))
      return set_error(VPD_ERR_INVALID, "vpd_surrogate_samples: non-finite material property");
  const JcParams jc = make_jc_params(props);
  TrainBuffers buf;
  float *X = nullptr, *Y = nullptr;
  double *R = nullptr;
  int rc;
  if ((rc = buf.alloc(&X, count * 16)) || (rc = buf.alloc(&Y, count * 16)) ||
      (records && (rc = buf.alloc(&R, count * VPD_SAMPLE_RECORD))))
    return rc;
  if ((rc = surrogate_samples_dev(jc, seed, count, X, Y, R, 0)))
    return rc;
  VPD_CUDA(cudaMemcpy(features, X, sizeof(float) * count * 16, cudaMemcpyDeviceToHost));
  VPD_CUDA(cudaMemcpy(targets, Y, sizeof(float) * count * 16, cudaMemcpyDeviceToHost));
  if (records)
    VPD_CUDA(cudaMemcpy(records, R, sizeof(double) * count * VPD_SAMPLE_RECORD, cudaMemcpyDeviceToHost));
  return VPD_OK;
}

extern "C" int vpd_train_surrogate(const vpd_surrogate_config *cfg, uint16_t *weights, float *biases,
                                   vpd_surrogate_report *report) {
  int rc = check_config(cfg);
  if (rc)
    return rc;
  if (!weights || !biases)
    return set_error(VPD_ERR_INVALID, "vpd_train_surrogate: null output buffer");
  return train_surrogate(*cfg, weights, biases, report);
}
