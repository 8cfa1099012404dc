// Device helpers shared by the mixed-precision bond kernels (vpd_mixed.cu, vpd_tiled.cu).
#pragma once

#include "vpd_math.cuh"
#include "vpd_step.cuh"

namespace vpd {

__device__ __forceinline__ float4 ldgf4(const float4 *p) { return __ldg(p); }

__device__ __forceinline__ int64_t clamp_index(int64_t j, int64_t n) {
  return j < 0 ? 0 : (j >= n ? n - 1 : j);
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float x) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}

// Packed FP32 pairs: one sm_100a paired instruction (FADD2, FMUL2, FFMA2) applies the same
// operation to both lanes, each lane rounded as the scalar operation.
__device__ __forceinline__ float2 bcast2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {  // a - b: b (-1) is exact, one rounding
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ void kahan_add2(float2 &s, float2 &c, float2 x) {  // kahan_add on each lane
  const float2 y = sub2(x, c);
  const float2 t = __fadd2_rn(s, y);
  c = sub2(sub2(t, s), y);
  s = t;
}

static __device__ __noinline__ bool exact_break_mixed(const double4 *xv, const double4 *U, int64_t i,
                                               int64_t j, double initiation, double failure,
                                               int use_compression) {
  const double4 xi = xv[i], xj = xv[j], ui = U[i], uj = U[j];
  const double yi0 = __dadd_rn(xi.x, ui.x), yi1 = __dadd_rn(xi.y, ui.y), yi2 = __dadd_rn(xi.z, ui.z);
  const double y0 = __dsub_rn(__dadd_rn(xj.x, uj.x), yi0);
  const double y1 = __dsub_rn(__dadd_rn(xj.y, uj.y), yi1);
  const double y2 = __dsub_rn(__dadd_rn(xj.z, uj.z), yi2);
  const double e0 = __dsub_rn(xj.x, xi.x), e1 = __dsub_rn(xj.y, xi.y), e2 = __dsub_rn(xj.z, xi.z);
  const double initial =
      __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(e0, e0), __dmul_rn(e1, e1)), __dmul_rn(e2, e2)));
  const double cur =
      __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(y0, y0), __dmul_rn(y1, y1)), __dmul_rn(y2, y2)));
  const double stretch = __ddiv_rn(__dsub_rn(cur, initial), initial);
  return stretch > initiation || (use_compression && stretch < -failure);
}

}  // namespace vpd
