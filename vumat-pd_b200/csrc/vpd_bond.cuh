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

// The FP32 force map of point j as the mixed force kernels gather it: three float4 records
// (fmapf[j], fmapf[n + j], fmapf[2 n + j]) holding VM = V_j M_j (row r, column c: VM_rc) and
// R = VM J_j (J_j: the point's jitter, its reference position less its lattice position):
//   rec0 = (VM_00, VM_10, VM_01, VM_11)   rec1 = (VM_02, VM_12, R_0, R_1)
//   rec2 = (VM_20, VM_21, VM_22, R_2)
// A bond term is VM xi = VM (o + J_j - J_i) = VM e + R with e = o - J_i, which depends on the
// neighbour only through its own record: rows 0 and 1 of it are three paired multiply-adds of
// the loaded pairs (VM_0c, VM_1c) with e_c on both lanes, plus the pair (R_0, R_1); row 2 is
// scalar.
struct FmapRecord {
  float2 c0, c1, c2, r01;  // (VM_0c, VM_1c) for c = 0, 1, 2; (R_0, R_1)
  float m20, m21, m22, r2;  // row 2 and R_2
};
__device__ __forceinline__ FmapRecord fmap_record(const float4 &a, const float4 &b, const float4 &c) {
  return {make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y), make_float2(b.z, b.w),
          c.x, c.y, c.z, c.w};
}
// VM e + R for bond reference offset e = o - J_i: rows 0 and 1 as a pair, row 2 scalar
__device__ __forceinline__ float2 fmap_rows01(const FmapRecord &m, float2 e0, float2 e1, float2 e2) {
  return __ffma2_rn(m.c2, e2, __ffma2_rn(m.c1, e1, __ffma2_rn(m.c0, e0, m.r01)));
}
__device__ __forceinline__ float fmap_row2(const FmapRecord &m, float e0, float e1, float e2) {
  return fmaf(m.m22, e2, fmaf(m.m21, e1, fmaf(m.m20, e0, m.r2)));
}
// Row r of VM (the point's own record, for the M_i s_i term)
__device__ __forceinline__ void fmap_rows(const float4 &a, const float4 &b, const float4 &c, float (&VM)[9]) {
  VM[0] = a.x, VM[1] = a.z, VM[2] = b.x;
  VM[3] = a.y, VM[4] = a.w, VM[5] = b.y;
  VM[6] = c.x, VM[7] = c.y, VM[8] = c.z;
}

// FP64 bond arithmetic shared by the per-slot (vpd_stencil.cu) and tiled (vpd_tiled64.cu)
// kernels, every rounding spelled out so both produce the same bits.
// G += (v d) (x) e for one bond (v: the neighbour's volume, or 0 without a bond).
__device__ __forceinline__ void bond_deform64(double (&G)[9], double v, double d0, double d1, double d2, double e0,
                                              double e1, double e2) {
  const double w0 = __dmul_rn(v, d0), w1 = __dmul_rn(v, d1), w2 = __dmul_rn(v, d2);
  G[0] = __fma_rn(w0, e0, G[0]), G[1] = __fma_rn(w0, e1, G[1]), G[2] = __fma_rn(w0, e2, G[2]);
  G[3] = __fma_rn(w1, e0, G[3]), G[4] = __fma_rn(w1, e1, G[4]), G[5] = __fma_rn(w1, e2, G[5]);
  G[6] = __fma_rn(w2, e0, G[6]), G[7] = __fma_rn(w2, e1, G[7]), G[8] = __fma_rn(w2, e2, G[8]);
}
// r . e, left to right
__device__ __forceinline__ double dot3_rn(double r0, double r1, double r2, double e0, double e1, double e2) {
  return __fma_rn(r2, e2, __fma_rn(r1, e1, __dmul_rn(r0, e0)));
}
// F = I + G K^-1 (row-major 3x3), each entry a left-to-right dot product
__device__ __forceinline__ void deformation_from_g(const double (&G)[9], const double (&K)[9], double (&F)[9]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      F[3 * a + b] = __dadd_rn(a == b ? 1.0 : 0.0, dot3_rn(G[3 * a], G[3 * a + 1], G[3 * a + 2], K[b], K[3 + b], K[6 + b]));
}

// The exact FP64 critical-stretch decision of bond (i, j) (the reference's stretch formula,
// every operation rounded as written).
static __device__ __noinline__ bool exact_break(const double4 *xv, const double4 *U, int64_t i,
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

// ------------------------------------------------------------------ lattice tiling
// Helpers of the tiled bond kernels (vpd_tiled.cu, vpd_tiled64.cu): a thread owns kTileP
// points of one lattice column along y and walks the stencil's groups (runs of slots that
// differ only in the y offset) as windows of consecutive lattice points.
constexpr int kUnrolledSlots = 12;  // the switches below list counts 1 .. 12

// Lattice coordinates of thread tau's column: z fastest, then the y-block, then x. Threads
// past the lattice get the last column (their points are marked invalid).
template <int kTileP>
__device__ __forceinline__ bool tile_coords(const StepParams &p, int64_t tau, int &x, int &yb, int &z) {
  const int nz = p.lat_nz, nyb = (p.lat_ny + kTileP - 1) / kTileP;
  z = (int)(tau % nz);
  const int64_t r = tau / nz;
  yb = (int)(r % nyb);
  x = (int)(r / nyb);
  const bool inb = x < p.lat_nx;
  x = inb ? x : p.lat_nx - 1;
  return inb;
}

__device__ __forceinline__ uint32_t group_bits(uint32_t word, int shift, uint32_t cm) {
  return (word >> shift) & cm;
}

template <typename I> __device__ __forceinline__ I clamp_to(I j, I n) { return j < 0 ? 0 : (j >= n ? n - 1 : j); }

// Point i's bonds of one group (first slot pos, mask word wd, shift sh) that the stretch tests
// flagged: `near` ones decided by the exact FP64 test, then both directed bonds of every
// broken pair marked (bit k: slot pos + k).
__device__ __forceinline__ void commit_breaks(const StepParams &p, int64_t i, int pos, int wd, int sh, uint32_t fr,
                                              uint32_t nr) {
  const int64_t n = p.n;
  if (nr) {
    const int64_t step = *p.step;
    const double4 *U = (step & 1) ? p.u1 : p.u0;
    for (uint32_t f = nr; f; f &= f - 1) {
      const int k = __ffs(f) - 1;
      if (exact_break(p.xv, U, i, i + p.st.delta[pos + k], p.dmg_initiation, p.dmg_failure, p.use_compression))
        fr |= 1u << k;
    }
  }
  if (fr) {
    atomicOr(p.st.broken + (int64_t)wd * n + i, fr << sh);
    for (uint32_t f = fr; f; f &= f - 1) {
      const int sl = pos + __ffs(f) - 1;
      const int r = p.st.reverse[sl];
      atomicOr(p.st.broken + (int64_t)(r >> 5) * n + (i + p.st.delta[sl]), 1u << (r & 31));
    }
  }
}

template <int kTileP> static unsigned tiled_grid(const StepParams &p) {
  const int64_t threads = (int64_t)p.lat_nx * ((p.lat_ny + kTileP - 1) / kTileP) * p.lat_nz;
  return (unsigned)((threads + kBondThreads - 1) / kBondThreads);
}

// 32-bit window indices need every index within a stencil reach of the lattice below 2^31
static inline bool index32(const StepParams &p) { return p.n < (int64_t(1) << 30); }

}  // namespace vpd
