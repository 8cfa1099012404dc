// Shared-window mixed-precision deformation kernel (no bond damage): the default FP32 bond sum
// of the deformation gradient when no bond can break.
//
// Tiling as the packed-pair kernels of vpd_tiled.cu: a thread owns two points of one lattice
// column along y (y = 2 yb + q) and walks the stencil's groups as windows of consecutive
// lattice points along y; point 0 holds window positions 0..cnt-1, point 1 positions 1..cnt.
//
// The bond sum is rewritten about a reference displacement, the thread's point 0:
//   G_q = sum_j V_j (u_j - u_q) (x) xi_qj,   xi_qj = a_j - e_q
//       = sum_j w_j (x) a_j  -  (sum_j w_j) (x) e_q  -  (u_q - u_0) (x) sum_j V_j xi_qj
// with w_j = V_j (u_j - u_0), a_j the neighbour's position relative to the tile's base row and
// e_q the point's own (its jitter, plus q h along y). w_j and a_j no longer depend on the point,
// so a window position that holds a bond of both points contributes one term w_j (x) a_j to
// both: where a group's bonds are all present for both points of every thread of the warp (the
// interior, away from the horizon's jitter-dependent fringe), the window's shared positions
// 1..cnt-1 are summed once in scalar FP32 and only its two ends (one point each) run as a
// packed pair. Groups with missing bonds take the masked packed-pair form of the same sums.
// The last term uses sum_j V_j xi_qj over all bonds, the FP64 vector the layout keeps (vxi);
// every bond of the mask enters the sum, as in the reference's F (it reads no bond damage).
//
// Accumulation: window sums in FP32, added into a partial per stencil plane (the groups with
// the same x offset, which come in order), and each plane's partial folded into the point's
// sum with Kahan compensation. The corrections and the compensation are applied in FP64 once
// per point; G is stored in FP32, as by the other mixed kernels.
#include "vpd_bond.cuh"

namespace vpd {

namespace {

struct WindowPoints {
  float ux, uy, uz;       // reference displacement: point 0's
  float2 ex, ey, ez;      // lane q: e_q (ey includes q h)
};

// A window's shared positions t = 1..CNT-1 (a bond of both points): S += w (x) a, Sw += w.
template <int CNT, typename I>
__device__ __forceinline__ void shared_core(const StepParams &p, I jb, I nz, float gx, float gz, float by0, float h,
                                            const WindowPoints &pt, float (&S)[9], float (&Sw)[3]) {
#pragma unroll
  for (int t = 1; t < CNT; ++t) {
    const I j = jb + (I)t * nz;
    const float4 a = ldgf4(p.jit + j), b = ldgf4(p.uf + j);
    const float ax = a.x + gx, ay = a.y + fmaf((float)t, h, by0), az = a.z + gz;
    const float w0 = a.w * (b.x - pt.ux), w1 = a.w * (b.y - pt.uy), w2 = a.w * (b.z - pt.uz);
    S[0] = fmaf(w0, ax, S[0]), S[1] = fmaf(w0, ay, S[1]), S[2] = fmaf(w0, az, S[2]);
    S[3] = fmaf(w1, ax, S[3]), S[4] = fmaf(w1, ay, S[4]), S[5] = fmaf(w1, az, S[5]);
    S[6] = fmaf(w2, ax, S[6]), S[7] = fmaf(w2, ay, S[7]), S[8] = fmaf(w2, az, S[8]);
    Sw[0] += w0, Sw[1] += w1, Sw[2] += w2;
  }
}

// One packed element: lane q takes the neighbour at window position tq (record j_q) with bond
// weight v_q (the volume, or 0 without a bond); P += w (x) a, W += w per lane.
__device__ __forceinline__ void window_pair(const float4 &a0, const float4 &b0, const float4 &a1, const float4 &b1,
                                            float t0, float t1, float v0, float v1, float gx, float gz, float by0,
                                            float h, const WindowPoints &pt, float2 (&P)[9], float2 (&W)[3]) {
  const float2 ax = make_float2(a0.x + gx, a1.x + gx);
  const float2 ay = make_float2(a0.y + fmaf(t0, h, by0), a1.y + fmaf(t1, h, by0));
  const float2 az = make_float2(a0.z + gz, a1.z + gz);
  const float2 v = make_float2(v0, v1);
  const float2 w0 = __fmul2_rn(v, make_float2(b0.x - pt.ux, b1.x - pt.ux));
  const float2 w1 = __fmul2_rn(v, make_float2(b0.y - pt.uy, b1.y - pt.uy));
  const float2 w2 = __fmul2_rn(v, make_float2(b0.z - pt.uz, b1.z - pt.uz));
  P[0] = __ffma2_rn(w0, ax, P[0]), P[1] = __ffma2_rn(w0, ay, P[1]), P[2] = __ffma2_rn(w0, az, P[2]);
  P[3] = __ffma2_rn(w1, ax, P[3]), P[4] = __ffma2_rn(w1, ay, P[4]), P[5] = __ffma2_rn(w1, az, P[5]);
  P[6] = __ffma2_rn(w2, ax, P[6]), P[7] = __ffma2_rn(w2, ay, P[7]), P[8] = __ffma2_rn(w2, az, P[8]);
  W[0] = __fadd2_rn(W[0], w0), W[1] = __fadd2_rn(W[1], w1), W[2] = __fadd2_rn(W[2], w2);
}

// A full group: the shared core once, then the two ends (point 0 at position 0, point 1 at
// position CNT) as one pair on top of it.
template <int CNT, typename I>
__device__ __forceinline__ void full_window(const StepParams &p, int cnt, I jb, I nz, float gx, float gz, float by0,
                                            float h, const WindowPoints &pt, float2 (&P)[9], float2 (&W)[3]) {
  float S[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, Sw[3] = {0.f, 0.f, 0.f};
  if constexpr (CNT > 0) {
    shared_core<CNT, I>(p, jb, nz, gx, gz, by0, h, pt, S, Sw);
  } else {
    for (int t = 1; t < cnt; ++t) {
      const I j = jb + (I)t * nz;  // within the zero halo of the neighbour arrays
      const float4 a = ldgf4(p.jit + j), b = ldgf4(p.uf + j);
      const float ax = a.x + gx, ay = a.y + fmaf((float)t, h, by0), az = a.z + gz;
      const float w0 = a.w * (b.x - pt.ux), w1 = a.w * (b.y - pt.uy), w2 = a.w * (b.z - pt.uz);
      S[0] = fmaf(w0, ax, S[0]), S[1] = fmaf(w0, ay, S[1]), S[2] = fmaf(w0, az, S[2]);
      S[3] = fmaf(w1, ax, S[3]), S[4] = fmaf(w1, ay, S[4]), S[5] = fmaf(w1, az, S[5]);
      S[6] = fmaf(w2, ax, S[6]), S[7] = fmaf(w2, ay, S[7]), S[8] = fmaf(w2, az, S[8]);
      Sw[0] += w0, Sw[1] += w1, Sw[2] += w2;
    }
  }
  const int c = CNT > 0 ? CNT : cnt;
  const I j0 = jb, j1 = jb + (I)c * nz;
  const float4 a0 = ldgf4(p.jit + j0), b0 = ldgf4(p.uf + j0), a1 = ldgf4(p.jit + j1), b1 = ldgf4(p.uf + j1);
  float2 Q[9], Qw[3];
#pragma unroll
  for (int k = 0; k < 9; ++k)
    Q[k] = bcast2(S[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k)
    Qw[k] = bcast2(Sw[k]);
  window_pair(a0, b0, a1, b1, 0.0f, (float)c, a0.w, a1.w, gx, gz, by0, h, pt, Q, Qw);
#pragma unroll
  for (int k = 0; k < 9; ++k)
    P[k] = __fadd2_rn(P[k], Q[k]);
#pragma unroll
  for (int k = 0; k < 3; ++k)
    W[k] = __fadd2_rn(W[k], Qw[k]);
}

// A group with missing bonds: every window position as one pair element, each lane's bond
// weight zero where its point has no bond there (bits[q] bit t: position t is a bond of q).
template <typename I>
__device__ __forceinline__ void masked_window(const StepParams &p, int cnt, I jb, I nz, float gx, float gz,
                                              float by0, float h, const WindowPoints &pt, const uint32_t (&bits)[2],
                                              float2 (&P)[9], float2 (&W)[3]) {
  for (int t = 0; t <= cnt; ++t) {
    const I j = jb + (I)t * nz;  // within the zero halo of the neighbour arrays
    const float4 a = ldgf4(p.jit + j), b = ldgf4(p.uf + j);
    window_pair(a, b, a, b, (float)t, (float)t, ((bits[0] >> t) & 1u) ? a.w : 0.0f,
                ((bits[1] >> t) & 1u) ? a.w : 0.0f, gx, gz, by0, h, pt, P, W);
  }
}

template <bool UNROLL>
__global__ void __launch_bounds__(kBondThreads, 2) k_deformation_window(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  const float h = (float)p.lat_h;
  int x, yb, z;
  const bool inb = tile_coords<2>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  int64_t ip[2];
  bool vp[2];
  float4 pa[2], pb[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int y = yb * 2 + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    pa[q] = ldgf4(p.jit + ip[q]), pb[q] = ldgf4(p.uf + ip[q]);
  }
  WindowPoints pt;
  pt.ux = pb[0].x, pt.uy = pb[0].y, pt.uz = pb[0].z;
  pt.ex = make_float2(pa[0].x, pa[1].x), pt.ey = make_float2(pa[0].y, pa[1].y + h);
  pt.ez = make_float2(pa[0].z, pa[1].z);
  float2 G[9], Gc[9], P[9], W[3];
#pragma unroll
  for (int k = 0; k < 9; ++k)
    G[k] = Gc[k] = P[k] = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int k = 0; k < 3; ++k)
    W[k] = make_float2(0.0f, 0.0f);
  int word = -1, plane = INT_MIN;
  uint32_t mw[2] = {0u, 0u};
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);  // dx, dz, lowest dy, (slots << 16) | first slot
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    if (gr.x != plane) {  // uniform: a new stencil plane; fold the last one's partial
      plane = gr.x;
#pragma unroll
      for (int k = 0; k < 9; ++k)
        kahan_add2(G[k], Gc[k], P[k]), P[k] = make_float2(0.0f, 0.0f);
    }
    if (wd != word) {  // uniform: groups come in slot order, several per mask word
      word = wd;
#pragma unroll
      for (int q = 0; q < 2; ++q)
        mw[q] = vp[q] ? __ldg(p.st.mask + (int64_t)wd * n + ip[q]) : 0u;
    }
    const uint32_t m0 = group_bits(mw[0], sh, cm), m1 = group_bits(mw[1], sh, cm);
    // a point past the lattice (vp false) counts as full: it takes whatever its lane computes
    const bool full = (m0 == cm || !vp[0]) && (m1 == cm || !vp[1]);
    const uint32_t bits[2] = {m0, m1 << 1};  // bit t: the neighbour at window position t
    if (__all_sync(0xffffffffu, (bits[0] | bits[1]) == 0u))
      continue;
    const float gx = (float)gr.x * h, gz = (float)gr.y * h, by0 = (float)gr.z * h;
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * 2 + gr.z)) * nz + (z + gr.y);
    if (__all_sync(0xffffffffu, full)) {
      if (UNROLL) {
        static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
        const int jb32 = (int)jb, nz32 = nz;
#define VPD_FULL_CASE(C)                                                             \
  case C:                                                                            \
    full_window<C, int>(p, cnt, jb32, nz32, gx, gz, by0, h, pt, P, W);               \
    break;
        switch (cnt) {
          VPD_FULL_CASE(1) VPD_FULL_CASE(2) VPD_FULL_CASE(3) VPD_FULL_CASE(4)
          VPD_FULL_CASE(5) VPD_FULL_CASE(6) VPD_FULL_CASE(7) VPD_FULL_CASE(8)
          VPD_FULL_CASE(9) VPD_FULL_CASE(10) VPD_FULL_CASE(11) VPD_FULL_CASE(12)
        default:
          full_window<0, int>(p, cnt, jb32, nz32, gx, gz, by0, h, pt, P, W);
        }
#undef VPD_FULL_CASE
      } else {
        full_window<0, int64_t>(p, cnt, jb, (int64_t)nz, gx, gz, by0, h, pt, P, W);
      }
    } else {
      masked_window<int64_t>(p, cnt, jb, (int64_t)nz, gx, gz, by0, h, pt, bits, P, W);
    }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k)
    kahan_add2(G[k], Gc[k], P[k]);
  // G_q = (sum w (x) a, compensated) - W_q (x) e_q - (u_q - u_0) (x) vxi_q, in FP64
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (!vp[q])
      continue;
    const int64_t i = ip[q];
    const double e[3] = {q ? pt.ex.y : pt.ex.x, q ? pt.ey.y : pt.ey.x, q ? pt.ez.y : pt.ez.x};
    const double w[3] = {q ? W[0].y : W[0].x, q ? W[1].y : W[1].x, q ? W[2].y : W[2].x};
    const double du[3] = {(double)pb[q].x - pt.ux, (double)pb[q].y - pt.uy, (double)pb[q].z - pt.uz};
    const double4 s = p.vxi[i];
    const double sv[3] = {s.x, s.y, s.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const int k = 3 * a + b;
        const double sum = q ? (double)G[k].y - (double)Gc[k].y : (double)G[k].x - (double)Gc[k].x;
        p.Gf[k * n + i] = (float)(sum - w[a] * e[b] - du[a] * sv[b]);
      }
  }
}

}  // namespace

// The shared-window kernel for increments without bond damage (the damaged increments keep
// the packed-pair kernel, whose stretch tests need each bond's own terms).
int launch_deformation_window(const StepParams &p, cudaStream_t s) {
  const unsigned grid = tiled_grid<2>(p);
  if (index32(p))
    k_deformation_window<true><<<grid, kBondThreads, 0, s>>>(p);
  else
    k_deformation_window<false><<<grid, kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
