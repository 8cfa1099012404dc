// Tiled mixed-precision bond kernels: the deformation gradient (with critical-stretch bond
// breaking) and the force bond sum, with each thread owning kTileP points of one lattice
// column along y (same x and z, y = kTileP yb + q).
//
// The stencil's slots are grouped by the offset's (x, z) components (vpd_stencil.cu): the
// offsets of a group differ only in y, so the neighbours that the kTileP points reach through
// one group form a single run of cnt + kTileP - 1 consecutive lattice points along y (the
// group's window). The thread loads each neighbour record of the window once and applies it
// to every one of its points that has the matching bond: the loads fall by about
// cnt kTileP / (cnt + kTileP - 1). Consecutive threads take consecutive z, so each load of a
// warp is one contiguous range.
//
// A group's window is walked fully unrolled for each slot count up to kUnrolledSlots (a switch
// over the count picks the instance): which (window position, point) pairs hold a slot, the
// bit each one tests and the lattice offset along y are then compile-time constants, and the
// neighbour index is 32-bit. Larger groups, and lattices of 2^30 points or more, take the same
// body in a runtime loop with 64-bit indices.
//
// Arithmetic is that of vpd_mixed.cu: FP32 bond terms, partial sums per group (per stencil
// plane in the packed-pair kernels) folded with Kahan compensation into the force (and in the
// packed-pair kernels into the deformation sum),
// the FP32 stretch test with a 1e-5 margin and the exact FP64 test inside it (in the packed
// kernel: for every bond not clearly intact), pairs broken once by the lower-index point.
#include "vpd_bond.cuh"

namespace vpd {

template <bool B> struct BoolConstant {
  static constexpr bool value = B;
};

// FP32 critical-stretch test of one live bond (reference xi = e, displacement difference d):
// bit t of `fresh` when the bond is clearly broken, of `near` when it is within the 1e-5 margin
// of a threshold and the exact FP64 test decides.
__device__ __forceinline__ void stretch_test(const StepParams &p, int t, float e0, float e1, float e2, float d0,
                                             float d1, float d2, uint32_t &fresh, uint32_t &near) {
  const float lo = 1.0f - 1.0e-5f, hi = 1.0f + 1.0e-5f;
  const float y0 = e0 + d0, y1 = e1 + d1, y2 = e2 + d2;
  const float yy = y0 * y0 + y1 * y1 + y2 * y2;
  const float xx = e0 * e0 + e1 * e1 + e2 * e2;
  const float tt = p.tension2f * xx;
  if (yy > tt * hi)
    fresh |= 1u << t;
  else if (yy >= tt * lo)
    near |= 1u << t;
  else if (p.use_compression) {
    const float c = p.compression2f * xx;
    if (yy < c * lo)
      fresh |= 1u << t;
    else if (yy <= c * hi)
      near |= 1u << t;
  }
}

// The stretch tests of the two lanes of a packed element, paired: lane q holds a bond at window
// position tq, tested when bit tq of live[q] is set. A bond whose FP32 stretch is not clearly
// below the threshold (|y|^2 >= tension2f |xi|^2 (1 - 1e-5), or with compression not clearly
// above its bound) sets bit tq of near[q], and the exact FP64 test (commit_breaks) decides it:
// the same decisions as stretch_test's, whose clearly broken bonds the exact test confirms, with
// one bit and one or two comparisons per lane.
__device__ __forceinline__ void stretch_test2(const StepParams &p, int t0, int t1, float2 e0, float2 e1, float2 e2,
                                              float2 d0, float2 d1, float2 d2, const uint32_t (&live)[2],
                                              uint32_t (&near)[2]) {
  const bool l0 = (live[0] >> t0) & 1u, l1 = (live[1] >> t1) & 1u;
  if (!(l0 || l1))
    return;
  const float2 y0 = __fadd2_rn(e0, d0), y1 = __fadd2_rn(e1, d1), y2 = __fadd2_rn(e2, d2);
  const float2 yy = __ffma2_rn(y2, y2, __ffma2_rn(y1, y1, __fmul2_rn(y0, y0)));
  const float2 xx = __ffma2_rn(e2, e2, __ffma2_rn(e1, e1, __fmul2_rn(e0, e0)));
  const float2 tlo = __fmul2_rn(__fmul2_rn(bcast2(p.tension2f), xx), bcast2(1.0f - 1.0e-5f));
  bool c0 = yy.x >= tlo.x, c1 = yy.y >= tlo.y;
  if (p.use_compression) {  // uniform
    const float2 chi = __fmul2_rn(__fmul2_rn(bcast2(p.compression2f), xx), bcast2(1.0f + 1.0e-5f));
    c0 = c0 || yy.x <= chi.x, c1 = c1 || yy.y <= chi.y;
  }
  near[0] |= (uint32_t)(l0 && c0) << t0;
  near[1] |= (uint32_t)(l1 && c1) << t1;
}

// ------------------------------------------------------------------ deformation
template <int P> struct DeformPoints {
  float jx[P], jy[P], jz[P], ux[P], uy[P], uz[P];  // jy includes q h (y relative to the tile's base row)
};

// One window position t of a group: the neighbour record and its bonds to the tile's points.
template <bool DAMAGE, int P, typename I>
__device__ __forceinline__ void deform_element(const StepParams &p, int t, int cnt, I j, float gx, float gz,
                                               float by0, float h, const DeformPoints<P> &pt,
                                               const uint32_t (&bits)[P], const uint32_t (&live)[P],
                                               float (&part)[P][9], uint32_t (&fresh)[P], uint32_t (&near)[P]) {
  const float4 a = ldgf4(p.jit + j), b = ldgf4(p.uf + j);
  const float bx = a.x + gx, by = a.y + fmaf((float)t, h, by0), bz = a.z + gz;
#pragma unroll
  for (int q = 0; q < P; ++q) {
    if (t < q || t - q >= cnt)  // window position t holds no slot of point q
      continue;
    const float e0 = bx - pt.jx[q], e1 = by - pt.jy[q], e2 = bz - pt.jz[q];
    const float d0 = b.x - pt.ux[q], d1 = b.y - pt.uy[q], d2 = b.z - pt.uz[q];
    const float v = (bits[q] & (1u << t)) ? a.w : 0.0f;  // no bond: no contribution
    const float w0 = v * d0, w1 = v * d1, w2 = v * d2;
    part[q][0] += w0 * e0, part[q][1] += w0 * e1, part[q][2] += w0 * e2;
    part[q][3] += w1 * e0, part[q][4] += w1 * e1, part[q][5] += w1 * e2;
    part[q][6] += w2 * e0, part[q][7] += w2 * e1, part[q][8] += w2 * e2;
    if (DAMAGE && (live[q] & (1u << t)))
      stretch_test(p, t, e0, e1, e2, d0, d1, d2, fresh[q], near[q]);
  }
}

// The window of one group: CNT > 0 unrolled with 32-bit indices, CNT == 0 a runtime loop.
template <int CNT, bool DAMAGE, int P, typename I>
__device__ __forceinline__ void deform_window(const StepParams &p, int cnt, I jb, I nz, I n, float gx, float gz,
                                              float by0, float h, const DeformPoints<P> &pt,
                                              const uint32_t (&bits)[P], const uint32_t (&live)[P],
                                              float (&part)[P][9], uint32_t (&fresh)[P], uint32_t (&near)[P]) {
  if constexpr (CNT > 0) {
#pragma unroll
    for (int t = 0; t < CNT + P - 1; ++t)
      deform_element<DAMAGE, P, I>(p, t, CNT, clamp_to<I>(jb + (I)t * nz, n), gx, gz, by0, h, pt, bits, live,
                                   part, fresh, near);
  } else {
    for (int t = 0; t < cnt + P - 1; ++t)
      deform_element<DAMAGE, P, I>(p, t, cnt, clamp_to<I>(jb + (I)t * nz, n), gx, gz, by0, h, pt, bits, live,
                                   part, fresh, near);
  }
}

template <bool DAMAGE, int kTileP, bool UNROLL>
__global__ void __launch_bounds__(kBondThreads, 2) k_deformation_tiled(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  const float h = (float)p.lat_h;
  int x, yb, z;
  const bool inb = tile_coords<kTileP>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  int64_t ip[kTileP];
  bool vp[kTileP];
  DeformPoints<kTileP> pt;
#pragma unroll
  for (int q = 0; q < kTileP; ++q) {
    const int y = yb * kTileP + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const float4 a = ldgf4(p.jit + ip[q]), b = ldgf4(p.uf + ip[q]);
    pt.jx[q] = a.x, pt.jy[q] = a.y + (float)q * h, pt.jz[q] = a.z;
    pt.ux[q] = b.x, pt.uy[q] = b.y, pt.uz[q] = b.z;
  }
  float G[kTileP][9];
#pragma unroll
  for (int q = 0; q < kTileP; ++q)
#pragma unroll
    for (int c = 0; c < 9; ++c)
      G[q][c] = 0.0f;
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);  // dx, dz, lowest dy, (slots << 16) | first slot
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    uint32_t bits[kTileP], live[kTileP];
    uint32_t any = 0u;
    const uint32_t fw = DAMAGE ? group_bits(__ldg(p.st.forward + wd), sh, cm) : 0u;
#pragma unroll
    for (int q = 0; q < kTileP; ++q) {
      const uint32_t m = vp[q] ? group_bits(__ldg(p.st.mask + (int64_t)wd * n + ip[q]), sh, cm) : 0u;
      bits[q] = m << q;  // bit t: the neighbour at window position t (slot pos + t - q)
      live[q] = 0u;
      if (DAMAGE) {
        const uint32_t bk = vp[q] ? group_bits(p.st.broken[(int64_t)wd * n + ip[q]], sh, cm) : 0u;
        live[q] = (m & fw & ~bk) << q;
      }
      any |= bits[q];
    }
    if (__all_sync(0xffffffffu, any == 0u))
      continue;
    const float gx = (float)gr.x * h, gz = (float)gr.y * h, by0 = (float)gr.z * h;
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * kTileP + gr.z)) * nz + (z + gr.y);
    float part[kTileP][9];
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
#pragma unroll
      for (int c = 0; c < 9; ++c)
        part[q][c] = 0.0f;
    uint32_t fresh[kTileP], near[kTileP];
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
      fresh[q] = 0u, near[q] = 0u;
    if (UNROLL) {
      static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
      const int jb32 = (int)jb, nz32 = nz, n32 = (int)n;
#define VPD_DEFORM_CASE(C)                                                                                \
  case C:                                                                                                 \
    deform_window<C, DAMAGE, kTileP, int>(p, cnt, jb32, nz32, n32, gx, gz, by0, h, pt, bits, live, part, \
                                          fresh, near);                                                   \
    break;
      switch (cnt) {
        VPD_DEFORM_CASE(1) VPD_DEFORM_CASE(2) VPD_DEFORM_CASE(3) VPD_DEFORM_CASE(4)
        VPD_DEFORM_CASE(5) VPD_DEFORM_CASE(6) VPD_DEFORM_CASE(7) VPD_DEFORM_CASE(8)
        VPD_DEFORM_CASE(9) VPD_DEFORM_CASE(10) VPD_DEFORM_CASE(11) VPD_DEFORM_CASE(12)
      default:
        deform_window<0, DAMAGE, kTileP, int>(p, cnt, jb32, nz32, n32, gx, gz, by0, h, pt, bits, live, part,
                                              fresh, near);
      }
#undef VPD_DEFORM_CASE
    } else {
      deform_window<0, DAMAGE, kTileP, int64_t>(p, cnt, jb, (int64_t)nz, n, gx, gz, by0, h, pt, bits, live,
                                                part, fresh, near);
    }
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
#pragma unroll
      for (int c = 0; c < 9; ++c)
        G[q][c] += part[q][c];
    if (DAMAGE)
#pragma unroll
      for (int q = 0; q < kTileP; ++q)  // window positions -> slot offsets within the group
        commit_breaks(p, ip[q], pos, wd, sh, fresh[q] >> q, near[q] >> q);
  }
#pragma unroll
  for (int q = 0; q < kTileP; ++q)
    if (vp[q])
#pragma unroll
      for (int c = 0; c < 9; ++c)
        p.Gf[c * n + ip[q]] = G[q][c];
}

// ------------------------------------------------------------------ force
template <int P> struct ForcePoints {
  float jx[P], jy[P], jz[P];
};

template <int P, typename I>
__device__ __forceinline__ void force_element(const StepParams &p, int t, int cnt, I j, float gx, float gz,
                                              float by0, float h, const ForcePoints<P> &pt,
                                              const uint32_t (&bits)[P], float (&part)[P][3]) {
  const FmapRecord r = fmap_record(ldgf4(p.fmapf + j), ldgf4(p.fmapf + p.n + j), ldgf4(p.fmapf + 2 * p.n + j));
  const float oy = fmaf((float)t, h, by0);
#pragma unroll
  for (int q = 0; q < P; ++q) {
    if (t < q || t - q >= cnt)  // window position t holds no slot of point q
      continue;
    if (bits[q] & (1u << t)) {  // VM_j (o - J_q) + R_j, row by row
      const float e0 = gx - pt.jx[q], e1 = oy - pt.jy[q], e2 = gz - pt.jz[q];
      part[q][0] += fmaf(r.c2.x, e2, fmaf(r.c1.x, e1, fmaf(r.c0.x, e0, r.r01.x)));
      part[q][1] += fmaf(r.c2.y, e2, fmaf(r.c1.y, e1, fmaf(r.c0.y, e0, r.r01.y)));
      part[q][2] += fmap_row2(r, e0, e1, e2);
    }
  }
}

template <int CNT, int P, typename I>
__device__ __forceinline__ void force_window(const StepParams &p, int cnt, I jb, I nz, I n, float gx, float gz,
                                             float by0, float h, const ForcePoints<P> &pt,
                                             const uint32_t (&bits)[P], float (&part)[P][3]) {
  if constexpr (CNT > 0) {
#pragma unroll
    for (int t = 0; t < CNT + P - 1; ++t)
      force_element<P, I>(p, t, CNT, clamp_to<I>(jb + (I)t * nz, n), gx, gz, by0, h, pt, bits, part);
  } else {
    for (int t = 0; t < cnt + P - 1; ++t)
      force_element<P, I>(p, t, cnt, clamp_to<I>(jb + (I)t * nz, n), gx, gz, by0, h, pt, bits, part);
  }
}

// f = sum (V_j M_j) xi over intact bonds + M_i s_i with s_i = vxi_i - sum_{broken j} V_j xi.
template <int kTileP, bool UNROLL>
__global__ void __launch_bounds__(kBondThreads, 2) k_force_tiled(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  const float h = (float)p.lat_h;
  int x, yb, z;
  const bool inb = tile_coords<kTileP>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  const float4 *P0 = p.fmapf, *P1 = p.fmapf + n, *P2 = p.fmapf + 2 * n;
  int64_t ip[kTileP];
  bool vp[kTileP];
  ForcePoints<kTileP> pt;
#pragma unroll
  for (int q = 0; q < kTileP; ++q) {
    const int y = yb * kTileP + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const float4 a = ldgf4(p.jit + ip[q]);
    pt.jx[q] = a.x, pt.jy[q] = a.y + (float)q * h, pt.jz[q] = a.z;
  }
  float fs[kTileP][3], fc[kTileP][3];
  double corr[kTileP][3];
#pragma unroll
  for (int q = 0; q < kTileP; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      fs[q][c] = 0.0f, fc[q][c] = 0.0f, corr[q][c] = 0.0;
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    uint32_t bits[kTileP];
    uint32_t any = 0u;
#pragma unroll
    for (int q = 0; q < kTileP; ++q) {
      uint32_t m = vp[q] ? group_bits(__ldg(p.st.mask + (int64_t)wd * n + ip[q]), sh, cm) : 0u;
      if (p.damage && m) {
        const uint32_t bk = m & group_bits(p.st.broken[(int64_t)wd * n + ip[q]], sh, cm);
        for (uint32_t f = bk; f; f &= f - 1) {  // broken bonds leave s_i
          const int sl = pos + __ffs(f) - 1;
          const float4 jj = p.jit[ip[q] + p.st.delta[sl]], o = p.st.e0[sl];
          const float4 ji = p.jit[ip[q]];
          corr[q][0] += (double)(jj.w * (o.x + (jj.x - ji.x)));
          corr[q][1] += (double)(jj.w * (o.y + (jj.y - ji.y)));
          corr[q][2] += (double)(jj.w * (o.z + (jj.z - ji.z)));
        }
        m &= ~bk;
      }
      bits[q] = m << q;
      any |= bits[q];
    }
    if (__all_sync(0xffffffffu, any == 0u))
      continue;
    const float gx = (float)gr.x * h, gz = (float)gr.y * h, by0 = (float)gr.z * h;
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * kTileP + gr.z)) * nz + (z + gr.y);
    float part[kTileP][3];
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
      part[q][0] = part[q][1] = part[q][2] = 0.0f;
    if (UNROLL) {
      static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
      const int jb32 = (int)jb, nz32 = nz, n32 = (int)n;
#define VPD_FORCE_CASE(C)                                                                               \
  case C:                                                                                               \
    force_window<C, kTileP, int>(p, cnt, jb32, nz32, n32, gx, gz, by0, h, pt, bits, part);             \
    break;
      switch (cnt) {
        VPD_FORCE_CASE(1) VPD_FORCE_CASE(2) VPD_FORCE_CASE(3) VPD_FORCE_CASE(4)
        VPD_FORCE_CASE(5) VPD_FORCE_CASE(6) VPD_FORCE_CASE(7) VPD_FORCE_CASE(8)
        VPD_FORCE_CASE(9) VPD_FORCE_CASE(10) VPD_FORCE_CASE(11) VPD_FORCE_CASE(12)
      default:
        force_window<0, kTileP, int>(p, cnt, jb32, nz32, n32, gx, gz, by0, h, pt, bits, part);
      }
#undef VPD_FORCE_CASE
    } else {
      force_window<0, kTileP, int64_t>(p, cnt, jb, (int64_t)nz, n, gx, gz, by0, h, pt, bits, part);
    }
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        kahan_add(fs[q][c], fc[q][c], part[q][c]);
  }
#pragma unroll
  for (int q = 0; q < kTileP; ++q) {
    if (!vp[q])
      continue;
    const int64_t i = ip[q];
    float VM[9];
    fmap_rows(P0[i], P1[i], P2[i], VM);
    const double4 s = p.vxi[i];
    const double s0 = s.x - corr[q][0], s1 = s.y - corr[q][1], s2 = s.z - corr[q][2];
    const double rv = 1.0 / (double)p.jit[i].w;
    const double f0 = (double)fs[q][0] + (VM[0] * s0 + VM[1] * s1 + VM[2] * s2) * rv;
    const double f1 = (double)fs[q][1] + (VM[3] * s0 + VM[4] * s1 + VM[5] * s2) * rv;
    const double f2 = (double)fs[q][2] + (VM[6] * s0 + VM[7] * s1 + VM[8] * s2) * rv;
    p.force[i] = make_double4(f0, f1, f2, 0.0);
  }
}

// ------------------------------------------------------------------ packed pairs
// The default bond kernels: kTileP = 2 with the thread's two points held as the two lanes of
// packed FP32 pairs, so each bond term of both points is one paired instruction (half the
// arithmetic issue of the scalar kernels above). Windows, masks, operation order and rounding
// per lane are those of the scalar kernels; the unrolled windows index their neighbours without
// clamping (the neighbour arrays carry zero halos as deep as a window reaches, st.halo). The
// window's two ends, each a slot of only one
// point (t = 0: point 0, t = cnt: point 1), share one pair element in the unrolled windows; the
// runtime loop runs them as separate elements with the other lane's bond weight zero.
struct DeformPair {
  float2 jx, jy, jz, ux, uy, uz;  // lane q: point q (jy includes q h)
};

// The group's offsets of a neighbour from the thread's points: lane q of cx is gx - x_q (the
// group's x offset times h less point q's jitter), cy the same along y at window position 0
// (lowest dy times h less y_q, which includes q h), cz along z; window position t adds t h to
// cy. A bond's reference vector is then the neighbour's jitter plus these, one paired add per
// component. (The force kernel keeps its per-position adds: at its 85-register budget the three
// pairs spilled and cost it 11 %, 0.457 against 0.411 ms at 1M points; the deformation kernel
// gained 2.5 %.)
struct GroupOffsets {
  float2 cx, cy, cz;
};

template <bool DAMAGE, typename I>
__device__ __forceinline__ void deform_pair_element(const StepParams &p, int t, I j, const GroupOffsets &o,
                                                    float h, const DeformPair &pt, const uint32_t (&bits)[2],
                                                    const uint32_t (&live)[2], float2 (&part)[9],
                                                    uint32_t (&fresh)[2], uint32_t (&near)[2]) {
  const float4 a = ldgf4(p.jit + j), b = ldgf4(p.uf + j);
  const float2 e0 = __fadd2_rn(bcast2(a.x), o.cx);
  const float2 e1 = __fadd2_rn(bcast2(a.y), __ffma2_rn(bcast2((float)t), bcast2(h), o.cy));
  const float2 e2 = __fadd2_rn(bcast2(a.z), o.cz);
  const float2 d0 = sub2(bcast2(b.x), pt.ux), d1 = sub2(bcast2(b.y), pt.uy), d2 = sub2(bcast2(b.z), pt.uz);
  // bit t of bits[q]: window position t is a bond of point q (clear where it holds no slot of q)
  const float2 v = make_float2(((bits[0] >> t) & 1u) ? a.w : 0.0f, ((bits[1] >> t) & 1u) ? a.w : 0.0f);
  const float2 w0 = __fmul2_rn(v, d0), w1 = __fmul2_rn(v, d1), w2 = __fmul2_rn(v, d2);
  part[0] = __ffma2_rn(w0, e0, part[0]), part[1] = __ffma2_rn(w0, e1, part[1]);
  part[2] = __ffma2_rn(w0, e2, part[2]), part[3] = __ffma2_rn(w1, e0, part[3]);
  part[4] = __ffma2_rn(w1, e1, part[4]), part[5] = __ffma2_rn(w1, e2, part[5]);
  part[6] = __ffma2_rn(w2, e0, part[6]), part[7] = __ffma2_rn(w2, e1, part[7]);
  part[8] = __ffma2_rn(w2, e2, part[8]);
  if (DAMAGE)
    stretch_test2(p, t, t, e0, e1, e2, d0, d1, d2, live, near);
}

// The two ends of a window of CNT slots as one pair: lane 0 takes position 0 (point 0's first
// slot), lane 1 position CNT (point 1's last slot), each with the operations of
// deform_pair_element, so a window costs CNT pair elements instead of CNT + 1.
template <int CNT, bool DAMAGE, typename I>
__device__ __forceinline__ void deform_pair_ends(const StepParams &p, I j0, I j1, const GroupOffsets &o, float h,
                                                 const DeformPair &pt, const uint32_t (&bits)[2],
                                                 const uint32_t (&live)[2], float2 (&part)[9], uint32_t (&fresh)[2],
                                                 uint32_t (&near)[2]) {
  const float4 a0 = ldgf4(p.jit + j0), b0 = ldgf4(p.uf + j0), a1 = ldgf4(p.jit + j1), b1 = ldgf4(p.uf + j1);
  const float2 e0 = __fadd2_rn(make_float2(a0.x, a1.x), o.cx);
  const float2 e1 = __fadd2_rn(make_float2(a0.y, a1.y), __ffma2_rn(make_float2(0.0f, (float)CNT), bcast2(h), o.cy));
  const float2 e2 = __fadd2_rn(make_float2(a0.z, a1.z), o.cz);
  const float2 d0 = make_float2(b0.x - pt.ux.x, b1.x - pt.ux.y), d1 = make_float2(b0.y - pt.uy.x, b1.y - pt.uy.y);
  const float2 d2 = make_float2(b0.z - pt.uz.x, b1.z - pt.uz.y);
  const float2 v = make_float2((bits[0] & 1u) ? a0.w : 0.0f, ((bits[1] >> CNT) & 1u) ? a1.w : 0.0f);
  const float2 w0 = __fmul2_rn(v, d0), w1 = __fmul2_rn(v, d1), w2 = __fmul2_rn(v, d2);
  part[0] = __ffma2_rn(w0, e0, part[0]), part[1] = __ffma2_rn(w0, e1, part[1]);
  part[2] = __ffma2_rn(w0, e2, part[2]), part[3] = __ffma2_rn(w1, e0, part[3]);
  part[4] = __ffma2_rn(w1, e1, part[4]), part[5] = __ffma2_rn(w1, e2, part[5]);
  part[6] = __ffma2_rn(w2, e0, part[6]), part[7] = __ffma2_rn(w2, e1, part[7]);
  part[8] = __ffma2_rn(w2, e2, part[8]);
  if (DAMAGE)
    stretch_test2(p, 0, CNT, e0, e1, e2, d0, d1, d2, live, near);
}

template <int CNT, bool DAMAGE, typename I>
__device__ __forceinline__ void deform_pair_window(const StepParams &p, int cnt, I jb, I nz, I n,
                                                   const GroupOffsets &o, float h, const DeformPair &pt,
                                                   const uint32_t (&bits)[2], const uint32_t (&live)[2],
                                                   float2 (&part)[9], uint32_t (&fresh)[2], uint32_t (&near)[2]) {
  if constexpr (CNT > 0) {
#pragma unroll
    for (int t = 1; t < CNT; ++t)  // positions that hold a slot of both points (unclamped: halo)
      deform_pair_element<DAMAGE, I>(p, t, jb + (I)t * nz, o, h, pt, bits, live, part, fresh, near);
    deform_pair_ends<CNT, DAMAGE, I>(p, jb, jb + (I)CNT * nz, o, h, pt, bits, live, part, fresh, near);
  } else {
    for (int t = 0; t < cnt + 1; ++t)
      deform_pair_element<DAMAGE, I>(p, t, clamp_to<I>(jb + (I)t * nz, n), o, h, pt, bits, live, part, fresh,
                                     near);
  }
}

template <bool DAMAGE, bool UNROLL>
__global__ void __launch_bounds__(kBondThreads, 2) k_deformation_pair(const __grid_constant__ StepParams p) {
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
  DeformPair pt;
  pt.jx = make_float2(pa[0].x, pa[1].x), pt.jy = make_float2(pa[0].y, pa[1].y + h);
  pt.jz = make_float2(pa[0].z, pa[1].z);
  pt.ux = make_float2(pb[0].x, pb[1].x), pt.uy = make_float2(pb[0].y, pb[1].y);
  pt.uz = make_float2(pb[0].z, pb[1].z);
  // The windows of one stencil plane (the groups with the same x offset, which come in order)
  // sum into the plane partial `part`; each plane's partial is folded into G with Kahan
  // compensation (Gc).
  float2 G[9], Gc[9], part[9];
#pragma unroll
  for (int c = 0; c < 9; ++c)
    G[c] = Gc[c] = part[c] = make_float2(0.0f, 0.0f);
  int word = -1;  // the mask word held in mw (groups come in slot order: several per word)
  int plane = INT_MIN;
  // mw: the mask words; bw: the broken-bond words, read with them (only this thread sets the
  // bits of its points' forward slots, the only ones tested, and each slot is in one group)
  uint32_t mw[2] = {0u, 0u}, bw[2] = {0u, 0u};
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);  // dx, dz, lowest dy, (slots << 16) | first slot
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    if (gr.x != plane) {  // uniform: a new plane; fold the last one's partial
      plane = gr.x;
#pragma unroll
      for (int c = 0; c < 9; ++c)
        kahan_add2(G[c], Gc[c], part[c]), part[c] = make_float2(0.0f, 0.0f);
    }
    if (wd != word) {  // uniform: the group table is the same for every thread
      word = wd;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        mw[q] = vp[q] ? __ldg(p.st.mask + (int64_t)wd * n + ip[q]) : 0u;
        if (DAMAGE)
          bw[q] = vp[q] ? p.st.broken[(int64_t)wd * n + ip[q]] : 0u;
      }
    }
    uint32_t bits[2], live[2];
    const uint32_t fw = DAMAGE ? group_bits(__ldg(p.st.forward + wd), sh, cm) : 0u;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t m = group_bits(mw[q], sh, cm);
      bits[q] = m << q;  // bit t: the neighbour at window position t (slot pos + t - q)
      live[q] = DAMAGE ? (m & fw & ~group_bits(bw[q], sh, cm)) << q : 0u;
    }
    if (__all_sync(0xffffffffu, (bits[0] | bits[1]) == 0u))
      continue;
    const float gx = (float)gr.x * h, gz = (float)gr.y * h, by0 = (float)gr.z * h;
    const GroupOffsets o{sub2(bcast2(gx), pt.jx), sub2(bcast2(by0), pt.jy), sub2(bcast2(gz), pt.jz)};
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * 2 + gr.z)) * nz + (z + gr.y);
    uint32_t fresh[2] = {0u, 0u}, near[2] = {0u, 0u};
    // windows with stretch tests only where some lane of the warp has a live bond in the group
    // (with damage: the forward groups, less their broken bonds)
    const bool tests = DAMAGE && __any_sync(0xffffffffu, (live[0] | live[1]) != 0u);
    auto windows = [&](auto tested) {
      constexpr bool D = decltype(tested)::value;
      if (UNROLL) {
        static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
        const int jb32 = (int)jb, nz32 = nz, n32 = (int)n;
#define VPD_DEFORM_CASE(C)                                                                                   \
  case C:                                                                                                    \
    deform_pair_window<C, D, int>(p, cnt, jb32, nz32, n32, o, h, pt, bits, live, part, fresh, near);         \
    break;
        switch (cnt) {
          VPD_DEFORM_CASE(1) VPD_DEFORM_CASE(2) VPD_DEFORM_CASE(3) VPD_DEFORM_CASE(4)
          VPD_DEFORM_CASE(5) VPD_DEFORM_CASE(6) VPD_DEFORM_CASE(7) VPD_DEFORM_CASE(8)
          VPD_DEFORM_CASE(9) VPD_DEFORM_CASE(10) VPD_DEFORM_CASE(11) VPD_DEFORM_CASE(12)
        default:
          deform_pair_window<0, D, int>(p, cnt, jb32, nz32, n32, o, h, pt, bits, live, part, fresh, near);
        }
#undef VPD_DEFORM_CASE
      } else {
        deform_pair_window<0, D, int64_t>(p, cnt, jb, (int64_t)nz, n, o, h, pt, bits, live, part, fresh, near);
      }
    };
    if (tests)
      windows(BoolConstant<DAMAGE>{});
    else
      windows(BoolConstant<false>{});
    if (DAMAGE)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        commit_breaks(p, ip[q], pos, wd, sh, fresh[q] >> q, near[q] >> q);
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    kahan_add2(G[c], Gc[c], part[c]);
    const float2 g = sub2(G[c], Gc[c]);
    if (vp[0])
      p.Gf[c * n + ip[0]] = g.x;
    if (vp[1])
      p.Gf[c * n + ip[1]] = g.y;
  }
}

// The packed force kernel pairs the rows of a neighbour's force map, not the thread's points:
// a neighbour's records load as the pairs (VM_0c, VM_1c) and (R_0, R_1) (fmap_record), so rows 0
// and 1 of a bond term are three paired multiply-adds with the point's reference offset on both
// lanes, and row 2 is three scalar ones; no neighbour value is copied to both lanes of a pair.
// Point q's offsets from the group's window position 0, o - J_q, on both lanes of a pair
// (ey at window position t adds t h):
struct ForceOffsets {
  float2 ex[2], ey[2], ez[2];
};

// Point Q's bond at window position t (if its bit is set): rows 0, 1 into part01, row 2 into part2.
template <int Q>
__device__ __forceinline__ void force_pair_point(const FmapRecord &r, int t, float2 th, const ForceOffsets &o,
                                                 const uint32_t (&bits)[2], float2 (&part01)[2],
                                                 float (&part2)[2]) {
  const float2 ey = __fadd2_rn(o.ey[Q], th);
  const float2 v01 = fmap_rows01(r, o.ex[Q], ey, o.ez[Q]);
  const float v2 = fmap_row2(r, o.ex[Q].x, ey.x, o.ez[Q].x);
  if ((bits[Q] >> t) & 1u) {
    part01[Q] = __fadd2_rn(part01[Q], v01);
    part2[Q] += v2;
  }
}

// Window position t: the neighbour record and its bonds to the points whose slots it holds
// (Q < 0: both, else point Q only).
template <int Q, typename I>
__device__ __forceinline__ void force_pair_element(const StepParams &p, int t, I j, float h, const ForceOffsets &o,
                                                   const uint32_t (&bits)[2], float2 (&part01)[2],
                                                   float (&part2)[2]) {
  const FmapRecord r = fmap_record(ldgf4(p.fmapf + j), ldgf4(p.fmapf + p.n + j), ldgf4(p.fmapf + 2 * p.n + j));
  const float2 th = bcast2((float)t * h);
  if (Q <= 0)
    force_pair_point<0>(r, t, th, o, bits, part01, part2);
  if (Q != 0)
    force_pair_point<1>(r, t, th, o, bits, part01, part2);
}

template <int CNT, typename I>
__device__ __forceinline__ void force_pair_window(const StepParams &p, int cnt, I jb, I nz, I n, float h,
                                                  const ForceOffsets &o, const uint32_t (&bits)[2],
                                                  float2 (&part01)[2], float (&part2)[2]) {
  if constexpr (CNT > 0) {  // unclamped: the records carry zero halos
    force_pair_element<0, I>(p, 0, jb, h, o, bits, part01, part2);  // point 0's first slot
#pragma unroll
    for (int t = 1; t < CNT; ++t)  // positions that hold a slot of both points
      force_pair_element<-1, I>(p, t, jb + (I)t * nz, h, o, bits, part01, part2);
    force_pair_element<1, I>(p, CNT, jb + (I)CNT * nz, h, o, bits, part01, part2);  // point 1's last
  } else {
    for (int t = 0; t < cnt + 1; ++t)  // the bits are clear where a position holds no slot of a point
      force_pair_element<-1, I>(p, t, clamp_to<I>(jb + (I)t * nz, n), h, o, bits, part01, part2);
  }
}

// f = sum (V_j M_j) xi over intact bonds + M_i s_i with s_i = vxi_i - sum_{broken j} V_j xi.
// Two blocks per SM (128 registers, no spills): 0.375 against 0.393 ms at three blocks (80
// registers and spills) on the 1M-point bar in plastic flow.
template <bool DAMAGE, bool UNROLL>
__global__ void __launch_bounds__(kBondThreads, 2) k_force_pair(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  const float h = (float)p.lat_h;
  int x, yb, z;
  const bool inb = tile_coords<2>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  const float4 *P0 = p.fmapf, *P1 = p.fmapf + n, *P2 = p.fmapf + 2 * n;
  int64_t ip[2];
  bool vp[2];
  float jx[2], jy[2], jz[2];  // jy includes q h (y relative to the thread's first point)
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int y = yb * 2 + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const float4 a = ldgf4(p.jit + ip[q]);
    jx[q] = a.x, jy[q] = a.y + (float)q * h, jz[q] = a.z;
  }
  // the windows of one stencil plane sum into part01/part2, folded into fs01/fs2 with Kahan
  // compensation (fc01/fc2)
  float2 fs01[2], fc01[2], part01[2];
  float fs2[2], fc2[2], part2[2];
  bool any_broken = false;  // broken bonds' corrections are rare: gathered after the sum
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    fs01[q] = fc01[q] = part01[q] = make_float2(0.0f, 0.0f);
    fs2[q] = fc2[q] = part2[q] = 0.0f;
  }
  int word = -1;  // the mask (and broken-bond) words held in mw (bw): several groups per word
  int plane = INT_MIN;
  uint32_t mw[2] = {0u, 0u}, bw[2] = {0u, 0u};
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    if (gr.x != plane) {  // uniform: a new plane
      plane = gr.x;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        kahan_add2(fs01[q], fc01[q], part01[q]), kahan_add(fs2[q], fc2[q], part2[q]);
        part01[q] = make_float2(0.0f, 0.0f), part2[q] = 0.0f;
      }
    }
    if (wd != word) {  // uniform: the group table is the same for every thread
      word = wd;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        mw[q] = vp[q] ? __ldg(p.st.mask + (int64_t)wd * n + ip[q]) : 0u;
        if (DAMAGE)  // written by the deformation kernel, read-only here
          bw[q] = vp[q] ? __ldg(p.st.broken + (int64_t)wd * n + ip[q]) : 0u;
      }
    }
    uint32_t bits[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      uint32_t m = group_bits(mw[q], sh, cm);
      if (DAMAGE && m) {
        const uint32_t bk = m & group_bits(bw[q], sh, cm);
        any_broken |= bk != 0u;
        m &= ~bk;
      }
      bits[q] = m << q;
    }
    if (__all_sync(0xffffffffu, (bits[0] | bits[1]) == 0u))
      continue;
    const float gx = (float)gr.x * h, gz = (float)gr.y * h, by0 = (float)gr.z * h;
    ForceOffsets o;
#pragma unroll
    for (int q = 0; q < 2; ++q)
      o.ex[q] = bcast2(gx - jx[q]), o.ey[q] = bcast2(by0 - jy[q]), o.ez[q] = bcast2(gz - jz[q]);
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * 2 + gr.z)) * nz + (z + gr.y);
    if (UNROLL) {
      static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
      const int jb32 = (int)jb, nz32 = nz, n32 = (int)n;
#define VPD_FORCE_CASE(C)                                                                 \
  case C:                                                                                 \
    force_pair_window<C, int>(p, cnt, jb32, nz32, n32, h, o, bits, part01, part2);        \
    break;
      switch (cnt) {
        VPD_FORCE_CASE(1) VPD_FORCE_CASE(2) VPD_FORCE_CASE(3) VPD_FORCE_CASE(4)
        VPD_FORCE_CASE(5) VPD_FORCE_CASE(6) VPD_FORCE_CASE(7) VPD_FORCE_CASE(8)
        VPD_FORCE_CASE(9) VPD_FORCE_CASE(10) VPD_FORCE_CASE(11) VPD_FORCE_CASE(12)
      default:
        force_pair_window<0, int>(p, cnt, jb32, nz32, n32, h, o, bits, part01, part2);
      }
#undef VPD_FORCE_CASE
    } else {
      force_pair_window<0, int64_t>(p, cnt, jb, (int64_t)nz, n, h, o, bits, part01, part2);
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    kahan_add2(fs01[q], fc01[q], part01[q]), kahan_add(fs2[q], fc2[q], part2[q]);
    if (!vp[q])
      continue;
    const int64_t i = ip[q];
    // s_i less the broken bonds' V_j xi, summed in slot order
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
    if (DAMAGE && any_broken) {
      const float4 ji = p.jit[i];
      for (int w = 0; w < p.st.nw; ++w)
        for (uint32_t f = p.st.mask[(int64_t)w * n + i] & p.st.broken[(int64_t)w * n + i]; f; f &= f - 1) {
          const int sl = 32 * w + __ffs(f) - 1;
          const float4 jj = p.jit[i + p.st.delta[sl]], o = p.st.e0[sl];
          c0 += (double)(jj.w * (o.x + (jj.x - ji.x)));
          c1 += (double)(jj.w * (o.y + (jj.y - ji.y)));
          c2 += (double)(jj.w * (o.z + (jj.z - ji.z)));
        }
    }
    float VM[9];
    fmap_rows(P0[i], P1[i], P2[i], VM);
    const double4 s = p.vxi[i];
    const double s0 = s.x - c0, s1 = s.y - c1, s2 = s.z - c2;
    const double rv = 1.0 / (double)p.jit[i].w;
    const double f0 = (double)fs01[q].x + (VM[0] * s0 + VM[1] * s1 + VM[2] * s2) * rv;
    const double f1 = (double)fs01[q].y + (VM[3] * s0 + VM[4] * s1 + VM[5] * s2) * rv;
    const double f2 = (double)fs2[q] + (VM[6] * s0 + VM[7] * s1 + VM[8] * s2) * rv;
    p.force[i] = make_double4(f0, f1, f2, 0.0);
  }
}

// ------------------------------------------------------------------ launchers
// With damage the scalar deformation kernel keeps the runtime window loop (unrolled, its
// stretch tests made it slower: 0.28 against 0.25 ms on the 250k-point bar); the packed-pair
// kernel unrolls its windows with damage too (0.698 against 0.783 ms on the 1M-point bar).
template <bool UNROLL> static void launch_deformation(const StepParams &p, cudaStream_t s) {
  const unsigned grid = tiled_grid<2>(p);
  if (p.tiled == 1) {
    if (p.damage)
      k_deformation_tiled<true, 2, false><<<grid, kBondThreads, 0, s>>>(p);
    else
      k_deformation_tiled<false, 2, UNROLL><<<grid, kBondThreads, 0, s>>>(p);
  } else {
    if (p.damage)
      k_deformation_pair<true, UNROLL><<<grid, kBondThreads, 0, s>>>(p);
    else
      k_deformation_pair<false, UNROLL><<<grid, kBondThreads, 0, s>>>(p);
  }
}

// p.tiled: 1 the scalar two-point kernels, else the packed-pair ones (VPD_BOND_KERNEL, read
// when the handle is created)
int launch_deformation_tiled(const StepParams &p, cudaStream_t s) {
  index32(p) ? launch_deformation<true>(p, s) : launch_deformation<false>(p, s);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int launch_force_tiled(const StepParams &p, cudaStream_t s) {
  const bool u = index32(p);
  const unsigned grid = tiled_grid<2>(p);
  if (p.tiled == 1) {
    if (u)
      k_force_tiled<2, true><<<grid, kBondThreads, 0, s>>>(p);
    else
      k_force_tiled<2, false><<<grid, kBondThreads, 0, s>>>(p);
  } else {
    if (p.damage)
      u ? k_force_pair<true, true><<<grid, kBondThreads, 0, s>>>(p)
        : k_force_pair<true, false><<<grid, kBondThreads, 0, s>>>(p);
    else
      u ? k_force_pair<false, true><<<grid, kBondThreads, 0, s>>>(p)
        : k_force_pair<false, false><<<grid, kBondThreads, 0, s>>>(p);
  }
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
