// Tiled FP64 bond kernels of the plain path: the deformation gradient (with critical-stretch
// bond breaking), two points per thread along y, and the force bond sum, three points per
// thread along y (the tiling of vpd_tiled.cu: one load of each neighbour record per
// stencil-group window, consecutive threads on consecutive z).
//
// Each point sums its bonds in slot order with the operations of the per-slot kernels
// (k_deformation_stencil, k_force_stencil in vpd_stencil.cu; both spell out every rounding
// through the helpers of vpd_bond.cuh): a window position that holds no slot of the point is
// skipped and a slot without a bond adds a zero term, as there. The results are therefore
// bit-identical to theirs; what changes is that a neighbour's records are read once for all of
// a thread's points instead of once per point, and padding slots are not visited.
#include "vpd_bond.cuh"

namespace vpd {

// ------------------------------------------------------------------ deformation
struct Deform64 {
  double xx[2], xy[2], xz[2], ux[2], uy[2], uz[2];  // the thread's two points
};

// Window position t of a group: neighbour j and its bonds to the thread's points (point q holds
// slot t - q of the group, 0 <= t - q < cnt).
template <bool DAMAGE, typename I>
__device__ __forceinline__ void deform64_element(const StepParams &p, const double4 *U, int t, int cnt, I j,
                                                 const Deform64 &pt, const int64_t (&ip)[2],
                                                 const uint32_t (&bits)[2], const uint32_t (&live)[2],
                                                 double (&G)[2][9], uint32_t (&fresh)[2]) {
  const double4 xj = ldg256(p.xv + j), uj = ldg256(U + j);
  const double lo = 1.0 - 1.0e-9, hi = 1.0 + 1.0e-9;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (t < q || t - q >= cnt)
      continue;
    const double v = ((bits[q] >> t) & 1u) ? xj.w : 0.0;
    const double e0 = xj.x - pt.xx[q], e1 = xj.y - pt.xy[q], e2 = xj.z - pt.xz[q];
    const double d0 = uj.x - pt.ux[q], d1 = uj.y - pt.uy[q], d2 = uj.z - pt.uz[q];
    bond_deform64(G[q], v, d0, d1, d2, e0, e1, e2);
    if (DAMAGE && ((live[q] >> t) & 1u)) {
      const double y0 = e0 + d0, y1 = e1 + d1, y2 = e2 + d2;
      const double yy = y0 * y0 + y1 * y1 + y2 * y2;
      const double xx = e0 * e0 + e1 * e1 + e2 * e2;
      const double tt = p.tension2 * xx;
      bool broke = false;
      if (yy > tt * hi)
        broke = true;
      else if (yy >= tt * lo)
        broke = exact_break(p.xv, U, ip[q], (int64_t)j, p.dmg_initiation, p.dmg_failure, p.use_compression);
      else if (p.use_compression) {
        const double c = p.compression2 * xx;
        if (yy < c * lo)
          broke = true;
        else if (yy <= c * hi)
          broke = exact_break(p.xv, U, ip[q], (int64_t)j, p.dmg_initiation, p.dmg_failure, 1);
      }
      if (broke)
        fresh[q] |= 1u << t;
    }
  }
}

template <int CNT, bool DAMAGE, typename I>
__device__ __forceinline__ void deform64_window(const StepParams &p, const double4 *U, int cnt, I jb, I nz, I n,
                                                const Deform64 &pt, const int64_t (&ip)[2],
                                                const uint32_t (&bits)[2], const uint32_t (&live)[2],
                                                double (&G)[2][9], uint32_t (&fresh)[2]) {
  if constexpr (CNT > 0) {
#pragma unroll
    for (int t = 0; t < CNT + 1; ++t)
      deform64_element<DAMAGE, I>(p, U, t, CNT, clamp_to<I>(jb + (I)t * nz, n), pt, ip, bits, live, G, fresh);
  } else {
    for (int t = 0; t < cnt + 1; ++t)
      deform64_element<DAMAGE, I>(p, U, t, cnt, clamp_to<I>(jb + (I)t * nz, n), pt, ip, bits, live, G, fresh);
  }
}

// F = I + [sum_j V_j (u_j - u_i) (x) xi] K^-1 over all bonds; with damage, the FP64
// critical-stretch test on each intact forward bond, breaking both directed bonds of a pair.
template <bool DAMAGE, bool UNROLL>
__global__ void __launch_bounds__(kBondThreads, 2) k_deformation_tiled64(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  int x, yb, z;
  const bool inb = tile_coords<2>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  const int64_t step = *p.step;
  const double4 *U = (step & 1) ? p.u1 : p.u0;
  int64_t ip[2];
  bool vp[2];
  Deform64 pt;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int y = yb * 2 + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const double4 xi = ldg256(p.xv + ip[q]), ui = ldg256(U + ip[q]);
    pt.xx[q] = xi.x, pt.xy[q] = xi.y, pt.xz[q] = xi.z;
    pt.ux[q] = ui.x, pt.uy[q] = ui.y, pt.uz[q] = ui.z;
  }
  double G[2][9];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int c = 0; c < 9; ++c)
      G[q][c] = 0.0;
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);  // dx, dz, lowest dy, (slots << 16) | first slot
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    uint32_t bits[2], live[2];
    const uint32_t fw = DAMAGE ? group_bits(__ldg(p.st.forward + wd), sh, cm) : 0u;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t m = vp[q] ? group_bits(__ldg(p.st.mask + (int64_t)wd * n + ip[q]), sh, cm) : 0u;
      bits[q] = m << q;  // bit t: the neighbour at window position t (slot pos + t - q)
      live[q] = 0u;
      if (DAMAGE) {
        const uint32_t bk = vp[q] ? group_bits(p.st.broken[(int64_t)wd * n + ip[q]], sh, cm) : 0u;
        live[q] = (m & fw & ~bk) << q;
      }
    }
    if (__all_sync(0xffffffffu, (bits[0] | bits[1]) == 0u))
      continue;
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * 2 + gr.z)) * nz + (z + gr.y);
    uint32_t fresh[2] = {0u, 0u};
    // With damage, the stretch tests run (in the runtime window loop: unrolled, they spill) only
    // for the groups where a lane of the warp has a live bond, the forward groups less their
    // broken bonds; the other groups take the unrolled windows without tests.
    if (DAMAGE && __any_sync(0xffffffffu, (live[0] | live[1]) != 0u)) {
      deform64_window<0, DAMAGE, int64_t>(p, U, cnt, jb, (int64_t)nz, n, pt, ip, bits, live, G, fresh);
    } else if (UNROLL) {
      static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
      const int jb32 = (int)jb, nz32 = nz, n32 = (int)n;
#define VPD_DEFORM64_CASE(C)                                                                        \
  case C:                                                                                           \
    deform64_window<C, false, int>(p, U, cnt, jb32, nz32, n32, pt, ip, bits, live, G, fresh);       \
    break;
      switch (cnt) {
        VPD_DEFORM64_CASE(1) VPD_DEFORM64_CASE(2) VPD_DEFORM64_CASE(3) VPD_DEFORM64_CASE(4)
        VPD_DEFORM64_CASE(5) VPD_DEFORM64_CASE(6) VPD_DEFORM64_CASE(7) VPD_DEFORM64_CASE(8)
        VPD_DEFORM64_CASE(9) VPD_DEFORM64_CASE(10) VPD_DEFORM64_CASE(11) VPD_DEFORM64_CASE(12)
      default:
        deform64_window<0, false, int>(p, U, cnt, jb32, nz32, n32, pt, ip, bits, live, G, fresh);
      }
#undef VPD_DEFORM64_CASE
    } else {
      deform64_window<0, false, int64_t>(p, U, cnt, jb, (int64_t)nz, n, pt, ip, bits, live, G, fresh);
    }
    if (DAMAGE)
#pragma unroll
      for (int q = 0; q < 2; ++q)  // window positions -> slot offsets within the group
        commit_breaks(p, ip[q], pos, wd, sh, fresh[q] >> q, 0u);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (!vp[q])
      continue;
    const int64_t i = ip[q];
    double K[9], F[9];
#pragma unroll
    for (int c = 0; c < 9; ++c)
      K[c] = p.kinv[c * n + i];
    deformation_from_g(G[q], K, F);
#pragma unroll
    for (int c = 0; c < 9; ++c)
      p.F[c * n + i] = F[c];
  }
}

// ------------------------------------------------------------------ force
template <int P, typename I>
__device__ __forceinline__ void force64_element(const StepParams &p, int t, int cnt, I j, const double (&px)[P],
                                                const double (&py)[P], const double (&pz)[P],
                                                const uint32_t (&bits)[P], double (&f)[P][3]) {
  const double4 *P0 = p.fmap, *P1 = p.fmap + p.n, *P2 = p.fmap + 2 * p.n;
  const double4 a = ldg256(P0 + j), c = ldg256(P1 + j), d = ldg256(P2 + j);
#pragma unroll
  for (int q = 0; q < P; ++q) {
    if (t < q || t - q >= cnt)
      continue;
    const bool bond = (bits[q] >> t) & 1u;
    const double e0 = bond ? a.w - px[q] : 0.0, e1 = bond ? c.w - py[q] : 0.0, e2 = bond ? d.w - pz[q] : 0.0;
    f[q][0] = __dadd_rn(f[q][0], dot3_rn(a.x, a.y, a.z, e0, e1, e2));
    f[q][1] = __dadd_rn(f[q][1], dot3_rn(c.x, c.y, c.z, e0, e1, e2));
    f[q][2] = __dadd_rn(f[q][2], dot3_rn(d.x, d.y, d.z, e0, e1, e2));
  }
}

template <int CNT, int P, typename I>
__device__ __forceinline__ void force64_window(const StepParams &p, int cnt, I jb, I nz, I n, const double (&px)[P],
                                               const double (&py)[P], const double (&pz)[P],
                                               const uint32_t (&bits)[P], double (&f)[P][3]) {
  if constexpr (CNT > 0) {
#pragma unroll
    for (int t = 0; t < CNT + P - 1; ++t)
      force64_element<P, I>(p, t, CNT, clamp_to<I>(jb + (I)t * nz, n), px, py, pz, bits, f);
  } else {
    for (int t = 0; t < cnt + P - 1; ++t)
      force64_element<P, I>(p, t, cnt, clamp_to<I>(jb + (I)t * nz, n), px, py, pz, bits, f);
  }
}

// f_i = sum_j V_j M_j xi over intact bonds + M_i s_i, s_i = vxi_i - sum_{broken j} V_j xi: a
// bond reads the three force-map records of j (its coordinates ride in their fourth lane).
// kTileP points per thread along y.
template <int kTileP, bool UNROLL, int TPB = kBondThreads, int MINB = 2>
__global__ void __launch_bounds__(TPB, MINB) k_force_tiled64(const __grid_constant__ StepParams p) {
  constexpr int P = kTileP;
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  int x, yb, z;
  const bool inb = tile_coords<P>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  int64_t ip[P];
  bool vp[P];
  double px[P], py[P], pz[P], f[P][3];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int y = yb * P + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const double4 xi = ldg256(p.xv + ip[q]);
    px[q] = xi.x, py[q] = xi.y, pz[q] = xi.z;
    f[q][0] = f[q][1] = f[q][2] = 0.0;
  }
  bool any_broken = false;  // corrections for broken bonds are rare: gathered after the sum
  for (int g = 0; g < p.st.ngroups; ++g) {
    const int4 gr = __ldg(p.st.groups + g);
    const int cnt = gr.w >> 16, pos = gr.w & 0xffff, wd = pos >> 5, sh = pos & 31;
    const uint32_t cm = cnt >= 32 ? ~0u : ((1u << cnt) - 1u);
    uint32_t bits[P], any = 0u;
#pragma unroll
    for (int q = 0; q < P; ++q) {
      uint32_t m = vp[q] ? group_bits(__ldg(p.st.mask + (int64_t)wd * n + ip[q]), sh, cm) : 0u;
      if (p.damage && m) {
        const uint32_t bk = m & group_bits(p.st.broken[(int64_t)wd * n + ip[q]], sh, cm);
        any_broken |= bk != 0u;
        m &= ~bk;
      }
      bits[q] = m << q;  // bit t: the neighbour at window position t (slot pos + t - q)
      any |= bits[q];
    }
    if (__all_sync(0xffffffffu, any == 0u))
      continue;
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * P + gr.z)) * nz + (z + gr.y);
    if (UNROLL) {
      static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
      const int jb32 = (int)jb, nz32 = nz, n32 = (int)n;
#define VPD_FORCE64_CASE(C)                                                       \
  case C:                                                                         \
    force64_window<C, P, int>(p, cnt, jb32, nz32, n32, px, py, pz, bits, f);      \
    break;
      switch (cnt) {
        VPD_FORCE64_CASE(1) VPD_FORCE64_CASE(2) VPD_FORCE64_CASE(3) VPD_FORCE64_CASE(4)
        VPD_FORCE64_CASE(5) VPD_FORCE64_CASE(6) VPD_FORCE64_CASE(7) VPD_FORCE64_CASE(8)
        VPD_FORCE64_CASE(9) VPD_FORCE64_CASE(10) VPD_FORCE64_CASE(11) VPD_FORCE64_CASE(12)
      default:
        force64_window<0, P, int>(p, cnt, jb32, nz32, n32, px, py, pz, bits, f);
      }
#undef VPD_FORCE64_CASE
    } else {
      force64_window<0, P, int64_t>(p, cnt, jb, (int64_t)nz, n, px, py, pz, bits, f);
    }
  }
  const double4 *P0 = p.fmap, *P1 = p.fmap + n, *P2 = p.fmap + 2 * n;
#pragma unroll
  for (int q = 0; q < P; ++q) {
    if (!vp[q])
      continue;
    const int64_t i = ip[q];
    // s_i less the broken bonds' V_j xi, summed in slot order
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
    if (any_broken)
      for (int w = 0; w < p.st.nw; ++w)
        for (uint32_t b = p.st.mask[(int64_t)w * n + i] & p.st.broken[(int64_t)w * n + i]; b; b &= b - 1) {
          const double4 xj = p.xv[i + p.st.delta[32 * w + __ffs(b) - 1]];
          c0 += xj.w * (xj.x - px[q]), c1 += xj.w * (xj.y - py[q]), c2 += xj.w * (xj.z - pz[q]);
        }
    const double4 a = P0[i], c = P1[i], d = P2[i], s = p.vxi[i];
    const double s0 = s.x - c0, s1 = s.y - c1, s2 = s.z - c2;
    const double r = 1.0 / p.xv[i].w;  // M_i = (V_i M_i) / V_i
    const double f0 = __dadd_rn(f[q][0], __dmul_rn(dot3_rn(a.x, a.y, a.z, s0, s1, s2), r));
    const double f1 = __dadd_rn(f[q][1], __dmul_rn(dot3_rn(c.x, c.y, c.z, s0, s1, s2), r));
    const double f2 = __dadd_rn(f[q][2], __dmul_rn(dot3_rn(d.x, d.y, d.z, s0, s1, s2), r));
    p.force[i] = make_double4(f0, f1, f2, 0.0);
  }
}

// ------------------------------------------------------------------ launchers
// With damage the groups with live bonds keep the runtime window loop (unrolled, the FP64 stretch
// tests spill about 1 KB per thread and the kernel slowed from 0.96 to 1.29 ms at 1M points); the
// groups without take the unrolled windows without tests (0.975 to 0.90 ms from rest at 1M).
int launch_deformation_tiled64(const StepParams &p, cudaStream_t s) {
  const unsigned grid = tiled_grid<2>(p);
  if (p.damage)
    index32(p) ? k_deformation_tiled64<true, true><<<grid, kBondThreads, 0, s>>>(p)
               : k_deformation_tiled64<true, false><<<grid, kBondThreads, 0, s>>>(p);
  else if (index32(p))
    k_deformation_tiled64<false, true><<<grid, kBondThreads, 0, s>>>(p);
  else
    k_deformation_tiled64<false, false><<<grid, kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

// three points per thread in one 384-thread block per SM (two points in 256-thread blocks with
// VPD_BOND_KERNEL=tiled2; the TMA-staged kernel of vpd_staged64.cu with VPD_BOND_KERNEL=staged
// where its box fits)
int launch_force_tiled64(const StepParams &p, cudaStream_t s) {
  if (p.tiled == 6 && p.staged.bytes)
    return launch_force_staged64(p, s);
  if (p.tiled == 3) {
    const unsigned grid = tiled_grid<2>(p);
    if (index32(p))
      k_force_tiled64<2, true><<<grid, kBondThreads, 0, s>>>(p);
    else
      k_force_tiled64<2, false><<<grid, kBondThreads, 0, s>>>(p);
  } else {
    // A block's neighbourhood of force-map records for one stencil plane (its y-z range plus the
    // stencil's reach, 96 bytes a point) is re-read for every group of the plane, so it should
    // stay in L1: three points per thread in one 384-thread block per SM (about 1150 points,
    // a neighbourhood of about 175 KB on a 50 x 50 cross-section). On the 1M-point bar that grid
    // is also 5.98 waves of 148 blocks. 0.616 ms at 1M points, against 0.787 for four points in
    // 512-thread blocks (3.43 waves) and 0.821 for four points in two 256-thread blocks per SM.
    const int64_t threads = (int64_t)tiled_grid<3>(p) * kBondThreads;
    const unsigned grid = (unsigned)((threads + 383) / 384);
    if (index32(p))
      k_force_tiled64<3, true, 384, 1><<<grid, 384, 0, s>>>(p);
    else
      k_force_tiled64<3, false, 384, 1><<<grid, 384, 0, s>>>(p);
  }
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
