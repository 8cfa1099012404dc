// Tiled mixed-precision bond kernels: the deformation gradient (with critical-stretch bond
// breaking) and the force bond sum, with each thread owning kTileP points of one lattice
// column along y (same x and z, y = kTileP yb + q).
//
// The stencil's slots are grouped by the offset's (x, z) components (vpd_stencil.cu): the
// offsets of a group differ only in y, so the neighbours that the kTileP points reach through
// one group form a single run of cnt + kTileP - 1 consecutive lattice points along y. The
// thread loads each of those neighbour records once and applies it to every one of its
// points that has the matching bond, instead of loading it once per bond: the loads fall by
// about cnt kTileP / (cnt + kTileP - 1). Consecutive threads take consecutive z, so each load
// of a warp is one contiguous range.
//
// Arithmetic is that of vpd_mixed.cu: FP32 bond terms, per-group partial sums (folded with
// Kahan compensation into the force), the FP32 stretch test with a 1e-5 margin and the exact
// FP64 test inside it, pairs broken once by the lower-index point.
#include "vpd_bond.cuh"

namespace vpd {

// Lattice coordinates of thread tau's column: z fastest, then the y-block, then x.
template <int kTileP>
__device__ __forceinline__ bool tile_coords(const StepParams &p, int64_t tau, int &x, int &yb, int &z) {
  const int nz = p.lat_nz, nyb = (p.lat_ny + kTileP - 1) / kTileP;
  z = (int)(tau % nz);
  const int64_t r = tau / nz;
  yb = (int)(r % nyb);
  x = (int)(r / nyb);
  return x < p.lat_nx;
}

__device__ __forceinline__ uint32_t group_bits(uint32_t word, int shift, uint32_t cm) {
  return (word >> shift) & cm;
}

template <bool DAMAGE, int kTileP>
__global__ void __launch_bounds__(kBondThreads, 2) k_deformation_tiled(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  const float h = (float)p.lat_h;
  int x, yb, z;
  const bool inb = tile_coords<kTileP>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  int64_t ip[kTileP];
  bool vp[kTileP];
  float jx[kTileP], jy[kTileP], jz[kTileP], ux[kTileP], uy[kTileP], uz[kTileP];
#pragma unroll
  for (int q = 0; q < kTileP; ++q) {
    const int y = yb * kTileP + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const float4 a = ldgf4(p.jit + ip[q]), b = ldgf4(p.uf + ip[q]);
    jx[q] = a.x, jy[q] = a.y + (float)q * h, jz[q] = a.z;  // y relative to the tile's base row
    ux[q] = b.x, uy[q] = b.y, uz[q] = b.z;
  }
  float G[kTileP][9];
#pragma unroll
  for (int q = 0; q < kTileP; ++q)
#pragma unroll
    for (int c = 0; c < 9; ++c)
      G[q][c] = 0.0f;
  const float lo = 1.0f - 1.0e-5f, hi = 1.0f + 1.0e-5f;
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
      if (DAMAGE) {
        const uint32_t bk = vp[q] ? group_bits(p.st.broken[(int64_t)wd * n + ip[q]], sh, cm) : 0u;
        live[q] = (m & fw & ~bk) << q;
      }
      any |= bits[q];
    }
    if (__all_sync(0xffffffffu, any == 0u))
      continue;
    const float gx = (float)gr.x * h, gz = (float)gr.y * h;
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
    const int T = cnt + kTileP - 1;
    for (int t = 0; t < T; ++t) {
      const int64_t j = clamp_index(jb + (int64_t)t * nz, n);
      const float4 a = ldgf4(p.jit + j), b = ldgf4(p.uf + j);
      const float bx = a.x + gx, by = a.y + (float)(gr.z + t) * h, bz = a.z + gz;
#pragma unroll
      for (int q = 0; q < kTileP; ++q) {
        if (t < q || t - q >= cnt)  // window position t holds no slot of point q (uniform)
          continue;
        const float e0 = bx - jx[q], e1 = by - jy[q], e2 = bz - jz[q];
        const float d0 = b.x - ux[q], d1 = b.y - uy[q], d2 = b.z - uz[q];
        const float v = ((bits[q] >> t) & 1u) ? a.w : 0.0f;  // no bond: no contribution
        const float w0 = v * d0, w1 = v * d1, w2 = v * d2;
        part[q][0] += w0 * e0, part[q][1] += w0 * e1, part[q][2] += w0 * e2;
        part[q][3] += w1 * e0, part[q][4] += w1 * e1, part[q][5] += w1 * e2;
        part[q][6] += w2 * e0, part[q][7] += w2 * e1, part[q][8] += w2 * e2;
        if (DAMAGE && ((live[q] >> t) & 1u)) {
          const float y0 = e0 + d0, y1 = e1 + d1, y2 = e2 + d2;
          const float yy = y0 * y0 + y1 * y1 + y2 * y2;
          const float xx = e0 * e0 + e1 * e1 + e2 * e2;
          const float tt = p.tension2f * xx;
          if (yy > tt * hi)
            fresh[q] |= 1u << t;
          else if (yy >= tt * lo)
            near[q] |= 1u << t;
          else if (p.use_compression) {
            const float c = p.compression2f * xx;
            if (yy < c * lo)
              fresh[q] |= 1u << t;
            else if (yy <= c * hi)
              near[q] |= 1u << t;
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
#pragma unroll
      for (int c = 0; c < 9; ++c)
        G[q][c] += part[q][c];
    if (DAMAGE) {
#pragma unroll
      for (int q = 0; q < kTileP; ++q) {
        uint32_t fr = fresh[q] >> q;  // slot offsets within the group
        if (near[q]) {
          const int64_t step = *p.step;
          const double4 *U = (step & 1) ? p.u1 : p.u0;
          for (uint32_t f = near[q] >> q; f; f &= f - 1) {
            const int k = __ffs(f) - 1;
            if (exact_break_mixed(p.xv, U, ip[q], ip[q] + p.st.delta[pos + k], p.dmg_initiation,
                                  p.dmg_failure, p.use_compression))
              fr |= 1u << k;
          }
        }
        if (fr) {
          atomicOr(p.st.broken + (int64_t)wd * n + ip[q], fr << sh);
          for (uint32_t f = fr; f; f &= f - 1) {
            const int sl = pos + __ffs(f) - 1;
            const int r = p.st.reverse[sl];
            atomicOr(p.st.broken + (int64_t)(r >> 5) * n + (ip[q] + p.st.delta[sl]), 1u << (r & 31));
          }
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kTileP; ++q)
    if (vp[q])
#pragma unroll
      for (int c = 0; c < 9; ++c)
        p.Gf[c * n + ip[q]] = G[q][c];
}

// f = sum (V_j M_j) xi over intact bonds + M_i s_i with s_i = vxi_i - sum_{broken j} V_j xi.
template <int kTileP>
__global__ void __launch_bounds__(kBondThreads, 2) k_force_tiled(const __grid_constant__ StepParams p) {
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  const float h = (float)p.lat_h;
  int x, yb, z;
  const bool inb = tile_coords<kTileP>(p, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, x, yb, z);
  const float4 *P0 = p.fmapf, *P1 = p.fmapf + n, *P2 = p.fmapf + 2 * n;
  int64_t ip[kTileP];
  bool vp[kTileP];
  float jx[kTileP], jy[kTileP], jz[kTileP];
#pragma unroll
  for (int q = 0; q < kTileP; ++q) {
    const int y = yb * kTileP + q;
    vp[q] = inb && y < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y) * nz + z : 0;
    const float4 a = ldgf4(p.jit + ip[q]);
    jx[q] = a.x, jy[q] = a.y + (float)q * h, jz[q] = a.z;
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
    const float gx = (float)gr.x * h, gz = (float)gr.y * h;
    const int64_t jb = ((int64_t)(x + gr.x) * ny + (yb * kTileP + gr.z)) * nz + (z + gr.y);
    float part[kTileP][3];
#pragma unroll
    for (int q = 0; q < kTileP; ++q)
      part[q][0] = part[q][1] = part[q][2] = 0.0f;
    const int T = cnt + kTileP - 1;
    for (int t = 0; t < T; ++t) {
      const int64_t j = clamp_index(jb + (int64_t)t * nz, n);
      const float4 a = ldgf4(P0 + j), b = ldgf4(P1 + j), c = ldgf4(P2 + j);
      const float bx = a.w + gx, by = b.w + (float)(gr.z + t) * h, bz = c.w + gz;
#pragma unroll
      for (int q = 0; q < kTileP; ++q) {
        if (t < q || t - q >= cnt)  // window position t holds no slot of point q (uniform)
          continue;
        const bool bond = (bits[q] >> t) & 1u;
        const float e0 = bond ? bx - jx[q] : 0.0f, e1 = bond ? by - jy[q] : 0.0f;
        const float e2 = bond ? bz - jz[q] : 0.0f;
        part[q][0] += a.x * e0 + a.y * e1 + a.z * e2;
        part[q][1] += b.x * e0 + b.y * e1 + b.z * e2;
        part[q][2] += c.x * e0 + c.y * e1 + c.z * e2;
      }
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
    const float4 a = P0[i], b = P1[i], c = P2[i], ji = p.jit[i];
    const double4 s = p.vxi[i];
    const double s0 = s.x - corr[q][0], s1 = s.y - corr[q][1], s2 = s.z - corr[q][2];
    const double rv = 1.0 / (double)ji.w;
    const double f0 = (double)fs[q][0] + (a.x * s0 + a.y * s1 + a.z * s2) * rv;
    const double f1 = (double)fs[q][1] + (b.x * s0 + b.y * s1 + b.z * s2) * rv;
    const double f2 = (double)fs[q][2] + (c.x * s0 + c.y * s1 + c.z * s2) * rv;
    p.force[i] = make_double4(f0, f1, f2, 0.0);
  }
}

template <int kTileP> static unsigned tiled_grid(const StepParams &p) {
  const int64_t threads = (int64_t)p.lat_nx * ((p.lat_ny + kTileP - 1) / kTileP) * p.lat_nz;
  return (unsigned)((threads + kBondThreads - 1) / kBondThreads);
}

// points per thread: 2 unless VPD_BOND_KERNEL=tiled3 (read when the handle is created)
int launch_deformation_tiled(const StepParams &p, cudaStream_t s) {
  if (p.tiled == 3) {
    if (p.damage)
      k_deformation_tiled<true, 3><<<tiled_grid<3>(p), kBondThreads, 0, s>>>(p);
    else
      k_deformation_tiled<false, 3><<<tiled_grid<3>(p), kBondThreads, 0, s>>>(p);
  } else {
    if (p.damage)
      k_deformation_tiled<true, 2><<<tiled_grid<2>(p), kBondThreads, 0, s>>>(p);
    else
      k_deformation_tiled<false, 2><<<tiled_grid<2>(p), kBondThreads, 0, s>>>(p);
  }
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int launch_force_tiled(const StepParams &p, cudaStream_t s) {
  if (p.tiled == 3)
    k_force_tiled<3><<<tiled_grid<3>(p), kBondThreads, 0, s>>>(p);
  else
    k_force_tiled<2><<<tiled_grid<2>(p), kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
