// Mixed-precision bond kernels (VPD_PRECISION_MIXED), lattice-stencil layout only.
//
// The bond sums run in FP32 on FP32 copies of the data they gather:
//   jit[i] = (X_i - lattice_i, V_i) as float4, so a bond vector is
//            xi = (o h) + (jit_j - jit_i) with the slot's lattice offset o h (float, per slot);
//   uf[i]  = the predicted displacement as float4, written by the integrator;
//   fmapf[i], fmapf[n + i], fmapf[2 n + i] = V_i M_i (force map scaled by volume) and
//            (V_i M_i) jit_i, so a bond term V_j M_j xi is V_j M_j (o h - jit_i) + (V_j M_j) jit_j
//            (fmap_record in vpd_bond.cuh).
// Each 32-slot word is summed in plain FP32 and the word sums are added with Kahan
// compensation, so the result carries ~1 FP32 ulp of error (relative ~6e-8) rather than the
// bond count times it. FP64 stays where the update integrates: K^-1, F = I + G K^-1, the
// polar/rotation update, the Johnson-Cook return map and the integrator (k_material,
// k_integrate). The critical-stretch test runs in FP32 with a 1e-5 relative margin and falls
// back to the reference's exact FP64 arithmetic inside the margin, so bond breaking decides
// exactly as the FP64 path would on the same displacements.
#include "vpd_bond.cuh"

namespace vpd {

// G = sum_j V_j (u_j - u_i) (x) xi in FP32 (written as 9 floats, structure of arrays); the
// material kernel forms F = I + G K^-1 in FP64.
template <bool DAMAGE>
__global__ void __launch_bounds__(kBondThreads, 3) k_deformation_mixed(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int64_t ii = valid ? i : n - 1;
  const float4 ji = ldgf4(p.jit + ii), ui = ldgf4(p.uf + ii);
  float Gs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Gc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const float lo = 1.0f - 1.0e-5f, hi = 1.0f + 1.0e-5f;
  for (int w = 0; w < p.st.nw; ++w) {
    const uint32_t m = valid ? __ldg(p.st.mask + (int64_t)w * n + i) : 0u;
    if (__all_sync(0xffffffffu, m == 0u))
      continue;
    const int32_t *dl = p.st.delta + 32 * w;
    const float4 *ol = p.st.e0 + 32 * w;
    uint32_t live = 0u, fresh = 0u, near = 0u;
    if (DAMAGE)
      live = m & __ldg(p.st.forward + w) & ~p.st.broken[(int64_t)w * n + ii];
    float G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
      const int64_t j = clamp_index(ii + __ldg(dl + b), n);  // contiguous across the warp
      const float4 o = __ldg(ol + b);
      const float4 jj = ldgf4(p.jit + j), uj = ldgf4(p.uf + j);
      const float e0 = o.x + (jj.x - ji.x), e1 = o.y + (jj.y - ji.y), e2 = o.z + (jj.z - ji.z);
      const float d0 = uj.x - ui.x, d1 = uj.y - ui.y, d2 = uj.z - ui.z;
      const float v = ((m >> b) & 1u) ? jj.w : 0.0f;  // lanes without this bond add nothing
      const float w0 = v * d0, w1 = v * d1, w2 = v * d2;
      G[0] += w0 * e0, G[1] += w0 * e1, G[2] += w0 * e2;
      G[3] += w1 * e0, G[4] += w1 * e1, G[5] += w1 * e2;
      G[6] += w2 * e0, G[7] += w2 * e1, G[8] += w2 * e2;
      if (DAMAGE && ((live >> b) & 1u)) {
        const float y0 = e0 + d0, y1 = e1 + d1, y2 = e2 + d2;
        const float yy = y0 * y0 + y1 * y1 + y2 * y2;
        const float xx = e0 * e0 + e1 * e1 + e2 * e2;
        const float t = p.tension2f * xx;
        if (yy > t * hi)
          fresh |= 1u << b;
        else if (yy >= t * lo)
          near |= 1u << b;
        else if (p.use_compression) {
          const float c = p.compression2f * xx;
          if (yy < c * lo)
            fresh |= 1u << b;
          else if (yy <= c * hi)
            near |= 1u << b;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 9; ++c)
      kahan_add(Gs[c], Gc[c], G[c]);
    if (DAMAGE && near) {
      const int64_t step = *p.step;
      const double4 *U = (step & 1) ? p.u1 : p.u0;
      for (uint32_t f = near; f; f &= f - 1) {
        const int b = __ffs(f) - 1;
        if (exact_break(p.xv, U, i, i + dl[b], p.dmg_initiation, p.dmg_failure,
                              p.use_compression))
          fresh |= 1u << b;
      }
    }
    if (DAMAGE && fresh) {
      atomicOr(p.st.broken + (int64_t)w * n + i, fresh);
      for (uint32_t f = fresh; f; f &= f - 1) {
        const int b = __ffs(f) - 1;
        const int r = p.st.reverse[32 * w + b];
        atomicOr(p.st.broken + (int64_t)(r >> 5) * n + (i + dl[b]), 1u << (r & 31));
      }
    }
  }
  if (!valid)
    return;
#pragma unroll
  for (int c = 0; c < 9; ++c)
    p.Gf[c * n + i] = Gs[c];
}

// f = sum (V_j M_j) xi over intact bonds + M_i s_i with s_i = vxi_i - sum_{broken j} V_j xi.
// A bond reads the three FP32 force-map records of j (VM_j and VM_j jit_j); the bond sum is
// FP32 with Kahan-folded words, s_i and the M_i term are FP64.
__global__ void __launch_bounds__(kBondThreads, 3) k_force_mixed(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int64_t ii = valid ? i : n - 1;
  const float4 ji = ldgf4(p.jit + ii);
  const float4 *P0 = p.fmapf, *P1 = p.fmapf + n, *P2 = p.fmapf + 2 * n;
  float fs[3] = {0, 0, 0}, fc[3] = {0, 0, 0};
  double c0 = 0, c1 = 0, c2 = 0;
  for (int w = 0; w < p.st.nw; ++w) {
    uint32_t m = valid ? __ldg(p.st.mask + (int64_t)w * n + i) : 0u;
    const int32_t *dl = p.st.delta + 32 * w;
    const float4 *ol = p.st.e0 + 32 * w;
    if (p.damage) {
      const uint32_t bk = m & p.st.broken[(int64_t)w * n + ii];
      for (uint32_t f = bk; f; f &= f - 1) {  // broken bonds leave s_i
        const int b = __ffs(f) - 1;
        const float4 jj = p.jit[i + dl[b]], o = ol[b];
        c0 += (double)(jj.w * (o.x + (jj.x - ji.x)));
        c1 += (double)(jj.w * (o.y + (jj.y - ji.y)));
        c2 += (double)(jj.w * (o.z + (jj.z - ji.z)));
      }
      m &= ~bk;
    }
    if (__all_sync(0xffffffffu, m == 0u))
      continue;
    float2 f01 = make_float2(0.0f, 0.0f);
    float f2 = 0.0f;
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
      const bool bond = (m >> b) & 1u;
      const int64_t j = clamp_index(ii + __ldg(dl + b), n);  // contiguous across the warp
      const float4 o = __ldg(ol + b);
      const FmapRecord r = fmap_record(ldgf4(P0 + j), ldgf4(P1 + j), ldgf4(P2 + j));
      const float e0 = o.x - ji.x, e1 = o.y - ji.y, e2 = o.z - ji.z;  // xi less the neighbour's jitter
      if (bond) {
        f01 = __fadd2_rn(f01, fmap_rows01(r, bcast2(e0), bcast2(e1), bcast2(e2)));
        f2 += fmap_row2(r, e0, e1, e2);
      }
    }
    kahan_add(fs[0], fc[0], f01.x), kahan_add(fs[1], fc[1], f01.y), kahan_add(fs[2], fc[2], f2);
  }
  if (!valid)
    return;
  float VM[9];
  fmap_rows(P0[i], P1[i], P2[i], VM);
  const double4 s = p.vxi[i];
  const double s0 = s.x - c0, s1 = s.y - c1, s2 = s.z - c2;
  const double rv = 1.0 / (double)ji.w;
  const double f0 = (double)fs[0] + (VM[0] * s0 + VM[1] * s1 + VM[2] * s2) * rv;
  const double f1 = (double)fs[1] + (VM[3] * s0 + VM[4] * s1 + VM[5] * s2) * rv;
  const double f2 = (double)fs[2] + (VM[6] * s0 + VM[7] * s1 + VM[8] * s2) * rv;
  p.force[i] = make_double4(f0, f1, f2, 0.0);
}

// FP32 copies for the mixed kernels: jit = (X - lattice position, V), uf = u[1] (the first
// predicted displacement).
__global__ void k_mixed_setup(StepParams p, int ny, int nz, double h, double yoff, double zoff) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n)
    return;
  const int iz = (int)(i % nz), iy = (int)((i / nz) % ny), ix = (int)(i / ((int64_t)ny * nz));
  const double4 x = p.xv[i];
  p.jit[i] = make_float4((float)(x.x - (double)ix * h), (float)(x.y - ((double)iy * h - yoff)),
                         (float)(x.z - ((double)iz * h - zoff)), (float)x.w);
  const double4 u = p.u1[i];
  p.uf[i] = make_float4((float)u.x, (float)u.y, (float)u.z, 0.0f);
}

int launch_deformation_mixed(const StepParams &p, cudaStream_t s) {
  const unsigned blocks = (unsigned)((p.n + kBondThreads - 1) / kBondThreads);
  if (p.damage)
    k_deformation_mixed<true><<<blocks, kBondThreads, 0, s>>>(p);
  else
    k_deformation_mixed<false><<<blocks, kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int launch_force_mixed(const StepParams &p, cudaStream_t s) {
  k_force_mixed<<<(unsigned)((p.n + kBondThreads - 1) / kBondThreads), kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int launch_mixed_setup(const StepParams &p, int ny, int nz, double h, double yoff, double zoff,
                       cudaStream_t s) {
  k_mixed_setup<<<(unsigned)((p.n + 255) / 256), 256, 0, s>>>(p, ny, nz, h, yoff, zoff);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
