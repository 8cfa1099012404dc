// Lattice-stencil bond layout and the bond kernels that stream it.
//
// Every point of a patch sits on an nx*ny*nz lattice (index (ix*ny + iy)*nz + iz), jittered or
// not, so each bond (i, j) is a lattice offset o = (jx-ix, jy-iy, jz-iz) with index difference
// delta(o) = (ox*ny + oy)*nz + oz. The set of offsets that occur in the sorted CSR (built
// bit-exactly by vpd_neighbors.cu) is the stencil; each point stores one bit per stencil
// slot (32 slots per word, words as structure of arrays). The bond set is exactly the CSR's;
// the kernels visit it slot by slot, all 32 threads of a warp on the same slot, so neighbour
// j = i + delta(slot) of consecutive points are consecutive addresses and no index is loaded.
// A point without a bond in a slot still reads i + delta (clamped to the array) so the warp's
// loads stay one contiguous range, and its contribution is masked to zero.
//
// Stencil slots are grouped by the (x, z) components of the offset: the offsets of one group
// differ only in y, take consecutive slots in ascending y (gaps in y become padding slots whose
// bits are never set), and a group never straddles a 32-bit word, so one word load and a
// shift give a point's bits of one group. The tiled bond kernels (vpd_tiled.cu) walk the
// groups; the slot kernels below walk the slots.
// Bond stretch is symmetric bit for bit ((i,j) and (j,i) see y and -y, xi and -xi), so the
// critical-stretch test runs once per pair, by the point with the lower index ("forward"
// slots, delta > 0), which sets the broken bit of both directed bonds.
#include "vpd_bond.cuh"

#include <algorithm>
#include <vector>

namespace vpd {

__device__ __forceinline__ void lattice_coords(int64_t i, int ny, int nz, int &x, int &y, int &z) {
  z = (int)(i % nz);
  y = (int)((i / nz) % ny);
  x = (int)(i / ((int64_t)ny * nz));
}

// ------------------------------------------------------------------ stencil construction
__global__ void k_offset_extent(const int64_t *row_ptr, const int32_t *col, int64_t n, int ny,
                                int nz, int *ext) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int m[3] = {0, 0, 0};
  if (i < n) {
    int ix, iy, iz;
    lattice_coords(i, ny, nz, ix, iy, iz);
    for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
      int jx, jy, jz;
      lattice_coords(col[q], ny, nz, jx, jy, jz);
      m[0] = max(m[0], abs(jx - ix)), m[1] = max(m[1], abs(jy - iy)), m[2] = max(m[2], abs(jz - iz));
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      m[d] = max(m[d], __shfl_xor_sync(0xffffffffu, m[d], o));
    if ((threadIdx.x & 31) == 0)
      atomicMax(&ext[d], m[d]);
  }
}

struct Extent {
  int rx, ry, rz;
  __host__ __device__ int code(int dx, int dy, int dz) const {
    return ((dx + rx) * (2 * ry + 1) + (dy + ry)) * (2 * rz + 1) + (dz + rz);
  }
  __host__ __device__ int size() const { return (2 * rx + 1) * (2 * ry + 1) * (2 * rz + 1); }
};

__global__ void k_offset_mark(const int64_t *row_ptr, const int32_t *col, int64_t n, int ny,
                              int nz, Extent ex, int *table) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  int ix, iy, iz;
  lattice_coords(i, ny, nz, ix, iy, iz);
  for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
    int jx, jy, jz;
    lattice_coords(col[q], ny, nz, jx, jy, jz);
    table[ex.code(jx - ix, jy - iy, jz - iz)] = 1;
  }
}

// One thread per point: its bond bits. The index difference of each bond must equal the
// slot's delta; a mismatch (points not in lattice order) is reported and the caller falls
// back to the sliced-ELL layout.
__global__ void k_mask_build(const int64_t *row_ptr, const int32_t *col, int64_t n, int ny, int nz,
                             Extent ex, const int *slot_of_code, const int32_t *delta, int nw,
                             uint32_t *mask, int *bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  uint32_t words[kMaxStencilWords];
  for (int w = 0; w < nw; ++w)
    words[w] = 0u;
  int ix, iy, iz;
  lattice_coords(i, ny, nz, ix, iy, iz);
  for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
    const int64_t j = col[q];
    int jx, jy, jz;
    lattice_coords(j, ny, nz, jx, jy, jz);
    const int slot = slot_of_code[ex.code(jx - ix, jy - iy, jz - iz)];
    if (slot < 0 || (int64_t)delta[slot] != j - i) {
      atomicOr(bad, 1);
      continue;
    }
    words[slot >> 5] |= 1u << (slot & 31);
  }
  for (int w = 0; w < nw; ++w)
    mask[(int64_t)w * n + i] = words[w];
}

int build_stencil(const int64_t *row_ptr, const int32_t *col, int64_t n, int ny, int nz,
                  double spacing, StencilLayout &st, cudaStream_t s) {
  st = StencilLayout{};
  int *dext = nullptr;
  VPD_CUDA(cudaMalloc(&dext, 4 * sizeof(int)));
  VPD_CUDA(cudaMemsetAsync(dext, 0, 4 * sizeof(int), s));
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_offset_extent<<<blocks, 256, 0, s>>>(row_ptr, col, n, ny, nz, dext);
  int ext[4];
  VPD_CUDA(cudaMemcpyAsync(ext, dext, sizeof ext, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  const Extent ex{ext[0], ext[1], ext[2]};
  // j - i == delta(offset) holds for every bond by construction; two slots may share a
  // delta on thin lattices, which is harmless because a point sets only its own offsets
  if (ex.size() > (1 << 16)) {
    cudaFree(dext);
    return VPD_OK;
  }
  int *table = nullptr, *slot_of = nullptr;
  VPD_CUDA(cudaMalloc(&table, sizeof(int) * ex.size()));
  VPD_CUDA(cudaMemsetAsync(table, 0, sizeof(int) * ex.size(), s));
  k_offset_mark<<<blocks, 256, 0, s>>>(row_ptr, col, n, ny, nz, ex, table);
  std::vector<int> used(ex.size());
  VPD_CUDA(cudaMemcpyAsync(used.data(), table, sizeof(int) * ex.size(), cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  std::vector<int> slot(ex.size(), -1);
  std::vector<int4> groups;  // (dx, dz, lowest dy, (slots << 16) | first slot)
  int S = 0;                 // slots including padding
  for (int dx = -ex.rx; dx <= ex.rx; ++dx)
    for (int dz = -ex.rz; dz <= ex.rz; ++dz) {
      int lo = ex.ry + 1, hi = -ex.ry - 1;
      for (int dy = -ex.ry; dy <= ex.ry; ++dy)
        if (used[ex.code(dx, dy, dz)])
          lo = std::min(lo, dy), hi = std::max(hi, dy);
      if (lo > hi)
        continue;
      const int count = hi - lo + 1;
      if (count > kMaxGroupSlots) {  // a horizon above ~14 spacings: the generic layout serves it
        cudaFree(dext), cudaFree(table);
        return VPD_OK;
      }
      if ((S & 31) + count > 32)
        S = (S + 31) & ~31;  // start the group in the next word
      for (int dy = lo; dy <= hi; ++dy)
        if (used[ex.code(dx, dy, dz)])
          slot[ex.code(dx, dy, dz)] = S + (dy - lo);
      groups.push_back(make_int4(dx, dz, lo, (count << 16) | S));
      S += count;
    }
  if (S == 0 || S > 32 * kMaxStencilWords) {
    cudaFree(dext), cudaFree(table);
    return VPD_OK;
  }
  const int nw = (S + 31) / 32;
  std::vector<int32_t> delta(32 * nw, 0), reverse(32 * nw, -1);
  std::vector<uint32_t> forward(nw, 0u);
  std::vector<float4> e0(32 * nw, make_float4(0.f, 0.f, 0.f, 0.f));
  for (int dx = -ex.rx; dx <= ex.rx; ++dx)
    for (int dy = -ex.ry; dy <= ex.ry; ++dy)
      for (int dz = -ex.rz; dz <= ex.rz; ++dz) {
        const int sl = slot[ex.code(dx, dy, dz)];
        if (sl < 0)
          continue;
        delta[sl] = (dx * ny + dy) * nz + dz;
        reverse[sl] = slot[ex.code(-dx, -dy, -dz)];  // bonds come in pairs, so it exists
        if (delta[sl] > 0)
          forward[sl >> 5] |= 1u << (sl & 31);
        e0[sl] = make_float4((float)(dx * spacing), (float)(dy * spacing), (float)(dz * spacing), 0.f);
      }
  for (int sl = 0; sl < 32 * nw; ++sl)
    if (reverse[sl] < 0)
      reverse[sl] = sl;  // padding slots
  VPD_CUDA(cudaMalloc(&slot_of, sizeof(int) * ex.size()));
  VPD_CUDA(cudaMemcpyAsync(slot_of, slot.data(), sizeof(int) * ex.size(), cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMalloc(&st.delta, sizeof(int32_t) * 32 * nw));
  VPD_CUDA(cudaMalloc(&st.reverse, sizeof(int32_t) * 32 * nw));
  VPD_CUDA(cudaMalloc(&st.forward, sizeof(uint32_t) * nw));
  VPD_CUDA(cudaMalloc(&st.mask, sizeof(uint32_t) * nw * n));
  VPD_CUDA(cudaMalloc(&st.broken, sizeof(uint32_t) * nw * n));
  VPD_CUDA(cudaMemcpyAsync(st.delta, delta.data(), sizeof(int32_t) * 32 * nw, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemcpyAsync(st.reverse, reverse.data(), sizeof(int32_t) * 32 * nw, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemcpyAsync(st.forward, forward.data(), sizeof(uint32_t) * nw, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemsetAsync(st.broken, 0, sizeof(uint32_t) * nw * n, s));
  VPD_CUDA(cudaMalloc(&st.e0, sizeof(float4) * 32 * nw));
  VPD_CUDA(cudaMemcpyAsync(st.e0, e0.data(), sizeof(float4) * 32 * nw, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMalloc(&st.groups, sizeof(int4) * groups.size()));
  VPD_CUDA(cudaMemcpyAsync(st.groups, groups.data(), sizeof(int4) * groups.size(), cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemsetAsync(dext, 0, sizeof(int), s));
  k_mask_build<<<blocks, 256, 0, s>>>(row_ptr, col, n, ny, nz, ex, slot_of, st.delta, nw, st.mask, dext);
  int bad = 0;
  VPD_CUDA(cudaMemcpyAsync(&bad, dext, sizeof bad, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  cudaFree(dext), cudaFree(table), cudaFree(slot_of);
  if (bad) {
    free_stencil(st);
    return VPD_OK;
  }
  st.slots = S;
  st.nw = nw;
  st.ngroups = (int)groups.size();
  // a two-point tile's window reaches y in [-ry, ny + ry], x and z within the extent
  st.halo = (int64_t)ex.rx * ny * nz + (int64_t)(ex.ry + 2) * nz + ex.rz + 1;
  st.rx = ex.rx, st.ry = ex.ry, st.rz = ex.rz;
  return VPD_OK;
}

void free_stencil(StencilLayout &st) {
  cudaFree(st.delta), cudaFree(st.reverse), cudaFree(st.forward), cudaFree(st.mask), cudaFree(st.broken);
  cudaFree(st.e0), cudaFree(st.groups);
  st = StencilLayout{};
}

// ------------------------------------------------------------------ K^-1 and s = sum V xi
__global__ void __launch_bounds__(kBondThreads) k_shape_stencil(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const double4 xi = p.xv[i];
  double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, s[3] = {0, 0, 0};
  for (int w = 0; w < p.st.nw; ++w) {
    const uint32_t m = p.st.mask[(int64_t)w * n + i];
    for (int b = 0; b < 32; ++b)
      if ((m >> b) & 1u) {
        const double4 xj = p.xv[i + p.st.delta[32 * w + b]];
        const double e[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          s[a] += xj.w * e[a];
#pragma unroll
          for (int c = 0; c < 3; ++c)
            K[3 * a + c] += xj.w * e[a] * e[c];
        }
      }
  }
  p.vxi[i] = make_double4(s[0], s[1], s[2], 0.0);
  double Kinv[9];
  if (!m_inv(K, Kinv)) {
    atomicOr(p.status, STATUS_SINGULAR_K);
#pragma unroll
    for (int c = 0; c < 9; ++c)
      Kinv[c] = 0.0;
  }
  double *kinv = const_cast<double *>(p.kinv);
#pragma unroll
  for (int c = 0; c < 9; ++c)
    kinv[c * n + i] = Kinv[c];
}

// ------------------------------------------------------------------ bond kernels
// F = I + [sum_j V_j (u_j - u_i) (x) xi] K^-1 over all bonds; with damage, the critical-stretch
// test on each intact forward bond, breaking both directed bonds of a pair.
template <bool DAMAGE>
__global__ void __launch_bounds__(kBondThreads, DAMAGE ? 2 : 3) k_deformation_stencil(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int64_t ii = valid ? i : n - 1;
  const int64_t step = *p.step;
  const double4 *U = (step & 1) ? p.u1 : p.u0;
  const double4 xi = ldg256(p.xv + ii), ui = ldg256(U + ii);
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double lo = 1.0 - 1.0e-9, hi = 1.0 + 1.0e-9;
  for (int w = 0; w < p.st.nw; ++w) {
    const uint32_t m = valid ? __ldg(p.st.mask + (int64_t)w * n + i) : 0u;
    if (__all_sync(0xffffffffu, m == 0u))
      continue;
    const int32_t *dl = p.st.delta + 32 * w;
    uint32_t live = 0u, fresh = 0u;
    if (DAMAGE)
      live = m & __ldg(p.st.forward + w) & ~p.st.broken[(int64_t)w * n + ii];
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
      // every lane reads i + delta (clamped), so the warp's loads stay one contiguous range;
      // lanes without this bond are masked by a zero weight
      const int64_t j = clamp_index(ii + __ldg(dl + b), n);
      const double4 xj = ldg256(p.xv + j), uj = ldg256(U + j);
      const double v = ((m >> b) & 1u) ? xj.w : 0.0;
      const double e0 = xj.x - xi.x, e1 = xj.y - xi.y, e2 = xj.z - xi.z;
      const double d0 = uj.x - ui.x, d1 = uj.y - ui.y, d2 = uj.z - ui.z;
      bond_deform64(G, v, d0, d1, d2, e0, e1, e2);
      if (DAMAGE && ((live >> b) & 1u)) {
        const double y0 = e0 + d0, y1 = e1 + d1, y2 = e2 + d2;
        const double yy = y0 * y0 + y1 * y1 + y2 * y2;
        const double xx = e0 * e0 + e1 * e1 + e2 * e2;
        const double t = p.tension2 * xx;
        bool broke = false;
        if (yy > t * hi)
          broke = true;
        else if (yy >= t * lo)
          broke = exact_break(p.xv, U, ii, j, p.dmg_initiation, p.dmg_failure, p.use_compression);
        else if (p.use_compression) {
          const double c = p.compression2 * xx;
          if (yy < c * lo)
            broke = true;
          else if (yy <= c * hi)
            broke = exact_break(p.xv, U, ii, j, p.dmg_initiation, p.dmg_failure, 1);
        }
        if (broke)
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
  double K[9], F[9];
#pragma unroll
  for (int c = 0; c < 9; ++c)
    K[c] = p.kinv[c * n + i];
  deformation_from_g(G, K, F);
#pragma unroll
  for (int c = 0; c < 9; ++c)
    p.F[c * n + i] = F[c];
}

// Bond sum of the force density over intact bonds,
//   f_i = sum_j V_j M_j xi + M_i s_i,   s_i = sum_j V_j xi = vxi_i - sum_{broken j} V_j xi,
// so a bond reads only the three force-map records of j (its coordinates ride in their fourth
// lane); broken bonds, rare, are taken out of the precomputed s_i one by one.
// Writes f into p.force; the integrator runs in k_integrate (vpd_step.cu).
__global__ void __launch_bounds__(kBondThreads, 3) k_force_stencil(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const int64_t ii = valid ? i : n - 1;
  const double4 xi = ldg256(p.xv + ii);
  const double4 *P0 = p.fmap, *P1 = p.fmap + n, *P2 = p.fmap + 2 * n;
  double f0 = 0, f1 = 0, f2 = 0, c0 = 0, c1 = 0, c2 = 0;
  for (int w = 0; w < p.st.nw; ++w) {
    uint32_t m = valid ? __ldg(p.st.mask + (int64_t)w * n + i) : 0u;
    const int32_t *dl = p.st.delta + 32 * w;
    if (p.damage) {
      const uint32_t bk = m & p.st.broken[(int64_t)w * n + ii];
      for (uint32_t f = bk; f; f &= f - 1) {  // broken bonds leave s_i
        const double4 xj = p.xv[i + dl[__ffs(f) - 1]];
        c0 += xj.w * (xj.x - xi.x), c1 += xj.w * (xj.y - xi.y), c2 += xj.w * (xj.z - xi.z);
      }
      m &= ~bk;
    }
    if (__all_sync(0xffffffffu, m == 0u))
      continue;
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
      const bool bond = (m >> b) & 1u;
      const int64_t j = clamp_index(ii + __ldg(dl + b), n);  // contiguous across the warp
      const double4 a = ldg256(P0 + j), c = ldg256(P1 + j), d = ldg256(P2 + j);
      const double e0 = bond ? a.w - xi.x : 0.0, e1 = bond ? c.w - xi.y : 0.0,
                   e2 = bond ? d.w - xi.z : 0.0;
      f0 = __dadd_rn(f0, dot3_rn(a.x, a.y, a.z, e0, e1, e2));
      f1 = __dadd_rn(f1, dot3_rn(c.x, c.y, c.z, e0, e1, e2));
      f2 = __dadd_rn(f2, dot3_rn(d.x, d.y, d.z, e0, e1, e2));
    }
  }
  if (!valid)
    return;
  const double4 a = P0[i], c = P1[i], d = P2[i], s = p.vxi[i];
  const double s0 = s.x - c0, s1 = s.y - c1, s2 = s.z - c2;
  const double rv = 1.0 / xi.w;  // M_i = (V_i M_i) / V_i
  f0 = __dadd_rn(f0, __dmul_rn(dot3_rn(a.x, a.y, a.z, s0, s1, s2), rv));
  f1 = __dadd_rn(f1, __dmul_rn(dot3_rn(c.x, c.y, c.z, s0, s1, s2), rv));
  f2 = __dadd_rn(f2, __dmul_rn(dot3_rn(d.x, d.y, d.z, s0, s1, s2), rv));
  p.force[i] = make_double4(f0, f1, f2, 0.0);
}

__global__ void k_damage_index_stencil(StepParams p, double *out) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double damaged = 0.0, total = 0.0;
  for (int w = 0; w < p.st.nw; ++w) {
    const uint32_t m = p.st.mask[(int64_t)w * n + i], bk = p.st.broken[(int64_t)w * n + i];
    for (int b = 0; b < 32; ++b)
      if ((m >> b) & 1u) {
        const double v = p.xv[i + p.st.delta[32 * w + b]].w;
        total += v;
        if ((bk >> b) & 1u)
          damaged += v;
      }
  }
  out[i] = total > 0.0 ? damaged / total : 0.0;
}

int launch_shape_stencil(const StepParams &p, cudaStream_t s) {
  k_shape_stencil<<<(unsigned)((p.n + kBondThreads - 1) / kBondThreads), kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}
int launch_deformation_stencil(const StepParams &p, cudaStream_t s) {
  const unsigned blocks = (unsigned)((p.n + kBondThreads - 1) / kBondThreads);
  if (p.damage)
    k_deformation_stencil<true><<<blocks, kBondThreads, 0, s>>>(p);
  else
    k_deformation_stencil<false><<<blocks, kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}
int launch_force_stencil(const StepParams &p, cudaStream_t s) {
  k_force_stencil<<<(unsigned)((p.n + kBondThreads - 1) / kBondThreads), kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}
int launch_damage_index_stencil(const StepParams &p, double *out, cudaStream_t s) {
  k_damage_index_stencil<<<(unsigned)((p.n + 255) / 256), 256, 0, s>>>(p, out);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
