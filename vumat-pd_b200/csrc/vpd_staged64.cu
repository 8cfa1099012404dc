// TMA-staged FP64 force bond sum of the plain path: k_force_tiled64's arithmetic with the
// neighbours' force-map records read from shared memory instead of through L1.
//
// Selected with VPD_BOND_KERNEL=staged; the default FP64 force kernel is k_force_tiled64<4>,
// which reads the same records through L1: on the 1M-point bar this kernel takes 0.85 ms per
// increment against 0.81 ms for the L1 kernel (measured on a B200; the box of 96-byte records
// with its halo limits the block to two per SM, and the L1 already serves the gathers).
//
// A block owns a tile of one lattice plane x: Ty x Tz points (y, z), each thread P consecutive
// y of one z (the tiling of k_force_tiled64<P>, whose window arithmetic and slot order it
// keeps, so the result is bit-identical to the per-slot kernel k_force_stencil).
// The stencil's groups come plane by plane (ascending x offset dx). For each plane x + dx one
// thread issues a single cp.async.bulk.tensor load of the tile's neighbourhood of that plane:
// a box of (Ty + 2 ry) x (Tz + 2 rz) points of all three force-map rows (a 5-D tensor map over
// fmap: double lane, z, y, x, row; 96 bytes per point), zero-filled where it reaches past the
// lattice, completing on an mbarrier. The block then sums every group of that plane from the
// box and, after a barrier, the next plane's load overwrites it. Planes past either end of
// the bar are skipped. Two blocks per SM keep one block's load in flight while the other sums.
// Planes are loaded in x-offset order (dx ascending) because the groups, and so the slot order
// the sums keep, come that way.
//
// Every wait is bounded: a timed-out wait sets STATUS_STAGED_WAIT, waits once more (bounded)
// for the copy in flight and the block returns; the host reports VPD_ERR_CUDA. A box base that
// is not 16-byte aligned is reported the same way before any copy is issued.
//
// The records are 32 bytes, so a warp reading consecutive records with 16-byte loads would
// hit every bank twice; each thread reads the two halves of its record in an order that
// alternates every four lanes, which makes each load conflict-free.
#include "vpd_bond.cuh"
#include "vpd_umma.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <string>

namespace vpd {

namespace {

constexpr uint32_t kStagedWaitLimit = 1u << 24;  // mbarrier polls before a wait is declared failed

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// One tile of a 5-D tensor map into shared memory, completing on the mbarrier (no multicast).
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5, %6}], [%7];" ::"r"(umma::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(umma::smem_u32(mbar))
      : "memory");
}

// A 32-byte record of the box, its halves read in the lane's order (see the file comment);
// without SWAP in their natural order.
template <bool SWAP>
__device__ __forceinline__ double4 lds_record(const double4 *rec, int swap) {
  if (!SWAP)
    return *rec;
  const double2 *h = reinterpret_cast<const double2 *>(rec);
  const double2 first = h[swap], second = h[swap ^ 1];
  const double2 lo = swap ? second : first, hi = swap ? first : second;
  return make_double4(lo.x, lo.y, hi.x, hi.y);
}

template <int P, bool SWAP>
__device__ __forceinline__ void staged_element(const double4 *r0, const double4 *r1, const double4 *r2, int swap,
                                               int t, int cnt, const double (&px)[P], const double (&py)[P],
                                               const double (&pz)[P], const uint32_t (&bits)[P], double (&f)[P][3]) {
  const double4 a = lds_record<SWAP>(r0, swap), c = lds_record<SWAP>(r1, swap), d = lds_record<SWAP>(r2, swap);
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

// The window of one group from the box: record of window position t at box row yy0 + t.
template <int CNT, int P, bool SWAP>
__device__ __forceinline__ void staged_window(const double4 *box, int plane, int bz, int cnt, int yy0, int zz,
                                              int swap, const double (&px)[P], const double (&py)[P],
                                              const double (&pz)[P], const uint32_t (&bits)[P], double (&f)[P][3]) {
  if constexpr (CNT > 0) {
#pragma unroll
    for (int t = 0; t < CNT + P - 1; ++t) {
      const int k = (yy0 + t) * bz + zz;
      staged_element<P, SWAP>(box + k, box + plane + k, box + 2 * plane + k, swap, t, CNT, px, py, pz, bits, f);
    }
  } else {
    for (int t = 0; t < cnt + P - 1; ++t) {
      const int k = (yy0 + t) * bz + zz;
      staged_element<P, SWAP>(box + k, box + plane + k, box + 2 * plane + k, swap, t, cnt, px, py, pz, bits, f);
    }
  }
}

template <int P, int THREADS, bool SWAP>
__global__ void __launch_bounds__(THREADS, 2) k_force_staged64(const __grid_constant__ StepParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  const double4 *box = reinterpret_cast<const double4 *>(smem);
  const StagedTiles &T = p.staged;
  const int64_t n = p.n;
  const int ny = p.lat_ny, nz = p.lat_nz;
  int b = blockIdx.x;
  const int tzi = b % T.tiles_z;
  b /= T.tiles_z;
  const int tyi = b % T.tiles_y, x = b / T.tiles_y;
  const int ty0 = tyi * T.ty, tz0 = tzi * T.tz;
  const int tid = threadIdx.x;
  // the thread's column: z = tz0 + zl, y = y0 .. y0 + P - 1; threads past the tile's columns
  // take column 0 (their points are invalid), so every box index stays inside the box
  int zl = tid % T.tz, ql = tid / T.tz;
  const bool active = ql < T.qy;
  if (!active)
    zl = 0, ql = 0;
  const int z = tz0 + zl, y0 = ty0 + P * ql;
  int64_t ip[P];
  bool vp[P];
  double px[P], py[P], pz[P], f[P][3];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    vp[q] = active && z < nz && y0 + q < ny;
    ip[q] = vp[q] ? ((int64_t)x * ny + y0 + q) * nz + z : 0;
    const double4 xi = ldg256(p.xv + ip[q]);
    px[q] = xi.x, py[q] = xi.y, pz[q] = xi.z;
    f[q][0] = f[q][1] = f[q][2] = 0.0;
  }
  const int plane = T.by * T.bz;  // records per force-map row in the box
  const int swap = (tid >> 2) & 1;
  // a TMA destination must be 16-byte aligned: refuse to run (and report) otherwise
  if (umma::smem_u32(smem) & 15u) {
    if (tid == 0)
      atomicOr(p.status, STATUS_STAGED_WAIT);
    return;
  }
  if (tid == 0)
    umma::mbar_init(&mbar, 1);
  __syncthreads();
  uint32_t phase = 0;
  bool ok = true, any_broken = false;
  int g = 0;
  while (g < p.st.ngroups) {
    const int dx = __ldg(&p.st.groups[g].x);
    int gend = g + 1;
    while (gend < p.st.ngroups && __ldg(&p.st.groups[gend].x) == dx)
      ++gend;
    if (x + dx < 0 || x + dx >= p.lat_nx) {  // the plane lies past an end of the bar: no bonds
      g = gend;
      continue;
    }
    if (tid == 0) {
      umma::fence_proxy_async();  // the previous plane's reads come before the copy's writes
      mbar_expect_tx(&mbar, T.bytes);
      tma_load_5d(smem, &p.fmap_tmap, 0, tz0 - T.rz, ty0 - T.ry, x + dx, 0, &mbar);
    }
    const bool got = umma::mbar_wait(&mbar, phase, kStagedWaitLimit);
    ok = __syncthreads_and(got) != 0;
    if (!ok) {
      if (tid == 0) {
        atomicOr(p.status, STATUS_STAGED_WAIT);
        umma::mbar_wait(&mbar, phase, kStagedWaitLimit);  // the copy in flight, once more
      }
      return;
    }
    phase ^= 1u;
    for (; g < gend; ++g) {
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
      const int yy0 = (y0 - ty0) + gr.z + T.ry, zz = zl + gr.y + T.rz;
      {
        static_assert(kUnrolledSlots == 12, "the cases below list the unrolled slot counts");
#define VPD_STAGED_CASE(C)                                                                  \
  case C:                                                                                   \
    staged_window<C, P, SWAP>(box, plane, T.bz, cnt, yy0, zz, swap, px, py, pz, bits, f);   \
    break;
        switch (cnt) {
          VPD_STAGED_CASE(1) VPD_STAGED_CASE(2) VPD_STAGED_CASE(3) VPD_STAGED_CASE(4)
          VPD_STAGED_CASE(5) VPD_STAGED_CASE(6) VPD_STAGED_CASE(7) VPD_STAGED_CASE(8)
          VPD_STAGED_CASE(9) VPD_STAGED_CASE(10) VPD_STAGED_CASE(11) VPD_STAGED_CASE(12)
        default:
          staged_window<0, P, SWAP>(box, plane, T.bz, cnt, yy0, zz, swap, px, py, pz, bits, f);
        }
#undef VPD_STAGED_CASE
      }
    }
    __syncthreads();  // every thread is done with the box before the next plane's copy
  }
  const double4 *P0 = p.fmap, *P1 = p.fmap + n, *P2 = p.fmap + 2 * n;
#pragma unroll
  for (int q = 0; q < P; ++q) {
    if (!vp[q])
      continue;
    const int64_t i = ip[q];
    // s_i less the broken bonds' V_j xi, summed in slot order (k_force_tiled64)
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
    if (any_broken)
      for (int w = 0; w < p.st.nw; ++w)
        for (uint32_t bb = p.st.mask[(int64_t)w * n + i] & p.st.broken[(int64_t)w * n + i]; bb; bb &= bb - 1) {
          const double4 xj = p.xv[i + p.st.delta[32 * w + __ffs(bb) - 1]];
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

}  // namespace

// The kernel's variants: two points per thread along y and 256 threads (the default), or four
// and 128 (VPD_STAGED=4x128); the record halves are read in alternating order in both (without
// it the 1M-point bar's force pass took 1.19 against 0.85 ms with two points per thread).
struct StagedVariant {
  int p, threads;
};

static StagedVariant staged_variant() {
  const char *v = getenv("VPD_STAGED");
  if (v && std::string(v) == "4x128")
    return {4, 128};
  return {2, 256};
}

template <int P, int THREADS, bool SWAP> static int set_smem(size_t bytes) {
  VPD_CUDA(cudaFuncSetAttribute(k_force_staged64<P, THREADS, SWAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes));
  return VPD_OK;
}

// Tile shape and tensor map for the staged kernel: tiles span the whole z extent up to 64
// points (else 32) and as many P-point y columns as fit the block's threads; the box adds the
// stencil's reach on each side. Leaves p.staged.bytes 0 (the tiled kernel runs) when the box
// would not fit two blocks per SM or the driver entry point is missing.
int setup_staged_force64(StepParams &p, int rx, int ry, int rz) {
  (void)rx;
  p.staged = StagedTiles{};
  if (!p.fmap || p.st.nw == 0)
    return VPD_OK;
  const StagedVariant V = staged_variant();
  StagedTiles T{};
  T.p = V.p;
  T.tz = p.lat_nz <= 64 ? p.lat_nz : 32;
  const int cols_y = (p.lat_ny + V.p - 1) / V.p;
  T.qy = std::max(1, std::min(V.threads / T.tz, cols_y));
  T.ty = V.p * T.qy;
  T.ry = ry, T.rz = rz;
  T.by = T.ty + 2 * ry, T.bz = T.tz + 2 * rz;
  T.tiles_y = (p.lat_ny + T.ty - 1) / T.ty;
  T.tiles_z = (p.lat_nz + T.tz - 1) / T.tz;
  const size_t bytes = (size_t)3 * T.by * T.bz * sizeof(double4);
  if (T.by > 256 || T.bz > 256 || bytes > kStagedMaxBytes || T.qy * T.tz > V.threads)
    return VPD_OK;
  T.threads = ((T.qy * T.tz + 31) / 32) * 32;
  T.bytes = (uint32_t)bytes;

  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return VPD_OK;
  }
  // fmap[r * n + i] = double4: dims (lane, z, y, x, row), innermost first
  const cuuint64_t dims[5] = {4, (cuuint64_t)p.lat_nz, (cuuint64_t)p.lat_ny, (cuuint64_t)p.lat_nx, 3};
  const cuuint64_t strides[4] = {32, (cuuint64_t)32 * p.lat_nz, (cuuint64_t)32 * p.lat_nz * p.lat_ny,
                                 (cuuint64_t)32 * p.n};
  const cuuint32_t box[5] = {4, (cuuint32_t)T.bz, (cuuint32_t)T.by, 1, 3};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn)(
      &p.fmap_tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, (void *)p.fmap, dims, strides, box, estr,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(VPD_ERR_CUDA, "cuTensorMapEncodeTiled failed for the force map");
  int rc = V.p == 4 ? set_smem<4, 128, true>(bytes) : set_smem<2, 256, true>(bytes);
  if (rc)
    return rc;
  p.staged = T;
  return VPD_OK;
}

int launch_force_staged64(const StepParams &p, cudaStream_t s) {
  const StagedTiles &T = p.staged;
  const unsigned grid = (unsigned)((int64_t)p.lat_nx * T.tiles_y * T.tiles_z);
  if (T.p == 4)
    k_force_staged64<4, 128, true><<<grid, T.threads, T.bytes, s>>>(p);
  else
    k_force_staged64<2, 256, true><<<grid, T.threads, T.bytes, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

}  // namespace vpd
