// GPU cell-list neighbour search emitting the reference's sorted neighbour lists as CSR,
// and the sliced-ELL copy the bond kernels stream.
//
// Same result as buildNeighborList (src/pd/PdCorrespondenceSkeleton.cpp:95-129), element
// for element: tolerance 64 eps max(delta, max|x|) (:30-39), cells of width delta + 2 tol,
// the 27 surrounding cells searched, a candidate kept when sqrt(dx^2+dy^2+dz^2) <= delta+tol
// with the reference's operation order and IEEE rounding (no FMA contraction), each row in
// ascending index order. Because correctly rounded sqrt is monotone, the test
// RN(sqrt(s)) <= r is replaced by the equivalent s <= s*, s* the largest double whose
// rounded root does not exceed r (found once on the host).
//
// Device passes: |x| max reduction; cell coordinates and their bounding box; counting sort
// of points into a dense cell grid; a warp per point counts its matches; an exclusive scan
// gives row_ptr; a warp per point gathers its matches with ballot compaction into shared
// memory and bitonic-sorts the row before writing it.
#include "vpd_internal.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <vector>

namespace vpd {

// ------------------------------------------------------------------ exclusive scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

int64_t scan_tmp_elems(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

// Exclusive scan across a block of kScanThreads threads; *total gets the block sum.
__device__ int64_t block_exclusive_scan(int64_t v, int64_t *total) {
  __shared__ int64_t warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o)
      x += y;
  }
  if (lane == 31)
    warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int64_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o)
        w += y;
    }
    if (lane < kScanThreads / 32)
      warp_sums[lane] = w;
  }
  __syncthreads();
  const int64_t excl = x - v + (wid > 0 ? warp_sums[wid - 1] : 0);
  *total = warp_sums[kScanThreads / 32 - 1];
  __syncthreads();
  return excl;
}

__global__ void k_scan_reduce(const int32_t *in, int64_t n, int64_t *sums) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n)
      s += in[base + k];
  int64_t total;
  block_exclusive_scan(s, &total);
  if (threadIdx.x == 0)
    sums[blockIdx.x] = total;
}

// Single block: exclusive scan of the per-tile sums in place; sums[nb] = grand total.
__global__ void k_scan_top(int64_t *sums, int64_t nb) {
  int64_t carry = 0;
  for (int64_t base = 0; base < nb; base += kScanTile) {
    int64_t v[kScanItems];
    int64_t local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int64_t idx = base + (int64_t)threadIdx.x * kScanItems + k;
      v[k] = idx < nb ? sums[idx] : 0;
      local += v[k];
    }
    int64_t total;
    int64_t run = block_exclusive_scan(local, &total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int64_t idx = base + (int64_t)threadIdx.x * kScanItems + k;
      if (idx < nb)
        sums[idx] = run;
      run += v[k];
    }
    carry += total;
  }
  if (threadIdx.x == 0)
    sums[nb] = carry;
}

__global__ void k_scan_apply(const int32_t *in, int64_t n, const int64_t *sums, int64_t nb,
                             int64_t *out) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    local += v[k];
  }
  int64_t total;
  int64_t run = block_exclusive_scan(local, &total) + sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n)
      out[base + k] = run;
    run += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0)
    out[n] = sums[nb];
}

int scan_exclusive_i32(const int32_t *in, int64_t n, int64_t *out, int64_t *tmp,
                       cudaStream_t s) {
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    VPD_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    return VPD_OK;
  }
  k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, tmp);
  k_scan_top<<<1, kScanThreads, 0, s>>>(tmp, nb);
  k_scan_apply<<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, tmp, nb, out);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

// ------------------------------------------------------------------ neighbour kernels
// reduce words: [0] max |x| bits, [1] non-finite flag, [2..4] min cell, [5..7] max cell,
// [8] max row length.
constexpr int kReduceWords = 9;

__global__ void k_abs_max(const double4 *xv, int64_t n, unsigned long long *red) {
  unsigned long long m = 0;
  unsigned int bad = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = xv[i];
    const double c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (!isfinite(c[d]))
        bad = 1;
      const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(c[d]));
      m = b > m ? b : m;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
    m = y > m ? y : m;
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&red[0], m);
    if (bad)
      atomicOr(&red[1], 1ull);
  }
}

__device__ __forceinline__ long long cell_coord(double x, double cw) {
  return (long long)floor(__ddiv_rn(x, cw));
}

__global__ void k_cell_coords(const double4 *xv, int64_t n, double cw, long long *cc,
                              long long *red) {
  long long lo[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, hi[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = xv[i];
    const long long c[3] = {cell_coord(p.x, cw), cell_coord(p.y, cw), cell_coord(p.z, cw)};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cc[3 * i + d] = c[d];
      lo[d] = c[d] < lo[d] ? c[d] : lo[d];
      hi[d] = c[d] > hi[d] ? c[d] : hi[d];
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const long long a = __shfl_xor_sync(0xffffffffu, lo[d], o);
      const long long b = __shfl_xor_sync(0xffffffffu, hi[d], o);
      lo[d] = a < lo[d] ? a : lo[d];
      hi[d] = b > hi[d] ? b : hi[d];
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&red[2 + d], lo[d]);
      atomicMax(&red[5 + d], hi[d]);
    }
  }
}

struct GridDev {
  long long lo0, lo1, lo2, d0, d1, d2;
};

__global__ void k_cell_assign(const long long *cc, int64_t n, GridDev g, int32_t *cell_of,
                              int32_t *count) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const long long c =
      ((cc[3 * i] - g.lo0) * g.d1 + (cc[3 * i + 1] - g.lo1)) * g.d2 + (cc[3 * i + 2] - g.lo2);
  cell_of[i] = (int32_t)c;
  atomicAdd(&count[c], 1);
}

__global__ void k_cell_scatter(const int32_t *cell_of, int64_t n, const int64_t *cell_start,
                               int32_t *cursor, int32_t *sorted) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int32_t c = cell_of[i];
  sorted[cell_start[c] + atomicAdd(&cursor[c], 1)] = (int32_t)i;
}

// |xj - xi|^2 in the reference's order ((a0 a0 + a1 a1) + a2 a2), every operation rounded.
__device__ __forceinline__ bool within(const double4 &pj, const double4 &pi, double dist2_max) {
  const double a0 = __dsub_rn(pj.x, pi.x), a1 = __dsub_rn(pj.y, pi.y), a2 = __dsub_rn(pj.z, pi.z);
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(a0, a0), __dmul_rn(a1, a1)), __dmul_rn(a2, a2));
  return s <= dist2_max;
}

constexpr int kNbWarps = 8;

// One warp per point: number of neighbours.
__global__ void k_nb_count(const double4 *xv, int64_t n, const long long *cc, GridDev g,
                           const int64_t *cell_start, const int32_t *sorted, double dist2_max,
                           int32_t *len, unsigned long long *red) {
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * kNbWarps + (threadIdx.x >> 5);
  if (i >= n)
    return;
  const double4 pi = xv[i];
  const long long c0 = cc[3 * i] - g.lo0, c1 = cc[3 * i + 1] - g.lo1, c2 = cc[3 * i + 2] - g.lo2;
  int cnt = 0;
  for (int dx = -1; dx <= 1; ++dx) {
    const long long x0 = c0 + dx;
    if (x0 < 0 || x0 >= g.d0)
      continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const long long x1 = c1 + dy;
      if (x1 < 0 || x1 >= g.d1)
        continue;
      for (int dz = -1; dz <= 1; ++dz) {
        const long long x2 = c2 + dz;
        if (x2 < 0 || x2 >= g.d2)
          continue;
        const long long cell = (x0 * g.d1 + x1) * g.d2 + x2;
        const int64_t end = cell_start[cell + 1];
        for (int64_t p = cell_start[cell] + lane; p < end; p += 32) {
          const int32_t j = sorted[p];
          if (j != i && within(xv[j], pi, dist2_max))
            ++cnt;
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) {
    len[i] = cnt;
    atomicMax(&red[8], (unsigned long long)cnt);
  }
}

// One warp per point: gather matches into shared memory, bitonic sort, write the row.
__global__ void k_nb_fill(const double4 *xv, int64_t n, const long long *cc, GridDev g,
                          const int64_t *cell_start, const int32_t *sorted, double dist2_max,
                          const int64_t *row_ptr, int32_t *col, int cap,
                          unsigned long long *red) {
  extern __shared__ int32_t nb_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (i >= n)
    return;
  int32_t *buf = nb_smem + (size_t)warp * cap;
  const double4 pi = xv[i];
  const long long c0 = cc[3 * i] - g.lo0, c1 = cc[3 * i + 1] - g.lo1, c2 = cc[3 * i + 2] - g.lo2;
  const unsigned lt = (1u << lane) - 1u;
  int cnt = 0;
  for (int dx = -1; dx <= 1; ++dx) {
    const long long x0 = c0 + dx;
    if (x0 < 0 || x0 >= g.d0)
      continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const long long x1 = c1 + dy;
      if (x1 < 0 || x1 >= g.d1)
        continue;
      for (int dz = -1; dz <= 1; ++dz) {
        const long long x2 = c2 + dz;
        if (x2 < 0 || x2 >= g.d2)
          continue;
        const long long cell = (x0 * g.d1 + x1) * g.d2 + x2;
        const int64_t start = cell_start[cell], end = cell_start[cell + 1];
        for (int64_t base = start; base < end; base += 32) {
          const int64_t p = base + lane;
          bool keep = false;
          int32_t j = 0;
          if (p < end) {
            j = sorted[p];
            keep = j != i && within(xv[j], pi, dist2_max);
          }
          const unsigned mask = __ballot_sync(0xffffffffu, keep);
          const int slot = cnt + __popc(mask & lt);
          if (keep && slot < cap)
            buf[slot] = j;
          cnt += __popc(mask);
        }
      }
    }
  }
  if (cnt > cap) {  // cannot happen when cap >= the count pass's maximum; reported, not written
    if (lane == 0)
      atomicOr(&red[1], 2ull);
    return;
  }
  int width = 32;
  while (width < cnt)
    width <<= 1;
  for (int t = cnt + lane; t < width; t += 32)
    buf[t] = INT_MAX;
  __syncwarp();
  for (int k = 2; k <= width; k <<= 1)
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int t = lane; t < width; t += 32) {
        const int partner = t ^ jj;
        if (partner > t) {
          const int32_t a = buf[t], b = buf[partner];
          const bool ascending = (t & k) == 0;
          if ((a > b) == ascending) {
            buf[t] = b;
            buf[partner] = a;
          }
        }
      }
      __syncwarp();
    }
  int32_t *row = col + row_ptr[i];
  for (int t = lane; t < cnt; t += 32)
    row[t] = buf[t];
}

// ------------------------------------------------------------------ host orchestration
int neighbor_scratch_alloc(NeighborScratch &scr, int64_t n) {
  VPD_CUDA(cudaMalloc(&scr.cell_coords, sizeof(long long) * 3 * (size_t)std::max<int64_t>(n, 1)));
  VPD_CUDA(cudaMalloc(&scr.cell_of, sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)));
  VPD_CUDA(cudaMalloc(&scr.sorted, sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)));
  VPD_CUDA(cudaMalloc(&scr.len, sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)));
  VPD_CUDA(cudaMalloc(&scr.reduce, sizeof(unsigned long long) * kReduceWords));
  return VPD_OK;
}

int neighbor_scratch_alloc_cells(NeighborScratch &scr, int64_t ncells) {
  const int64_t tmp = std::max(scan_tmp_elems(ncells), scan_tmp_elems(0)) + 8;
  VPD_CUDA(cudaMalloc(&scr.cell_count, sizeof(int32_t) * (size_t)(ncells + 1)));
  VPD_CUDA(cudaMalloc(&scr.cell_start, sizeof(int64_t) * (size_t)(ncells + 1)));
  VPD_CUDA(cudaMalloc(&scr.scan_tmp, sizeof(int64_t) * (size_t)tmp));
  return VPD_OK;
}

void neighbor_scratch_free(NeighborScratch &scr) {
  cudaFree(scr.cell_coords), cudaFree(scr.cell_of), cudaFree(scr.sorted), cudaFree(scr.len);
  cudaFree(scr.reduce), cudaFree(scr.cell_count), cudaFree(scr.cell_start), cudaFree(scr.scan_tmp);
  scr = NeighborScratch{};
}

static unsigned grid_for(int64_t n, int threads) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

int neighbor_count(const double4 *xv, int64_t n, double horizon, int64_t *row_ptr,
                   NeighborGrid &grid, NeighborScratch &scr, cudaStream_t s) {
  if (!(horizon > 0.0))
    return set_error(VPD_ERR_INVALID, "PD horizon must be positive.");
  if (n <= 0 || n > INT32_MAX)
    return set_error(VPD_ERR_INVALID, "neighbour search needs 1 <= n < 2^31 points");
  unsigned long long init[kReduceWords] = {0, 0,
                                           (unsigned long long)LLONG_MAX, (unsigned long long)LLONG_MAX,
                                           (unsigned long long)LLONG_MAX, (unsigned long long)LLONG_MIN,
                                           (unsigned long long)LLONG_MIN, (unsigned long long)LLONG_MIN, 0};
  VPD_CUDA(cudaMemcpyAsync(scr.reduce, init, sizeof init, cudaMemcpyHostToDevice, s));
  k_abs_max<<<grid_for(n, 256), 256, 0, s>>>(xv, n, scr.reduce);
  unsigned long long red[kReduceWords];
  VPD_CUDA(cudaMemcpyAsync(red, scr.reduce, sizeof red, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (red[1])
    return set_error(VPD_ERR_NONFINITE, "Nonfinite PD coordinate.");
  double maxabs;
  memcpy(&maxabs, &red[0], sizeof maxabs);
  const double scale = std::max(horizon, maxabs);
  grid.tolerance = 64.0 * DBL_EPSILON * scale;
  grid.radius = horizon + grid.tolerance;
  grid.cell_width = horizon + 2.0 * grid.tolerance;
  double s2 = grid.radius * grid.radius;
  while (std::sqrt(std::nextafter(s2, INFINITY)) <= grid.radius)
    s2 = std::nextafter(s2, INFINITY);
  while (std::sqrt(s2) > grid.radius)
    s2 = std::nextafter(s2, 0.0);
  grid.dist2_max = s2;

  k_cell_coords<<<grid_for(n, 256), 256, 0, s>>>(xv, n, grid.cell_width, scr.cell_coords,
                                                 (long long *)scr.reduce);
  VPD_CUDA(cudaMemcpyAsync(red, scr.reduce, sizeof red, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  long long lo[3], hi[3];
  memcpy(lo, &red[2], sizeof lo);
  memcpy(hi, &red[5], sizeof hi);
  double cells = 1.0;
  for (int d = 0; d < 3; ++d) {
    grid.lo[d] = lo[d];
    grid.dims[d] = hi[d] - lo[d] + 1;
    cells *= (double)grid.dims[d];
  }
  if (cells > (double)kMaxCells)
    return set_error(VPD_ERR_CAPACITY, "neighbour cell grid exceeds 2^28 cells; the points are "
                                       "too spread out relative to the horizon");
  grid.ncells = grid.dims[0] * grid.dims[1] * grid.dims[2];
  if (!scr.cell_count) {
    int rc = neighbor_scratch_alloc_cells(scr, grid.ncells);
    if (rc)
      return rc;
  }
  const GridDev g{grid.lo[0], grid.lo[1], grid.lo[2], grid.dims[0], grid.dims[1], grid.dims[2]};
  VPD_CUDA(cudaMemsetAsync(scr.cell_count, 0, sizeof(int32_t) * (size_t)(grid.ncells + 1), s));
  const unsigned pb = (unsigned)((n + 255) / 256);
  k_cell_assign<<<pb, 256, 0, s>>>(scr.cell_coords, n, g, scr.cell_of, scr.cell_count);
  int rc = scan_exclusive_i32(scr.cell_count, grid.ncells, scr.cell_start, scr.scan_tmp, s);
  if (rc)
    return rc;
  VPD_CUDA(cudaMemsetAsync(scr.cell_count, 0, sizeof(int32_t) * (size_t)(grid.ncells + 1), s));
  k_cell_scatter<<<pb, 256, 0, s>>>(scr.cell_of, n, scr.cell_start, scr.cell_count, scr.sorted);
  const unsigned wb = (unsigned)((n + kNbWarps - 1) / kNbWarps);
  k_nb_count<<<wb, 32 * kNbWarps, 0, s>>>(xv, n, scr.cell_coords, g, scr.cell_start, scr.sorted,
                                          grid.dist2_max, scr.len, scr.reduce);
  // reuse the cell scan scratch when large enough, else the row scan needs its own
  int64_t *tmp = scr.scan_tmp;
  int64_t *own = nullptr;
  if (scan_tmp_elems(n) > std::max(scan_tmp_elems(grid.ncells), scan_tmp_elems(0)) + 8) {
    VPD_CUDA(cudaMalloc(&own, sizeof(int64_t) * (size_t)scan_tmp_elems(n)));
    tmp = own;
  }
  rc = scan_exclusive_i32(scr.len, n, row_ptr, tmp, s);
  VPD_CUDA(cudaMemcpyAsync(red, scr.reduce, sizeof red, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (own)
    cudaFree(own);
  if (rc)
    return rc;
  grid.max_len = (int)red[8];
  if (grid.max_len > kMaxRow)
    return set_error(VPD_ERR_CAPACITY, "a point has more than 8192 neighbours");
  return VPD_OK;
}

int neighbor_fill(const double4 *xv, int64_t n, const int64_t *row_ptr, int32_t *col,
                  const NeighborGrid &grid, const NeighborScratch &scr, cudaStream_t s) {
  int cap = 32;
  while (cap < grid.max_len)
    cap <<= 1;
  const int warps = std::max(1, std::min(8, (48 * 1024) / (cap * 4)));
  const size_t smem = (size_t)warps * cap * sizeof(int32_t);
  const GridDev g{grid.lo[0], grid.lo[1], grid.lo[2], grid.dims[0], grid.dims[1], grid.dims[2]};
  const unsigned blocks = (unsigned)((n + warps - 1) / warps);
  k_nb_fill<<<blocks, 32 * warps, smem, s>>>(xv, n, scr.cell_coords, g, scr.cell_start,
                                             scr.sorted, grid.dist2_max, row_ptr, col, cap,
                                             scr.reduce);
  VPD_CUDA(cudaGetLastError());
  unsigned long long red[kReduceWords];
  VPD_CUDA(cudaMemcpyAsync(red, scr.reduce, sizeof red, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (red[1] & 2ull)
    return set_error(VPD_ERR_CAPACITY, "neighbour row exceeded its buffer");
  return VPD_OK;
}

// ------------------------------------------------------------------ sliced ELL
__global__ void k_sell_width(const int64_t *row_ptr, int64_t n, int64_t nslices, int32_t *len,
                             int32_t *width32) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nslices * 32)
    return;
  int l = 0;
  if (i < n) {
    l = (int)(row_ptr[i + 1] - row_ptr[i]);
    len[i] = l;
  }
  int m = l;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int y = __shfl_xor_sync(0xffffffffu, m, o);
    m = y > m ? y : m;
  }
  if ((threadIdx.x & 31) == 0)
    width32[i >> 5] = 32 * m;
}

__global__ void k_sell_fill(const int64_t *row_ptr, const int32_t *col, int64_t n,
                            int64_t nslices, const int64_t *slice_off, int32_t *sell) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nslices * 32)
    return;
  const int64_t sl = i >> 5;
  const int lane = (int)(i & 31);
  const int width = (int)((slice_off[sl + 1] - slice_off[sl]) >> 5);
  const int l = i < n ? (int)(row_ptr[i + 1] - row_ptr[i]) : 0;
  const int32_t self = i < n ? (int32_t)i : 0;
  int32_t *out = sell + slice_off[sl] + lane;
  for (int k = 0; k < width; ++k)
    out[32 * k] = k < l ? col[row_ptr[i] + k] : self;
}

int build_sell(const int64_t *row_ptr, const int32_t *col, int64_t n, int32_t **len_out,
               int64_t **slice_off_out, int32_t **sell_out, int64_t *sell_total,
               cudaStream_t s) {
  const int64_t nslices = (n + 31) / 32;
  int32_t *len = nullptr, *width32 = nullptr, *sell = nullptr;
  int64_t *slice_off = nullptr, *tmp = nullptr;
  VPD_CUDA(cudaMalloc(&len, sizeof(int32_t) * (size_t)(nslices * 32)));
  VPD_CUDA(cudaMemsetAsync(len, 0, sizeof(int32_t) * (size_t)(nslices * 32), s));
  VPD_CUDA(cudaMalloc(&width32, sizeof(int32_t) * (size_t)nslices));
  VPD_CUDA(cudaMalloc(&slice_off, sizeof(int64_t) * (size_t)(nslices + 1)));
  VPD_CUDA(cudaMalloc(&tmp, sizeof(int64_t) * (size_t)scan_tmp_elems(nslices)));
  const unsigned blocks = (unsigned)((nslices * 32 + 255) / 256);
  k_sell_width<<<blocks, 256, 0, s>>>(row_ptr, n, nslices, len, width32);
  int rc = scan_exclusive_i32(width32, nslices, slice_off, tmp, s);
  if (rc)
    return rc;
  int64_t total = 0;
  VPD_CUDA(cudaMemcpyAsync(&total, slice_off + nslices, sizeof total, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  VPD_CUDA(cudaMalloc(&sell, sizeof(int32_t) * (size_t)std::max<int64_t>(total, 32)));
  k_sell_fill<<<blocks, 256, 0, s>>>(row_ptr, col, n, nslices, slice_off, sell);
  VPD_CUDA(cudaGetLastError());
  VPD_CUDA(cudaStreamSynchronize(s));
  cudaFree(width32);
  cudaFree(tmp);
  *len_out = len;
  *slice_off_out = slice_off;
  *sell_out = sell;
  *sell_total = total;
  return VPD_OK;
}

}  // namespace vpd
