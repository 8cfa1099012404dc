// Internal declarations shared by the libvpd_gpu.so translation units.
#pragma once

#include "../../include/vpd_gpu.h"
#include "vpd_jc.cuh"

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace vpd {

// ---- error reporting (thread-local message behind vpd_last_error) ----
int set_error(int status, const std::string &message);
int cuda_error(cudaError_t e, const char *what);
#define VPD_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return ::vpd::cuda_error(e_, #call);                                                  \
  } while (0)

// ---- device status word bits (ORed by kernels, read by the host) ----
enum : unsigned int {
  STATUS_SINGULAR_K = 1u,
  STATUS_SINGULAR_F = 2u,
  STATUS_SINGULAR_KINEMATICS = 4u,
  STATUS_SURROGATE_WAIT = 8u,  // a tensor-core wait of the surrogate material kernel timed out
  STATUS_STAGED_WAIT = 16u,    // a TMA wait of the staged FP64 force kernel timed out
};

// ---- point flags ----
enum : uint8_t {
  FLAG_SUPPORT = 1,
  FLAG_LOADED = 2,
  FLAG_ANCHOR = 4,
  FLAG_ROTATION_PIN = 8,
  FLAG_LATERAL_NEG = 16,
  FLAG_LATERAL_POS = 32,
};

// ---- neighbour build (vpd_neighbors.cu) ----
// Scratch for one build; every pointer is device memory.
struct NeighborScratch {
  long long *cell_coords = nullptr;  // 3n
  int32_t *cell_of = nullptr;        // n
  int32_t *cell_count = nullptr;     // ncells (+1)
  int64_t *cell_start = nullptr;     // ncells + 1
  int32_t *sorted = nullptr;         // n
  int32_t *len = nullptr;            // n
  int64_t *scan_tmp = nullptr;       // scan block sums
  unsigned long long *reduce = nullptr;  // small reduction words
};

struct NeighborGrid {
  double radius = 0, cell_width = 0, dist2_max = 0, tolerance = 0;
  long long lo[3] = {0, 0, 0};
  long long dims[3] = {0, 0, 0};
  int64_t ncells = 0;
  int max_len = 0;
};

// Maximum neighbours per point the sorted fill supports (shared-memory row buffer).
constexpr int kMaxRow = 8192;
// Upper bound on the dense cell grid.
constexpr int64_t kMaxCells = int64_t(1) << 28;

// Exclusive scan of n values into out[0..n] (out[n] = total). tmp needs
// scan_tmp_elems(n) int64 values.
int64_t scan_tmp_elems(int64_t n);
int scan_exclusive_i32(const int32_t *in, int64_t n, int64_t *out, int64_t *tmp,
                       cudaStream_t s);

// Builds the sorted CSR of n points (x,y,z in .x/.y/.z). Two phases share the grid:
//   neighbor_count: fills grid, scratch.len and row_ptr[0..n];
//   neighbor_fill: writes col using row_ptr.
// The caller provides scratch sized by neighbor_scratch_bytes (cells unknown until the
// count phase: neighbor_count allocates cell arrays itself when alloc is true).
int neighbor_count(const double4 *xv, int64_t n, double horizon, int64_t *row_ptr,
                   NeighborGrid &grid, NeighborScratch &scr, cudaStream_t s);
int neighbor_fill(const double4 *xv, int64_t n, const int64_t *row_ptr, int32_t *col,
                  const NeighborGrid &grid, const NeighborScratch &scr, cudaStream_t s);
int neighbor_scratch_alloc(NeighborScratch &scr, int64_t n);
int neighbor_scratch_alloc_cells(NeighborScratch &scr, int64_t ncells);
void neighbor_scratch_free(NeighborScratch &scr);

// Sliced-ELL (32 rows per slice) copy of a CSR: for point i in slice s = i/32, entry k sits
// at sell[slice_off[s] + 32 k + (i % 32)]; rows shorter than the slice width are padded
// with the point's own index.
int build_sell(const int64_t *row_ptr, const int32_t *col, int64_t n, int32_t **len_out,
               int64_t **slice_off_out, int32_t **sell_out, int64_t *sell_total,
               cudaStream_t s);

}  // namespace vpd
