// vpd_force_density_noalloc: the force-density evaluation for callers that must not
// allocate device memory.
//
// Some hosts cannot call cudaMalloc while they run a time step: a solver that hands all of
// the device memory to its own pool before the run starts, or a step loop that drives other
// streams concurrently and cannot accept the device-wide synchronisation cudaMalloc and
// cudaFree imply. vpd_force_density allocates its force-map scratch (9 doubles per point)
// and a status word on every call; this variant uses a fixed scratch array compiled into the
// library instead, so it allocates nothing. The caller still passes every input and output.
//
// Limits and sharing:
//   * at most kNoAllocMaxPoints = 65,536 points per call; larger calls are rejected with
//     VPD_ERR_CAPACITY before any device work;
//   * the scratch (65,536 x 9 doubles plus a status word, about 4.7 MB) lives in every GPU
//     that loads the library until the process exits;
//   * all calls share the one array and it keeps the last call's contents: the status word
//     is cleared at the start of every call (the force map is fully overwritten), and calls
//     that overlap on the GPU -- on different streams or from different host threads without
//     ordering between them -- race on it;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress)
//     with that device current and caches it. With CUDA's lazy module loading (the default
//     since CUDA 12.2) that lookup is also what loads this file's device code on the device,
//     and loading it reserves the 4.7 MB array in device memory at that moment. So the first
//     call on each device must come before the host hands its device memory to its own pool
//     (or the load fails with cudaErrorMemoryAllocation, returned as VPD_ERR_CUDA) and before
//     any stream capture. Later calls reserve nothing.
#include "vpd_internal.h"

#include <mutex>

namespace vpd {
// The module kernels of vpd_modules.cu: the force map M = J sigma F^-T K^-1 and the bond sum.
__global__ void k_csr_force_map(const double *sigma, const double *F, const double *kinv,
                                int64_t n, double *M, unsigned *status);
__global__ void k_csr_force(const double *pos, const double *vol, int64_t n,
                            const int64_t *row_ptr, const int32_t *col, const double *M,
                            const double *bond_damage, double *force);
}  // namespace vpd

namespace {

constexpr int64_t kNoAllocMaxPoints = 65536;
constexpr int64_t kStatusOffset = kNoAllocMaxPoints * 9;  // status word after the force map

// Force map (9 doubles per point) followed by one status word.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxPoints * 9 + 32];

constexpr int kMaxDevices = 64;
std::mutex g_bind_mutex;
double *g_bound[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device, looked up once per device.
int bound_scratch(double **out) {
  int dev = 0;
  VPD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return vpd::set_error(VPD_ERR_UNSUPPORTED, "device ordinal beyond 64");
  std::lock_guard<std::mutex> lock(g_bind_mutex);
  if (!g_bound[dev]) {
    double *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess)
      return vpd::cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_bound[dev] = ptr;
  }
  *out = g_bound[dev];
  return VPD_OK;
}

}  // namespace

using namespace vpd;

extern "C" int vpd_force_density_noalloc(const double *positions, const double *volumes, int64_t n,
                                         const int64_t *row_ptr, const int32_t *col,
                                         const double *kinv, const double *defgrad,
                                         const double *cauchy_stress, const double *bond_damage,
                                         double *force, void *stream) {
  if (!positions || !volumes || !row_ptr || !col || !kinv || !defgrad || !cauchy_stress || !force)
    return set_error(VPD_ERR_INVALID, "vpd_force_density_noalloc: NULL argument");
  if (n < 1)
    return set_error(VPD_ERR_INVALID, "vpd_force_density_noalloc: needs at least one point");
  if (n > kNoAllocMaxPoints)
    return set_error(VPD_ERR_CAPACITY,
                     "vpd_force_density_noalloc handles at most 65536 points per call; use "
                     "vpd_force_density for larger blocks");
  double *scratch = nullptr;
  int rc = bound_scratch(&scratch);
  if (rc)
    return rc;
  double *M = scratch;
  unsigned *status = reinterpret_cast<unsigned *>(scratch + kStatusOffset);
  cudaStream_t s = (cudaStream_t)stream;
  VPD_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned), s));
  const unsigned blocks = (unsigned)((n + 127) / 128);
  k_csr_force_map<<<blocks, 128, 0, s>>>(cauchy_stress, defgrad, kinv, n, M, status);
  k_csr_force<<<blocks, 128, 0, s>>>(positions, volumes, n, row_ptr, col, M, bond_damage, force);
  VPD_CUDA(cudaGetLastError());
  unsigned st = 0;
  VPD_CUDA(cudaMemcpyAsync(&st, status, sizeof st, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (st & STATUS_SINGULAR_F)
    return set_error(VPD_ERR_SINGULAR, "Invalid deformation gradient determinant.");
  return VPD_OK;
}
