// Material update through a host VUMAT plugin: the reference's VUMAT-PD bridge
// (src/material/VumatPdCorrespondenceMaterial.cpp:72-176 driving
// src/material/VumatMaterialAdapter.cpp:238-362) with everything but the plugin call on the GPU.
//
//   k_vumat_pack    F (or I + G K^-1), the corotational update and every point's plugin
//                   arguments, packed into 256-row column-major blocks in the adapter's
//                   legacy_vumat_pd order; the kinematic history is committed as k_material does
//   host function   pads the short last block with its last row (the bridge's padding, :138-153),
//                   then calls the plugin once per block, blocks spread over OpenMP threads
//   k_vumat_unpack  stress, state, temperature and energies back into the point arrays, the
//                   rotation to the spatial frame, the force map and the diagnostic partials
//                   (material_store / material_reduce, shared with k_material)
//
// The copies between them are ordered on the handle's stream, so an increment with a plugin is
// still one launch sequence and is captured in the handle's CUDA graph (the host function
// becomes a host node).
#include "vpd_material.cuh"
#include "vpd_step.cuh"

#include <dlfcn.h>
#include <omp.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace vpd {

namespace {

constexpr int kRows = 256;  // rows of one plugin call (VumatPdCorrespondenceMaterial.cpp:90)

// Columns of one packed input block, each kRows doubles, in the order the adapter fills its
// work arrays (VumatMaterialAdapter.cpp:300-344). The state block has max(nstatev, 1) columns
// (stateSize, :262); the energies, the new stretch and the new F follow it.
enum {
  IN_STRAIN_INC = 0,    // 6: unrotated rate of deformation x dt, Voigt with averaged shears
  IN_REL_SPIN = 6,      // 3: relative spin increment, components (2,3), (3,1), (1,2)
  IN_TEMP_OLD = 9,      // 1
  IN_STRETCH_OLD = 10,  // 6: V_n, Voigt
  IN_DEFGRAD_OLD = 16,  // 9: F_n in the order 11 22 33 12 23 31 21 32 13
  IN_STRESS_OLD = 25,   // 6
  IN_STATE_OLD = 31,    // state, then: internal energy, inelastic energy, V_n+1 (6), F_n+1 (9)
};
// Columns of one output block: stress (6), state, temperature, internal and inelastic energy.
enum { OUT_STRESS = 0, OUT_STATE = 6 };

__host__ __device__ constexpr int state_cols(int nsv) { return nsv > 0 ? nsv : 1; }
__host__ __device__ constexpr int in_cols(int nsv) { return IN_STATE_OLD + state_cols(nsv) + 17; }
__host__ __device__ constexpr int out_cols(int nsv) { return OUT_STATE + state_cols(nsv) + 3; }

using VumatCall = void (*)(int *, int *, int *, int *, int *, int *, int *, double *, double *, double *,
                           char *, double *, double *, double *, double *, double *, double *, double *,
                           double *, double *, double *, double *, double *, double *, double *, double *,
                           double *, double *, double *, double *, double *, double *, double *);

// Host side of an attached plugin.
struct HostVumat {
  void *lib = nullptr;
  VumatCall call = nullptr;
  int nsv = 0;
  int threads = 1;  // OpenMP team of the host function
  int64_t n = 0, blocks = 0, in_stride = 0, out_stride = 0;
  double dt = 0.0, density = 0.0, char_length = 0.0;
  char cmname[80];
  std::vector<double> props;
  double *in_host = nullptr, *out_host = nullptr;  // pinned
  double *in_dev = nullptr, *out_dev = nullptr, *temp_dev = nullptr, *stash_dev = nullptr;
};

__device__ __forceinline__ void voigt_of(const double *t, double *v) {  // fullTensorToVumatVoigt
  v[0] = t[0], v[1] = t[4], v[2] = t[8];
  v[3] = 0.5 * (t[5] + t[7]), v[4] = 0.5 * (t[2] + t[6]), v[5] = 0.5 * (t[1] + t[3]);
}

__device__ __forceinline__ void defgrad_of(const double *t, double *v) {  // fullTensorToVumatDefgrad
  v[0] = t[0], v[1] = t[4], v[2] = t[8], v[3] = t[1], v[4] = t[5], v[5] = t[6], v[6] = t[3], v[7] = t[7], v[8] = t[2];
}

// One thread per point: kinematics and the packed plugin arguments. Thread 0 also writes the
// step and total time of the increment ((step - 1) dt, DemoCaseRunner.cpp:343-345) after the
// last block, where the host function reads it.
__global__ void __launch_bounds__(kMaterialThreads) k_vumat_pack(const __grid_constant__ StepParams p, int nsv,
                                                                 int64_t in_stride) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = p.n;
  if (i == 0)
    p.pack_in[(n + kRows - 1) / kRows * in_stride] = (double)(*p.step - 1) * p.dt;
  if (i >= n)
    return;
  double F[9], Fn[9], Vn[9], Rn[9], Eold[6];
  if (p.mixed) {  // F = I + G K^-1 in FP64 from the FP32 bond sum, as material_load forms it
    double G[9], K[9];
#pragma unroll
    for (int c = 0; c < 9; ++c)
      G[c] = (double)p.Gf[c * n + i], K[c] = p.kinv[c * n + i];
    m_mul(G, K, F);
#pragma unroll
    for (int c = 0; c < 9; c += 4)
      F[c] += 1.0;
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c)
      F[c] = p.F[c * n + i];
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    Fn[c] = p.Fn[c * n + i];
    Vn[c] = p.Vn[c * n + i];
    Rn[c] = p.Rn[c * n + i];
  }
#pragma unroll
  for (int c = 0; c < 6; ++c)
    Eold[c] = p.En[c * n + i];
  Corotational co;
  if (!corotational_update(Fn, F, Vn, Rn, p.dt, co)) {
    atomicOr(p.status, STATUS_SINGULAR_KINEMATICS);
#pragma unroll
    for (int c = 0; c < 9; ++c)
      co.dbar[c] = 0.0, co.spin[c] = 0.0, co.r[c] = Rn[c], co.v[c] = Vn[c];
  }
  double E[6];
  green_lagrange6(F, E);

  double *b = p.pack_in + (i / kRows) * in_stride + (i % kRows);
  const auto put = [b](int column, double v) { b[(int64_t)column * kRows] = v; };
  double v6[6], v9[9];
  voigt_of(co.dbar, v6);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    put(IN_STRAIN_INC + c, v6[c] * p.dt);
  put(IN_REL_SPIN + 0, co.spin[5]);
  put(IN_REL_SPIN + 1, co.spin[6]);
  put(IN_REL_SPIN + 2, co.spin[1]);
  put(IN_TEMP_OLD, p.temp[i]);
  voigt_of(Vn, v6);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    put(IN_STRETCH_OLD + c, v6[c]);
  defgrad_of(Fn, v9);
#pragma unroll
  for (int c = 0; c < 9; ++c)
    put(IN_DEFGRAD_OLD + c, v9[c]);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    put(IN_STRESS_OLD + c, p.sig[c * n + i]);
  const int nsc = state_cols(nsv);
  for (int c = 0; c < nsc; ++c)
    put(IN_STATE_OLD + c, c < nsv ? p.state[c * n + i] : 0.0);
  const int tail = IN_STATE_OLD + nsc;
  put(tail, p.eI[i]);
  put(tail + 1, p.eP[i]);
  voigt_of(co.v, v6);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    put(tail + 2 + c, v6[c]);
  defgrad_of(F, v9);
#pragma unroll
  for (int c = 0; c < 9; ++c)
    put(tail + 8 + c, v9[c]);

  // kinematic history of this increment, and what the diagnostics need from it
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    p.Fn[c * n + i] = F[c];
    p.Vn[c * n + i] = co.v[c];
    p.Rn[c * n + i] = co.r[c];
  }
  bool fin = true;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    p.En[c * n + i] = E[c];
    p.mstash[c * n + i] = E[c] - Eold[c];
    fin = fin && isfinite(E[c]);
  }
  const int ax = p.bc.axis;
  p.mstash[6 * n + i] = ax == 0 ? E[0] : (ax == 1 ? E[1] : E[2]);
  p.mstash[7 * n + i] = fin ? 1.0 : 0.0;
}

// One thread per point, k_material's grid: the plugin's results into the point arrays, then
// the same store and reduction as the device update.
__global__ void __launch_bounds__(kMaterialThreads, 4) k_vumat_unpack(const __grid_constant__ StepParams p, int nsv,
                                                                      int64_t out_stride) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double part[PM_COUNT] = {};
  double maxEqps = 0.0;
  if (i < p.n) {
    const int64_t n = p.n;
    const int nsc = state_cols(nsv);
    const double *o = p.pack_out + (i / kRows) * out_stride + (i % kRows);
    const auto get = [o](int column) { return o[(int64_t)column * kRows]; };
    MaterialPoint m;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      m.F[c] = p.Fn[c * n + i];  // committed by k_vumat_pack
      m.R[c] = p.Rn[c * n + i];
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      m.dE[c] = p.mstash[c * n + i];
      m.inc[c] = 0.0;
      m.pt.stress[c] = get(OUT_STRESS + c);
      m.pt.state[c] = c < nsv ? get(OUT_STATE + c) : p.state[c * n + i];  // beyond the plugin's: kept
    }
    m.eAxis = p.mstash[6 * n + i];
    m.eFinite = p.mstash[7 * n + i] != 0.0;
    for (int c = 6; c < nsv; ++c)
      p.state[c * n + i] = get(OUT_STATE + c);
    p.temp[i] = get(OUT_STATE + nsc);
    m.pt.eInternal = get(OUT_STATE + nsc + 1);
    m.pt.eInelastic = get(OUT_STATE + nsc + 2);
    material_store<true>(p, i, m, part, maxEqps);
  }
  material_reduce(p, part, maxEqps, blockIdx.x);
}

// Runs on the stream's host-function thread once the packed blocks have reached host memory.
// No CUDA call is made here.
void CUDART_CB run_plugin(void *arg) {
  HostVumat &h = *static_cast<HostVumat *>(arg);
  const double time = h.in_host[h.blocks * h.in_stride];
  const int64_t last = h.n - (h.blocks - 1) * kRows;  // rows of the last block
  if (last < kRows) {  // pad by duplicating the last row; its results are discarded
    double *b = h.in_host + (h.blocks - 1) * h.in_stride;
    for (int c = 0; c < in_cols(h.nsv); ++c)
      std::fill(b + (int64_t)c * kRows + last, b + (int64_t)(c + 1) * kRows, b[(int64_t)c * kRows + last - 1]);
  }
  const int nsc = state_cols(h.nsv);
#pragma omp parallel num_threads(h.threads)
  {
    // per-thread copies of the arguments every block shares, refilled before each call as the
    // adapter refills its work arrays (VumatMaterialAdapter.cpp:271-290)
    std::vector<double> coord(3 * kRows), charLength(kRows), density(kRows), fieldOld(kRows),
        fieldNew(kRows), props(h.props.size());
#pragma omp for schedule(static)
    for (int64_t blk = 0; blk < h.blocks; ++blk) {
      double *in = h.in_host + blk * h.in_stride, *out = h.out_host + blk * h.out_stride;
      const auto col_in = [in](int c) { return in + (int64_t)c * kRows; };
      const auto col_out = [out](int c) { return out + (int64_t)c * kRows; };
      std::fill(coord.begin(), coord.end(), 0.0);
      std::fill(charLength.begin(), charLength.end(), h.char_length);
      std::fill(density.begin(), density.end(), h.density);
      std::fill(fieldOld.begin(), fieldOld.end(), 0.0);
      std::fill(fieldNew.begin(), fieldNew.end(), 0.0);
      std::copy(h.props.begin(), h.props.end(), props.begin());
      std::fill(col_out(OUT_STRESS), col_out(OUT_STATE + nsc), 0.0);  // stressNew, stateNew
      std::copy(col_in(IN_TEMP_OLD), col_in(IN_TEMP_OLD + 1), col_out(OUT_STATE + nsc));
      std::copy(col_in(IN_STATE_OLD + nsc), col_in(IN_STATE_OLD + nsc + 2), col_out(OUT_STATE + nsc + 1));
      int nblock = kRows, ndir = 3, nshr = 3, nstatev = h.nsv, nfieldv = 0, nprops = (int)h.props.size();
      int lanneal = 0;
      double stepTime = time, totalTime = time, dt = h.dt;
      char cmname[80];
      std::memcpy(cmname, h.cmname, sizeof(cmname));
      const int tail = IN_STATE_OLD + nsc;
      h.call(&nblock, &ndir, &nshr, &nstatev, &nfieldv, &nprops, &lanneal, &stepTime, &totalTime, &dt, cmname,
             coord.data(), charLength.data(), props.data(), density.data(), col_in(IN_STRAIN_INC),
             col_in(IN_REL_SPIN), col_in(IN_TEMP_OLD), col_in(IN_STRETCH_OLD), col_in(IN_DEFGRAD_OLD),
             fieldOld.data(), col_in(IN_STRESS_OLD), col_in(IN_STATE_OLD), col_in(tail), col_in(tail + 1),
             col_out(OUT_STATE + nsc), col_in(tail + 2), col_in(tail + 8), fieldNew.data(), col_out(OUT_STRESS),
             col_out(OUT_STATE), col_out(OUT_STATE + nsc + 1), col_out(OUT_STATE + nsc + 2));
    }
  }
}

}  // namespace

int launch_material_host(const StepParams &p, cudaStream_t s) {
  HostVumat &h = *static_cast<HostVumat *>(p.host_vumat);
  const size_t in_bytes = sizeof(double) * (size_t)(h.blocks * h.in_stride + 1);
  const size_t out_bytes = sizeof(double) * (size_t)(h.blocks * h.out_stride);
  k_vumat_pack<<<(unsigned)material_grid(p.n), kMaterialThreads, 0, s>>>(p, h.nsv, h.in_stride);
  VPD_CUDA(cudaGetLastError());
  VPD_CUDA(cudaMemcpyAsync(h.in_host, p.pack_in, in_bytes, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaLaunchHostFunc(s, run_plugin, &h));
  VPD_CUDA(cudaMemcpyAsync(p.pack_out, h.out_host, out_bytes, cudaMemcpyHostToDevice, s));
  k_vumat_unpack<<<(unsigned)material_grid(p.n), kMaterialThreads, 0, s>>>(p, h.nsv, h.out_stride);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

void host_vumat_detach(StepParams &p) {
  HostVumat *h = static_cast<HostVumat *>(p.host_vumat);
  if (!h)
    return;
  cudaFreeHost(h->in_host);
  cudaFreeHost(h->out_host);
  cudaFree(h->in_dev);
  cudaFree(h->out_dev);
  cudaFree(h->temp_dev);
  cudaFree(h->stash_dev);
  if (h->lib)
    dlclose(h->lib);
  delete h;
  p.host_vumat = nullptr;
  p.pack_in = p.pack_out = p.temp = p.mstash = nullptr;
}

int host_vumat_attach(StepParams &p, const char *path, const char *symbol, const char *cmname, const double *props,
                      int nprops, int nstatev, double density, double char_length, double temperature,
                      cudaStream_t s) {
  // VumatMaterialAdapter's constructor checks (VumatMaterialAdapter.cpp:27-75), same messages
  if (nstatev < 0)
    return set_error(VPD_ERR_INVALID, "nstatev must be non-negative.");
  if (nprops < 1 || !props)
    return set_error(VPD_ERR_INVALID, "VUMAT props cannot be empty.");
  if (!path)
    return set_error(VPD_ERR_INVALID, "Failed to load VUMAT plugin: no path");
  auto *h = new HostVumat();
  h->lib = dlopen(path, RTLD_NOW);
  if (!h->lib) {
    const char *why = dlerror();
    delete h;
    return set_error(VPD_ERR_INVALID, std::string("Failed to load VUMAT plugin: ") + (why ? why : path));
  }
  const std::string name = symbol && *symbol ? symbol : "vumat_adapter_call";
  h->call = reinterpret_cast<VumatCall>(dlsym(h->lib, name.c_str()));
  if (!h->call) {
    dlclose(h->lib);
    delete h;
    return set_error(VPD_ERR_INVALID, "Failed to resolve symbol in VUMAT plugin: " + name);
  }
  std::memset(h->cmname, ' ', sizeof(h->cmname));
  if (cmname)
    std::memcpy(h->cmname, cmname, std::min(sizeof(h->cmname), std::strlen(cmname)));
  h->props.assign(props, props + nprops);
  h->nsv = nstatev;
  h->n = p.n;
  h->blocks = (p.n + kRows - 1) / kRows;
  h->in_stride = (int64_t)kRows * in_cols(nstatev);
  h->out_stride = (int64_t)kRows * out_cols(nstatev);
  h->dt = p.dt, h->density = density, h->char_length = char_length;
  // Half the processors unless OMP_NUM_THREADS says otherwise: a team on every core competes
  // with the CUDA driver's threads and the host thread waiting on the stream, and a barrier
  // that waits for a preempted thread cost ~10 ms per increment on a 16-core host (against
  // 0.4 ms with 8 threads, 4000 points).
  const char *env = std::getenv("OMP_NUM_THREADS");
  const int threads = env && *env ? omp_get_max_threads() : std::max(1, omp_get_num_procs() / 2);
  h->threads = (int)std::max<int64_t>(1, std::min<int64_t>(h->blocks, threads));
  p.host_vumat = h;  // from here on host_vumat_detach frees what has been allocated
  const size_t in_count = (size_t)(h->blocks * h->in_stride + 1), out_count = (size_t)(h->blocks * h->out_stride);
  cudaError_t e = cudaMallocHost(&h->in_host, sizeof(double) * in_count);
  if (e == cudaSuccess)
    e = cudaMallocHost(&h->out_host, sizeof(double) * out_count);
  if (e == cudaSuccess)
    e = cudaMalloc(&h->in_dev, sizeof(double) * in_count);
  if (e == cudaSuccess)
    e = cudaMalloc(&h->out_dev, sizeof(double) * out_count);
  if (e == cudaSuccess)
    e = cudaMalloc(&h->temp_dev, sizeof(double) * (size_t)p.n);
  if (e == cudaSuccess)
    e = cudaMalloc(&h->stash_dev, sizeof(double) * 8 * (size_t)p.n);
  if (e == cudaSuccess) {  // temperatures start at the reference temperature (:67)
    std::vector<double> t((size_t)p.n, temperature);
    e = cudaMemcpyAsync(h->temp_dev, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) {
    host_vumat_detach(p);
    return cuda_error(e, "vpd_set_host_vumat");
  }
  p.pack_in = h->in_dev, p.pack_out = h->out_dev, p.temp = h->temp_dev, p.mstash = h->stash_dev;
  return VPD_OK;
}

}  // namespace vpd
