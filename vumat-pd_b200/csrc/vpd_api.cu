// C ABI of libvpd_gpu.so: the simulation handle (create / step / download / destroy).
//
// vpd_create mirrors runMaterial's set-up (src/host/BoundaryValueCaseRunner.cpp:142-190):
// the lattice of makeParticlePatch (src/host/Geometry.cpp:10-34) generated on the device,
// the sorted neighbour lists, K^-1, the boundary bands, pins and observation weights
// (src/host/ParticleSets.cpp:12-71, src/host/BoundaryConditions.cpp:54-68,96-110,
// include/ObservationWindow.hpp:13-56), the initial material state and the constraints at
// t = 0. vpd_step runs the step loop (:207-306) as device kernels, captured in a CUDA graph.
#include "vpd_math.cuh"
#include "vpd_step.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace vpd {

thread_local std::string g_error;

int set_error(int status, const std::string &message) {
  g_error = message;
  return status;
}
int cuda_error(cudaError_t e, const char *what) {
  return set_error(VPD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Position generator: the lattice of makeParticlePatch plus the seeded jitter, every
// operation rounded as the host formula (no FMA contraction) so hosts reproduce it exactly.
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct LatticeParams {
  int nx, ny, nz;
  double h, yoff, zoff, volume, amp;
  uint64_t seed;
  int jitter;
};

__global__ void k_lattice(LatticeParams L, double4 *xv) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = (int64_t)L.nx * L.ny * L.nz;
  if (p >= n)
    return;
  const int k = (int)(p % L.nz), j = (int)((p / L.nz) % L.ny), i = (int)(p / ((int64_t)L.ny * L.nz));
  double x[3] = {__dmul_rn((double)i, L.h), __dsub_rn(__dmul_rn((double)j, L.h), L.yoff),
                 __dsub_rn(__dmul_rn((double)k, L.h), L.zoff)};
  if (L.jitter) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const uint64_t r =
          splitmix64(L.seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(3 * p + d + 1)));
      const double u = (double)(r >> 11) * 0x1.0p-53;
      x[d] = __dadd_rn(x[d], __dmul_rn(__dadd_rn(2.0 * u, -1.0), L.amp));
    }
  }
  const double v = L.volume * ((i == 0 || i == L.nx - 1) ? 0.5 : 1.0) *
                   ((j == 0 || j == L.ny - 1) ? 0.5 : 1.0) * ((k == 0 || k == L.nz - 1) ? 0.5 : 1.0);
  xv[p] = make_double4(x[0], x[1], x[2], v);
}

__global__ void k_pack_xv(const double *pos, const double *vol, int64_t n, double4 *xv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    xv[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], vol[i]);
}

// Volume-weighted broken-bond fraction (damageIndex, PdSimpleDamage.cpp:23-36).
__global__ void k_damage_index(int64_t n, const double4 *xv, const int32_t *len,
                               const int64_t *slice_off, const int32_t *sell,
                               const uint32_t *words, double *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const int64_t s = i >> 5, off = slice_off[s];
  const int lane = (int)(i & 31);
  double damaged = 0.0, total = 0.0;
  for (int k = 0; k < len[i]; ++k) {
    const double v = xv[sell[off + 32 * k + lane]].w;
    if ((words[(off >> 5) + k] >> lane) & 1u)
      damaged += v;
    total += v;
  }
  out[i] = total > 0.0 ? damaged / total : 0.0;
}

// ------------------------------------------------------------------ host-side sets
struct Sets {
  std::vector<uint8_t> flags;
  std::vector<double> obsw;
  double interior = 0, gauge = 0, lat_gauge = 0, area = 0, n_lat_pos = 0, n_lat_neg = 0;
  int axis = 0, lateral = 1;
};

// selectBoundaryRegion (ParticleSets.cpp:12-50)
static bool select_region(const std::vector<double> &x, int64_t n, int comp, bool selectMin,
                          double width, std::vector<uint8_t> &flags, uint8_t bit) {
  double extreme = selectMin ? std::numeric_limits<double>::infinity()
                             : -std::numeric_limits<double>::infinity();
  for (int64_t i = 0; i < n; ++i)
    extreme = selectMin ? std::min(extreme, x[3 * i + comp]) : std::max(extreme, x[3 * i + comp]);
  const double tol = 1.0e-10 * std::max(1.0, std::abs(extreme));
  bool any = false;
  for (int64_t i = 0; i < n; ++i) {
    const double dist = selectMin ? x[3 * i + comp] - extreme : extreme - x[3 * i + comp];
    if (dist <= width + tol) {
      flags[i] |= bit;
      any = true;
    }
  }
  return any;
}

static int build_sets(const vpd_case &c, const std::vector<double> &x, const std::vector<double> &vol,
                      Sets &s) {
  const int64_t n = (int64_t)vol.size();
  const double h = c.spacing;
  s.axis = c.load_axis;
  s.lateral = s.axis == 0 ? 1 : 0;
  s.flags.assign((size_t)n, 0);
  s.obsw.assign((size_t)n, 0.0);
  const double width = (double)(c.region_layers - 1) * h + 1.0e-9 * h;
  if (!select_region(x, n, s.axis, true, width, s.flags, FLAG_SUPPORT) ||
      !select_region(x, n, s.axis, false, width, s.flags, FLAG_LOADED))
    return set_error(VPD_ERR_INVALID, "Boundary-region selection returned no particles.");
  // anchor: support point closest to the centroid (BoundaryConditions.cpp:58-67)
  double centre[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d)
      centre[d] += x[3 * i + d];
  for (double &v : centre)
    v /= (double)n;
  int64_t anchor = -1;
  double best = std::numeric_limits<double>::infinity();
  for (int64_t i = 0; i < n; ++i)
    if (s.flags[i] & FLAG_SUPPORT) {
      double dist = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double delta = x[3 * i + d] - centre[d];
        dist += delta * delta;
      }
      if (dist < best)
        best = dist, anchor = i;
    }
  if (anchor < 0)
    return set_error(VPD_ERR_INVALID, "Closest-particle selection requires candidates.");
  int64_t pin = anchor;
  double greatestY = -1.0e100;
  for (int64_t i = 0; i < n; ++i)
    if (s.flags[i] & FLAG_SUPPORT) {
      if (std::abs(x[3 * i] - x[3 * anchor]) < 1e-8 && std::abs(x[3 * i + 2] - x[3 * anchor + 2]) < 1e-8 &&
          x[3 * i + 1] > greatestY)
        greatestY = x[3 * i + 1], pin = i;
    }
  s.flags[anchor] |= FLAG_ANCHOR;
  s.flags[pin] |= FLAG_ROTATION_PIN;
  double sl = 0, ss = 0, nl = 0, ns = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (s.flags[i] & FLAG_LOADED) sl += x[3 * i + s.axis], nl += 1;
    if (s.flags[i] & FLAG_SUPPORT) ss += x[3 * i + s.axis], ns += 1;
  }
  s.gauge = std::abs(sl / nl - ss / ns);
  select_region(x, n, s.lateral, true, 1.0e-9 * h, s.flags, FLAG_LATERAL_NEG);
  select_region(x, n, s.lateral, false, 1.0e-9 * h, s.flags, FLAG_LATERAL_POS);
  double sp = 0, sn = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (s.flags[i] & FLAG_LATERAL_POS) sp += x[3 * i + s.lateral], s.n_lat_pos += 1;
    if (s.flags[i] & FLAG_LATERAL_NEG) sn += x[3 * i + s.lateral], s.n_lat_neg += 1;
  }
  s.lat_gauge = std::abs(sp / s.n_lat_pos - sn / s.n_lat_neg);
  // observation window (ObservationWindow.hpp:13-56)
  double lo = x[s.axis], hi = lo;
  for (int64_t i = 0; i < n; ++i)
    lo = std::min(lo, x[3 * i + s.axis]), hi = std::max(hi, x[3 * i + s.axis]);
  const double band = (double)(c.region_layers - 1) * h;
  const double a = std::isnan(c.observation_min) ? lo + band : c.observation_min;
  const double b = std::isnan(c.observation_max) ? hi - band : c.observation_max;
  if (!std::isfinite(a) || !std::isfinite(b) || a < lo || b > hi || a >= b)
    return set_error(VPD_ERR_INVALID,
                     "Observation window must lie within the body and have positive length.");
  const double tol = 1e-8 * h;
  bool foundA = false, foundB = false;
  for (int64_t i = 0; i < n; ++i) {
    const double v = x[3 * i + s.axis];
    const bool atA = std::abs(v - a) < tol, atB = std::abs(v - b) < tol;
    foundA = foundA || atA;
    foundB = foundB || atB;
    if (v < a - tol || v > b + tol)
      continue;
    const bool interiorEnd = (atA && a > lo + tol) || (atB && b < hi - tol);
    s.obsw[i] = vol[i] * (interiorEnd ? 0.5 : 1.0);
    s.interior += s.obsw[i];
  }
  if (!foundA || !foundB)
    return set_error(VPD_ERR_INVALID, "Observation bounds must coincide with reference nodal planes.");
  const int cross = s.axis == 0 ? c.ny : c.nx;
  s.area = (double)((cross - 1) * (c.nz - 1)) * h * h;
  return VPD_OK;
}

}  // namespace vpd

using namespace vpd;

struct vpd_handle {
  vpd_case c{};
  int64_t n = 0, nbonds = 0, sell_total = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  float last_ms = 0.0f;
  int64_t step = 0;  // increments completed
  std::vector<void *> allocations;
  double4 *xv = nullptr, *u0 = nullptr, *u1 = nullptr, *vel = nullptr, *acc = nullptr, *force = nullptr;
  int64_t *row_ptr = nullptr, *slice_off = nullptr, *step_dev = nullptr;
  int32_t *col = nullptr, *len = nullptr, *sell = nullptr;
  uint32_t *words = nullptr;
  double *kinv = nullptr, *F = nullptr, *Fn = nullptr, *Vn = nullptr, *Rn = nullptr, *En = nullptr;
  double *sig = nullptr, *state = nullptr, *eI = nullptr, *eP = nullptr, *Mt = nullptr, *obsw = nullptr;
  StencilLayout st;
  double *part_mat = nullptr, *part_force = nullptr, *accum = nullptr, *diag = nullptr;
  double *part_group = nullptr;
  unsigned *group_counter = nullptr;
  uint8_t *flags = nullptr;
  unsigned *status_dev = nullptr, *counter = nullptr;
  double *pdmg = nullptr;      // point damage (point damage modes only)
  double *field_buf = nullptr;  // device buffer of vpd_download's point-major layouts
  int64_t field_cap = 0;        // its doubles
  uint16_t *surr_w = nullptr;  // surrogate network (device copies)
  float *surr_b = nullptr;
  bool surrogate_ready = false;
  StepParams params{};
};

namespace {

template <typename T> int dalloc(vpd_handle *h, T **p, size_t count) {
  void *q = nullptr;
  VPD_CUDA(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
  h->allocations.push_back(q);
  *p = static_cast<T *>(q);
  return VPD_OK;
}

int check_case(const vpd_case *c) {
  if (!c)
    return set_error(VPD_ERR_INVALID, "case is NULL");
  if (c->nx < 2 || c->ny < 2 || c->nz < 2)
    return set_error(VPD_ERR_INVALID, "PD patch geometry requires nx/ny/nz >= 2.");
  if (!(c->spacing > 0.0) || !(c->horizon > 0.0))
    return set_error(VPD_ERR_INVALID, "PD geometry requires positive spacing and horizon.");
  if (!(c->dt > 0.0) || !std::isfinite(c->dt))
    return set_error(VPD_ERR_INVALID, "time_integration requires dt > 0.");
  if (!(c->density > 0.0))
    return set_error(VPD_ERR_INVALID, "Explicit dynamics requires density > 0.");
  if (c->nstatev < 6 || c->nstatev > 64)
    return set_error(VPD_ERR_INVALID, "JohnsonCook VUMAT requires 6 <= nstatev <= 64");
  if (c->region_layers < 1 || (c->load_axis != 0 && c->load_axis != 1))
    return set_error(VPD_ERR_INVALID, "regional loading needs regionLayers >= 1 and axis x or y");
  if (c->bc_mode == VPD_BC_SMOOTH_DISPLACEMENT) {
    if (c->amplitude == 0.0 || !(c->rise_time > 0.0))
      return set_error(VPD_ERR_INVALID, "smooth displacement needs amplitude != 0 and riseTime > 0");
  } else if (c->bc_mode == VPD_BC_VELOCITY_RAMP) {
    if (c->grip_velocity == 0.0 || !(c->ramp_time > 0.0))
      return set_error(VPD_ERR_INVALID, "velocity ramp needs grip_velocity != 0 and ramp_time > 0");
  } else {
    return set_error(VPD_ERR_INVALID, "unknown boundary-condition mode");
  }
  if (c->damage_mode == VPD_DAMAGE_CRITICAL_STRETCH && !(c->damage_initiation > 0.0))
    return set_error(VPD_ERR_INVALID, "critical_stretch requires initiation > 0.");
  if (c->damage_mode < VPD_DAMAGE_NONE || c->damage_mode > VPD_DAMAGE_MAX_PRINCIPAL_STRAIN)
    return set_error(VPD_ERR_INVALID, "unknown damage mode");
  if (c->damage_mode >= VPD_DAMAGE_EQPS_THRESHOLD && !(c->damage_failure - c->damage_initiation > 0.0))
    return set_error(VPD_ERR_INVALID, "SimpleDamageModel requires failure > initiation.");
  if (c->precision != VPD_PRECISION_FP64 && c->precision != VPD_PRECISION_MIXED)
    return set_error(VPD_ERR_INVALID, "unknown precision mode");
  if (c->material_mode != VPD_MATERIAL_VUMAT && c->material_mode != VPD_MATERIAL_SURROGATE)
    return set_error(VPD_ERR_INVALID, "unknown material mode");
  if (c->material_mode == VPD_MATERIAL_SURROGATE && c->damage_mode >= VPD_DAMAGE_EQPS_THRESHOLD)
    return set_error(VPD_ERR_UNSUPPORTED, "the point damage modes run with material_mode VPD_MATERIAL_VUMAT");
  for (int k = 0; k < 14; ++k)
    if (!std::isfinite(c->props[k]))
      return set_error(VPD_ERR_INVALID, "Johnson-Cook props must be finite");
  return VPD_OK;
}

int read_status(vpd_handle *h) {
  unsigned st = 0;
  VPD_CUDA(cudaMemcpyAsync(&st, h->status_dev, sizeof st, cudaMemcpyDeviceToHost, h->stream));
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  if (st & STATUS_SINGULAR_K)
    return set_error(VPD_ERR_SINGULAR, "Singular tensor in PD shape tensor.");
  if (st & STATUS_SINGULAR_F)
    return set_error(VPD_ERR_SINGULAR, "Invalid deformation gradient determinant.");
  if (st & STATUS_SINGULAR_KINEMATICS)
    return set_error(VPD_ERR_SINGULAR, "Corotational update encountered a singular tensor.");
  if (st & STATUS_SURROGATE_WAIT)
    return set_error(VPD_ERR_CUDA, "surrogate material kernel: tensor-core wait timed out");
  if (st & STATUS_STAGED_WAIT)
    return set_error(VPD_ERR_CUDA, "staged force kernel: TMA wait timed out");
  return VPD_OK;
}

// VPD_TRACE=1: the wall-clock time of each phase of vpd_create (the stream synchronised at every
// mark) on stderr.
struct CreateTrace {
  bool on = false;
  cudaStream_t stream = nullptr;
  std::chrono::steady_clock::time_point last = std::chrono::steady_clock::now();
  CreateTrace() {
    const char *t = getenv("VPD_TRACE");
    on = t && t[0] == '1';
  }
  void mark(const char *phase) {
    if (!on)
      return;
    if (stream)
      cudaStreamSynchronize(stream);
    const auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "vpd_create %-28s %9.2f ms\n", phase,
            std::chrono::duration<double, std::milli>(now - last).count());
    last = now;
  }
};

int create_impl(vpd_handle *h, const vpd_case *c, const double *positions, const double *volumes) {
  CreateTrace trace;
  int rc = check_case(c);
  if (rc)
    return rc;
  h->c = *c;
  const int64_t n = (int64_t)c->nx * c->ny * c->nz;
  if (n > INT32_MAX)
    return set_error(VPD_ERR_CAPACITY, "more than 2^31 points");
  h->n = n;

  // nominal lattice on the host: bands, pins and observation weights (all host-side checks
  // finish before the first CUDA call)
  const double hsp = c->spacing;
  const double yoff = 0.5 * (double)(c->ny - 1) * hsp, zoff = 0.5 * (double)(c->nz - 1) * hsp;
  const double volume = hsp * hsp * hsp;
  std::vector<double> nominal((size_t)(3 * n)), vol((size_t)n);
  {
    int64_t p = 0;
    for (int i = 0; i < c->nx; ++i)
      for (int j = 0; j < c->ny; ++j)
        for (int k = 0; k < c->nz; ++k, ++p) {
          nominal[3 * p] = (double)i * hsp;
          nominal[3 * p + 1] = (double)j * hsp - yoff;
          nominal[3 * p + 2] = (double)k * hsp - zoff;
          vol[p] = volume * ((i == 0 || i == c->nx - 1) ? 0.5 : 1.0) *
                   ((j == 0 || j == c->ny - 1) ? 0.5 : 1.0) * ((k == 0 || k == c->nz - 1) ? 0.5 : 1.0);
        }
  }
  Sets sets;
  if ((rc = build_sets(*c, nominal, vol, sets)))
    return rc;
  trace.mark("host sets");
  VPD_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  VPD_CUDA(cudaEventCreate(&h->ev0));
  VPD_CUDA(cudaEventCreate(&h->ev1));
  cudaStream_t s = h->stream;

  // device arrays
  if ((rc = dalloc(h, &h->xv, n)) || (rc = dalloc(h, &h->u0, n)) || (rc = dalloc(h, &h->u1, n)) ||
      (rc = dalloc(h, &h->vel, n)) || (rc = dalloc(h, &h->acc, n)) || (rc = dalloc(h, &h->force, n)) ||
      (rc = dalloc(h, &h->kinv, 9 * n)) || (rc = dalloc(h, &h->F, 9 * n)) ||
      (rc = dalloc(h, &h->Fn, 9 * n)) || (rc = dalloc(h, &h->Vn, 9 * n)) ||
      (rc = dalloc(h, &h->Rn, 9 * n)) || (rc = dalloc(h, &h->En, 6 * n)) ||
      (rc = dalloc(h, &h->sig, 6 * n)) || (rc = dalloc(h, &h->state, (size_t)c->nstatev * n)) ||
      (rc = dalloc(h, &h->eI, n)) || (rc = dalloc(h, &h->eP, n)) ||
      (rc = dalloc(h, &h->obsw, n)) || (rc = dalloc(h, &h->flags, n)) ||
      (rc = dalloc(h, &h->row_ptr, n + 1)) || (rc = dalloc(h, &h->step_dev, 1)) ||
      (rc = dalloc(h, &h->status_dev, 1)) || (rc = dalloc(h, &h->counter, 1)) ||
      (rc = dalloc(h, &h->accum, ACC_COUNT)) || (rc = dalloc(h, &h->diag, (size_t)kDiagRing * VPD_DIAG_COLS)))
    return rc;
  if (c->damage_mode >= VPD_DAMAGE_EQPS_THRESHOLD) {
    if ((rc = dalloc(h, &h->pdmg, n)))
      return rc;
    VPD_CUDA(cudaMemsetAsync(h->pdmg, 0, sizeof(double) * n, s));
  }
  trace.stream = s;
  trace.mark("device arrays");
  VPD_CUDA(cudaMemsetAsync(h->u0, 0, sizeof(double4) * n, s));
  VPD_CUDA(cudaMemsetAsync(h->status_dev, 0, sizeof(unsigned), s));
  VPD_CUDA(cudaMemsetAsync(h->counter, 0, sizeof(unsigned), s));

  // positions
  if (positions) {
    double *dpos = nullptr, *dvol = nullptr;
    VPD_CUDA(cudaMalloc(&dpos, sizeof(double) * 3 * n));
    VPD_CUDA(cudaMalloc(&dvol, sizeof(double) * n));
    VPD_CUDA(cudaMemcpyAsync(dpos, positions, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
    VPD_CUDA(cudaMemcpyAsync(dvol, volumes ? volumes : vol.data(), sizeof(double) * n,
                             cudaMemcpyHostToDevice, s));
    k_pack_xv<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dpos, dvol, n, h->xv);
    VPD_CUDA(cudaStreamSynchronize(s));
    cudaFree(dpos);
    cudaFree(dvol);
  } else {
    LatticeParams L{c->nx, c->ny, c->nz, hsp, yoff, zoff, volume, c->jitter * hsp, c->jitter_seed,
                    c->jitter != 0.0};
    k_lattice<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(L, h->xv);
  }
  trace.mark("positions");
  VPD_CUDA(cudaMemcpyAsync(h->flags, sets.flags.data(), n, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemcpyAsync(h->obsw, sets.obsw.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));

  // neighbour lists: sorted CSR, then the sliced-ELL copy the kernels stream
  {
    NeighborScratch scr;
    NeighborGrid grid;
    if ((rc = neighbor_scratch_alloc(scr, n)) == VPD_OK) {
      trace.mark("neighbour scratch");
      if ((rc = neighbor_count(h->xv, n, c->horizon, h->row_ptr, grid, scr, s)) == VPD_OK) {
        VPD_CUDA(cudaMemcpyAsync(&h->nbonds, h->row_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        VPD_CUDA(cudaStreamSynchronize(s));
        trace.mark("neighbour count");
        if ((rc = dalloc(h, &h->col, (size_t)h->nbonds)) == VPD_OK) {
          trace.mark("neighbour list allocation");
          rc = neighbor_fill(h->xv, n, h->row_ptr, h->col, grid, scr, s);
        }
      }
    }
    neighbor_scratch_free(scr);
    if (rc)
      return rc;
  }
  trace.mark("neighbour fill, scratch freed");
  // the bond layout the kernels stream: lattice-stencil bit masks when the points form the
  // lattice in index order (every generated patch), else the sliced ELL
  // (VPD_BOND_LAYOUT=ell selects the sliced ELL for any case)
  const char *layout = getenv("VPD_BOND_LAYOUT");
  if (!(layout && std::string(layout) == "ell") &&
      (rc = build_stencil(h->row_ptr, h->col, n, c->ny, c->nz, c->spacing, h->st, s)))
    return rc;
  if (h->st.nw == 0) {
    if ((rc = build_sell(h->row_ptr, h->col, n, &h->len, &h->slice_off, &h->sell, &h->sell_total, s)))
      return rc;
    h->allocations.push_back(h->len);
    h->allocations.push_back(h->slice_off);
    h->allocations.push_back(h->sell);
    if ((rc = dalloc(h, &h->words, (size_t)(h->sell_total / 32))) || (rc = dalloc(h, &h->Mt, 10 * n)))
      return rc;
    VPD_CUDA(cudaMemsetAsync(h->words, 0, sizeof(uint32_t) * std::max<int64_t>(h->sell_total / 32, 1), s));
  }
  trace.mark("bond layout");
  const int mat_blocks = material_grid(n);
  const int force_blocks = integrate_grid(n);
  const int groups = (force_blocks + kGroupBlocks - 1) / kGroupBlocks;
  if ((rc = dalloc(h, &h->part_mat, (size_t)mat_blocks * PM_COUNT)) ||
      (rc = dalloc(h, &h->part_force, (size_t)force_blocks * PF_COUNT)) ||
      (rc = dalloc(h, &h->part_group, (size_t)groups * (PM_COUNT + PF_COUNT))) ||
      (rc = dalloc(h, &h->group_counter, (size_t)groups)))
    return rc;
  VPD_CUDA(cudaMemsetAsync(h->group_counter, 0, sizeof(unsigned) * groups, s));

  // step parameters
  StepParams &p = h->params;
  p.n = n;
  p.dt = c->dt;
  p.rho = c->density;
  p.xv = h->xv, p.len = h->len, p.slice_off = h->slice_off, p.sell = h->sell, p.words = h->words;
  p.u0 = h->u0, p.u1 = h->u1, p.vel = h->vel, p.acc = h->acc, p.force = h->force;
  p.kinv = h->kinv, p.F = h->F, p.Fn = h->Fn, p.Vn = h->Vn, p.Rn = h->Rn, p.En = h->En;
  p.sig = h->sig, p.state = h->state, p.eI = h->eI, p.eP = h->eP, p.Mt = h->Mt;
  p.st = h->st;
  p.lat_nx = c->nx, p.lat_ny = c->ny, p.lat_nz = c->nz, p.lat_h = c->spacing;
  {
    // VPD_BOND_KERNEL=slot selects the per-slot bond kernels (both precisions), scalar the
    // two-point tiled mixed kernels in scalar FP32, tiled2 the two-point FP64 force kernel,
    // staged the TMA-staged FP64 force kernel (default: tiled; packed pairs when mixed, four
    // points per thread reading through L1 in the FP64 force)
    const char *bk = getenv("VPD_BOND_KERNEL");
    const std::string kind = bk ? bk : "";
    p.tiled = kind == "slot" ? 0 : kind == "scalar" ? 1 : kind == "tiled2" ? 3 : kind == "staged" ? 6 : 2;
    // VPD_RETURN_MAP=bisection: the material kernel evaluates every bisection iteration (the
    // default decides most of them from two anchor evaluations; the results are the same)
    const char *rm = getenv("VPD_RETURN_MAP");
    p.literal_bisection = rm && std::string(rm) == "bisection";
  }
  if (p.st.nw && ((rc = dalloc(h, &p.vxi, n)) ||
                  (c->precision != VPD_PRECISION_MIXED && (rc = dalloc(h, &p.fmap, 3 * n)))))
    return rc;
  if (p.st.nw && p.fmap && p.tiled == 6 && (rc = setup_staged_force64(p, p.st.rx, p.st.ry, p.st.rz)))
    return rc;
  p.nstatev = c->nstatev;
  p.flags = h->flags, p.obsw = h->obsw;
  p.jc = make_jc_params(c->props);
  p.bc = BcParams{c->bc_mode, c->amplitude, c->rise_time, c->grip_velocity, c->ramp_time,
                  sets.axis, sets.lateral, c->plane_strain};
  p.damage = c->damage_mode == VPD_DAMAGE_CRITICAL_STRETCH;
  p.dmg_initiation = c->damage_initiation;
  p.dmg_failure = c->damage_failure;
  p.use_compression = c->damage_failure > 0.0 && std::isfinite(c->damage_failure);
  p.tension2 = (1.0 + c->damage_initiation) * (1.0 + c->damage_initiation);
  p.compression2 = c->damage_failure < 1.0 ? (1.0 - c->damage_failure) * (1.0 - c->damage_failure) : 0.0;
  p.tension2f = (float)p.tension2, p.compression2f = (float)p.compression2;
  p.point_damage = c->damage_mode >= VPD_DAMAGE_EQPS_THRESHOLD ? c->damage_mode : 0;
  p.dmg_deletion = c->damage_deletion != 0;
  p.pdmg = h->pdmg;
  p.surrogate = c->material_mode == VPD_MATERIAL_SURROGATE;
  if (c->precision == VPD_PRECISION_MIXED) {
    if (!h->st.nw)
      return set_error(VPD_ERR_UNSUPPORTED,
                       "mixed precision needs the points in lattice order (lattice-stencil bonds)");
    // neighbour records with zero halos (StepParams): the packed bond kernels' window loads
    // stay in bounds without clamping, and a masked-out lane reads finite zeros
    const int64_t H = h->st.halo;
    float4 *jit = nullptr, *uf = nullptr, *fmapf = nullptr;
    if ((rc = dalloc(h, &jit, n + 2 * H)) || (rc = dalloc(h, &uf, n + 2 * H)) || (rc = dalloc(h, &p.Gf, 9 * n)) ||
        (rc = dalloc(h, &fmapf, 3 * n + 2 * H)))
      return rc;
    VPD_CUDA(cudaMemsetAsync(jit, 0, sizeof(float4) * (n + 2 * H), s));
    VPD_CUDA(cudaMemsetAsync(uf, 0, sizeof(float4) * (n + 2 * H), s));
    VPD_CUDA(cudaMemsetAsync(fmapf, 0, sizeof(float4) * (3 * n + 2 * H), s));
    p.jit = jit + H, p.uf = uf + H, p.fmapf = fmapf + H;
    p.mixed = 1;
  }
  p.step = h->step_dev, p.status = h->status_dev;
  p.part_mat = h->part_mat, p.part_force = h->part_force, p.accum = h->accum, p.diag = h->diag;
  p.part_group = h->part_group, p.group_counter = h->group_counter;
  p.counter = h->counter;
  p.mat_blocks = mat_blocks;
  p.interior = sets.interior, p.gauge = sets.gauge, p.lat_gauge = sets.lat_gauge;
  p.area = sets.area, p.n_lat_pos = sets.n_lat_pos, p.n_lat_neg = sets.n_lat_neg;
  p.sign = (c->bc_mode == VPD_BC_SMOOTH_DISPLACEMENT ? c->amplitude : c->grip_velocity) > 0.0 ? 1.0 : -1.0;

  trace.mark("parameters, mixed arrays");
  if ((rc = p.st.nw ? launch_shape_stencil(p, s) : launch_shape_inverse_sell(p, s)))
    return rc;
  if ((rc = launch_init(p, s)))
    return rc;
  if (p.mixed && (rc = launch_mixed_setup(p, c->ny, c->nz, hsp, yoff, zoff, s)))
    return rc;
  const double acc0[ACC_COUNT] = {0.0, 0.0, 0.0, 1.0};
  const int64_t one = 1;
  VPD_CUDA(cudaMemcpyAsync(h->accum, acc0, sizeof acc0, cudaMemcpyHostToDevice, s));
  VPD_CUDA(cudaMemcpyAsync(h->step_dev, &one, sizeof one, cudaMemcpyHostToDevice, s));
  const int status = read_status(h);
  trace.mark("shape tensors, initial state");
  return status;
}

void destroy_impl(vpd_handle *h) {
  if (h->graph)
    cudaGraphExecDestroy(h->graph);
  if (h->stream)
    cudaStreamSynchronize(h->stream);
  host_vumat_detach(h->params);
  for (void *p : h->allocations)
    cudaFree(p);
  cudaFree(h->field_buf);
  free_stencil(h->st);
  if (h->ev0)
    cudaEventDestroy(h->ev0);
  if (h->ev1)
    cudaEventDestroy(h->ev1);
  if (h->stream)
    cudaStreamDestroy(h->stream);
  delete h;
}

constexpr int kGraphSteps = 8;

int ensure_graph(vpd_handle *h) {
  if (h->graph)
    return VPD_OK;
  cudaGraph_t g = nullptr;
  VPD_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = VPD_OK;
  for (int k = 0; k < kGraphSteps && rc == VPD_OK; ++k)
    rc = launch_increment(h->params, h->stream);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc)
    return rc;
  if (e != cudaSuccess)
    return cuda_error(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return cuda_error(e, "cudaGraphInstantiate");
  h->graph_steps = kGraphSteps;
  return VPD_OK;
}

int copy_rows(vpd_handle *h, int64_t first_step, int64_t count, double *out) {
  // rows of increments first_step .. first_step+count-1 sit at (step-1) % ring
  int64_t done = 0;
  while (done < count) {
    const int64_t slot = (first_step - 1 + done) % kDiagRing;
    const int64_t m = std::min<int64_t>(count - done, kDiagRing - slot);
    VPD_CUDA(cudaMemcpyAsync(out + done * VPD_DIAG_COLS, h->diag + slot * VPD_DIAG_COLS,
                             sizeof(double) * VPD_DIAG_COLS * m, cudaMemcpyDeviceToHost, h->stream));
    done += m;
  }
  return VPD_OK;
}

template <typename Fn> int with_host_buffer(size_t count, Fn &&fn) {
  std::vector<double> buf(count);
  return fn(buf);
}

// ---- checkpoint / resume ----
// The state an increment carries to the next, as (device pointer, bytes) sections in a fixed
// order: everything else is either fixed at creation (geometry, bonds, K^-1, the sets) or
// recomputed inside every increment (F, the force map, the mixed-precision sums, the
// diagnostic partials and counters).
struct Section {
  void *ptr;
  size_t bytes;
};

std::vector<Section> checkpoint_sections(vpd_handle *h) {
  const size_t n = (size_t)h->n, d4 = sizeof(double4) * n, d1 = sizeof(double) * n;
  const StepParams &p = h->params;
  std::vector<Section> v = {{h->u0, d4}, {h->u1, d4},     {h->vel, d4},     {h->acc, d4},
                            {h->force, d4}, {h->Fn, 9 * d1}, {h->Vn, 9 * d1}, {h->Rn, 9 * d1},
                            {h->En, 6 * d1}, {h->sig, 6 * d1}, {h->state, (size_t)h->c.nstatev * d1},
                            {h->eI, d1},     {h->eP, d1},     {h->accum, sizeof(double) * ACC_COUNT},
                            {h->step_dev, sizeof(int64_t)}};
  if (h->words)
    v.push_back({h->words, sizeof(uint32_t) * (size_t)(h->sell_total / 32)});
  if (h->st.nw)
    v.push_back({h->st.broken, sizeof(uint32_t) * (size_t)h->st.nw * n});
  if (p.mixed)
    v.push_back({p.uf, sizeof(float4) * n});
  if (h->pdmg)
    v.push_back({h->pdmg, d1});
  if (p.host_vumat)
    v.push_back({p.temp, d1});
  return v;
}

// What the loading handle must share with the saving one.
struct CheckpointHeader {
  char magic[8];
  uint32_t version, sections;
  int64_t step, n, nbonds, sell_total;
  int32_t stencil_words, mixed, host_vumat, surrogate;
  uint64_t payload;
  vpd_case c;
};

// Field by field, bitwise (NaN observation bounds compare equal); padding is not compared.
bool same_case(const vpd_case &a, const vpd_case &b) {
#define VPD_SAME(f) (std::memcmp(&a.f, &b.f, sizeof(a.f)) == 0)
  return VPD_SAME(nx) && VPD_SAME(ny) && VPD_SAME(nz) && VPD_SAME(spacing) && VPD_SAME(horizon) &&
         VPD_SAME(jitter) && VPD_SAME(jitter_seed) && VPD_SAME(dt) && VPD_SAME(density) && VPD_SAME(bc_mode) &&
         VPD_SAME(load_axis) && VPD_SAME(region_layers) && VPD_SAME(plane_strain) && VPD_SAME(amplitude) &&
         VPD_SAME(rise_time) && VPD_SAME(grip_velocity) && VPD_SAME(ramp_time) && VPD_SAME(observation_min) &&
         VPD_SAME(observation_max) && VPD_SAME(props) && VPD_SAME(nstatev) && VPD_SAME(reference_temperature) &&
         VPD_SAME(damage_mode) && VPD_SAME(damage_initiation) && VPD_SAME(damage_failure) &&
         VPD_SAME(precision) && VPD_SAME(material_mode) && VPD_SAME(damage_deletion);
#undef VPD_SAME
}

CheckpointHeader checkpoint_header(vpd_handle *h, const std::vector<Section> &v) {
  CheckpointHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  std::memcpy(hd.magic, "VPDCKPT", 8);
  hd.version = 1;
  hd.sections = (uint32_t)v.size();
  hd.step = h->step, hd.n = h->n, hd.nbonds = h->nbonds, hd.sell_total = h->sell_total;
  hd.stencil_words = h->st.nw, hd.mixed = h->params.mixed;
  hd.host_vumat = h->params.host_vumat != nullptr, hd.surrogate = h->params.surrogate;
  for (const Section &sec : v)
    hd.payload += sec.bytes;
  hd.c = h->c;
  return hd;
}

}  // namespace

namespace {
// Point-major layouts of vpd_download, formed on the device (one copy to the host follows).
// MODE 0: components 0..comps-1 (or the fourth, comps == 1) of a double4 array; 1: a structure
// of arrays; 2: a Voigt tensor (11,22,33,23,13,12) as the full 3x3; 3: the spatial stress
// R sigma R^T from the Voigt corotational stress and R, rounded as the host loop it replaces
// (separate products and sums, left to right).
template <int MODE>
__global__ void k_field_pack(int64_t n, int comps, const double4 *v4, const double *a, const double *b,
                             double *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  if (MODE == 0) {
    const double4 v = v4[i];
    if (comps == 1) {
      out[i] = v.w;
    } else {
      out[3 * i] = v.x, out[3 * i + 1] = v.y, out[3 * i + 2] = v.z;
    }
  } else if (MODE == 1) {
    for (int c = 0; c < comps; ++c)
      out[comps * i + c] = a[c * n + i];
  } else {
    double v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
      v[c] = a[c * n + i];
    const double f[9] = {v[0], v[5], v[4], v[5], v[1], v[3], v[4], v[3], v[2]};
    double *o = out + 9 * i;
    if (MODE == 2) {
#pragma unroll
      for (int c = 0; c < 9; ++c)
        o[c] = f[c];
    } else {
      double R[9], t[9];
#pragma unroll
      for (int c = 0; c < 9; ++c)
        R[c] = b[c * n + i];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          t[3 * r + c] = __dadd_rn(__dadd_rn(__dmul_rn(f[3 * r], R[3 * c]), __dmul_rn(f[3 * r + 1], R[3 * c + 1])),
                                   __dmul_rn(f[3 * r + 2], R[3 * c + 2]));
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          o[3 * r + c] = __dadd_rn(__dadd_rn(__dmul_rn(R[3 * r], t[c]), __dmul_rn(R[3 * r + 1], t[3 + c])),
                                   __dmul_rn(R[3 * r + 2], t[6 + c]));
    }
  }
}

}  // namespace

extern "C" {

int vpd_abi_version(void) { return VPD_ABI_VERSION; }
const char *vpd_last_error(void) { return g_error.c_str(); }

int vpd_field_width(const vpd_handle *h, int field) {
  switch (field) {
  case VPD_FIELD_VOLUME: case VPD_FIELD_TEMPERATURE: case VPD_FIELD_ENERGY_INTERNAL:
  case VPD_FIELD_ENERGY_INELASTIC: case VPD_FIELD_DAMAGE_INDEX:
    return 1;
  case VPD_FIELD_POSITION: case VPD_FIELD_DISPLACEMENT: case VPD_FIELD_VELOCITY:
  case VPD_FIELD_ACCELERATION: case VPD_FIELD_FORCE_DENSITY:
    return 3;
  case VPD_FIELD_STATE:
    return h ? h->c.nstatev : -1;
  case VPD_FIELD_DEFGRAD: case VPD_FIELD_STRESS_COROTATIONAL: case VPD_FIELD_STRESS_SPATIAL:
  case VPD_FIELD_STRAIN: case VPD_FIELD_ROTATION: case VPD_FIELD_LEFT_STRETCH: case VPD_FIELD_SHAPE_INVERSE:
    return 9;
  default:
    return -1;
  }
}

int vpd_create(const vpd_case *c, const double *positions, const double *volumes, vpd_handle **out) {
  if (!out)
    return set_error(VPD_ERR_INVALID, "out is NULL");
  *out = nullptr;
  vpd_handle *h = new vpd_handle();
  const int rc = create_impl(h, c, positions, volumes);
  if (rc) {
    const std::string msg = g_error;
    destroy_impl(h);
    g_error = msg;
    return rc;
  }
  *out = h;
  return VPD_OK;
}

int vpd_destroy(vpd_handle *h) {
  if (h)
    destroy_impl(h);
  return VPD_OK;
}

int64_t vpd_num_points(const vpd_handle *h) { return h ? h->n : -1; }
int64_t vpd_num_bonds(const vpd_handle *h) { return h ? h->nbonds : -1; }
int vpd_bond_layout_words(const vpd_handle *h) { return h ? h->st.nw : -1; }
void *vpd_stream(vpd_handle *h) { return h ? (void *)h->stream : nullptr; }
int vpd_last_step_ms(const vpd_handle *h, double *ms) {
  if (!h || !ms)
    return set_error(VPD_ERR_INVALID, "NULL argument");
  *ms = h->last_ms;
  return VPD_OK;
}

int vpd_step(vpd_handle *h, int32_t nsteps, double *diag_out) {
  if (!h || nsteps < 0)
    return set_error(VPD_ERR_INVALID, "vpd_step needs a handle and nsteps >= 0");
  if (h->params.surrogate && !h->surrogate_ready)
    return set_error(VPD_ERR_INVALID, "material_mode is VPD_MATERIAL_SURROGATE: call vpd_set_surrogate first");
  if (nsteps == 0)
    return VPD_OK;
  int rc = ensure_graph(h);
  if (rc)
    return rc;
  VPD_CUDA(cudaEventRecord(h->ev0, h->stream));
  int64_t done = 0;
  while (done < nsteps) {
    const int64_t chunk = std::min<int64_t>(nsteps - done, kDiagRing);
    int64_t k = 0;
    for (; k + h->graph_steps <= chunk; k += h->graph_steps)
      VPD_CUDA(cudaGraphLaunch(h->graph, h->stream));
    for (; k < chunk; ++k)
      if ((rc = launch_increment(h->params, h->stream)))
        return rc;
    if (diag_out && (rc = copy_rows(h, h->step + done + 1, chunk, diag_out + done * VPD_DIAG_COLS)))
      return rc;
    done += chunk;
    if (done < nsteps && diag_out)
      VPD_CUDA(cudaStreamSynchronize(h->stream));  // ring slots are reused by the next chunk
  }
  VPD_CUDA(cudaEventRecord(h->ev1, h->stream));
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  VPD_CUDA(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  h->step += nsteps;
  return read_status(h);
}

int vpd_set_surrogate(vpd_handle *h, const uint16_t *weights, const float *biases, int32_t guess,
                      int32_t newton_steps) {
  if (!h)
    return set_error(VPD_ERR_INVALID, "vpd_set_surrogate: null handle");
  if (!h->params.surrogate)
    return set_error(VPD_ERR_INVALID, "vpd_set_surrogate: the case's material_mode is not VPD_MATERIAL_SURROGATE");
  if (guess != VPD_GUESS_NETWORK && guess != VPD_GUESS_WARM_START && guess != VPD_GUESS_HYBRID)
    return set_error(VPD_ERR_INVALID, "vpd_set_surrogate: unknown guess mode");
  if (newton_steps < 0 || newton_steps > 50)
    return set_error(VPD_ERR_INVALID, "vpd_set_surrogate: newton_steps must be in [0, 50]");
  if (guess != VPD_GUESS_WARM_START && (!weights || !biases))
    return set_error(VPD_ERR_INVALID, "vpd_set_surrogate: the network guess needs weights and biases");
  if (guess != VPD_GUESS_WARM_START) {
    for (int k = 0; k < VPD_MLP_PARAMS - VPD_MLP_WEIGHTS; ++k)
      if (!std::isfinite(biases[k]))
        return set_error(VPD_ERR_NONFINITE, "vpd_set_surrogate: non-finite bias");
    int rc;
    if (!h->surr_w && ((rc = dalloc(h, &h->surr_w, VPD_MLP_WEIGHTS)) ||
                       (rc = dalloc(h, &h->surr_b, VPD_MLP_PARAMS - VPD_MLP_WEIGHTS))))
      return rc;
    VPD_CUDA(cudaMemcpyAsync(h->surr_w, weights, sizeof(uint16_t) * VPD_MLP_WEIGHTS, cudaMemcpyHostToDevice,
                             h->stream));
    VPD_CUDA(cudaMemcpyAsync(h->surr_b, biases, sizeof(float) * (VPD_MLP_PARAMS - VPD_MLP_WEIGHTS),
                             cudaMemcpyHostToDevice, h->stream));
    VPD_CUDA(cudaStreamSynchronize(h->stream));
    int rc2 = prepare_material_surrogate();
    if (rc2)
      return rc2;
  }
  h->params.surr_guess = guess;
  h->params.surr_steps = newton_steps;
  h->params.sw = h->surr_w;
  h->params.sb = h->surr_b;
  h->surrogate_ready = true;
  if (h->graph) {  // recaptured with the new parameters at the next vpd_step
    VPD_CUDA(cudaStreamSynchronize(h->stream));
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return VPD_OK;
}

int vpd_set_host_vumat(vpd_handle *h, const char *plugin_path, const char *symbol, const char *cmname,
                       const double *props, int32_t nprops, int32_t nstatev, double density) {
  if (!h)
    return set_error(VPD_ERR_INVALID, "vpd_set_host_vumat: null handle");
  if (h->c.material_mode != VPD_MATERIAL_VUMAT)
    return set_error(VPD_ERR_INVALID, "vpd_set_host_vumat: the case's material_mode is not VPD_MATERIAL_VUMAT");
  if (h->params.host_vumat)
    return set_error(VPD_ERR_INVALID, "vpd_set_host_vumat: a plugin is already attached to this handle");
  if (h->step != 0)
    return set_error(VPD_ERR_INVALID, "vpd_set_host_vumat: call before the first vpd_step");
  if (nstatev > h->c.nstatev)
    return set_error(VPD_ERR_INVALID, "vpd_set_host_vumat: nstatev exceeds the case's nstatev");
  if (!std::isfinite(density))
    return set_error(VPD_ERR_INVALID, "vpd_set_host_vumat: density must be finite");
  if (h->c.damage_mode == VPD_DAMAGE_EQPS_THRESHOLD && nstatev < 2)  // SimpleDamageModel.cpp:22-25
    return set_error(VPD_ERR_INVALID, "eqpsStateIndex is outside the VUMAT state vector.");
  if (h->graph) {  // recaptured with the plugin's launches at the next vpd_step
    VPD_CUDA(cudaStreamSynchronize(h->stream));
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return host_vumat_attach(h->params, plugin_path, symbol, cmname, props, nprops, nstatev, density, h->c.spacing,
                           h->c.reference_temperature, h->stream);
}

int vpd_set_internal_indicator(vpd_handle *h, const int32_t *indices, int32_t count, int32_t reduction_min,
                               int32_t one_minus) {
  if (!h || (!indices && count > 0))
    return set_error(VPD_ERR_INVALID, "vpd_set_internal_indicator: null argument");
  if (count < 0 || count > 8)
    return set_error(VPD_ERR_UNSUPPORTED, "vpd_set_internal_indicator: at most 8 state variables");
  for (int k = 0; k < count; ++k)
    if (indices[k] < 0 || indices[k] >= h->c.nstatev)
      return set_error(VPD_ERR_INVALID, "internalIndicator index is outside nstatev");
  h->params.ind_count = count;
  h->params.ind_min = reduction_min != 0;
  h->params.ind_one_minus = one_minus != 0;
  for (int k = 0; k < 8; ++k)
    h->params.ind_idx[k] = k < count ? indices[k] : 0;
  if (h->graph) {  // recaptured with the indicator's launch at the next vpd_step
    VPD_CUDA(cudaStreamSynchronize(h->stream));
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return VPD_OK;
}

int vpd_set_initial_state(vpd_handle *h, const double *state, int32_t nstatev) {
  if (!h || (!state && nstatev > 0))
    return set_error(VPD_ERR_INVALID, "vpd_set_initial_state: null argument");
  if (h->step != 0)
    return set_error(VPD_ERR_INVALID, "vpd_set_initial_state: call before the first vpd_step");
  if (nstatev < 0 || nstatev > h->c.nstatev)
    return set_error(VPD_ERR_INVALID, "Initial VUMAT state size does not match nstatev.");
  for (int c = 0; c < nstatev; ++c)
    if (!std::isfinite(state[c]))
      return set_error(VPD_ERR_NONFINITE, "vpd_set_initial_state: non-finite state value");
  std::vector<double> column((size_t)h->n);
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  for (int c = 0; c < nstatev; ++c) {  // every point starts from the same state (:62-66)
    std::fill(column.begin(), column.end(), state[c]);
    VPD_CUDA(cudaMemcpy(h->state + (size_t)c * h->n, column.data(), sizeof(double) * column.size(),
                        cudaMemcpyHostToDevice));
  }
  return VPD_OK;
}

int64_t vpd_checkpoint_bytes(vpd_handle *h) {
  if (!h)
    return -1;
  const auto v = checkpoint_sections(h);
  return (int64_t)(sizeof(CheckpointHeader) + checkpoint_header(h, v).payload);
}

int vpd_checkpoint_save(vpd_handle *h, void *buffer, int64_t bytes) {
  if (!h || !buffer)
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_save: null argument");
  const auto v = checkpoint_sections(h);
  const CheckpointHeader hd = checkpoint_header(h, v);
  if (bytes != (int64_t)(sizeof(hd) + hd.payload))
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_save: buffer size is not vpd_checkpoint_bytes");
  char *out = static_cast<char *>(buffer);
  std::memcpy(out, &hd, sizeof(hd));
  size_t at = sizeof(hd);
  for (const Section &sec : v) {
    VPD_CUDA(cudaMemcpyAsync(out + at, sec.ptr, sec.bytes, cudaMemcpyDeviceToHost, h->stream));
    at += sec.bytes;
  }
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  return VPD_OK;
}

int vpd_checkpoint_load(vpd_handle *h, const void *buffer, int64_t bytes) {
  if (!h || !buffer)
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_load: null argument");
  const auto v = checkpoint_sections(h);
  CheckpointHeader mine = checkpoint_header(h, v), theirs;
  if (bytes < (int64_t)sizeof(theirs))
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_load: buffer too small for a checkpoint");
  std::memcpy(&theirs, buffer, sizeof(theirs));
  if (std::memcmp(theirs.magic, "VPDCKPT", 8) != 0 || theirs.version != 1)
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_load: not a checkpoint of this library");
  mine.step = theirs.step;  // the one field the loading handle takes over
  const bool case_matches = same_case(mine.c, theirs.c);
  std::memset(&mine.c, 0, sizeof(mine.c));
  std::memset(&theirs.c, 0, sizeof(theirs.c));
  if (!case_matches || std::memcmp(&mine, &theirs, sizeof(mine)) != 0)
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_load: the checkpoint was saved from a handle with another "
                                      "case, layout, precision or material path");
  if (bytes != (int64_t)(sizeof(theirs) + theirs.payload))
    return set_error(VPD_ERR_INVALID, "vpd_checkpoint_load: buffer size does not match the checkpoint");
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  const char *in = static_cast<const char *>(buffer);
  size_t at = sizeof(theirs);
  for (const Section &sec : v) {
    VPD_CUDA(cudaMemcpyAsync(sec.ptr, in + at, sec.bytes, cudaMemcpyHostToDevice, h->stream));
    at += sec.bytes;
  }
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  h->step = theirs.step;
  return VPD_OK;
}

int vpd_profile_increment(vpd_handle *h, int32_t nsteps, double *stage_ms) {
  if (!h || !stage_ms || nsteps < 1)
    return set_error(VPD_ERR_INVALID, "vpd_profile_increment needs a handle, nsteps >= 1 and an output");
  cudaEvent_t ev[kStages + 1];
  for (auto &e : ev)
    VPD_CUDA(cudaEventCreate(&e));
  for (int k = 0; k < kStages; ++k)
    stage_ms[k] = 0.0;
  int rc = VPD_OK;
  for (int32_t it = 0; it < nsteps && rc == VPD_OK; ++it) {
    VPD_CUDA(cudaEventRecord(ev[0], h->stream));
    for (int k = 0; k < kStages && rc == VPD_OK; ++k) {
      rc = launch_stage(k, h->params, h->stream);
      VPD_CUDA(cudaEventRecord(ev[k + 1], h->stream));
    }
    VPD_CUDA(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < kStages; ++k) {
      float ms = 0.0f;
      VPD_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      stage_ms[k] += ms / nsteps;
    }
  }
  for (auto &e : ev)
    cudaEventDestroy(e);
  if (rc)
    return rc;
  h->step += nsteps;
  return read_status(h);
}

int vpd_neighbors(vpd_handle *h, int64_t *row_ptr, int32_t *col) {
  if (!h || !row_ptr || !col)
    return set_error(VPD_ERR_INVALID, "NULL argument");
  VPD_CUDA(cudaMemcpyAsync(row_ptr, h->row_ptr, sizeof(int64_t) * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
  VPD_CUDA(cudaMemcpyAsync(col, h->col, sizeof(int32_t) * h->nbonds, cudaMemcpyDeviceToHost, h->stream));
  VPD_CUDA(cudaStreamSynchronize(h->stream));
  return VPD_OK;
}

int vpd_download(vpd_handle *h, int32_t field, double *out) {
  if (!h || !out)
    return set_error(VPD_ERR_INVALID, "NULL argument");
  const int64_t n = h->n;
  cudaStream_t s = h->stream;
  // a point-major field of `comps` doubles per point packed by k_field_pack<MODE> into the
  // handle's device buffer, then one copy into the caller's array
  auto packed = [&](auto kernel, int comps, const double4 *v4, const double *a, const double *b) -> int {
    const int64_t need = (int64_t)comps * n;
    if (need > h->field_cap) {  // sized once for the widest field
      cudaFree(h->field_buf);
      h->field_buf = nullptr, h->field_cap = 0;
      const int64_t cap = std::max<int64_t>(need, (int64_t)std::max(9, h->c.nstatev) * n);
      VPD_CUDA(cudaMalloc(&h->field_buf, sizeof(double) * cap));
      h->field_cap = cap;
    }
    kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, comps, v4, a, b, h->field_buf);
    VPD_CUDA(cudaGetLastError());
    VPD_CUDA(cudaMemcpyAsync(out, h->field_buf, sizeof(double) * need, cudaMemcpyDeviceToHost, s));
    VPD_CUDA(cudaStreamSynchronize(s));
    return VPD_OK;
  };
  auto get4 = [&](const double4 *src, int comps) -> int {
    return packed(k_field_pack<0>, comps == 1 ? 1 : 3, src, nullptr, nullptr);
  };
  auto getSoA = [&](const double *src, int comps, std::vector<double> &buf) -> int {
    buf.resize((size_t)(comps * n));
    VPD_CUDA(cudaMemcpyAsync(buf.data(), src, sizeof(double) * comps * n, cudaMemcpyDeviceToHost, s));
    VPD_CUDA(cudaStreamSynchronize(s));
    return VPD_OK;
  };
  auto aos = [&](const double *src, int comps) -> int {
    return packed(k_field_pack<1>, comps, nullptr, src, nullptr);
  };
  auto sym = [&](const double *src) -> int {  // Voigt 11,22,33,23,13,12 -> full 3x3
    return packed(k_field_pack<2>, 9, nullptr, src, nullptr);
  };
  switch (field) {
  case VPD_FIELD_POSITION: return get4(h->xv, 3);
  case VPD_FIELD_VOLUME: return get4(h->xv, 1);
  case VPD_FIELD_DISPLACEMENT: return get4((h->step & 1) ? h->u1 : h->u0, 3);
  case VPD_FIELD_VELOCITY: return get4(h->vel, 3);
  case VPD_FIELD_ACCELERATION: return get4(h->acc, 3);
  case VPD_FIELD_FORCE_DENSITY: return get4(h->force, 3);
  case VPD_FIELD_DEFGRAD: return aos(h->Fn, 9);
  case VPD_FIELD_ROTATION: return aos(h->Rn, 9);
  case VPD_FIELD_LEFT_STRETCH: return aos(h->Vn, 9);
  case VPD_FIELD_SHAPE_INVERSE: return aos(h->kinv, 9);
  case VPD_FIELD_STATE: return aos(h->state, h->c.nstatev);
  case VPD_FIELD_ENERGY_INTERNAL: return aos(h->eI, 1);
  case VPD_FIELD_ENERGY_INELASTIC: return aos(h->eP, 1);
  case VPD_FIELD_STRESS_COROTATIONAL: return sym(h->sig);
  case VPD_FIELD_STRAIN: return sym(h->En);
  case VPD_FIELD_STRESS_SPATIAL:  // R sigma R^T
    return packed(k_field_pack<3>, 9, nullptr, h->sig, h->Rn);
  case VPD_FIELD_TEMPERATURE: {
    if (h->params.host_vumat) {  // the plugin's tempNew, kept per point
      VPD_CUDA(cudaMemcpyAsync(out, h->params.temp, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      VPD_CUDA(cudaStreamSynchronize(s));
      return VPD_OK;
    }
    std::vector<double> st;
    int rc = getSoA(h->state, 3, st);
    if (rc)
      return rc;
    for (int64_t i = 0; i < n; ++i)
      out[i] = st[i] != 0.0 ? st[2 * n + i] : h->c.reference_temperature;
    return VPD_OK;
  }
  case VPD_FIELD_DAMAGE_INDEX: {
    if (h->pdmg) {  // point modes: the point damage (PdSimpleDamage.cpp:86-92)
      VPD_CUDA(cudaMemcpyAsync(out, h->pdmg, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      VPD_CUDA(cudaStreamSynchronize(s));
      return VPD_OK;
    }
    double *d = nullptr;
    VPD_CUDA(cudaMalloc(&d, sizeof(double) * n));
    if (h->st.nw) {
      const int rc = launch_damage_index_stencil(h->params, d, s);
      if (rc) {
        cudaFree(d);
        return rc;
      }
    } else {
      k_damage_index<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, h->xv, h->len, h->slice_off, h->sell,
                                                                h->words, d);
    }
    cudaError_t e = cudaMemcpyAsync(out, d, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess)
      return cuda_error(e, "damage index");
    return VPD_OK;
  }
  default:
    return set_error(VPD_ERR_INVALID, "unknown field");
  }
}

}  // extern "C"
