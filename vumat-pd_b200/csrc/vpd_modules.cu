// Module-level entry points of libvpd_gpu.so: the reference's C++ module functions on
// caller-owned device arrays in the reference's point-major layout (Tensor3 row-major,
// neighbour lists as CSR), and the VUMAT plugin entry vumat_adapter_call evaluated on the GPU.
// Each kernel is one thread per point.
#include "vpd_math.cuh"
#include "vpd_step.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace vpd {

__global__ void k_pack_positions(const double *pos, int64_t n, double4 *xv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    xv[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.0);
}

// PdCorrespondenceSkeleton::initialize (:149-170)
__global__ void k_csr_shape_inverse(const double *pos, const double *vol, int64_t n,
                                    const int64_t *row_ptr, const int32_t *col, double *kinv,
                                    unsigned *status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
    const int64_t j = col[q];
    const double e[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                         pos[3 * j + 2] - pos[3 * i + 2]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        K[3 * a + b] += vol[j] * e[a] * e[b];
  }
  double Ki[9];
  if (!m_inv(K, Ki)) {
    atomicOr(status, STATUS_SINGULAR_K);
    for (int c = 0; c < 9; ++c)
      Ki[c] = 0.0;
  }
  for (int c = 0; c < 9; ++c)
    kinv[9 * i + c] = Ki[c];
}

// computeDeformationGradients (:172-197), in displacement-gradient form
// F = I + [sum_j V_j (u_j - u_i) (x) xi] K^-1.
__global__ void k_csr_deformation(const double *pos, const double *disp, const double *vol,
                                  int64_t n, const int64_t *row_ptr, const int32_t *col,
                                  const double *kinv, double *F) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
    const int64_t j = col[q];
    double e[3], d[3];
    for (int c = 0; c < 3; ++c) {
      e[c] = pos[3 * j + c] - pos[3 * i + c];
      d[c] = vol[j] * (disp[3 * j + c] - disp[3 * i + c]);
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        G[3 * a + b] += d[a] * e[b];
  }
  double K[9], GK[9];
  for (int c = 0; c < 9; ++c)
    K[c] = kinv[9 * i + c];
  m_mul(G, K, GK);
  for (int c = 0; c < 9; ++c)
    F[9 * i + c] = ((c % 4 == 0) ? 1.0 : 0.0) + GK[c];
}

__global__ void k_csr_force_map(const double *sigma, const double *F, const double *kinv,
                                int64_t n, double *M, unsigned *status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double s[9], f[9], k[9], m[9];
  for (int c = 0; c < 9; ++c)
    s[c] = sigma[9 * i + c], f[c] = F[9 * i + c], k[c] = kinv[9 * i + c];
  if (!force_map(s, f, k, m)) {
    atomicOr(status, STATUS_SINGULAR_F);
    for (int c = 0; c < 9; ++c)
      m[c] = 0.0;
  }
  for (int c = 0; c < 9; ++c)
    M[9 * i + c] = m[c];
}

// computeForceDensity (:199-230): f_i = sum (1 - clamp(d)) (M_i + M_j) xi V_j
__global__ void k_csr_force(const double *pos, const double *vol, int64_t n,
                            const int64_t *row_ptr, const int32_t *col, const double *M,
                            const double *bond_damage, double *force) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double f[3] = {0, 0, 0};
  const double *Mi = M + 9 * i;
  for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
    const int64_t j = col[q];
    const double *Mj = M + 9 * j;
    const double e[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                         pos[3 * j + 2] - pos[3 * i + 2]};
    double dmg = bond_damage ? bond_damage[q] : 0.0;
    dmg = dmg < 0.0 ? 0.0 : (dmg > 1.0 ? 1.0 : dmg);
    const double w = (1.0 - dmg) * vol[j];
    for (int a = 0; a < 3; ++a)
      f[a] += w * ((Mi[3 * a] + Mj[3 * a]) * e[0] + (Mi[3 * a + 1] + Mj[3 * a + 1]) * e[1] +
                   (Mi[3 * a + 2] + Mj[3 * a + 2]) * e[2]);
  }
  for (int a = 0; a < 3; ++a)
    force[3 * i + a] = f[a];
}

__global__ void k_corotational(int64_t n, const double *fN, const double *fNP1, const double *vN,
                               const double *rN, double dt, double *dbar, double *spin,
                               double *rNew, double *vNew, double *strain, unsigned *status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double a[9], b[9], v[9], r[9];
  for (int c = 0; c < 9; ++c)
    a[c] = fN[9 * i + c], b[c] = fNP1[9 * i + c], v[c] = vN[9 * i + c], r[c] = rN[9 * i + c];
  Corotational co;
  if (!corotational_update(a, b, v, r, dt, co))
    atomicOr(status, STATUS_SINGULAR_KINEMATICS);
  double e6[6], e[9];
  green_lagrange6(b, e6);
  voigt_to_full(e6, e);
  for (int c = 0; c < 9; ++c) {
    dbar[9 * i + c] = co.dbar[c];
    spin[9 * i + c] = co.spin[c];
    rNew[9 * i + c] = co.r[c];
    vNew[9 * i + c] = co.v[c];
    strain[9 * i + c] = e[c];
  }
}

// VumatPdCorrespondenceMaterial::update for one point (:155-170,195-210).
__global__ void k_material_update(int64_t n, JcParams jc, int nstatev, double dt, const double *Fnew,
                                  double *Fold, double *stretch, double *rotation, double *strain,
                                  double *sig, double *state, double *temp, double *eI, double *eP,
                                  double *spatial, unsigned *status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double F[9], Fn[9], Vn[9], Rn[9];
  for (int c = 0; c < 9; ++c)
    F[c] = Fnew[9 * i + c], Fn[c] = Fold[9 * i + c], Vn[c] = stretch[9 * i + c], Rn[c] = rotation[9 * i + c];
  Corotational co;
  if (!corotational_update(Fn, F, Vn, Rn, dt, co)) {
    atomicOr(status, STATUS_SINGULAR_KINEMATICS);
    return;
  }
  JcPoint pt;
  double s9[9];
  for (int c = 0; c < 9; ++c)
    s9[c] = sig[9 * i + c];
  full_to_voigt(s9, pt.stress);
  for (int c = 0; c < 6; ++c)
    pt.state[c] = state[(size_t)nstatev * i + c];
  pt.eInternal = eI[i];
  pt.eInelastic = eP[i];
  const double *d = co.dbar;
  const double inc[6] = {d[0] * dt, d[4] * dt, d[8] * dt, 0.5 * (d[5] + d[7]) * dt,
                         0.5 * (d[2] + d[6]) * dt, 0.5 * (d[1] + d[3]) * dt};
  jc_update(jc, dt, inc, pt);
  double full[9], sp[9], e6[6], e[9];
  voigt_to_full(pt.stress, full);
  rotate_to_spatial(full, co.r, sp);
  green_lagrange6(F, e6);
  voigt_to_full(e6, e);
  for (int c = 0; c < 9; ++c) {
    Fold[9 * i + c] = F[c];
    stretch[9 * i + c] = co.v[c];
    rotation[9 * i + c] = co.r[c];
    strain[9 * i + c] = e[c];
    sig[9 * i + c] = full[c];
    spatial[9 * i + c] = sp[c];
  }
  for (int c = 0; c < 6; ++c)
    state[(size_t)nstatev * i + c] = pt.state[c];
  temp[i] = pt.state[2];
  eI[i] = pt.eInternal;
  eP[i] = pt.eInelastic;
}

// The VUMAT's return map alone for one point (JohnsonCook.f90:74-136): the elastic trial from
// the old stress and state, then the bisection, certified (jc_return_map) or literal
// (jc_bisection). A point on its initialising call (state[0] == 0) reports 0 iterations.
template <bool CERTIFIED>
__global__ void k_jc_return_map(int64_t n, JcParams jc, double dt, const double *inc, const double *sig,
                                const double *state, int nstatev, double *epInc, double *yield, int32_t *iters) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  JcPoint pt;
  double d[6];
  for (int c = 0; c < 6; ++c)
    d[c] = inc[6 * i + c], pt.stress[c] = sig[6 * i + c], pt.state[c] = state[(size_t)nstatev * i + c];
  pt.eInternal = pt.eInelastic = 0.0;
  JcTrial t;
  double e = 0.0, y = 0.0;
  int it = 0;
  if (jc_trial(jc, d, pt, t))
    it = CERTIFIED ? jc_return_map(jc, dt, t, pt.state[4], e, y) : jc_bisection(jc, dt, t, pt.state[4], e, y);
  epInc[i] = e, yield[i] = y, iters[i] = it;
}

// PdSimpleDamage::update critical_stretch (:51-82) with the reference's rounding, and the
// damage index (:23-36).
__global__ void k_csr_damage(const double *pos, const double *disp, const double *vol, int64_t n,
                             const int64_t *row_ptr, const int32_t *col, double initiation,
                             double failure, int use_compression, double *bond_damage,
                             double *damage_index) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double yi[3];
  for (int c = 0; c < 3; ++c)
    yi[c] = __dadd_rn(pos[3 * i + c], disp[3 * i + c]);
  double damaged = 0.0, total = 0.0;
  for (int64_t q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
    const int64_t j = col[q];
    double e[3], y[3];
    for (int c = 0; c < 3; ++c) {
      e[c] = __dsub_rn(pos[3 * j + c], pos[3 * i + c]);
      y[c] = __dsub_rn(__dadd_rn(pos[3 * j + c], disp[3 * j + c]), yi[c]);
    }
    const double initial =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(e[0], e[0]), __dmul_rn(e[1], e[1])), __dmul_rn(e[2], e[2])));
    const double cur =
        __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(y[0], y[0]), __dmul_rn(y[1], y[1])), __dmul_rn(y[2], y[2])));
    const double stretch = __ddiv_rn(__dsub_rn(cur, initial), initial);
    if (stretch > initiation || (use_compression && stretch < -failure))
      bond_damage[q] = 1.0;
    damaged += bond_damage[q] * vol[j];
    total += vol[j];
  }
  if (damage_index)
    damage_index[i] = total > 0.0 ? damaged / total : 0.0;
}

// Johnson-Cook on one column-major block (the plugin ABI).
__global__ void k_vumat_block(int nb, JcParams jc, double dt, int nstatev, const double *strainInc,
                              const double *stressOld, const double *stateOld,
                              const double *enerInternOld, const double *enerInelasOld,
                              double *stressNew, double *stateNew, double *tempNew,
                              double *enerInternNew, double *enerInelasNew) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb)
    return;
  JcPoint pt;
  double inc[6];
  for (int c = 0; c < 6; ++c) {
    pt.stress[c] = stressOld[k + nb * c];
    inc[c] = strainInc[k + nb * c];
    pt.state[c] = stateOld[k + nb * c];
  }
  pt.eInternal = enerInternOld[k];
  pt.eInelastic = enerInelasOld[k];
  jc_update(jc, dt, inc, pt);
  for (int c = 0; c < 6; ++c) {
    stressNew[k + nb * c] = pt.stress[c];
    stateNew[k + nb * c] = pt.state[c];
  }
  for (int c = 6; c < nstatev; ++c)
    stateNew[k + nb * c] = stateOld[k + nb * c];
  tempNew[k] = pt.state[2];
  enerInternNew[k] = pt.eInternal;
  enerInelasNew[k] = pt.eInelastic;
}

static int check_status(unsigned *dstatus, cudaStream_t s) {
  unsigned st = 0;
  VPD_CUDA(cudaMemcpyAsync(&st, dstatus, sizeof st, cudaMemcpyDeviceToHost, s));
  VPD_CUDA(cudaStreamSynchronize(s));
  if (st & STATUS_SINGULAR_K)
    return set_error(VPD_ERR_SINGULAR, "Singular tensor in PD shape tensor.");
  if (st & STATUS_SINGULAR_F)
    return set_error(VPD_ERR_SINGULAR, "Invalid deformation gradient determinant.");
  if (st & STATUS_SINGULAR_KINEMATICS)
    return set_error(VPD_ERR_SINGULAR, "Corotational update encountered a singular tensor.");
  return VPD_OK;
}

// A device status word owned by the calling thread.
static unsigned *thread_status() {
  thread_local unsigned *word = nullptr;
  if (!word && cudaMalloc(&word, sizeof(unsigned)) != cudaSuccess)
    word = nullptr;
  return word;
}

static unsigned blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 127) / 128); }

}  // namespace vpd

using namespace vpd;

extern "C" {

int vpd_build_neighbor_list(const double *positions, int64_t n, double horizon, int64_t *row_ptr,
                            int32_t *col, int64_t *total, void *stream) {
  if (!positions || !row_ptr || !total || n <= 0)
    return set_error(VPD_ERR_INVALID, "vpd_build_neighbor_list: invalid argument");
  cudaStream_t s = (cudaStream_t)stream;
  double4 *xv = nullptr;
  VPD_CUDA(cudaMalloc(&xv, sizeof(double4) * n));
  k_pack_positions<<<blocks(n), 128, 0, s>>>(positions, n, xv);
  NeighborScratch scr;
  NeighborGrid grid;
  int rc = neighbor_scratch_alloc(scr, n);
  if (rc == VPD_OK)
    rc = neighbor_count(xv, n, horizon, row_ptr, grid, scr, s);
  if (rc == VPD_OK) {
    cudaError_t e = cudaMemcpyAsync(total, row_ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
      rc = cuda_error(e, "neighbour total");
  }
  if (rc == VPD_OK && col)
    rc = neighbor_fill(xv, n, row_ptr, col, grid, scr, s);
  neighbor_scratch_free(scr);
  cudaFree(xv);
  return rc;
}

int vpd_shape_tensor_inverse(const double *positions, const double *volumes, int64_t n,
                             const int64_t *row_ptr, const int32_t *col, double *kinv, void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  unsigned *st = thread_status();
  if (!st)
    return set_error(VPD_ERR_CUDA, "status word allocation failed");
  VPD_CUDA(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  k_csr_shape_inverse<<<blocks(n), 128, 0, s>>>(positions, volumes, n, row_ptr, col, kinv, st);
  VPD_CUDA(cudaGetLastError());
  return check_status(st, s);
}

int vpd_deformation_gradients(const double *positions, const double *displacement, const double *volumes,
                              int64_t n, const int64_t *row_ptr, const int32_t *col, const double *kinv,
                              double *defgrad, void *stream) {
  k_csr_deformation<<<blocks(n), 128, 0, (cudaStream_t)stream>>>(positions, displacement, volumes, n,
                                                                  row_ptr, col, kinv, defgrad);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int vpd_force_density(const double *positions, const double *volumes, int64_t n, const int64_t *row_ptr,
                      const int32_t *col, const double *kinv, const double *defgrad,
                      const double *cauchy_stress, const double *bond_damage, double *force,
                      void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  unsigned *st = thread_status();
  if (!st)
    return set_error(VPD_ERR_CUDA, "status word allocation failed");
  double *M = nullptr;
  VPD_CUDA(cudaMalloc(&M, sizeof(double) * 9 * std::max<int64_t>(n, 1)));
  VPD_CUDA(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  k_csr_force_map<<<blocks(n), 128, 0, s>>>(cauchy_stress, defgrad, kinv, n, M, st);
  k_csr_force<<<blocks(n), 128, 0, s>>>(positions, volumes, n, row_ptr, col, M, bond_damage, force);
  cudaError_t e = cudaGetLastError();
  const int rc = e == cudaSuccess ? check_status(st, s) : cuda_error(e, "force density");
  cudaFree(M);
  return rc;
}

int vpd_corotational_update(int64_t n, const double *defgrad_old, const double *defgrad_new,
                            const double *stretch_old, const double *rotation_old, double dt,
                            double *rate_of_deformation, double *relative_spin, double *rotation_new,
                            double *stretch_new, double *strain_new, void *stream) {
  if (!(dt > 0.0))
    return set_error(VPD_ERR_INVALID, "Corotational update requires dt > 0.");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned *st = thread_status();
  if (!st)
    return set_error(VPD_ERR_CUDA, "status word allocation failed");
  VPD_CUDA(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  k_corotational<<<blocks(n), 128, 0, s>>>(n, defgrad_old, defgrad_new, stretch_old, rotation_old, dt,
                                           rate_of_deformation, relative_spin, rotation_new, stretch_new,
                                           strain_new, st);
  VPD_CUDA(cudaGetLastError());
  return check_status(st, s);
}

int vpd_material_update(int64_t n, const double *props, int32_t nstatev, double dt, const double *defgrad_new,
                        double *defgrad_old, double *stretch, double *rotation, double *strain,
                        double *stress_corotational, double *state, double *temperature,
                        double *energy_internal, double *energy_inelastic, double *stress_spatial,
                        void *stream) {
  if (!props || nstatev < 6 || !(dt > 0.0))
    return set_error(VPD_ERR_INVALID, "VUMAT-PD material update requires props, nstatev >= 6 and dt > 0.");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned *st = thread_status();
  if (!st)
    return set_error(VPD_ERR_CUDA, "status word allocation failed");
  VPD_CUDA(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
  k_material_update<<<blocks(n), 128, 0, s>>>(n, make_jc_params(props), nstatev, dt, defgrad_new, defgrad_old,
                                              stretch, rotation, strain, stress_corotational, state,
                                              temperature, energy_internal, energy_inelastic, stress_spatial, st);
  VPD_CUDA(cudaGetLastError());
  return check_status(st, s);
}

int vpd_jc_return_map(int64_t n, const double *props, double dt, const double *strain_inc, const double *stress,
                      const double *state, int32_t nstatev, int32_t method, double *ep_inc, double *yield,
                      int32_t *iterations, void *stream) {
  if (!props || nstatev < 6 || !(dt > 0.0) || n < 0 || (method != 0 && method != 1))
    return set_error(VPD_ERR_INVALID, "JC return map requires props, nstatev >= 6, dt > 0, n >= 0 and method 0 or 1.");
  if (n == 0)
    return VPD_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const JcParams jc = make_jc_params(props);
  if (method == 0)
    k_jc_return_map<true><<<blocks(n), 128, 0, s>>>(n, jc, dt, strain_inc, stress, state, nstatev, ep_inc, yield,
                                                   iterations);
  else
    k_jc_return_map<false><<<blocks(n), 128, 0, s>>>(n, jc, dt, strain_inc, stress, state, nstatev, ep_inc, yield,
                                                    iterations);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int vpd_damage_update(const double *positions, const double *displacement, const double *volumes, int64_t n,
                      const int64_t *row_ptr, const int32_t *col, double initiation, double failure,
                      double *bond_damage, double *damage_index, void *stream) {
  if (!(initiation > 0.0))
    return set_error(VPD_ERR_INVALID, "critical_stretch requires initiation > 0.");
  const int use_compression = failure > 0.0 && std::isfinite(failure);
  k_csr_damage<<<blocks(n), 128, 0, (cudaStream_t)stream>>>(positions, displacement, volumes, n, row_ptr, col,
                                                            initiation, failure, use_compression, bond_damage,
                                                            damage_index);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

void vumat_adapter_call(int *nblock, int *ndir, int *nshr, int *nstatev, int *nfieldv, int *nprops,
                        int *lanneal, double *stepTime, double *totalTime, double *dt, char *cmname,
                        double *coordMp, double *charLength, double *props, double *density,
                        double *strainInc, double *relSpinInc, double *tempOld, double *stretchOld,
                        double *defgradOld, double *fieldOld, double *stressOld, double *stateOld,
                        double *enerInternOld, double *enerInelasOld, double *tempNew, double *stretchNew,
                        double *defgradNew, double *fieldNew, double *stressNew, double *stateNew,
                        double *enerInternNew, double *enerInelasNew) {
  (void)lanneal, (void)stepTime, (void)totalTime, (void)cmname, (void)coordMp, (void)charLength;
  (void)density, (void)relSpinInc, (void)tempOld;
  // The Fortran routine stops the process on these (JohnsonCook.f90:52-53); so does this entry.
  if (*ndir != 3 || *nshr != 3) {
    fprintf(stderr, "JohnsonCook VUMAT requires ndir=3,nshr=3\n");
    exit(1);
  }
  if (*nprops < 14 || *nstatev < 6) {
    fprintf(stderr, "JohnsonCook VUMAT requires 14 props and 6 states\n");
    exit(1);
  }
  const int nb = *nblock, nsv = *nstatev;
  // copy-through outputs (JohnsonCook.f90:84-90)
  std::memcpy(stretchNew, stretchOld, sizeof(double) * 6 * nb);
  std::memcpy(defgradNew, defgradOld, sizeof(double) * 9 * nb);
  if (*nfieldv > 0)
    std::memcpy(fieldNew, fieldOld, sizeof(double) * (size_t)(*nfieldv) * nb);
  // per-thread device block (the reference keeps one adapter per OpenMP thread)
  struct Block {
    cudaStream_t s = nullptr;
    double *buf = nullptr;
    size_t cap = 0;
  };
  thread_local Block blk;
  const size_t per = (size_t)(6 + 6 + nsv + 1 + 1 + 6 + nsv + 1 + 1 + 1);
  const size_t need = per * (size_t)nb;
  auto fail = [](cudaError_t e) {
    fprintf(stderr, "vumat_adapter_call: CUDA error %s\n", cudaGetErrorString(e));
    exit(1);
  };
  cudaError_t e = cudaSuccess;
  if (!blk.s && (e = cudaStreamCreateWithFlags(&blk.s, cudaStreamNonBlocking)) != cudaSuccess)
    fail(e);
  if (blk.cap < need) {
    cudaFree(blk.buf);
    if ((e = cudaMalloc(&blk.buf, need * sizeof(double))) != cudaSuccess)
      fail(e);
    blk.cap = need;
  }
  double *d_inc = blk.buf, *d_sold = d_inc + 6 * nb, *d_stold = d_sold + 6 * nb;
  double *d_eio = d_stold + (size_t)nsv * nb, *d_epo = d_eio + nb, *d_snew = d_epo + nb;
  double *d_stnew = d_snew + 6 * nb, *d_tnew = d_stnew + (size_t)nsv * nb, *d_ein = d_tnew + nb;
  double *d_epn = d_ein + nb;
  cudaStream_t s = blk.s;
  cudaMemcpyAsync(d_inc, strainInc, sizeof(double) * 6 * nb, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_sold, stressOld, sizeof(double) * 6 * nb, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_stold, stateOld, sizeof(double) * nsv * nb, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_eio, enerInternOld, sizeof(double) * nb, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_epo, enerInelasOld, sizeof(double) * nb, cudaMemcpyHostToDevice, s);
  k_vumat_block<<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(nb, make_jc_params(props), *dt, nsv, d_inc, d_sold,
                                                              d_stold, d_eio, d_epo, d_snew, d_stnew, d_tnew,
                                                              d_ein, d_epn);
  cudaMemcpyAsync(stressNew, d_snew, sizeof(double) * 6 * nb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(stateNew, d_stnew, sizeof(double) * nsv * nb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(tempNew, d_tnew, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(enerInternNew, d_ein, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(enerInelasNew, d_epn, sizeof(double) * nb, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
    fail(e);
}

}  // extern "C"
