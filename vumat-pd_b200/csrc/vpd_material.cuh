// Per-point body of the material stage, shared by k_material (vpd_step.cu) and the surrogate
// material kernel (vpd_surrogate.cu): F, the corotational update and the VUMAT's old state
// (material_load); then, after the constitutive update, the spatial stress, the force map,
// the history commit and the block's diagnostic partials (material_store).
// VumatPdCorrespondenceMaterial::update (src/pd/VumatPdCorrespondenceMaterial.cpp:72-176) with
// the kinematics of CorotationalKinematics.cpp:61-149.
#pragma once

#include "vpd_math.cuh"
#include "vpd_step.cuh"

namespace vpd {

// Block-wide sums of K doubles; thread 0 writes them to out[slot * K].
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double *out, int64_t slot) {
  __shared__ double red[32][K];
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k)
      red[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w)
      s += red[w][threadIdx.x];
    out[(size_t)slot * K + threadIdx.x] = s;
  }
}

// One point's material context across the constitutive update. The kinematic history (F, V,
// R, E) is written as soon as it is formed (material_load), so of the kinematics only F and R
// (the force map's and the stress rotation's inputs) stay live across the return map.
struct MaterialPoint {
  double F[9];    // deformation gradient of this increment
  double R[9];    // rotation R_{n+1}
  double inc[6];  // corotational strain increment (Voigt, tensor shear)
  double dE[6];   // E_{n+1} - E_n, for the internal-energy diagnostic
  double eAxis;   // E_{n+1} along the loading axis, for the observation-window mean
  bool eFinite;   // every component of E_{n+1} finite
  JcPoint pt;     // VUMAT stress, state and energies (old on entry to the update)
};

__device__ __forceinline__ void material_load(const StepParams &p, int64_t i, MaterialPoint &m) {
  const int64_t n = p.n;
  JcPoint &pt = m.pt;
  double(&F)[9] = m.F;
  double Fn[9], Vn[9], Rn[9], Eold[6];
  // every load first (one memory round trip; the stores below would otherwise order them)
  if (p.mixed) {  // F = I + G K^-1 in FP64 from the FP32 bond sum
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
  for (int c = 0; c < 6; ++c) {
    Eold[c] = p.En[c * n + i];
    pt.stress[c] = p.sig[c * n + i];
    pt.state[c] = p.state[c * n + i];
  }
  pt.eInternal = p.eI[i];
  pt.eInelastic = p.eP[i];
  Corotational co;
  if (!corotational_update(Fn, F, Vn, Rn, p.dt, co)) {
    atomicOr(p.status, STATUS_SINGULAR_KINEMATICS);
#pragma unroll
    for (int c = 0; c < 9; ++c)
      co.dbar[c] = 0.0, co.spin[c] = 0.0, co.r[c] = Rn[c], co.v[c] = Vn[c];
  }
  double E[6];
  green_lagrange6(F, E);
  // kinematic history of this increment, committed now
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    p.Fn[c * n + i] = F[c];
    p.Vn[c * n + i] = co.v[c];
    p.Rn[c * n + i] = co.r[c];
    m.R[c] = co.r[c];
  }
  m.eFinite = true;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    m.dE[c] = E[c] - Eold[c];
    p.En[c * n + i] = E[c];
    m.eFinite = m.eFinite && isfinite(E[c]);
  }
  // selects rather than a runtime index, which would put the array in local memory
  const int ax = p.bc.axis;
  m.eAxis = ax == 0 ? E[0] : (ax == 1 ? E[1] : E[2]);
  const double *d = co.dbar;
  m.inc[0] = d[0] * p.dt, m.inc[1] = d[4] * p.dt, m.inc[2] = d[8] * p.dt;
  m.inc[3] = 0.5 * (d[5] + d[7]) * p.dt, m.inc[4] = 0.5 * (d[2] + d[6]) * p.dt;
  m.inc[5] = 0.5 * (d[1] + d[3]) * p.dt;
}

// The point damage modes (SimpleDamageModel::update and degradeStress, SimpleDamageModel.cpp:14-50):
// the point's damage from this increment's metric (the new eqps, or the largest principal
// strain of E_n+1), kept non-decreasing, and the factor its spatial stress takes before the
// force map.
static __device__ __noinline__ double point_damage_factor(int mode, int deletion, double initiation, double failure,
                                                   double *pdmg, const double *En, int64_t n, int64_t i,
                                                   double eqps) {
  double metric = eqps;  // state variable 2 (eqpsStateIndex 1)
  if (mode == VPD_DAMAGE_MAX_PRINCIPAL_STRAIN) {
    double E[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
      E[c] = En[c * n + i];  // E_n+1, committed by material_load
    metric = max_principal6(E);
  }
  const double t = (metric - initiation) / (failure - initiation);
  const double clamped = t < 0.0 ? 0.0 : (1.0 < t ? 1.0 : t);
  const double prev = pdmg[i];
  const double dmg = prev < clamped ? clamped : prev;
  pdmg[i] = dmg;
  if (deletion && dmg >= 1.0)
    return 0.0;
  return 1.0 - (dmg < 0.0 ? 0.0 : (1.0 < dmg ? 1.0 : dmg));
}

// part[PM_*] and maxEqps receive this point's diagnostic contributions. POINT_DAMAGE compiles
// in the point damage modes (kernels without it keep their registers).
template <bool POINT_DAMAGE = false>
__device__ __forceinline__ void material_store(const StepParams &p, int64_t i, const MaterialPoint &m, double *part,
                                               double &maxEqps) {
  const int64_t n = p.n;
  const JcPoint &pt = m.pt;
  const double(&F)[9] = m.F;
  const double(&R)[9] = m.R;
  double K[9], old[6], oldFull[9], full[9], spatial[9], M[9];
#pragma unroll
  for (int c = 0; c < 9; ++c)
    K[c] = p.kinv[c * n + i];
#pragma unroll
  for (int c = 0; c < 6; ++c)
    old[c] = p.sig[c * n + i];  // the old stress, still in place
  voigt_to_full(old, oldFull);
  voigt_to_full(pt.stress, full);
  rotate_to_spatial(full, R, spatial);
  bool mapped;
  if (POINT_DAMAGE && p.point_damage) {
    // the effective stress of the force map (PdSimpleDamage.cpp:86-92); the diagnostics below
    // keep the undegraded stress, as the reference's runner reads rawStress
    // (BoundaryValueCaseRunner.cpp:231-259)
    const double factor = point_damage_factor(p.point_damage, p.dmg_deletion, p.dmg_initiation, p.dmg_failure,
                                              p.pdmg, p.En, n, i, pt.state[1]);
    double effective[9];
#pragma unroll
    for (int c = 0; c < 9; ++c)
      effective[c] = spatial[c] * factor;
    mapped = force_map(effective, F, K, M);
  } else {
    mapped = force_map(spatial, F, K, M);
  }
  if (!mapped) {
    atomicOr(p.status, STATUS_SINGULAR_F);
#pragma unroll
    for (int c = 0; c < 9; ++c)
      M[c] = 0.0;
  }
  // the force map scaled by the point's volume, in the layout the force kernel gathers
  const double4 xi = p.xv[i];
  const double vol = xi.w;
  if (p.mixed) {
    // the records of fmap_record (vpd_bond.cuh): VM = V M and R = VM J in FP32
    const float4 ji = p.jit[i];
    double VM[9], R[3];
#pragma unroll
    for (int c = 0; c < 9; ++c)
      VM[c] = vol * M[c];
#pragma unroll
    for (int r = 0; r < 3; ++r)
      R[r] = VM[3 * r] * (double)ji.x + VM[3 * r + 1] * (double)ji.y + VM[3 * r + 2] * (double)ji.z;
    p.fmapf[i] = make_float4((float)VM[0], (float)VM[3], (float)VM[1], (float)VM[4]);
    p.fmapf[n + i] = make_float4((float)VM[2], (float)VM[5], (float)R[0], (float)R[1]);
    p.fmapf[2 * n + i] = make_float4((float)VM[6], (float)VM[7], (float)VM[8], (float)R[2]);
  } else if (p.fmap) {
    const double xr[3] = {xi.x, xi.y, xi.z};
#pragma unroll
    for (int r = 0; r < 3; ++r)
      st256(p.fmap + r * n + i, make_double4(vol * M[3 * r], vol * M[3 * r + 1], vol * M[3 * r + 2], xr[r]));
  } else {
    double2 *Mt = reinterpret_cast<double2 *>(p.Mt + 10 * i);
    Mt[0] = make_double2(vol * M[0], vol * M[1]);
    Mt[1] = make_double2(vol * M[2], vol * M[3]);
    Mt[2] = make_double2(vol * M[4], vol * M[5]);
    Mt[3] = make_double2(vol * M[6], vol * M[7]);
    Mt[4] = make_double2(vol * M[8], 0.0);
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    p.sig[c * n + i] = pt.stress[c];
    p.state[c * n + i] = pt.state[c];
  }
  p.eI[i] = pt.eInternal;
  p.eP[i] = pt.eInelastic;
  // diagnostics: internal-energy increment with the reference's mixed-frame average
  // (BoundaryValueCaseRunner.cpp:231-238), observation-window means, max eqps, finiteness
  const double a0 = 0.5 * (oldFull[0] + spatial[0]), a4 = 0.5 * (oldFull[4] + spatial[4]);
  const double a8 = 0.5 * (oldFull[8] + spatial[8]), a1 = 0.5 * (oldFull[1] + spatial[1]);
  const double a2 = 0.5 * (oldFull[2] + spatial[2]), a5 = 0.5 * (oldFull[5] + spatial[5]);
  const double *dE = m.dE;
  part[PM_DU] = (a0 * dE[0] + a4 * dE[1] + a8 * dE[2] + 2.0 * (a1 * dE[5] + a2 * dE[4] + a5 * dE[3])) * vol;
  const double w = p.obsw[i];
  if (w > 0.0) {
    const int ax = p.bc.axis;
    const double sa = ax == 0 ? spatial[0] : (ax == 1 ? spatial[4] : spatial[8]);
    part[PM_AVG_STRESS] = p.sign * sa * w;
    part[PM_AVG_STRAIN] = p.sign * m.eAxis * w;
  }
  maxEqps = pt.state[1];
  bool fin = m.eFinite;
#pragma unroll
  for (int c = 0; c < 9; ++c)
    fin = fin && isfinite(spatial[c]);
#pragma unroll
  for (int c = 0; c < 6; ++c)
    fin = fin && isfinite(pt.state[c]);
  part[PM_NONFINITE] = fin ? 0.0 : 1.0;
  part[PM_PLASTIC] = pt.state[4] > 0.0 ? 1.0 : 0.0;
}

// Reduces the block's partials of one 128-point tile into p.part_mat[slot] (sums; max for
// PM_MAX_EQPS). Every thread of the block calls it (it contains __syncthreads).
__device__ __forceinline__ void material_reduce(const StepParams &p, double (&part)[PM_COUNT], double maxEqps,
                                                int64_t slot) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    maxEqps = fmax(maxEqps, __shfl_xor_sync(0xffffffffu, maxEqps, o));
  __shared__ double smax[32];
  if ((threadIdx.x & 31) == 0)
    smax[threadIdx.x >> 5] = maxEqps;
  block_partials<PM_COUNT>(part, p.part_mat, slot);  // contains __syncthreads
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      m = fmax(m, smax[w]);
    p.part_mat[(size_t)slot * PM_COUNT + PM_MAX_EQPS] = m;
  }
  __syncthreads();  // smax and block_partials' buffer are reused by the next tile
}

}  // namespace vpd
