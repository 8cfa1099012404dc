// The explicit increment on the device: three kernels per increment.
//
//   k_deformation  F = I + [sum_j V_j (u_j - u_i) (x) xi_ij] K^-1 over the sliced-ELL bonds,
//                  fused with critical-stretch bond breaking on the same gathered data
//                  (computeDeformationGradients :172-197, PdSimpleDamage::update :51-82)
//   k_material     corotational kinematics, the Johnson-Cook VUMAT, rotation to the spatial
//                  frame and the force map M = J sigma F^-T K^-1
//                  (VumatPdCorrespondenceMaterial::update :72-176, cauchyToFirstPiola :83-91)
//   k_force        f_i = sum_j (1 - d_ij) (M_i + M_j) xi_ij V_j (computeForceDensity :199-230)
//   k_integrate    velocity-Verlet correction, boundary conditions at t_n, diagnostics, then
//                  the next increment's displacement prediction with boundary conditions at
//                  t_n+1 (ExplicitTimeIntegrator.cpp:23-52, BoundaryConditions.cpp:81-115,
//                  BoundaryValueCaseRunner.cpp:231-306)
//
// One thread per point; the 32 points of a warp form one sliced-ELL slice, so the neighbour
// index loads are coalesced and the bond loop runs to the slice width with the tail masked.
// The increment number lives in device memory (*step), so the launch sequence is
// independent of the host and can be captured in a CUDA graph. Diagnostics are reduced
// deterministically: each block writes a partial, the last block of each group of k_integrate
// blocks sums its group's share, and the last group sums the groups in order and writes the
// increment's row.
#include "vpd_math.cuh"
#include <math_constants.h>
#include "vpd_material.cuh"
#include "vpd_step.cuh"

namespace vpd {

// Prescribed band kinematics: r[0..2] loaded band u, v, a; r[3..5] support band.
__device__ __forceinline__ void ramp(const BcParams &b, double t, double *r) {
  if (b.mode == VPD_BC_SMOOTH_DISPLACEMENT) {  // BoundaryConditions.cpp:70-79
    if (t >= b.rise_time) {
      r[0] = b.amplitude, r[1] = 0.0, r[2] = 0.0;
    } else {
      const double pi = 3.14159265358979323846;
      const double phase = pi * t / b.rise_time;
      r[0] = 0.5 * b.amplitude * (1.0 - cos(phase));
      r[1] = 0.5 * b.amplitude * pi / b.rise_time * sin(phase);
      r[2] = 0.5 * b.amplitude * pi * pi / (b.rise_time * b.rise_time) * cos(phase);
    }
    r[3] = r[4] = r[5] = 0.0;
    return;
  }
  // velocity ramp: +-v/2 per band, v rising linearly over ramp_time
  const double vh = 0.5 * b.grip_velocity, T = b.ramp_time;
  if (t < T) {
    r[0] = vh * (t * t / (2.0 * T));
    r[1] = vh * (t / T);
    r[2] = vh / T;
  } else {
    r[0] = vh * (t - 0.5 * T);
    r[1] = vh;
    r[2] = 0.0;
  }
  r[3] = -r[0], r[4] = -r[1], r[5] = -r[2];
}

// Read-only 32-byte load through the non-coherent path.
__device__ __forceinline__ double4 ldg4(const double4 *p) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
  const double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ double comp(const double4 &v, int d) {
  return d == 0 ? v.x : (d == 1 ? v.y : v.z);
}
__device__ __forceinline__ void set_comp(double4 &v, int d, double x) {
  if (d == 0) v.x = x; else if (d == 1) v.y = x; else v.z = x;
}

// RegionalConstraintSystem::apply order: support, loaded, anchor lateral, anchor z,
// rotation pin z, plane strain z.
__device__ __forceinline__ void apply_bc(const BcParams &b, uint8_t fl, const double *r,
                                         double4 &u, double4 &v, double4 &a) {
  if (fl & FLAG_SUPPORT)
    set_comp(u, b.axis, r[3]), set_comp(v, b.axis, r[4]), set_comp(a, b.axis, r[5]);
  if (fl & FLAG_LOADED)
    set_comp(u, b.axis, r[0]), set_comp(v, b.axis, r[1]), set_comp(a, b.axis, r[2]);
  if (fl & FLAG_ANCHOR) {
    set_comp(u, b.lateral, 0.0), set_comp(v, b.lateral, 0.0), set_comp(a, b.lateral, 0.0);
    if (!b.plane_strain)
      u.z = 0.0, v.z = 0.0, a.z = 0.0;
  }
  if ((fl & FLAG_ROTATION_PIN) && !b.plane_strain)
    u.z = 0.0, v.z = 0.0, a.z = 0.0;
  if (b.plane_strain)
    u.z = 0.0, v.z = 0.0, a.z = 0.0;
}

// ------------------------------------------------------------------ k_deformation
__device__ __noinline__ bool exact_break(const double4 &xi, const double4 &ui, const double4 &xj,
                                         const double4 &uj, double initiation, double failure,
                                         int use_compression) {
  // PdSimpleDamage.cpp:59-70 with every operation rounded as in the reference.
  const double yi0 = __dadd_rn(xi.x, ui.x), yi1 = __dadd_rn(xi.y, ui.y), yi2 = __dadd_rn(xi.z, ui.z);
  const double y0 = __dsub_rn(__dadd_rn(xj.x, uj.x), yi0);
  const double y1 = __dsub_rn(__dadd_rn(xj.y, uj.y), yi1);
  const double y2 = __dsub_rn(__dadd_rn(xj.z, uj.z), yi2);
  const double e0 = __dsub_rn(xj.x, xi.x), e1 = __dsub_rn(xj.y, xi.y), e2 = __dsub_rn(xj.z, xi.z);
  const double initial =
      __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(e0, e0), __dmul_rn(e1, e1)), __dmul_rn(e2, e2)));
  const double cur =
      __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(y0, y0), __dmul_rn(y1, y1)), __dmul_rn(y2, y2)));
  const double stretch = __ddiv_rn(__dsub_rn(cur, initial), initial);
  return stretch > initiation || (use_compression && stretch < -failure);
}

__global__ void __launch_bounds__(kBondThreads) k_deformation(StepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nsl = (p.n + 31) >> 5;
  if (i >= nsl * 32)
    return;
  const int64_t n = p.n;
  const int64_t s = i >> 5;
  const int lane = (int)(i & 31);
  const int64_t step = *p.step;
  const double4 *U = (step & 1) ? p.u1 : p.u0;
  const bool valid = i < n;
  const int64_t ii = valid ? i : 0;
  const double4 xi = p.xv[ii], ui = U[ii];
  const int len = valid ? p.len[i] : 0;
  const int64_t off = p.slice_off[s];
  const int width = (int)((p.slice_off[s + 1] - off) >> 5);
  const int32_t *idx = p.sell + off + lane;
  uint32_t *words = p.words + (off >> 5);
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double lo = 1.0 - 1.0e-9, hi = 1.0 + 1.0e-9;
  for (int k = 0; k < width; ++k) {
    const int32_t j = __ldg(idx + 32 * k);
    const double4 xj = ldg4(p.xv + j);
    const double4 uj = U[j];
    const bool act = k < len;
    const double w = act ? xj.w : 0.0;
    const double e0 = xj.x - xi.x, e1 = xj.y - xi.y, e2 = xj.z - xi.z;
    const double d0 = uj.x - ui.x, d1 = uj.y - ui.y, d2 = uj.z - ui.z;
    const double w0 = w * d0, w1 = w * d1, w2 = w * d2;
    G[0] += w0 * e0, G[1] += w0 * e1, G[2] += w0 * e2;
    G[3] += w1 * e0, G[4] += w1 * e1, G[5] += w1 * e2;
    G[6] += w2 * e0, G[7] += w2 * e1, G[8] += w2 * e2;
    if (p.damage) {
      const uint32_t word = words[k];
      bool broke = false;
      if (act && !((word >> lane) & 1u)) {
        const double y0 = e0 + d0, y1 = e1 + d1, y2 = e2 + d2;
        const double yy = y0 * y0 + y1 * y1 + y2 * y2;
        const double xx = e0 * e0 + e1 * e1 + e2 * e2;
        const double t = p.tension2 * xx;
        if (yy > t * hi)
          broke = true;
        else if (yy >= t * lo)
          broke = exact_break(xi, ui, xj, uj, p.dmg_initiation, p.dmg_failure, p.use_compression);
        else if (p.use_compression) {
          const double c = p.compression2 * xx;
          if (yy < c * lo)
            broke = true;
          else if (yy <= c * hi)
            broke = exact_break(xi, ui, xj, uj, p.dmg_initiation, p.dmg_failure, 1);
        }
      }
      const uint32_t fresh = __ballot_sync(0xffffffffu, broke);
      if (fresh && lane == 0)
        words[k] = word | fresh;
    }
  }
  if (!valid)
    return;
  double K[9];
#pragma unroll
  for (int c = 0; c < 9; ++c)
    K[c] = p.kinv[c * n + i];
  double GK[9];
  m_mul(G, K, GK);
#pragma unroll
  for (int c = 0; c < 9; ++c)
    p.F[c * n + i] = ((c % 4 == 0) ? 1.0 : 0.0) + GK[c];
}

// ------------------------------------------------------------------ k_material
// Four blocks per SM (128 registers, a few hundred bytes of spills to L1): the FP64 kinematics
// and return map are latency-bound, and the extra warps outweigh the spills (26 % faster on
// the 250k-point bar in plastic flow than at the unconstrained 196 registers; on the 1M-point
// bar in plastic flow 0.70 ms against 0.76 ms at three blocks per SM).
// POINT_DAMAGE: the point damage modes (a separate instance, so the plain one keeps its registers).
// CERTIFIED: the return map of jc_return_map (the bisection's results with fewer flow-stress
// evaluations); false, the literal bisection (VPD_RETURN_MAP=bisection).
template <bool POINT_DAMAGE, bool CERTIFIED>
__global__ void __launch_bounds__(kMaterialThreads, 4) k_material(const __grid_constant__ StepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double part[PM_COUNT] = {};
  double maxEqps = 0.0;
  if (i < p.n) {
    MaterialPoint m;
    material_load(p, i, m);
    jc_update<CERTIFIED>(p.jc, p.dt, m.inc, m.pt);
    material_store<POINT_DAMAGE>(p, i, m, part, maxEqps);
  }
  material_reduce(p, part, maxEqps, blockIdx.x);
}

// ------------------------------------------------------------------ k_force (sliced ELL)
// Bond sum of the force density: f = M_i sum V_j xi + sum (V_j M_j) xi over intact bonds.
__global__ void __launch_bounds__(kBondThreads) k_force(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nsl = (n + 31) >> 5;
  if (i >= nsl * 32)
    return;
  const int64_t s = i >> 5;
  const int lane = (int)(i & 31);
  const bool valid = i < n;
  const int64_t ii = valid ? i : 0;
  const double4 xi = p.xv[ii];
  const int len = valid ? p.len[i] : 0;
  const int64_t off = p.slice_off[s];
  const int width = (int)((p.slice_off[s + 1] - off) >> 5);
  const int32_t *idx = p.sell + off + lane;
  const uint32_t *words = p.words + (off >> 5);
  double f0 = 0, f1 = 0, f2 = 0, s0 = 0, s1 = 0, s2 = 0;
  for (int k = 0; k < width; ++k) {
    const int32_t j = __ldg(idx + 32 * k);
    const double4 xj = ldg4(p.xv + j);
    const bool intact = k < len && !(p.damage && ((words[k] >> lane) & 1u));
    const double w = intact ? xj.w : 0.0, g = intact ? 1.0 : 0.0;
    const double e0 = xj.x - xi.x, e1 = xj.y - xi.y, e2 = xj.z - xi.z;
    s0 += w * e0, s1 += w * e1, s2 += w * e2;
    const double2 *Mj = reinterpret_cast<const double2 *>(p.Mt + 10 * (int64_t)j);
    const double2 a = __ldg(Mj), b = __ldg(Mj + 1), c = __ldg(Mj + 2), d = __ldg(Mj + 3),
                  h = __ldg(Mj + 4);
    f0 += g * (a.x * e0 + a.y * e1 + b.x * e2);
    f1 += g * (b.y * e0 + c.x * e1 + c.y * e2);
    f2 += g * (d.x * e0 + d.y * e1 + h.x * e2);
  }
  if (!valid)
    return;
  const double *Mi = p.Mt + 10 * i;
  const double rv = 1.0 / xi.w;  // M_i = (V_i M_i) / V_i
  f0 += (Mi[0] * s0 + Mi[1] * s1 + Mi[2] * s2) * rv;
  f1 += (Mi[3] * s0 + Mi[4] * s1 + Mi[5] * s2) * rv;
  f2 += (Mi[6] * s0 + Mi[7] * s1 + Mi[8] * s2) * rv;
  p.force[i] = make_double4(f0, f1, f2, 0.0);
}

// ------------------------------------------------------------------ k_integrate
// Velocity-Verlet correction with the force density, constraints at t_n, diagnostics, then
// the next increment's prediction with constraints at t_n+1; the last block writes the row.
__global__ void __launch_bounds__(kBondThreads, 3) k_integrate(StepParams p) {
  const int64_t n = p.n;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t step = *p.step;
  double part[PF_COUNT] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double4 fv = p.force[i];
    const double f0 = fv.x, f1 = fv.y, f2 = fv.z;
    const double4 *Ucur = (step & 1) ? p.u1 : p.u0;
    double4 *Unext = (step & 1) ? p.u0 : p.u1;
    double4 u = Ucur[i], v = p.vel[i], a = p.acc[i];
    const uint8_t fl = p.flags[i];
    const double dt = p.dt, rho = p.rho;
    double4 an = make_double4(f0 / rho, f1 / rho, f2 / rho, 0.0);
    v.x += 0.5 * dt * (a.x + an.x);
    v.y += 0.5 * dt * (a.y + an.y);
    v.z += 0.5 * dt * (a.z + an.z);
    a = an;
    const double t = (double)step * dt;
    double r[6];
    if (fl & (FLAG_SUPPORT | FLAG_LOADED))
      ramp(p.bc, t, r);
    apply_bc(p.bc, fl, r, u, v, a);
    p.vel[i] = v;
    p.acc[i] = a;
    const double vol = p.xv[i].w;
    part[PF_NETX] = f0 * vol, part[PF_NETY] = f1 * vol, part[PF_NETZ] = f2 * vol;
    const double fax = p.bc.axis == 0 ? f0 : f1;
    if (fl & FLAG_LOADED)
      part[PF_REACTION] = (rho * r[2] - fax) * vol;
    if (fl & FLAG_SUPPORT)
      part[PF_SUPPORT_REACTION] = (rho * r[5] - fax) * vol;
    part[PF_KINETIC] = 0.5 * rho * vol * (v.x * v.x + v.y * v.y + v.z * v.z);
    const double ul = comp(u, p.bc.lateral);
    if (fl & FLAG_LATERAL_POS)
      part[PF_LAT_POS] = ul;
    if (fl & FLAG_LATERAL_NEG)
      part[PF_LAT_NEG] = ul;
    part[PF_NONFINITE] = (isfinite(f0) && isfinite(f1) && isfinite(f2)) ? 0.0 : 1.0;
    // predict the next increment (ExplicitTimeIntegrator.cpp:23-34) and constrain at t+dt
    double4 un = make_double4(u.x + (dt * v.x + 0.5 * dt * dt * a.x),
                              u.y + (dt * v.y + 0.5 * dt * dt * a.y),
                              u.z + (dt * v.z + 0.5 * dt * dt * a.z), 0.0);
    if (fl) {
      double rn[6];
      if (fl & (FLAG_SUPPORT | FLAG_LOADED))
        ramp(p.bc, (double)(step + 1) * dt, rn);
      double4 vv = v, aa = a;
      apply_bc(p.bc, fl, rn, un, vv, aa);
    }
    if (p.bc.plane_strain)
      un.z = 0.0;
    Unext[i] = un;
    if (p.mixed)
      p.uf[i] = make_float4((float)un.x, (float)un.y, (float)un.z, 0.0f);
  }
  block_partials<PF_COUNT>(part, p.part_force, blockIdx.x);

  // Two-level reduction, deterministic: the last block of each group of kGroupBlocks blocks sums
  // the group's force partials and its share of the material partials (each thread its slots in
  // slot order, then a fixed tree); the last group to finish sums the group partials in group
  // order and writes the diagnostic row. Every slot is read by one thread of one block, so the
  // reads run in parallel instead of one block walking all of them.
  constexpr int Q = PM_COUNT + PF_COUNT;
  const int ngroups = (int)((gridDim.x + kGroupBlocks - 1) / kGroupBlocks);
  const int g = (int)(blockIdx.x / kGroupBlocks), gfirst = g * kGroupBlocks;
  const int gcount = min(kGroupBlocks, (int)gridDim.x - gfirst);
  // the threads that wrote the block's partials make them visible device-wide, and the barrier
  // orders that before the block is counted
  __shared__ bool last;
  if (threadIdx.x < PF_COUNT)
    __threadfence();
  __syncthreads();
  if (threadIdx.x == 0)
    last = atomicAdd(p.group_counter + g, 1u) == (unsigned)gcount - 1u;
  __syncthreads();
  if (!last)
    return;
  double acc[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q)
    acc[q] = 0.0;
  const int ms = (p.mat_blocks + ngroups - 1) / ngroups;
  const int mlo = g * ms, mhi = min(p.mat_blocks, mlo + ms);
  for (int b = mlo + (int)threadIdx.x; b < mhi; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < PM_COUNT; ++q) {
      const double v = __ldcg(p.part_mat + (size_t)b * PM_COUNT + q);
      acc[q] = q == PM_MAX_EQPS ? fmax(acc[q], v) : acc[q] + v;
    }
  for (int b = gfirst + (int)threadIdx.x; b < gfirst + gcount; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < PF_COUNT; ++q)
      acc[PM_COUNT + q] += __ldcg(p.part_force + (size_t)b * PF_COUNT + q);
  __shared__ double red[kBondThreads / 32][Q];
  __shared__ double tot[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, acc[q], o);
      acc[q] = q == PM_MAX_EQPS ? fmax(acc[q], y) : acc[q] + y;
    }
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < Q; ++q)
      red[threadIdx.x >> 5][q] = acc[q];
  __syncthreads();
  if (threadIdx.x < Q) {
    const int q = threadIdx.x;
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      s = q == PM_MAX_EQPS ? fmax(s, red[w][q]) : s + red[w][q];
    p.part_group[(size_t)g * Q + q] = s;
  }
  if (threadIdx.x == 0)
    p.group_counter[g] = 0u;  // ready for the next increment
  __shared__ bool final_group;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0)
    final_group = atomicAdd(p.counter, 1u) == (unsigned)ngroups - 1u;
  __syncthreads();
  if (!final_group)
    return;
  if (threadIdx.x < Q) {
    const int q = threadIdx.x;
    double s = 0.0;
    for (int gg = 0; gg < ngroups; ++gg) {
      const double v = __ldcg(p.part_group + (size_t)gg * Q + q);
      s = q == PM_MAX_EQPS ? fmax(s, v) : s + v;
    }
    tot[q] = s;
  }
  __syncthreads();
  if (threadIdx.x != 0)
    return;
  const double *pm = tot, *pf = tot + PM_COUNT;
  double *A = p.accum;
  const double dt = p.dt, time = (double)step * dt;
  double r[6];
  ramp(p.bc, time, r);
  A[ACC_INTERNAL] += pm[PM_DU];
  const double avgS = pm[PM_AVG_STRESS] / p.interior, avgE = pm[PM_AVG_STRAIN] / p.interior;
  const double reaction = pf[PF_REACTION];
  const double power = reaction * r[1] +
                       (p.bc.mode == VPD_BC_VELOCITY_RAMP ? pf[PF_SUPPORT_REACTION] * r[4] : 0.0);
  A[ACC_EXTERNAL] += 0.5 * dt * (A[ACC_PREV_POWER] + power);
  A[ACC_PREV_POWER] = power;
  const double kinetic = pf[PF_KINETIC];
  double scale = fmax(fabs(A[ACC_EXTERNAL]), fabs(A[ACC_INTERNAL]) + kinetic);
  scale = fmax(scale, 1.0e-12);
  const double energyError = fabs(kinetic + A[ACC_INTERNAL] - A[ACC_EXTERNAL]) / scale;
  const bool finite = A[ACC_FINITE] != 0.0 && pm[PM_NONFINITE] == 0.0 &&
                      pf[PF_NONFINITE] == 0.0 && isfinite(kinetic) &&
                      isfinite(A[ACC_INTERNAL]) && isfinite(A[ACC_EXTERNAL]) &&
                      isfinite(energyError);
  A[ACC_FINITE] = finite ? 1.0 : 0.0;
  double *row = p.diag + (size_t)((step - 1) % kDiagRing) * VPD_DIAG_COLS;
  row[VPD_DIAG_STEP] = (double)step;
  row[VPD_DIAG_TIME] = time;
  row[VPD_DIAG_LOAD_DISPLACEMENT] = r[0];
  row[VPD_DIAG_LOAD_VELOCITY] = r[1];
  row[VPD_DIAG_REACTION] = reaction;
  row[VPD_DIAG_ENGINEERING_STRAIN] = p.sign * (r[0] - r[3]) / p.gauge;
  row[VPD_DIAG_LATERAL_STRAIN] =
      (pf[PF_LAT_POS] / p.n_lat_pos - pf[PF_LAT_NEG] / p.n_lat_neg) / p.lat_gauge;
  row[VPD_DIAG_NOMINAL_STRESS] = p.sign * reaction / p.area;
  row[VPD_DIAG_AVERAGE_AXIAL_STRAIN] = avgE;
  row[VPD_DIAG_AVERAGE_AXIAL_STRESS] = avgS;
  row[VPD_DIAG_MAX_EQPS] = pm[PM_MAX_EQPS];
  row[VPD_DIAG_MAX_INTERNAL_INDICATOR] = 0.0;
  row[VPD_DIAG_KINETIC_ENERGY] = kinetic;
  row[VPD_DIAG_INTERNAL_ENERGY] = A[ACC_INTERNAL];
  row[VPD_DIAG_EXTERNAL_WORK] = A[ACC_EXTERNAL];
  row[VPD_DIAG_ENERGY_ERROR] = energyError;
  row[VPD_DIAG_NET_INTERNAL_FORCE] =
      sqrt(pf[PF_NETX] * pf[PF_NETX] + pf[PF_NETY] * pf[PF_NETY] + pf[PF_NETZ] * pf[PF_NETZ]);
  row[VPD_DIAG_FINITE] = finite ? 1.0 : 0.0;
  row[VPD_DIAG_PLASTIC_POINTS] = pm[PM_PLASTIC];
  row[VPD_DIAG_FALLBACK_POINTS] = pm[PM_FALLBACK];
  *p.counter = 0u;
  *p.step = step + 1;
}

// ------------------------------------------------------------------ k_indicator
// The case's internal indicator (internalIndicator, BoundaryValueCaseRunner.cpp:93-107,
// :258-263): per point the min or max of the chosen state variables (optionally 1 - it), and
// per increment the largest of them and 0, into the row k_integrate has just written (which
// holds 0 there). Launched after k_integrate, only when the case configures an indicator.
// The running value starts at 0 and takes no NaN (std::max keeps its first argument), so it is
// never negative, and the IEEE bits of non-negative doubles order as the numbers: the blocks
// combine with a 64-bit atomicMax.
__global__ void __launch_bounds__(kBondThreads) k_indicator(const __grid_constant__ StepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < p.n) {
    double value = p.ind_min ? CUDART_INF : -CUDART_INF;
    for (int k = 0; k < p.ind_count; ++k) {
      const double item = p.state[(int64_t)p.ind_idx[k] * p.n + i];
      value = p.ind_min ? (item < value ? item : value) : (value < item ? item : value);
    }
    if (p.ind_one_minus)
      value = 1.0 - value;
    v = v < value ? value : v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = v < w ? w : v;
  }
  __shared__ double warp_max[kBondThreads / 32];
  if ((threadIdx.x & 31) == 0)
    warp_max[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      v = v < warp_max[w] ? warp_max[w] : v;
    const int64_t step = *p.step - 1;  // the increment k_integrate has just closed
    double *slot = p.diag + (size_t)((step - 1) % kDiagRing) * VPD_DIAG_COLS + VPD_DIAG_MAX_INTERNAL_INDICATOR;
    atomicMax(reinterpret_cast<unsigned long long *>(slot), (unsigned long long)__double_as_longlong(v));
  }
}

// ------------------------------------------------------------------ set-up kernels
// Constraints at t = 0 and the first displacement prediction (BoundaryValueCaseRunner.cpp:190,
// then predictDisplacement + apply at t = dt).
__global__ void k_init(StepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n)
    return;
  const uint8_t fl = p.flags[i];
  double4 u = make_double4(0, 0, 0, 0), v = u, a = u;
  double r[6] = {0, 0, 0, 0, 0, 0};
  if (fl & (FLAG_SUPPORT | FLAG_LOADED))
    ramp(p.bc, 0.0, r);
  apply_bc(p.bc, fl, r, u, v, a);
  p.u0[i] = u;
  p.vel[i] = v;
  p.acc[i] = a;
  p.force[i] = make_double4(0, 0, 0, 0);
  const double dt = p.dt;
  double4 un = make_double4(u.x + (dt * v.x + 0.5 * dt * dt * a.x),
                            u.y + (dt * v.y + 0.5 * dt * dt * a.y),
                            u.z + (dt * v.z + 0.5 * dt * dt * a.z), 0.0);
  if (fl & (FLAG_SUPPORT | FLAG_LOADED))
    ramp(p.bc, dt, r);
  double4 vv = v, aa = a;
  apply_bc(p.bc, fl, r, un, vv, aa);
  if (p.bc.plane_strain)
    un.z = 0.0;
  p.u1[i] = un;
  // material state: F_n = V_n = R_n = I, zero strain, stress, state and energies
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    const double id = (c % 4 == 0) ? 1.0 : 0.0;
    p.Fn[c * p.n + i] = id;
    p.Vn[c * p.n + i] = id;
    p.Rn[c * p.n + i] = id;
  }
  if (p.Mt)
    for (int c = 0; c < 10; ++c)
      p.Mt[10 * i + c] = 0.0;
  for (int c = 0; c < 6; ++c)
    p.En[c * p.n + i] = 0.0, p.sig[c * p.n + i] = 0.0;
  for (int c = 0; c < p.nstatev; ++c)
    p.state[c * p.n + i] = 0.0;
  p.eI[i] = 0.0;
  p.eP[i] = 0.0;
}

// K_i = sum_j V_j xi (x) xi and its inverse (PdCorrespondenceSkeleton::initialize :149-170).
__global__ void __launch_bounds__(kBondThreads) k_shape_inverse(StepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = p.n;
  if (i >= n)
    return;
  const int64_t s = i >> 5;
  const int lane = (int)(i & 31);
  const double4 xi = p.xv[i];
  const int len = p.len[i];
  const int32_t *idx = p.sell + p.slice_off[s] + lane;
  double K[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < len; ++k) {
    const double4 xj = p.xv[idx[32 * k]];
    const double e[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
        K[3 * a + b] += xj.w * e[a] * e[b];
  }
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

int material_grid(int64_t n) { return (int)((n + kMaterialThreads - 1) / kMaterialThreads); }
static unsigned bond_grid(int64_t n) { return (unsigned)(((n + 31) / 32 * 32 + kBondThreads - 1) / kBondThreads); }

int launch_init(const StepParams &p, cudaStream_t s) {
  k_init<<<(unsigned)((p.n + 255) / 256), 256, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int launch_shape_inverse_sell(const StepParams &p, cudaStream_t s) {
  k_shape_inverse<<<(unsigned)((p.n + kBondThreads - 1) / kBondThreads), kBondThreads, 0, s>>>(p);
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int integrate_grid(int64_t n) { return (int)((n + kBondThreads - 1) / kBondThreads); }

int launch_stage(int stage, const StepParams &p, cudaStream_t s) {
  if (stage == 0) {
    if (p.mixed)
      return p.tiled ? launch_deformation_tiled(p, s) : launch_deformation_mixed(p, s);
    if (p.st.nw)
      return p.tiled ? launch_deformation_tiled64(p, s) : launch_deformation_stencil(p, s);
    k_deformation<<<bond_grid(p.n), kBondThreads, 0, s>>>(p);
  } else if (stage == 1) {
    if (p.host_vumat)
      return launch_material_host(p, s);
    if (p.surrogate)
      return launch_material_surrogate(p, s);
    const unsigned grid = (unsigned)material_grid(p.n);
    if (p.point_damage)
      p.literal_bisection ? k_material<true, false><<<grid, kMaterialThreads, 0, s>>>(p)
                          : k_material<true, true><<<grid, kMaterialThreads, 0, s>>>(p);
    else
      p.literal_bisection ? k_material<false, false><<<grid, kMaterialThreads, 0, s>>>(p)
                          : k_material<false, true><<<grid, kMaterialThreads, 0, s>>>(p);
  } else if (stage == 2) {
    if (p.mixed)
      return p.tiled ? launch_force_tiled(p, s) : launch_force_mixed(p, s);
    if (p.st.nw)
      return p.tiled ? launch_force_tiled64(p, s) : launch_force_stencil(p, s);
    k_force<<<bond_grid(p.n), kBondThreads, 0, s>>>(p);
  } else {
    k_integrate<<<(unsigned)integrate_grid(p.n), kBondThreads, 0, s>>>(p);
    if (p.ind_count)
      k_indicator<<<(unsigned)((p.n + kBondThreads - 1) / kBondThreads), kBondThreads, 0, s>>>(p);
  }
  VPD_CUDA(cudaGetLastError());
  return VPD_OK;
}

int launch_increment(const StepParams &p, cudaStream_t s) {
  for (int stage = 0; stage < kStages; ++stage) {
    int rc = launch_stage(stage, p, s);
    if (rc)
      return rc;
  }
  return VPD_OK;
}

}  // namespace vpd
