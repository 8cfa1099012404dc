// Parameters and launchers of the per-increment kernels (vpd_step.cu).
#pragma once

#include "vpd_internal.h"

namespace vpd {

struct BcParams {
  int mode;  // VPD_BC_*
  double amplitude, rise_time, grip_velocity, ramp_time;
  int axis, lateral, plane_strain;
};

// Quantities each material block reduces (sums except the max).
enum { PM_DU = 0, PM_AVG_STRESS, PM_AVG_STRAIN, PM_MAX_EQPS, PM_NONFINITE, PM_COUNT };
// Quantities each force block reduces (sums).
enum {
  PF_NETX = 0, PF_NETY, PF_NETZ, PF_REACTION, PF_SUPPORT_REACTION, PF_KINETIC, PF_LAT_POS,
  PF_LAT_NEG, PF_NONFINITE, PF_COUNT
};
// Running sums kept on the device between increments.
enum { ACC_INTERNAL = 0, ACC_EXTERNAL, ACC_PREV_POWER, ACC_FINITE, ACC_COUNT };

constexpr int kDiagRing = 4096;      // diagnostic rows buffered on the device
constexpr int kBondThreads = 256;    // threads per block of the bond kernels
constexpr int kMaterialThreads = 128;

struct StepParams {
  int64_t n;
  double dt, rho;
  // geometry and bonds
  const double4 *xv;          // x, y, z, volume
  const int32_t *len;         // neighbours per point
  const int64_t *slice_off;   // sliced-ELL slice offsets
  const int32_t *sell;        // sliced-ELL neighbour indices
  uint32_t *words;            // broken-bond bits, one word per (slice, column)
  // kinematic state
  double4 *u0, *u1;           // displacement ping-pong: increment s reads u[s & 1]
  double4 *vel, *acc, *force;
  // material state, structure of arrays (component c of point i at [c * n + i])
  const double *kinv;
  double *F, *Fn, *Vn, *Rn, *En, *sig, *state, *eI, *eP, *M;
  int nstatev;
  // boundary and diagnostics sets
  const uint8_t *flags;
  const double *obsw;
  JcParams jc;
  BcParams bc;
  int damage;
  double dmg_initiation, dmg_failure, tension2, compression2;
  int use_compression;
  // device bookkeeping
  int64_t *step;              // increment being computed (1-based)
  unsigned int *status;
  double *part_mat, *part_force, *accum, *diag;
  unsigned int *counter;
  int mat_blocks;
  // diagnostic constants
  double interior, gauge, lat_gauge, area, sign, n_lat_pos, n_lat_neg;
};

// The increment's kernels, in order: deformation (+ bond breaking), material, force.
constexpr int kStages = 3;
int launch_init(const StepParams &p, cudaStream_t s);
int launch_stage(int stage, const StepParams &p, cudaStream_t s);
int launch_increment(const StepParams &p, cudaStream_t s);
int launch_shape_inverse_sell(const StepParams &p, cudaStream_t s);
int material_grid(int64_t n);

}  // namespace vpd
