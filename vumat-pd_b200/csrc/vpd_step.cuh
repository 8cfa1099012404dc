// Parameters and launchers of the per-increment kernels (vpd_step.cu).
#pragma once

#include "vpd_internal.h"

#include <cuda.h>  // CUtensorMap (the staged FP64 force kernel's tensor map)

namespace vpd {

struct BcParams {
  int mode;  // VPD_BC_*
  double amplitude, rise_time, grip_velocity, ramp_time;
  int axis, lateral, plane_strain;
};

// Quantities each material block reduces (sums except the max).
enum { PM_DU = 0, PM_AVG_STRESS, PM_AVG_STRAIN, PM_MAX_EQPS, PM_NONFINITE, PM_PLASTIC, PM_FALLBACK, PM_COUNT };
// Quantities each force block reduces (sums).
enum {
  PF_NETX = 0, PF_NETY, PF_NETZ, PF_REACTION, PF_SUPPORT_REACTION, PF_KINETIC, PF_LAT_POS,
  PF_LAT_NEG, PF_NONFINITE, PF_COUNT
};
// Running sums kept on the device between increments.
enum { ACC_INTERNAL = 0, ACC_EXTERNAL, ACC_PREV_POWER, ACC_FINITE, ACC_COUNT };

constexpr int kDiagRing = 4096;      // diagnostic rows buffered on the device
constexpr int kGroupBlocks = 256;   // k_integrate blocks reduced together by the group's last block
constexpr int kBondThreads = 256;    // threads per block of the bond kernels
constexpr int kMaterialThreads = 128;
constexpr int kMaxStencilWords = 32; // at most 1024 lattice offsets per stencil
// At most this many slots per stencil group: the tiled bond kernels hold a group's window for
// their P <= 4 points per thread as bits 0 .. slots + P - 2 of one 32-bit word.
constexpr int kMaxGroupSlots = 29;
constexpr size_t kStagedMaxBytes = 110 * 1024;  // its box, so that two blocks fit an SM

// Tiles of the TMA-staged FP64 force kernel (vpd_staged64.cu); bytes == 0: not in use.
struct StagedTiles {
  int p = 2;                           // points per thread along y (2 or 4)
  int tz = 0, ty = 0, qy = 0;          // tile extent along z and y; p-point y columns
  int ry = 0, rz = 0;                  // the stencil's reach along y and z
  int by = 0, bz = 0;                  // box extent: tile plus reach on both sides
  int tiles_y = 0, tiles_z = 0, threads = 0;
  uint32_t bytes = 0;                  // box bytes: 3 rows x by x bz x 32
};

// Lattice-stencil bond layout (vpd_stencil.cu). nw == 0: not in use.
struct StencilLayout {
  int slots = 0, nw = 0, ngroups = 0;
  int4 *groups = nullptr;      // [ngroups] (dx, dz, lowest dy, (slots << 16) | first slot)
  int32_t *delta = nullptr;    // [32 nw] index difference j - i of each slot (0: padding)
  int32_t *reverse = nullptr;  // [32 nw] slot of the opposite offset
  uint32_t *forward = nullptr; // [nw] bits of the slots with delta > 0
  uint32_t *mask = nullptr;    // [nw][n] bond bits
  uint32_t *broken = nullptr;  // [nw][n] broken-bond bits
  float4 *e0 = nullptr;        // [32 nw] lattice offset of each slot times h (mixed precision)
  int64_t halo = 0;            // points a tile's window can reach beyond either end of the lattice
  int rx = 0, ry = 0, rz = 0;  // the largest |offset| along x, y, z
};

struct StepParams {
  int64_t n;
  double dt, rho;
  // geometry and bonds
  const double4 *xv;          // x, y, z, volume
  const int32_t *len;         // neighbours per point
  const int64_t *slice_off;   // sliced-ELL slice offsets
  const int32_t *sell;        // sliced-ELL neighbour indices
  uint32_t *words;            // broken-bond bits, one word per (slice, column)
  StencilLayout st;           // lattice-stencil layout; used instead of the ELL when st.nw > 0
  int lat_nx, lat_ny, lat_nz; // the lattice (points in index order (x ny + y) nz + z)
  double lat_h;               // lattice spacing
  int tiled;                  // bond kernels: 0 per slot; mixed 1 tiled scalar, else packed pairs; FP64
                              // tiled with the 4-point force, 3 with the 2-point force, 6 with the
                              // TMA-staged force
  int literal_bisection;      // 1: k_material runs the VUMAT's bisection literally (every iteration
                              // evaluated), 0: jc_return_map (same results)
  // kinematic state
  double4 *u0, *u1;           // displacement ping-pong: increment s reads u[s & 1]
  double4 *vel, *acc, *force;
  // material state, structure of arrays (component c of point i at [c * n + i])
  const double *kinv;
  double *F, *Fn, *Vn, *Rn, *En, *sig, *state, *eI, *eP;
  double *Mt;                 // V_i M_i, 10 doubles per point (point-major; sliced ELL only)
  // lattice-stencil force map: row r of V_i M_i with the point's coordinate r,
  // fmap[r * n + i] = (VM_r0, VM_r1, VM_r2, X_r), so one bond reads three 32-byte records
  double4 *fmap;
  double4 *vxi;               // sum over all bonds of V_j xi (FP64, set once; stencil layout)
  StagedTiles staged;         // the TMA-staged FP64 force kernel's tiles and box
  CUtensorMap fmap_tmap;      // ... and its tensor map over fmap (lane, z, y, x, row)
  // mixed precision (VPD_PRECISION_MIXED): FP32 copies gathered by the bond kernels
  int mixed;
  // mixed precision: jit, uf and fmapf carry st.halo zero records before and after their n
  // (3n) records, so the packed bond kernels read window neighbours unclamped
  float4 *jit;                // (X_i - lattice position, V_i)
  float4 *uf;                 // predicted displacement
  float *Gf;                  // sum V_j (u_j - u_i) (x) xi, 9 floats structure of arrays
  float4 *fmapf;              // V_i M_i and (V_i M_i) jit_i in FP32: three records (fmap_record)
  float tension2f, compression2f;
  // surrogate material update (VPD_MATERIAL_SURROGATE, vpd_surrogate.cu)
  int surrogate;              // 1: guess + Newton, bisection fallback, instead of the bisection
  int surr_guess;             // VPD_GUESS_*: the network, or the previous plastic increment
  int surr_steps;             // Newton steps allowed after the guess
  const uint16_t *sw;         // network weights (bf16 bits, VPD_MLP_WEIGHTS)
  const float *sb;            // network biases (400)
  // host VUMAT plugin (vpd_set_host_vumat, vpd_hostvumat.cu); null: the device update
  void *host_vumat;           // host-side context (never dereferenced on the device)
  double *pack_in, *pack_out; // device blocks of the plugin's inputs and outputs
  double *temp;               // temperature per point
  double *mstash;             // per point: E_{n+1} - E_n (6), E along the axis, E finite
  int nstatev;
  // boundary and diagnostics sets
  const uint8_t *flags;
  const double *obsw;
  JcParams jc;
  BcParams bc;
  int damage;
  double dmg_initiation, dmg_failure, tension2, compression2;
  int use_compression;
  // point damage (SimpleDamageModel::update): VPD_DAMAGE_EQPS_THRESHOLD or
  // VPD_DAMAGE_MAX_PRINCIPAL_STRAIN, 0 otherwise
  int point_damage, dmg_deletion;
  double *pdmg;               // damage per point, non-decreasing
  // internal indicator of the diagnostics (vpd_set_internal_indicator; 0 indices: none)
  int ind_count, ind_min, ind_one_minus;
  int ind_idx[8];
  // device bookkeeping
  int64_t *step;              // increment being computed (1-based)
  unsigned int *status;
  double *part_mat, *part_force, *accum, *diag;
  double *part_group;          // per group of kGroupBlocks integrate blocks: PM_COUNT + PF_COUNT sums
  unsigned int *counter;       // groups done (k_integrate)
  unsigned int *group_counter; // blocks done, per group
  int mat_blocks;
  // diagnostic constants
  double interior, gauge, lat_gauge, area, sign, n_lat_pos, n_lat_neg;
};

// The increment's kernels, in order: deformation (+ bond breaking), material, force bond sum,
// integration (+ boundary conditions, diagnostics, next prediction).
constexpr int kStages = 4;
int launch_init(const StepParams &p, cudaStream_t s);
int launch_stage(int stage, const StepParams &p, cudaStream_t s);
int launch_increment(const StepParams &p, cudaStream_t s);
int launch_shape_inverse_sell(const StepParams &p, cudaStream_t s);
int material_grid(int64_t n);
int integrate_grid(int64_t n);

// lattice-stencil layout (vpd_stencil.cu): st.nw stays 0 when the points do not form the
// lattice in index order or the stencil is too large
int build_stencil(const int64_t *row_ptr, const int32_t *col, int64_t n, int ny, int nz,
                  double spacing, StencilLayout &st, cudaStream_t s);
void free_stencil(StencilLayout &st);
int launch_shape_stencil(const StepParams &p, cudaStream_t s);
int launch_deformation_stencil(const StepParams &p, cudaStream_t s);
int launch_force_stencil(const StepParams &p, cudaStream_t s);
int launch_damage_index_stencil(const StepParams &p, double *out, cudaStream_t s);
// material update through a host VUMAT plugin (vpd_hostvumat.cu): attach loads the plugin and
// allocates its buffers into p (temperatures set to `temperature`); detach frees them
int launch_material_host(const StepParams &p, cudaStream_t s);
int host_vumat_attach(StepParams &p, const char *path, const char *symbol, const char *cmname, const double *props,
                      int nprops, int nstatev, double density, double char_length, double temperature,
                      cudaStream_t s);
void host_vumat_detach(StepParams &p);
// surrogate material update (vpd_surrogate.cu)
int launch_material_surrogate(const StepParams &p, cudaStream_t s);
int prepare_material_surrogate();  // kernel attributes; call before any capture
// mixed precision (vpd_mixed.cu)
int launch_deformation_mixed(const StepParams &p, cudaStream_t s);
int launch_force_mixed(const StepParams &p, cudaStream_t s);
int launch_mixed_setup(const StepParams &p, int ny, int nz, double h, double yoff, double zoff,
                       cudaStream_t s);
// tiled mixed-precision bond kernels (vpd_tiled.cu)
int launch_deformation_tiled(const StepParams &p, cudaStream_t s);
int launch_force_tiled(const StepParams &p, cudaStream_t s);
// tiled FP64 bond kernels (vpd_tiled64.cu)
int launch_deformation_tiled64(const StepParams &p, cudaStream_t s);
int launch_force_tiled64(const StepParams &p, cudaStream_t s);
// TMA-staged FP64 force kernel (vpd_staged64.cu): setup fills p.staged and p.fmap_tmap (left
// unused when the box does not fit or the driver lacks tensor maps)
int setup_staged_force64(StepParams &p, int rx, int ry, int rz);
int launch_force_staged64(const StepParams &p, cudaStream_t s);

}  // namespace vpd
