/*
 * vpd_gpu.h -- C ABI of the B200 correspondence-peridynamics increment (libvpd_gpu.so).
 *
 * Plain C types only: pointers, sizes and status codes. Every entry point returns an
 * int status (VPD_OK == 0); vpd_last_error() gives a message for the calling thread's
 * last failure. A handle owns device state and one CUDA stream; it is not thread-safe.
 *
 * Reference interfaces each entry point replaces (paths inside 1998yu/vumat-pd):
 *   vpd_create               makeParticlePatch (src/host/Geometry.cpp:10-34)
 *                            + buildNeighborList (src/pd/PdCorrespondenceSkeleton.cpp:95-129)
 *                            + PdCorrespondenceSkeleton::initialize (:149-170)
 *                            + RegionalConstraintSystem ctor (src/host/BoundaryConditions.cpp:54-68)
 *                            + VumatPdCorrespondenceMaterial::initialize
 *                              (src/material/VumatPdCorrespondenceMaterial.cpp:48-70)
 *                            + runMaterial set-up (src/host/BoundaryValueCaseRunner.cpp:142-190)
 *   vpd_step                 the step loop of runMaterial (BoundaryValueCaseRunner.cpp:207-306):
 *                            predictDisplacement, constraints.apply, computeDeformationGradients,
 *                            bridge.update (kinematics + VUMAT), PdSimpleDamage::update,
 *                            computeForceDensity, correctVelocity, constraints.apply, diagnostics
 *   vpd_download             the per-node fields written by writeSnapshot
 *                            (BoundaryValueCaseRunner.cpp:115-137) and the MaterialState /
 *                            ExplicitDynamicState members (include/PdTypes.hpp:25-47,
 *                            include/ExplicitTimeIntegrator.hpp:10-13)
 *   vpd_neighbors            ParticleBlock::neighbors (include/PdTypes.hpp:18) as CSR
 *   vpd_build_neighbor_list  buildNeighborList (PdCorrespondenceSkeleton.cpp:95-129)
 *   vpd_shape_tensor_inverse PdCorrespondenceSkeleton::initialize (:149-170)
 *   vpd_deformation_gradients PdCorrespondenceSkeleton::computeDeformationGradients (:172-197)
 *   vpd_force_density        PdCorrespondenceSkeleton::computeForceDensity (:199-230)
 *   vpd_corotational_update  updateCorotationalKinematics, greenLagrangeStrain
 *                            (src/pd/CorotationalKinematics.cpp:61-149)
 *   vpd_material_update      VumatPdCorrespondenceMaterial::update (:72-176) with the
 *                            Johnson-Cook VUMAT (materials/examples/JohnsonCook.f90:12-172)
 *   vpd_jc_return_map        the Johnson-Cook bisection alone (JohnsonCook.f90:74-136)
 *   vpd_damage_update        PdSimpleDamage::update, critical_stretch (src/damage/PdSimpleDamage.cpp:51-96);
 *                            the point modes run inside vpd_step (SimpleDamageModel.cpp:14-50)
 *   vpd_set_host_vumat       VumatMaterialAdapter (src/material/VumatMaterialAdapter.cpp:238-362)
 *                            driving any user VUMAT plugin on 256-row blocks, with the rest
 *                            of the increment on the GPU
 *   vpd_set_initial_state    a material's initialState in VumatPdCorrespondenceMaterial::initialize
 *                            (VumatPdCorrespondenceMaterial.cpp:62-66, src/config/DemoConfig.cpp:220-251)
 *   vpd_set_internal_indicator  the internalIndicator of the step diagnostics
 *                            (BoundaryValueCaseRunner.cpp:93-107, :258-263)
 *   vpd_checkpoint_*         no counterpart: the state an increment carries, saved and restored
 *   vumat_adapter_call       the plugin entry the reference dlopens
 *                            (materials/bridge/vumat_c_wrapper_jinfo.f90:1-17,
 *                             include/VumatMaterialAdapter.hpp:35-39), Johnson-Cook on the GPU
 *
 * Module-level entry points (vpd_build_neighbor_list ... vpd_damage_update) take DEVICE
 * pointers owned by the caller and a cudaStream_t passed as void*; they run on that stream
 * and return after the work is queued unless stated otherwise. Tensors are row-major 3x3
 * (9 doubles per point, point-major), vectors 3 doubles per point, as the reference's
 * Tensor3/Vec3 (include/PdTypes.hpp:9-10).
 */
#ifndef VPD_GPU_H
#define VPD_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VPD_ABI_VERSION 1

/* Status codes. */
enum {
  VPD_OK = 0,
  VPD_ERR_INVALID = 1,     /* bad argument or configuration (reference: std::runtime_error) */
  VPD_ERR_CUDA = 2,        /* CUDA runtime error */
  VPD_ERR_SINGULAR = 3,    /* |det| < 1e-14 in K, F or a kinematics inverse */
  VPD_ERR_NONFINITE = 4,   /* non-finite coordinate or state */
  VPD_ERR_CAPACITY = 5,    /* neighbour row or cell grid beyond the supported size */
  VPD_ERR_UNSUPPORTED = 6  /* configuration the device path does not implement */
};

enum { VPD_BC_SMOOTH_DISPLACEMENT = 0, VPD_BC_VELOCITY_RAMP = 1 };
/* damage modes (SimpleDamageConfig::mode, include/SimpleDamageModel.hpp:9-17): bond breaking by
   critical stretch, or one of the point modes of SimpleDamageModel::update
   (src/damage/SimpleDamageModel.cpp:14-40), which degrade the spatial stress the force map uses */
enum {
  VPD_DAMAGE_NONE = 0,
  VPD_DAMAGE_CRITICAL_STRETCH = 1,
  VPD_DAMAGE_EQPS_THRESHOLD = 2,        /* metric: state variable 2 (index 1, the JC eqps) */
  VPD_DAMAGE_MAX_PRINCIPAL_STRAIN = 3   /* metric: largest principal Green-Lagrange strain */
};
enum { VPD_PRECISION_FP64 = 0, VPD_PRECISION_MIXED = 1 };
enum { VPD_MATERIAL_VUMAT = 0, VPD_MATERIAL_SURROGATE = 1 };

/*
 * One regional boundary-value case (the fields of DemoCaseConfig that the PD increment uses,
 * include/DemoConfig.hpp:71-167), in the reference's mm-ms-N-MPa units.
 */
typedef struct vpd_case {
  /* geometry: a nx*ny*nz lattice, index (i*ny + j)*nz + k, x from 0, y and z centred */
  int32_t nx, ny, nz;
  double spacing;          /* h, mm */
  double horizon;          /* delta, mm */
  double jitter;           /* uniform position jitter amplitude as a fraction of h (0: none) */
  uint64_t jitter_seed;
  /* time integration */
  double dt;               /* ms */
  double density;          /* dynamics.density, N ms^2 / mm^4 */
  /* boundary conditions */
  int32_t bc_mode;         /* VPD_BC_* */
  int32_t load_axis;       /* 0: x, left support / right load; 1: y, bottom / top */
  int32_t region_layers;   /* constrained nodal planes per band */
  int32_t plane_strain;    /* 1: all z displacement constrained */
  double amplitude;        /* smooth displacement: end displacement, mm */
  double rise_time;        /* smooth displacement: half-cosine rise, ms */
  double grip_velocity;    /* velocity ramp: relative speed of the two bands, mm/ms */
  double ramp_time;        /* velocity ramp: linear ramp duration, ms */
  double observation_min;  /* observation window along the load axis, mm; NaN: band edges */
  double observation_max;
  /* material: Johnson-Cook props E, nu, A, B, C, n, m, rate0, Tref, Tmelt, rho, beta, Cp,
     workToHeat (materials/examples/JohnsonCook.f90:9) */
  double props[14];
  int32_t nstatev;         /* >= 6 */
  double reference_temperature;
  /* damage (PdSimpleDamage) */
  int32_t damage_mode;     /* VPD_DAMAGE_* */
  double damage_initiation;
  double damage_failure;   /* critical stretch: > 0 enables the compression threshold;
                              point modes: damage = (metric - initiation) / (failure - initiation) */
  /* numerics */
  int32_t precision;       /* VPD_PRECISION_* */
  int32_t material_mode;   /* VPD_MATERIAL_* */
  /* point damage modes: 1 deletes a fully damaged point (its stress no longer enters the force
     map; SimpleDamageConfig::deletionEnabled) */
  int32_t damage_deletion;
} vpd_case;

/* Per-step diagnostic row: the numeric columns of timeseries.csv in the reference's order
   (BoundaryValueCaseRunner.cpp:347-351, values :309-315). */
enum {
  VPD_DIAG_STEP = 0,
  VPD_DIAG_TIME,
  VPD_DIAG_LOAD_DISPLACEMENT,
  VPD_DIAG_LOAD_VELOCITY,
  VPD_DIAG_REACTION,
  VPD_DIAG_ENGINEERING_STRAIN,
  VPD_DIAG_LATERAL_STRAIN,
  VPD_DIAG_NOMINAL_STRESS,
  VPD_DIAG_AVERAGE_AXIAL_STRAIN,
  VPD_DIAG_AVERAGE_AXIAL_STRESS,
  VPD_DIAG_MAX_EQPS,
  VPD_DIAG_MAX_INTERNAL_INDICATOR,
  VPD_DIAG_KINETIC_ENERGY,
  VPD_DIAG_INTERNAL_ENERGY,
  VPD_DIAG_EXTERNAL_WORK,
  VPD_DIAG_ENERGY_ERROR,
  VPD_DIAG_NET_INTERNAL_FORCE,
  VPD_DIAG_FINITE,
  VPD_DIAG_PLASTIC_POINTS,   /* points whose return map gave a plastic increment (state 5 > 0) */
  VPD_DIAG_FALLBACK_POINTS,  /* surrogate mode: plastic points the gate sent to the VUMAT */
  VPD_DIAG_COLS
};

/* Fields for vpd_download; widths per point in brackets. */
enum {
  VPD_FIELD_POSITION = 0,     /* [3] reference position */
  VPD_FIELD_VOLUME,           /* [1] */
  VPD_FIELD_DISPLACEMENT,     /* [3] */
  VPD_FIELD_VELOCITY,         /* [3] */
  VPD_FIELD_ACCELERATION,     /* [3] */
  VPD_FIELD_DEFGRAD,          /* [9] F at the end of the last increment */
  VPD_FIELD_STRESS_COROTATIONAL, /* [9] VUMAT stress, corotational frame */
  VPD_FIELD_STRESS_SPATIAL,   /* [9] R sigma R^T, as used by the force state */
  VPD_FIELD_STRAIN,           /* [9] Green-Lagrange strain */
  VPD_FIELD_ROTATION,         /* [9] */
  VPD_FIELD_LEFT_STRETCH,     /* [9] */
  VPD_FIELD_STATE,            /* [nstatev] VUMAT state variables */
  VPD_FIELD_TEMPERATURE,      /* [1] */
  VPD_FIELD_ENERGY_INTERNAL,  /* [1] */
  VPD_FIELD_ENERGY_INELASTIC, /* [1] */
  VPD_FIELD_DAMAGE_INDEX,     /* [1] volume-weighted broken-bond fraction */
  VPD_FIELD_FORCE_DENSITY,    /* [3] force density of the last increment */
  VPD_FIELD_SHAPE_INVERSE,    /* [9] K^-1 */
  VPD_FIELD_COUNT
};

typedef struct vpd_handle vpd_handle;

int vpd_abi_version(void);
const char *vpd_last_error(void);
/* Width (doubles per point) of a field for a handle's case. */
int vpd_field_width(const vpd_handle *h, int field);

/* Builds the lattice, neighbour lists and K^-1 on the device and initialises the state.
   positions/volumes may be NULL (lattice from the case) or host arrays of n_points*3 and
   n_points doubles that replace the lattice's coordinates (the lattice still defines the
   boundary bands and observation window, which need nx*ny*nz == n_points). */
int vpd_create(const vpd_case *c, const double *positions, const double *volumes,
               vpd_handle **out);
int vpd_destroy(vpd_handle *h);
int64_t vpd_num_points(const vpd_handle *h);
int64_t vpd_num_bonds(const vpd_handle *h);
/* Bond layout the kernels stream: the number of 32-slot lattice-stencil bit-mask words per
   point, or 0 for the sliced-ELL index layout. (No reference counterpart.) */
int vpd_bond_layout_words(const vpd_handle *h);
/* Advances nsteps increments. diag_out (host, may be NULL) receives nsteps rows of
   VPD_DIAG_COLS doubles. Returns after the increments completed on the device. */
int vpd_step(vpd_handle *h, int32_t nsteps, double *diag_out);
/* Copies a field of every point into host memory (n_points * width doubles). */
int vpd_download(vpd_handle *h, int32_t field, double *host_out);
/* Canonical neighbour lists: row_ptr[n_points+1] and col[n_bonds], host memory, each row
   ascending as ParticleBlock::neighbors. */
int vpd_neighbors(vpd_handle *h, int64_t *row_ptr, int32_t *col);
/* The handle's CUDA stream (cudaStream_t) and device-side time of its last vpd_step. */
void *vpd_stream(vpd_handle *h);
int vpd_last_step_ms(const vpd_handle *h, double *ms);
/* Advances nsteps increments launching each kernel separately, with CUDA events between
   them on the handle's stream; stage_ms[4] receives the mean device time of the
   deformation, material, force and integration kernels. Diagnostics rows are kept on the
   device only.
   (No reference counterpart: per-stage timing of the step loop.) */
int vpd_profile_increment(vpd_handle *h, int32_t nsteps, double *stage_ms);
/* The VUMAT state every point starts from (VumatPdCorrespondenceMaterial::initialize with a
   configured initialState, src/material/VumatPdCorrespondenceMaterial.cpp:62-66): state[0..
   nstatev) for every point, the case's further components left at zero. Before the first
   vpd_step; nstatev at most the case's. */
int vpd_set_initial_state(vpd_handle *h, const double *state, int32_t nstatev);
/* The diagnostics' internal indicator (internalIndicator of a material entry,
   BoundaryValueCaseRunner.cpp:93-107): per point the minimum (reduction_min 1) or maximum of
   state variables indices[0..count), 1 minus that when one_minus is 1; the timeseries column
   VPD_DIAG_MAX_INTERNAL_INDICATOR then carries the largest over the points and 0 (0 without
   an indicator). count at most 8. */
int vpd_set_internal_indicator(vpd_handle *h, const int32_t *indices, int32_t count, int32_t reduction_min,
                               int32_t one_minus);
/* Checkpoint and resume between increments. A checkpoint holds the state one increment
   carries to the next: displacements, velocities, accelerations and forces; the material
   history (F, V, R, E, stress, state, energies); broken bonds; point damage and plugin
   temperatures where used; the running energy sums and the increment count. It does not
   hold what the case and the attached material determine (geometry, bonds, K^-1, the sets,
   the network). vpd_checkpoint_bytes gives the size; vpd_checkpoint_save fills a host buffer
   of exactly that size. vpd_checkpoint_load restores one into a handle created from the same
   case (and, before the load, given the same vpd_set_surrogate or vpd_set_host_vumat), which
   then continues bit for bit as the saved handle would have; a checkpoint of another case,
   layout, precision or material path is refused. The diagnostic rows of later vpd_step calls
   continue the saved run's step numbers.
   (No reference counterpart: the reference keeps no state between runs.) */
int64_t vpd_checkpoint_bytes(vpd_handle *h);
int vpd_checkpoint_save(vpd_handle *h, void *buffer, int64_t bytes);
int vpd_checkpoint_load(vpd_handle *h, const void *buffer, int64_t bytes);

/* ---- module-level entry points (device pointers, caller-owned) ---- */

/* Sorted neighbour lists of n points (positions n*3 doubles). First call with col == NULL:
   fills row_ptr[n+1] and *total. Second call with col of *total ints fills the rows. Both
   calls synchronise the stream. Scratch memory is allocated and freed internally. */
int vpd_build_neighbor_list(const double *positions, int64_t n, double horizon,
                            int64_t *row_ptr, int32_t *col, int64_t *total, void *stream);
int vpd_shape_tensor_inverse(const double *positions, const double *volumes, int64_t n,
                             const int64_t *row_ptr, const int32_t *col, double *kinv,
                             void *stream);
int vpd_deformation_gradients(const double *positions, const double *displacement,
                              const double *volumes, int64_t n, const int64_t *row_ptr,
                              const int32_t *col, const double *kinv, double *defgrad,
                              void *stream);
/* bond_damage: one double per CSR entry (PdDamageState::bondDamageN). */
int vpd_force_density(const double *positions, const double *volumes, int64_t n,
                      const int64_t *row_ptr, const int32_t *col, const double *kinv,
                      const double *defgrad, const double *cauchy_stress,
                      const double *bond_damage, double *force, void *stream);
/* vpd_force_density without any device allocation, for hosts that cannot allocate device
   memory during a step (all device memory handed to their own pool, or a step loop that
   cannot take the device-wide synchronisation of cudaMalloc/cudaFree). Same arguments,
   results and errors as vpd_force_density; its scratch is a fixed array inside the library
   (about 4.7 MB held on each GPU that loads it). At most 65536 points per call, else
   VPD_ERR_CAPACITY. Calls share the scratch: calls that overlap on the GPU race. The first
   call on a device looks up the scratch address, which (CUDA loads modules lazily) loads the
   library's code for this entry point and with it reserves the 4.7 MB scratch on that
   device: make that first call before the host's pool takes the device memory and before
   any stream capture. Synchronises the stream. (No counterpart in the reference.) */
int vpd_force_density_noalloc(const double *positions, const double *volumes, int64_t n,
                              const int64_t *row_ptr, const int32_t *col, const double *kinv,
                              const double *defgrad, const double *cauchy_stress,
                              const double *bond_damage, double *force, void *stream);
/* Per point: F_n, F_n+1, V_n, R_n -> D-bar (unrotated rate of deformation), relative spin
   increment, R_n+1, V_n+1, Green-Lagrange E(F_n+1); all [9] per point. */
int vpd_corotational_update(int64_t n, const double *defgrad_old, const double *defgrad_new,
                            const double *stretch_old, const double *rotation_old, double dt,
                            double *rate_of_deformation, double *relative_spin,
                            double *rotation_new, double *stretch_new, double *strain_new,
                            void *stream);
/* The material bridge on device state (updated in place): defgrad_old, stretch, rotation,
   strain, stress_corotational [9]; state [nstatev]; temperature, energies [1].
   stress_spatial [9] receives R sigma R^T. props: 14 Johnson-Cook properties (host). */
int vpd_material_update(int64_t n, const double *props, int32_t nstatev, double dt,
                        const double *defgrad_new, double *defgrad_old, double *stretch,
                        double *rotation, double *strain, double *stress_corotational,
                        double *state, double *temperature, double *energy_internal,
                        double *energy_inelastic, double *stress_spatial, void *stream);
/* The Johnson-Cook return map alone (replaces the bisection of JohnsonCook.f90:114-136, with its
   elastic trial :74-112) on device arrays of n points: strain_inc [n x 6] (Voigt 11,22,33,23,13,12,
   tensor shear), stress [n x 6] and state [n x nstatev] (the VUMAT's old values) -> ep_inc,
   yield [n] and iterations [n] (0 for a point on its initialising call). method 0: the certified
   bisection the increment kernels run (most iterations decided from two anchor evaluations of the
   flow stress); method 1: the literal bisection, every iteration evaluated. Both give the same
   bits. */
int vpd_jc_return_map(int64_t n, const double *props, double dt, const double *strain_inc,
                      const double *stress, const double *state, int32_t nstatev, int32_t method,
                      double *ep_inc, double *yield, int32_t *iterations, void *stream);
/* Critical-stretch bond breaking: bond_damage (per CSR entry, 0/1) updated in place,
   damage_index [n] written. */
int vpd_damage_update(const double *positions, const double *displacement,
                      const double *volumes, int64_t n, const int64_t *row_ptr,
                      const int32_t *col, double initiation, double failure,
                      double *bond_damage, double *damage_index, void *stream);

/* ---- surrogate network (no reference counterpart: the learned Johnson-Cook update) ----
   10 -> 128 -> 128 -> 128 -> 7, SiLU, BF16 weights, FP32 accumulation on the tensor cores.
   Parameters: `weights` are VPD_MLP_WEIGHTS bf16 values (uint16 bit patterns), w1 [128][16],
   w2 [128][128], w3 [128][128], w4 [16][128] row-major [out][in]; `biases` are b1 [128],
   b2 [128], b3 [128], b4 [16] floats. Inputs and outputs are padded to 16 columns. */
#define VPD_MLP_WEIGHTS 36864
#define VPD_MLP_PARAMS 37264
/* out [batch][16] = network(x [batch][16]). Synchronises the stream. */
int vpd_mlp_forward(const uint16_t *weights, const float *biases, const float *x, int64_t batch,
                    float *out, void *stream);
/* grad [VPD_MLP_PARAMS] (weights then biases, FP32) = d/dparams of sum(out * gout), i.e. the
   backward pass for the output gradient gout [batch][16]. Synchronises the stream. */
int vpd_mlp_gradients(const uint16_t *weights, const float *biases, const float *x,
                      const float *gout, int64_t batch, float *grad, void *stream);

/* ---- the learned Johnson-Cook update (no reference counterpart) ----
   Features and targets of one material-point increment (host arrays, 16 floats per row), with
   deq the equivalent deviatoric strain increment and xf = (qTrial - oldYield) / (3 mu) the
   increment of a return to the old yield stress (an upper bound of the plastic increment):
   features 0-5 strain increment / deq, 6 (log10 eqps + 3) / 3, 7 (log10(deq / dt in 1/s)
   - 1.5) / 3, 8 homologous temperature, 9 xf / deq (trial overstress, in [-2, 2]); targets
   0 the plastic increment / xf (in (0, 1]), 1-6 stress increment / (2 mu deq), 15 the row's
   training weight (1 when the trial state yields, else 0). */
#define VPD_SURROGATE_MAX_EPOCHS 64
#define VPD_SAMPLE_RECORD 26
typedef struct vpd_surrogate_config {
  double props[14];            /* Johnson-Cook properties, as vpd_case.props */
  int64_t samples;             /* increments generated by the device VUMAT */
  int32_t epochs;              /* 1 .. VPD_SURROGATE_MAX_EPOCHS */
  int32_t batch;               /* rows per Adam step (>= 128) */
  double learning_rate;        /* Adam */
  uint64_t seed;
  double validation_fraction;  /* held-out tail of the samples, [0, 0.5] */
} vpd_surrogate_config;

typedef struct vpd_surrogate_report {
  int32_t epochs_run;
  double epoch_loss[VPD_SURROGATE_MAX_EPOCHS]; /* mean weighted MSE of each epoch */
  double validation_loss;
  double ratio_rmse;           /* plastic validation rows: rms error of target 0 */
  double stress_rmse;          /* plastic validation rows: rms error of targets 1-6 */
  double plastic_fraction;     /* of all samples */
  double train_ms;             /* device time of the training loop */
} vpd_surrogate_report;

/* Generates `count` increments with the device VUMAT (seeded; strain increments N(0, 1e-4)
   per component for even rows, log-uniform magnitude 1e-8..1e-3 for odd rows; eqps
   log-uniform [1e-6, 0.5]; strain rate log-uniform [1e-3, 1e4] /s; T uniform [293, 1200] K;
   old stress on or inside the yield surface). features / targets: [count][16] floats;
   records (may be NULL): [count][VPD_SAMPLE_RECORD] doubles: strain increment (6), old stress
   (6), eqps, temperature, old yield stress, dt, new stress (6), plastic increment, bisection
   iterations (cold start), trial yields (0/1), yield stress at zero increment. Host buffers. */
int vpd_surrogate_samples(const double *props, uint64_t seed, int64_t count, float *features,
                          float *targets, double *records);

/* Generates cfg->samples increments with the device VUMAT and trains the network on them
   with the tensor-core forward/backward kernels and Adam (weighted MSE, target 0 weighted 4).
   weights [VPD_MLP_WEIGHTS] bf16 bits and biases [400] receive the trained parameters;
   report (may be NULL) the losses and validation errors. */
int vpd_train_surrogate(const vpd_surrogate_config *cfg, uint16_t *weights, float *biases,
                        vpd_surrogate_report *report);

enum { VPD_GUESS_NETWORK = 0, VPD_GUESS_WARM_START = 1, VPD_GUESS_HYBRID = 2 };
/* Attaches the surrogate to a handle created with material_mode VPD_MATERIAL_SURROGATE:
   each yielding point's plastic increment starts from the network's prediction
   (VPD_GUESS_NETWORK; weights and biases as above, host arrays), from the point's previous
   plastic increment (VPD_GUESS_WARM_START; weights may be NULL), or from the previous plastic
   increment where the previous increment was plastic and the network elsewhere
   (VPD_GUESS_HYBRID), takes at most newton_steps Newton steps (in ln of the increment) and is
   accepted when the residual is below the VUMAT's tolerance E 1e-9; the
   other points fall back to the VUMAT's bisection (VPD_DIAG_FALLBACK_POINTS). Required before
   the first vpd_step of such a handle. */
int vpd_set_surrogate(vpd_handle *h, const uint16_t *weights, const float *biases, int32_t guess,
                      int32_t newton_steps);

/* Runs the handle's material update through a host VUMAT plugin (any library exporting the
   reference's vumat_adapter_call ABI, include/VumatMaterialAdapter.hpp:35-39, found by dlopen
   and dlsym) in place of the device Johnson-Cook update. Each increment the GPU forms every
   point's kinematics and packs the plugin's arguments as the reference's adapter does
   (VumatMaterialAdapter.cpp:238-362: 256-row column-major blocks, legacy_vumat_pd order, a
   short last block padded with its last point; step and total time at the increment's start,
   charLength = spacing, coordinates and fields zero); the blocks are copied to pinned host
   memory, the plugin runs on them (blocks in parallel over OpenMP threads, so it must be
   reentrant, as the reference requires), and the stress, state, temperature and energies are
   copied back for the force map and the diagnostics. All of it is ordered on the handle's
   stream. cmname (blank-padded to 80), props [nprops] and density (kg/m^3, for the plugin's
   energy terms) are the material config's; nstatev, at most the case's, is the plugin's
   number of state variables (the case's extra ones are kept). The case's material_mode must
   be VPD_MATERIAL_VUMAT. Call before the first vpd_step; temperatures start at the case's
   reference_temperature. */
int vpd_set_host_vumat(vpd_handle *h, const char *plugin_path, const char *symbol, const char *cmname,
                       const double *props, int32_t nprops, int32_t nstatev, double density);

/* Plugin ABI: the Johnson-Cook VUMAT evaluated on the GPU for one block of host arrays
   in the reference's column-major [component][nblock] layout. Synchronous. A failure is
   reported on stderr and ends the process, as the Fortran routine's `stop` does. */
void vumat_adapter_call(int *nblock, int *ndir, int *nshr, int *nstatev, int *nfieldv,
                        int *nprops, int *lanneal, double *stepTime, double *totalTime,
                        double *dt, char *cmname, double *coordMp, double *charLength,
                        double *props, double *density, double *strainInc, double *relSpinInc,
                        double *tempOld, double *stretchOld, double *defgradOld, double *fieldOld,
                        double *stressOld, double *stateOld, double *enerInternOld,
                        double *enerInelasOld, double *tempNew, double *stretchNew,
                        double *defgradNew, double *fieldNew, double *stressNew, double *stateNew,
                        double *enerInternNew, double *enerInelasNew);

#ifdef __cplusplus
}
#endif

#endif /* VPD_GPU_H */
