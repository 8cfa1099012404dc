// ORACLE / TEST INFRASTRUCTURE ONLY -- drives the reference library, never the product.
//
// A C API over the reference's own module classes, compiled from its sources into
// oracle/_ref/libvumat_pd_ref.a: makeParticlePatch, buildNeighborList,
// PdCorrespondenceSkeleton, VumatPdCorrespondenceMaterial (loading a restated VUMAT plugin
// through the reference's dlopen adapter), PdSimpleDamage, ExplicitTimeIntegrator and
// RegionalConstraintSystem. The step order is runMaterial's
// (src/host/BoundaryValueCaseRunner.cpp:207-306). Two inputs the reference cannot express
// are added here: seeded lattice jitter and the velocity-ramp grips; for those the
// constraint application is this file's own, on the band sets the reference's
// RegionalConstraintSystem selects from the un-jittered lattice.
#include "../include/vpd_gpu.h"

#include "BoundaryConditions.hpp"
#include "ExplicitTimeIntegrator.hpp"
#include "Geometry.hpp"
#include "ObservationWindow.hpp"
#include "ParticleSets.hpp"
#include "PdCorrespondenceSkeleton.hpp"
#include "PdSimpleDamage.hpp"
#include "VumatPdCorrespondenceMaterial.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

using namespace vumat;

extern "C" double vo_jitter_value(uint64_t seed, int64_t p, int c, double amp);

namespace {
thread_local std::string g_error;

struct RefSim {
  vpd_case c{};
  pd::ParticleBlock block, nominal;
  demo::BoundaryConditionConfig bc;
  std::unique_ptr<demo::RegionalConstraintSystem> constraints;
  std::unique_ptr<pd::PdCorrespondenceSkeleton> skeleton;
  pd::CorrespondenceState cstate;
  std::unique_ptr<pd::VumatPdCorrespondenceMaterial> bridge;
  pd::MaterialState mstate;
  std::unique_ptr<pd::PdSimpleDamage> damage;
  pd::PdDamageState dstate;
  std::unique_ptr<pd::ExplicitTimeIntegrator> integrator;
  pd::ExplicitDynamicState dyn;
  pd::MaterialUpdateResult last;
  std::vector<pd::Vec3> force;
  std::vector<double> obsWeight, damageIndex;
  std::vector<size_t> latNeg, latPos;
  size_t rotationPin = 0;
  double gauge = 0, lateralGauge = 0, area = 0;
  int axis = 0, lateral = 1;
  int64_t step = 0;
  double internalEnergy = 0, externalWork = 0, previousPower = 0;
  bool finite = true;
  bool referenceApply = false;
  double stageSeconds[5] = {0, 0, 0, 0, 0}; // F, material, damage, force, rest
};

} // namespace

extern "C" void vo_ramp(const vpd_case *c, double t, double *out);

namespace {
void applyConstraints(RefSim &s, double t) {
  if (s.referenceApply) {
    s.constraints->apply(s.block, s.dyn, t);
    return;
  }
  double r[6];
  vo_ramp(&s.c, t, r);
  auto set = [&](size_t i, int d, double u, double v, double a) {
    s.block.displacement[i][d] = u;
    s.dyn.velocity[i][d] = v;
    s.dyn.acceleration[i][d] = a;
  };
  for (size_t i : s.constraints->support())
    set(i, s.axis, r[3], r[4], r[5]);
  for (size_t i : s.constraints->loaded())
    set(i, s.axis, r[0], r[1], r[2]);
  set(s.constraints->anchor(), s.lateral, 0, 0, 0);
  if (!s.c.plane_strain) {
    set(s.constraints->anchor(), 2, 0, 0, 0);
    set(s.rotationPin, 2, 0, 0, 0);
  } else {
    for (size_t i = 0; i < s.block.referencePosition.size(); ++i)
      set(i, 2, 0, 0, 0);
  }
}
double seconds(std::chrono::steady_clock::time_point a) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
}
} // namespace

extern "C" {

const char *vr_last_error() { return g_error.c_str(); }

// plugin_path: a restated VUMAT plugin exporting vumat_adapter_call.
void *vr_create(const vpd_case *c, const char *plugin_path) {
  try {
    auto s = std::make_unique<RefSim>();
    s->c = *c;
    s->nominal = demo::makeParticlePatch(c->nx, c->ny, c->nz, c->spacing, c->horizon);
    s->block = s->nominal;
    if (c->jitter != 0.0) {
      const double amp = c->jitter * c->spacing;
      for (size_t p = 0; p < s->block.referencePosition.size(); ++p)
        for (int d = 0; d < 3; ++d)
          s->block.referencePosition[p][d] =
              s->nominal.referencePosition[p][d] + vo_jitter_value(c->jitter_seed, (int64_t)p, d, amp);
      s->block.neighbors = pd::buildNeighborList(s->block.referencePosition, c->horizon);
    }
    auto &bc = s->bc;
    bc.type = "regional_smooth_displacement";
    bc.component = c->load_axis == 1 ? "y" : "x";
    bc.supportRegion = c->load_axis == 1 ? "bottom" : "left";
    bc.loadRegion = c->load_axis == 1 ? "top" : "right";
    bc.regionLayers = c->region_layers;
    bc.amplitude = c->amplitude;
    bc.riseTime = c->rise_time;
    bc.planeStrain = c->plane_strain != 0;
    bc.rigidBodySuppression = true;
    s->constraints = std::make_unique<demo::RegionalConstraintSystem>(s->nominal, bc, c->spacing);
    s->referenceApply = c->bc_mode == VPD_BC_SMOOTH_DISPLACEMENT && c->jitter == 0.0;
    s->axis = s->constraints->loadComponent();
    s->lateral = s->constraints->lateralComponent();
    // rotation pin as BoundaryConditions.cpp:96-110, on the nominal lattice
    s->rotationPin = s->constraints->anchor();
    double greatestY = -1.0e100;
    const auto &centre = s->nominal.referencePosition[s->constraints->anchor()];
    for (size_t i : s->constraints->support()) {
      const auto &x = s->nominal.referencePosition[i];
      if (std::abs(x[0] - centre[0]) < 1e-8 && std::abs(x[2] - centre[2]) < 1e-8 && x[1] > greatestY)
        greatestY = x[1], s->rotationPin = i;
    }
    auto mean = [&](const std::vector<size_t> &idx, int comp) {
      double sum = 0;
      for (size_t i : idx)
        sum += s->nominal.referencePosition[i][comp];
      return sum / (double)idx.size();
    };
    s->gauge = std::abs(mean(s->constraints->loaded(), s->axis) - mean(s->constraints->support(), s->axis));
    s->latNeg = demo::selectBoundaryRegion(s->nominal, s->lateral == 0 ? "left" : "bottom", 1e-9 * c->spacing);
    s->latPos = demo::selectBoundaryRegion(s->nominal, s->lateral == 0 ? "right" : "top", 1e-9 * c->spacing);
    s->lateralGauge = std::abs(mean(s->latPos, s->lateral) - mean(s->latNeg, s->lateral));
    const auto [lo, hi] = demo::observationBounds(s->nominal, s->axis, (c->region_layers - 1) * c->spacing,
                                                  c->observation_min, c->observation_max);
    s->obsWeight = demo::observationWeights(s->nominal, s->axis, lo, hi, 1e-8 * c->spacing);
    const int cross = s->axis == 0 ? c->ny : c->nx;
    s->area = (double)((cross - 1) * (c->nz - 1)) * c->spacing * c->spacing;

    s->skeleton = std::make_unique<pd::PdCorrespondenceSkeleton>(c->horizon);
    s->skeleton->initialize(s->block, s->cstate);
    pd::VumatPdCorrespondenceConfig mc;
    mc.material.name = "JC";
    mc.material.cmname = "JOHNSONCOOK";
    mc.material.pluginPath = plugin_path;
    mc.material.nstatev = c->nstatev;
    mc.material.props.assign(c->props, c->props + 14);
    mc.material.density = c->props[10];
    mc.charLength = c->spacing;
    mc.referenceTemperature = c->reference_temperature;
    s->bridge = std::make_unique<pd::VumatPdCorrespondenceMaterial>(mc);
    s->bridge->initialize(s->skeleton->computeDeformationGradients(s->block, s->cstate), s->mstate);
    SimpleDamageConfig dc;
    static const char *const modes[] = {"none", "critical_stretch", "eqps_threshold", "max_principal_strain"};
    dc.mode = c->damage_mode >= 0 && c->damage_mode <= VPD_DAMAGE_MAX_PRINCIPAL_STRAIN ? modes[c->damage_mode] : "?";
    dc.initiation = c->damage_initiation;
    dc.failure = c->damage_failure;
    dc.deletionEnabled = c->damage_deletion != 0;
    s->damage = std::make_unique<pd::PdSimpleDamage>(dc);
    s->damage->initialize(s->block, s->dstate);
    s->integrator = std::make_unique<pd::ExplicitTimeIntegrator>(c->density);
    s->integrator->initialize(s->block, s->dyn);
    applyConstraints(*s, 0.0);
    s->damageIndex.assign(s->block.referencePosition.size(), 0.0);
    return s.release();
  } catch (const std::exception &e) {
    g_error = e.what();
    return nullptr;
  }
}

void vr_destroy(void *h) { delete static_cast<RefSim *>(h); }
int64_t vr_num_points(void *h) { return (int64_t) static_cast<RefSim *>(h)->block.referencePosition.size(); }
int64_t vr_num_bonds(void *h) {
  int64_t t = 0;
  for (auto &row : static_cast<RefSim *>(h)->block.neighbors)
    t += (int64_t)row.size();
  return t;
}
int vr_neighbors(void *h, int64_t *row_ptr, int32_t *col) {
  auto *s = static_cast<RefSim *>(h);
  row_ptr[0] = 0;
  for (size_t i = 0; i < s->block.neighbors.size(); ++i) {
    row_ptr[i + 1] = row_ptr[i] + (int64_t)s->block.neighbors[i].size();
    std::copy(s->block.neighbors[i].begin(), s->block.neighbors[i].end(), col + row_ptr[i]);
  }
  return 0;
}
void vr_stage_seconds(void *h, double *out) { std::memcpy(out, static_cast<RefSim *>(h)->stageSeconds, 5 * sizeof(double)); }

// runMaterial's loop body, BoundaryValueCaseRunner.cpp:207-306.
int vr_step(void *h, int32_t nsteps, double *diag) {
  auto &s = *static_cast<RefSim *>(h);
  try {
    const auto &c = s.c;
    const double dt = c.dt, rho = c.density;
    const size_t n = s.block.referencePosition.size();
    for (int32_t it = 0; it < nsteps; ++it) {
      const int64_t step = ++s.step;
      const double time = (double)step * dt;
      auto t0 = std::chrono::steady_clock::now();
      s.integrator->predictDisplacement(s.block, s.dyn, dt);
      applyConstraints(s, time);
      const auto previousStress = s.mstate.rawStressN;
      const auto previousStrain = s.mstate.strainN;
      s.stageSeconds[4] += seconds(t0);
      t0 = std::chrono::steady_clock::now();
      const auto F = s.skeleton->computeDeformationGradients(s.block, s.cstate);
      s.stageSeconds[0] += seconds(t0);
      t0 = std::chrono::steady_clock::now();
      auto result = s.bridge->update(F, s.mstate, dt, (step - 1) * dt, (step - 1) * dt);
      s.stageSeconds[1] += seconds(t0);
      t0 = std::chrono::steady_clock::now();
      auto damage = s.damage->update(s.block, result.strain, result.rawStress, s.mstate.vumatStateN, s.dstate);
      s.stageSeconds[2] += seconds(t0);
      t0 = std::chrono::steady_clock::now();
      s.force = s.skeleton->computeForceDensity(s.block, s.cstate, result.deformationGradient,
                                                damage.effectiveStress, damage.bondDamage);
      s.stageSeconds[3] += seconds(t0);
      t0 = std::chrono::steady_clock::now();
      s.integrator->correctVelocity(s.dyn, s.force, dt);
      applyConstraints(s, time);
      // diagnostics (BoundaryValueCaseRunner.cpp:231-306)
      for (size_t i = 0; i < n; ++i) {
        double avg[9], inc[9];
        for (int k = 0; k < 9; ++k) {
          avg[k] = 0.5 * (previousStress[i][k] + result.rawStress[i][k]);
          inc[k] = result.strain[i][k] - previousStrain[i][k];
        }
        s.internalEnergy += (avg[0] * inc[0] + avg[4] * inc[4] + avg[8] * inc[8] +
                             2.0 * (avg[1] * inc[1] + avg[2] * inc[2] + avg[5] * inc[5])) *
                            s.block.volume[i];
      }
      const double sign = (c.bc_mode == VPD_BC_SMOOTH_DISPLACEMENT ? c.amplitude : c.grip_velocity) > 0 ? 1.0 : -1.0;
      double r[6];
      vo_ramp(&c, time, r);
      double net[3] = {0, 0, 0}, reaction = 0, supportReaction = 0, avgS = 0, avgE = 0, maxEqps = 0, interior = 0,
             plastic = 0;
      for (size_t i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d)
          net[d] += s.force[i][d] * s.block.volume[i];
        if (s.obsWeight[i] > 0.0) {
          avgS += sign * result.rawStress[i][4 * s.axis] * s.obsWeight[i];
          avgE += sign * result.strain[i][4 * s.axis] * s.obsWeight[i];
          interior += s.obsWeight[i];
        }
        maxEqps = std::max(maxEqps, s.mstate.vumatStateN[i][1]);
        if (s.mstate.vumatStateN[i].size() > 4 && s.mstate.vumatStateN[i][4] > 0.0)
          plastic += 1.0;
        for (int k = 0; k < 9; ++k)
          s.finite = s.finite && std::isfinite(result.rawStress[i][k]) && std::isfinite(result.strain[i][k]);
        for (int d = 0; d < 3; ++d)
          s.finite = s.finite && std::isfinite(s.force[i][d]);
        for (double v : s.mstate.vumatStateN[i])
          s.finite = s.finite && std::isfinite(v);
      }
      for (size_t i : s.constraints->loaded())
        reaction += (rho * r[2] - s.force[i][s.axis]) * s.block.volume[i];
      for (size_t i : s.constraints->support())
        supportReaction += (rho * r[5] - s.force[i][s.axis]) * s.block.volume[i];
      avgS /= interior;
      avgE /= interior;
      const double power = reaction * r[1] + (c.bc_mode == VPD_BC_VELOCITY_RAMP ? supportReaction * r[4] : 0.0);
      s.externalWork += 0.5 * dt * (s.previousPower + power);
      s.previousPower = power;
      double kinetic = 0;
      for (size_t i = 0; i < n; ++i) {
        const auto &v = s.dyn.velocity[i];
        kinetic += 0.5 * rho * s.block.volume[i] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      }
      const double scale = std::max({std::abs(s.externalWork), std::abs(s.internalEnergy) + kinetic, 1.0e-12});
      const double energyError = std::abs(kinetic + s.internalEnergy - s.externalWork) / scale;
      auto meanU = [&](const std::vector<size_t> &idx) {
        double sum = 0;
        for (size_t i : idx)
          sum += s.block.displacement[i][s.lateral];
        return sum / (double)idx.size();
      };
      const double lateralStrain = (meanU(s.latPos) - meanU(s.latNeg)) / s.lateralGauge;
      s.finite = s.finite && std::isfinite(kinetic) && std::isfinite(s.internalEnergy) &&
                 std::isfinite(s.externalWork) && std::isfinite(energyError);
      if (diag) {
        double *row = diag + (size_t)it * VPD_DIAG_COLS;
        row[VPD_DIAG_STEP] = (double)step;
        row[VPD_DIAG_TIME] = time;
        row[VPD_DIAG_LOAD_DISPLACEMENT] = r[0];
        row[VPD_DIAG_LOAD_VELOCITY] = r[1];
        row[VPD_DIAG_REACTION] = reaction;
        row[VPD_DIAG_ENGINEERING_STRAIN] = sign * (r[0] - r[3]) / s.gauge;
        row[VPD_DIAG_LATERAL_STRAIN] = lateralStrain;
        row[VPD_DIAG_NOMINAL_STRESS] = sign * reaction / s.area;
        row[VPD_DIAG_AVERAGE_AXIAL_STRAIN] = avgE;
        row[VPD_DIAG_AVERAGE_AXIAL_STRESS] = avgS;
        row[VPD_DIAG_MAX_EQPS] = maxEqps;
        row[VPD_DIAG_MAX_INTERNAL_INDICATOR] = 0.0;
        row[VPD_DIAG_KINETIC_ENERGY] = kinetic;
        row[VPD_DIAG_INTERNAL_ENERGY] = s.internalEnergy;
        row[VPD_DIAG_EXTERNAL_WORK] = s.externalWork;
        row[VPD_DIAG_ENERGY_ERROR] = energyError;
        row[VPD_DIAG_NET_INTERNAL_FORCE] = std::sqrt(net[0] * net[0] + net[1] * net[1] + net[2] * net[2]);
        row[VPD_DIAG_FINITE] = s.finite ? 1.0 : 0.0;
        row[VPD_DIAG_PLASTIC_POINTS] = plastic;
        row[VPD_DIAG_FALLBACK_POINTS] = 0.0;
      }
      s.damageIndex = damage.damageIndex;
      s.last = std::move(result);
      s.stageSeconds[4] += seconds(t0);
    }
    return 0;
  } catch (const std::exception &e) {
    g_error = e.what();
    return VPD_ERR_INVALID;
  }
}

int vr_get(void *h, int32_t field, double *out) {
  auto &s = *static_cast<RefSim *>(h);
  const size_t n = s.block.referencePosition.size();
  auto put3 = [&](const std::vector<pd::Vec3> &v) {
    for (size_t i = 0; i < n; ++i)
      std::memcpy(out + 3 * i, v[i].data(), 3 * sizeof(double));
  };
  auto put9 = [&](const std::vector<pd::Tensor3> &v) {
    for (size_t i = 0; i < n; ++i)
      std::memcpy(out + 9 * i, v[i].data(), 9 * sizeof(double));
  };
  auto put1 = [&](const std::vector<double> &v) { std::memcpy(out, v.data(), n * sizeof(double)); };
  switch (field) {
  case VPD_FIELD_POSITION: put3(s.block.referencePosition); return 0;
  case VPD_FIELD_VOLUME: put1(s.block.volume); return 0;
  case VPD_FIELD_DISPLACEMENT: put3(s.block.displacement); return 0;
  case VPD_FIELD_VELOCITY: put3(s.dyn.velocity); return 0;
  case VPD_FIELD_ACCELERATION: put3(s.dyn.acceleration); return 0;
  case VPD_FIELD_DEFGRAD: put9(s.mstate.deformationGradientN); return 0;
  case VPD_FIELD_STRESS_COROTATIONAL: put9(s.mstate.rawStressN); return 0;
  case VPD_FIELD_STRESS_SPATIAL:
    if (s.last.rawStress.size() != n) return VPD_ERR_INVALID;
    put9(s.last.rawStress); return 0;
  case VPD_FIELD_STRAIN: put9(s.mstate.strainN); return 0;
  case VPD_FIELD_ROTATION: put9(s.mstate.rotationN); return 0;
  case VPD_FIELD_LEFT_STRETCH: put9(s.mstate.leftStretchN); return 0;
  case VPD_FIELD_STATE:
    for (size_t i = 0; i < n; ++i)
      std::memcpy(out + (size_t)s.c.nstatev * i, s.mstate.vumatStateN[i].data(), s.c.nstatev * sizeof(double));
    return 0;
  case VPD_FIELD_TEMPERATURE: put1(s.mstate.temperatureN); return 0;
  case VPD_FIELD_ENERGY_INTERNAL: put1(s.mstate.internalEnergyN); return 0;
  case VPD_FIELD_ENERGY_INELASTIC: put1(s.mstate.inelasticEnergyN); return 0;
  case VPD_FIELD_DAMAGE_INDEX: put1(s.damageIndex); return 0;
  case VPD_FIELD_FORCE_DENSITY:
    if (s.force.size() != n) return VPD_ERR_INVALID;
    put3(s.force); return 0;
  case VPD_FIELD_SHAPE_INVERSE: put9(s.cstate.shapeTensorInverse); return 0;
  default: return VPD_ERR_INVALID;
  }
}

// buildNeighborList on arbitrary positions (two calls: col == nullptr gives row_ptr/total).
int64_t vr_build_neighbor_list(const double *pos, int64_t n, double horizon, int64_t *row_ptr, int32_t *col) {
  try {
    std::vector<pd::Vec3> x((size_t)n);
    for (int64_t i = 0; i < n; ++i)
      x[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    auto nb = pd::buildNeighborList(x, horizon);
    row_ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
      row_ptr[i + 1] = row_ptr[i] + (int64_t)nb[i].size();
      if (col)
        std::copy(nb[i].begin(), nb[i].end(), col + row_ptr[i]);
    }
    return row_ptr[n];
  } catch (const std::exception &e) {
    g_error = e.what();
    return -VPD_ERR_INVALID;
  }
}

} // extern "C"
