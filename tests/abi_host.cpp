// A compiled C++ host on the C ABI, the way the reference's host would drive the library in
// place of runMaterial's step loop (src/host/BoundaryValueCaseRunner.cpp:139-337). It
// includes include/vpd_gpu.h only and links libvpd_gpu.so; tests/test_abi.py and
// tests/test_gpu_abi_host.py build it with the system compiler.
//
//   abi_host layout          prints sizeof(vpd_case) and the offset of every field
//   abi_host run N OUT       runs the 40x10x10 steel bar for N increments (outputEvery 10)
//                            and writes the N diagnostic rows and the final displacement to
//                            OUT as raw doubles; prints the point count and dt
#include "vpd_gpu.h"

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// The parts of the reference's DemoCaseConfig / MaterialConfig a host reads, as plain fields.
struct GeometryConfig { int nx, ny, nz; double spacing, horizon; };
struct BoundaryConfig { std::string component; int regionLayers; double gripVelocity, rampTime; };
struct MaterialConfig { std::vector<double> props; int nstatev; double referenceTemperature; };
struct DamageConfig { std::string model; double initiation, failure; };
struct CaseConfig {
  GeometryConfig geometry;
  double dt, density;
  int steps, outputEvery;
  BoundaryConfig boundaryCondition;
  MaterialConfig material;
  DamageConfig damage;
};

// The 40x10x10 steel Johnson-Cook bar: h = 0.5 mm, horizon 3.015 h, grips at 1 m/s ramped
// over 200 increments, dt = 0.8 h / c_p.
CaseConfig steel_bar(int steps) {
  CaseConfig cfg{};
  cfg.geometry = {40, 10, 10, 0.5, 3.015 * 0.5};
  const double e = 200000.0, nu = 0.3;
  cfg.density = 7850.0e-6;
  const double cp = std::sqrt(e * (1.0 - nu) / (cfg.density * (1.0 + nu) * (1.0 - 2.0 * nu)));
  cfg.dt = 0.8 * cfg.geometry.spacing / cp;
  cfg.steps = steps;
  cfg.outputEvery = 10;
  cfg.boundaryCondition = {"x", 3, 1.0, 200 * cfg.dt};
  cfg.material = {{e, nu, 350.0, 275.0, 0.022, 0.36, 1.0, 1.0e-3, 293.0, 1793.0, 7850.0, 0.9,
                   477.0, 1.0},
                  6, 293.0};
  cfg.damage = {"none", 0.0, 0.0};
  return cfg;
}

void check(int rc) {
  if (rc != VPD_OK)
    throw std::runtime_error(vpd_last_error());
}

// runMaterial's loop on the GPU: create, step in outputEvery chunks, download, destroy.
void run(const CaseConfig &cfg, std::vector<double> &rows, std::vector<double> &u) {
  vpd_case c{};
  c.nx = cfg.geometry.nx; c.ny = cfg.geometry.ny; c.nz = cfg.geometry.nz;
  c.spacing = cfg.geometry.spacing; c.horizon = cfg.geometry.horizon;
  c.dt = cfg.dt; c.density = cfg.density;
  c.bc_mode = VPD_BC_VELOCITY_RAMP;
  c.load_axis = cfg.boundaryCondition.component == "y" ? 1 : 0;
  c.region_layers = cfg.boundaryCondition.regionLayers;
  c.grip_velocity = cfg.boundaryCondition.gripVelocity;
  c.ramp_time = cfg.boundaryCondition.rampTime;
  c.observation_min = NAN; c.observation_max = NAN;  // the band edges
  for (size_t i = 0; i < 14; ++i)
    c.props[i] = cfg.material.props.at(i);
  c.nstatev = cfg.material.nstatev;
  c.reference_temperature = cfg.material.referenceTemperature;
  c.damage_mode = cfg.damage.model == "critical_stretch" ? VPD_DAMAGE_CRITICAL_STRETCH : VPD_DAMAGE_NONE;
  c.damage_initiation = cfg.damage.initiation;
  c.damage_failure = cfg.damage.failure;
  c.precision = VPD_PRECISION_FP64;
  c.material_mode = VPD_MATERIAL_VUMAT;

  vpd_handle *h = nullptr;
  check(vpd_create(&c, nullptr, nullptr, &h));
  rows.assign((size_t)VPD_DIAG_COLS * cfg.steps, 0.0);
  for (int done = 0; done < cfg.steps; done += cfg.outputEvery) {
    const int n = cfg.steps - done < cfg.outputEvery ? cfg.steps - done : cfg.outputEvery;
    check(vpd_step(h, n, rows.data() + (size_t)VPD_DIAG_COLS * done));
  }
  u.assign(3 * (size_t)vpd_num_points(h), 0.0);
  check(vpd_download(h, VPD_FIELD_DISPLACEMENT, u.data()));
  check(vpd_destroy(h));
}

void print_layout() {
#define F(name) std::printf("%s %zu\n", #name, offsetof(vpd_case, name))
  std::printf("sizeof %zu\n", sizeof(vpd_case));
  F(nx); F(ny); F(nz); F(spacing); F(horizon); F(jitter); F(jitter_seed); F(dt); F(density);
  F(bc_mode); F(load_axis); F(region_layers); F(plane_strain); F(amplitude); F(rise_time);
  F(grip_velocity); F(ramp_time); F(observation_min); F(observation_max); F(props); F(nstatev);
  F(reference_temperature); F(damage_mode); F(damage_initiation); F(damage_failure);
  F(precision); F(material_mode); F(damage_deletion);
#undef F
}

}  // namespace

int main(int argc, char **argv) {
  if (argc >= 2 && std::string(argv[1]) == "layout") {
    print_layout();
    return 0;
  }
  if (argc != 4 || std::string(argv[1]) != "run") {
    std::fprintf(stderr, "usage: abi_host layout | abi_host run N OUT\n");
    return 1;
  }
  if (vpd_abi_version() != VPD_ABI_VERSION) {
    std::fprintf(stderr, "ABI version %d, header %d\n", vpd_abi_version(), VPD_ABI_VERSION);
    return 1;
  }
  try {
    const CaseConfig cfg = steel_bar(std::atoi(argv[2]));
    std::vector<double> rows, u;
    run(cfg, rows, u);
    FILE *f = std::fopen(argv[3], "wb");
    if (!f)
      throw std::runtime_error("cannot open output file");
    std::fwrite(rows.data(), sizeof(double), rows.size(), f);
    std::fwrite(u.data(), sizeof(double), u.size(), f);
    std::fclose(f);
    std::printf("points %zu dt %.17g\n", u.size() / 3, cfg.dt);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
