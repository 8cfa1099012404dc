/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- shared by the CPU oracle (vpd_oracle.c) and the
 * reference harness (ref_harness.cpp).
 *
 * The two case inputs the reference cannot express, defined once for the checkers; the GPU
 * path implements the same definitions independently:
 *   - seeded lattice jitter from a counter-based splitmix64 stream (vo_jitter_value);
 *   - prescribed band kinematics (vo_ramp): the reference's half-cosine displacement ramp
 *     and the velocity-ramp grips.
 */
#include "../include/vpd_gpu.h"

#include <math.h>
#include <stdint.h>

uint64_t vo_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  uint64_t z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
/* Jitter of coordinate c of point p: uniform in [-amp, amp), amp = jitter * spacing. */
double vo_jitter_value(uint64_t seed, int64_t p, int c, double amp) {
  const uint64_t r = vo_splitmix64(seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(3 * p + c + 1)));
  const double u = (double)(r >> 11) * 0x1.0p-53;
  return (2.0 * u - 1.0) * amp;
}

/* Prescribed band kinematics at time t. Smooth mode: RegionalConstraintSystem::ramp
   (BoundaryConditions.cpp:70-79), loaded band only. Velocity-ramp mode (extension): the
   loaded band moves at +v/2 and the support band at -v/2 along the axis, v rising linearly
   from 0 to grip_velocity over ramp_time. out[0..2] loaded u,v,a; out[3..5] support u,v,a. */
void vo_ramp(const vpd_case *c, double t, double *out) {
  if (c->bc_mode == VPD_BC_SMOOTH_DISPLACEMENT) {
    if (t >= c->rise_time) {
      out[0] = c->amplitude, out[1] = 0.0, out[2] = 0.0;
    } else {
      const double pi = 3.14159265358979323846;
      const double phase = pi * t / c->rise_time;
      out[0] = 0.5 * c->amplitude * (1.0 - cos(phase));
      out[1] = 0.5 * c->amplitude * pi / c->rise_time * sin(phase);
      out[2] = 0.5 * c->amplitude * pi * pi / (c->rise_time * c->rise_time) * cos(phase);
    }
    out[3] = out[4] = out[5] = 0.0;
    return;
  }
  const double vh = 0.5 * c->grip_velocity, T = c->ramp_time;
  if (t < T) {
    out[0] = vh * (t * t / (2.0 * T));
    out[1] = vh * (t / T);
    out[2] = vh / T;
  } else {
    out[0] = vh * (t - 0.5 * T);
    out[1] = vh;
    out[2] = 0.0;
  }
  out[3] = -out[0], out[4] = -out[1], out[5] = -out[2];
}

