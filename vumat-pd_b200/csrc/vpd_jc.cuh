// Johnson-Cook VUMAT as a device function, one material point per thread.
//
// Same update as materials/examples/JohnsonCook.f90:74-156 and the same state layout
// (init flag, eqps, temperature, yield stress, last plastic increment, cumulative
// iterations): elastic trial, first-call initialisation, the bracketed bisection return map
// (at most 50 iterations, warm start from the previous increment, |q - sigma_y| < E 1e-9),
// radial scaling, energies and adiabatic heating. Stress and strain increments use the
// legacy_vumat_pd Voigt order 11,22,33,23,13,12 with tensor shear.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace vpd {

struct JcParams {
  double young, poisson, a0, b0, rateC, hardN, thermalM, rate0, tref, tmelt, rho, beta, cp,
      workToHeat;
  double mu, lambda, tolerance;
};

inline JcParams make_jc_params(const double *props) {
  JcParams p;
  p.young = props[0], p.poisson = props[1], p.a0 = props[2], p.b0 = props[3];
  p.rateC = props[4], p.hardN = props[5], p.thermalM = props[6], p.rate0 = props[7];
  p.tref = props[8], p.tmelt = props[9], p.rho = props[10], p.beta = props[11];
  p.cp = props[12], p.workToHeat = props[13];
  p.mu = p.young / (2.0 * (1.0 + p.poisson));
  p.lambda = p.young * p.poisson / ((1.0 + p.poisson) * (1.0 - 2.0 * p.poisson));
  p.tolerance = p.young * 1.0e-9;
  return p;
}

// Flow stress (JohnsonCook.f90:160-170), split so that a return map evaluates the thermal
// factor once (the temperature stays the old one during a return) and pays one pow and one log
// per iteration. The values are bit for bit those of the one-line formula: pow(x, 1) is x and
// log(rate0 / rate0) is 0 exactly, so the m = 1 and zero-rate shortcuts change nothing.
__device__ __forceinline__ double jc_thermal(const JcParams &p, double temp) {
  double theta = (temp - p.tref) / (p.tmelt - p.tref);
  theta = theta > 0.0 ? theta : 0.0;
  theta = theta < 1.0 ? theta : 1.0;
  return 1.0 - (p.thermalM == 1.0 ? theta : pow(theta, p.thermalM));
}
__device__ __forceinline__ double jc_rate_term(const JcParams &p, double rate) {
  return rate == 0.0 ? 1.0 : 1.0 + p.rateC * log(rate / p.rate0);
}
__device__ __forceinline__ double jc_flow(const JcParams &p, double hardPow, double thermal, double rterm) {
  return (p.a0 + p.b0 * hardPow) * thermal * rterm;
}
__device__ __forceinline__ double jc_yield_t(const JcParams &p, double ep, double rate, double thermal) {
  return jc_flow(p, pow(ep, p.hardN), thermal, jc_rate_term(p, rate));
}
__device__ __forceinline__ double jc_yield(const JcParams &p, double ep, double rate, double temp) {
  return jc_yield_t(p, ep, rate, jc_thermal(p, temp));
}

struct JcPoint {
  double stress[6];   // in: old corotational stress; out: new
  double state[6];    // in/out: [init, eqps, T, sigma_y, last deps, sum iterations]
  double eInternal;   // in/out
  double eInelastic;  // in/out
};

// Elastic trial state of one increment (JohnsonCook.f90:74-112).
struct JcTrial {
  double trial[6], dev[6];
  double pressure, qTrial, epOld, temperature, oldYield;
  double thermal;  // 1 - theta^m at the old temperature
};

// Forms the trial state. On the first (initialising) call it completes the update of pt
// itself and returns false.
__device__ __forceinline__ bool jc_trial(const JcParams &p, const double *inc, JcPoint &pt, JcTrial &t) {
  const double traceInc = inc[0] + inc[1] + inc[2];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    t.trial[i] = pt.stress[i] + p.lambda * traceInc + 2.0 * p.mu * inc[i];
#pragma unroll
  for (int i = 3; i < 6; ++i)
    t.trial[i] = pt.stress[i] + 2.0 * p.mu * inc[i];

  if (pt.state[0] == 0.0) {  // first call (:92-102)
    pt.state[0] = 1.0, pt.state[1] = 0.0, pt.state[2] = p.tref;
    pt.state[3] = 0.0, pt.state[4] = 0.0, pt.state[5] = 1.0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
      pt.stress[i] = t.trial[i];
    return false;
  }
  t.epOld = pt.state[1], t.temperature = pt.state[2], t.oldYield = pt.state[3];
  t.thermal = jc_thermal(p, t.temperature);
  t.pressure = (t.trial[0] + t.trial[1] + t.trial[2]) / 3.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    t.dev[i] = t.trial[i] - t.pressure;
#pragma unroll
  for (int i = 3; i < 6; ++i)
    t.dev[i] = t.trial[i];
  t.qTrial = sqrt(1.5 * (t.dev[0] * t.dev[0] + t.dev[1] * t.dev[1] + t.dev[2] * t.dev[2] +
                         2.0 * (t.dev[3] * t.dev[3] + t.dev[4] * t.dev[4] + t.dev[5] * t.dev[5])));
  return true;
}

// Bracketed bisection with warm start (:114-136): plastic increment and yield stress; returns
// the iteration count.
__device__ __forceinline__ int jc_bisection(const JcParams &p, double dt, const JcTrial &t, double warmStart,
                                            double &epIncOut, double &yieldOut) {
  double epInc = 0.0, epLower = 0.0, epUpper = t.qTrial / (2.0 * p.mu), yield = t.oldYield;
  int iteration = 0;
  while (iteration < 50) {
    ++iteration;
    const double epRate = epInc / dt;
    yield = jc_yield_t(p, t.epOld + epInc, epRate, t.thermal);
    yield = yield > t.oldYield ? yield : t.oldYield;
    double qNew = t.qTrial - 3.0 * p.mu * epInc;
    qNew = qNew > 0.0 ? qNew : 0.0;
    const double residual = qNew - yield;
    if (fabs(residual) < p.tolerance)
      break;
    if (epInc == 0.0 && residual < 0.0)
      break;
    if (residual >= 0.0)
      epLower = epLower > epInc ? epLower : epInc;
    else
      epUpper = epUpper < epInc ? epUpper : epInc;
    epInc = 0.5 * (epLower + epUpper);
    if (iteration == 1) {
      double warm = warmStart;
      warm = warm > epLower ? warm : epLower;
      epInc = warm < epUpper ? warm : epUpper;
    }
  }
  epIncOut = epInc;
  yieldOut = yield;
  return iteration;
}

// Radial scaling, energies, heating and state for a given plastic increment (:138-156).
__device__ __forceinline__ void jc_finish(const JcParams &p, const double *inc, const JcTrial &t, double epInc,
                                          double yield, double iterations, JcPoint &pt) {
  double updated[6];
#pragma unroll
  for (int i = 0; i < 6; ++i)
    updated[i] = t.trial[i];
  if (t.qTrial > 0.0) {  // radial scaling (:138-142)
    double scale = 1.0 - 3.0 * p.mu * epInc / t.qTrial;
    scale = scale > 0.0 ? scale : 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
      updated[i] = t.pressure + scale * t.dev[i];
#pragma unroll
    for (int i = 3; i < 6; ++i)
      updated[i] = scale * t.dev[i];
  }
  double qNew = t.qTrial - 3.0 * p.mu * epInc;
  qNew = qNew > 0.0 ? qNew : 0.0;
  double work = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i)
    work += (pt.stress[i] + updated[i]) * inc[i];
  const double workInc = 0.5 * work;
  const double plasticWork = 0.5 * epInc * qNew;
#pragma unroll
  for (int i = 0; i < 6; ++i)
    pt.stress[i] = updated[i];
  pt.eInternal += workInc / p.rho;
  pt.eInelastic += plasticWork / p.rho;
  pt.state[0] = 1.0;
  pt.state[1] = t.epOld + epInc;
  pt.state[2] = t.temperature + p.workToHeat * p.beta * plasticWork / (p.rho * p.cp);
  pt.state[3] = yield;
  pt.state[4] = epInc;
  pt.state[5] = pt.state[5] + iterations;
}

// One increment for one point. inc: strain increment (Voigt, tensor shear). Returns the
// bisection iteration count (0 on the initialising call).
__device__ __forceinline__ int jc_update(const JcParams &p, double dt, const double *inc, JcPoint &pt) {
  JcTrial t;
  if (!jc_trial(p, inc, pt, t))
    return 0;
  double epInc, yield;
  const int iteration = jc_bisection(p, dt, t, pt.state[4], epInc, yield);
  jc_finish(p, inc, t, epInc, yield, (double)iteration, pt);
  return iteration;
}

}  // namespace vpd
