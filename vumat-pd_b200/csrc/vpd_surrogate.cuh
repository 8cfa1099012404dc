// The learned Johnson-Cook return map: input features, training targets and the Newton
// acceptance that gates the network's plastic increment (no counterpart in the reference; the
// VUMAT's bisection, jc_bisection, stays the fallback, and its residual decides acceptance).
//
// For a point whose elastic trial state yields (the VUMAT's first bisection iteration, at
// epInc = 0, leaves a residual of at least the tolerance E 1e-9), the plastic increment solves
//   r(x) = max(qTrial - 3 mu x, 0) - max(sigma_y(epOld + x, x / dt, T), oldYield) = 0,
// the equation the bisection brackets (JohnsonCook.f90:114-136). The yield is floored at
// oldYield, so the root lies in (0, xf] with xf = (qTrial - oldYield) / (3 mu), the increment
// of a return to the old yield stress. The network predicts rho = x / xf in (0, 1] from ten
// features of the increment and the state; Newton steps on r from x = rho xf must reach
// |r| < E 1e-9, the VUMAT's own convergence test, within a fixed number of steps, else the
// point falls back to the bisection. An accepted increment therefore meets the same tolerance
// as the VUMAT's, and the stress follows from it by the VUMAT's radial scaling (jc_finish).
#pragma once

#include "vpd_jc.cuh"

namespace vpd {

enum { SURROGATE_FEATURES = 10, SURROGATE_TARGETS = 7 };

// Equivalent deviatoric strain increment sqrt(2/3 e:e) (tensor shear in inc[3..5]).
__device__ __forceinline__ double equivalent_increment(const double *inc) {
  const double m = (inc[0] + inc[1] + inc[2]) / 3.0;
  const double d0 = inc[0] - m, d1 = inc[1] - m, d2 = inc[2] - m;
  return sqrt((2.0 / 3.0) * (d0 * d0 + d1 * d1 + d2 * d2 +
                             2.0 * (inc[3] * inc[3] + inc[4] * inc[4] + inc[5] * inc[5])));
}

// Increment of a return to the old yield stress: the upper end of the root's bracket.
__device__ __forceinline__ double floor_increment(const JcParams &p, const JcTrial &t) {
  return (t.qTrial - t.oldYield) / (3.0 * p.mu);
}

// The ten network inputs (all O(1)):
//   0-5 strain increment / deq (its direction; clamped to +-8)
//   6   (log10 epOld + 3) / 3
//   7   (log10(total equivalent strain rate in 1/s) - 1.5) / 3   (time unit of dt: ms)
//   8   homologous temperature (T - Tref) / (Tmelt - Tref)
//   9   trial overstress above the old yield stress, xf / deq, clamped to [-2, 2]: the
//       old-stress information the update depends on through the trial state
__device__ __forceinline__ void surrogate_features(const JcParams &p, double dt, const double *inc,
                                                   const JcTrial &t, float *f) {
  double deq = equivalent_increment(inc);
  deq = deq > 1.0e-300 ? deq : 1.0e-300;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double v = inc[c] / deq;
    v = v > 8.0 ? 8.0 : (v < -8.0 ? -8.0 : v);
    f[c] = (float)v;
  }
  const double ep = t.epOld > 1.0e-12 ? t.epOld : 1.0e-12;
  f[6] = (float)((log10(ep) + 3.0) / 3.0);
  double rate = deq / dt * 1.0e3;
  rate = rate > 1.0e-12 ? rate : 1.0e-12;
  f[7] = (float)((log10(rate) - 1.5) / 3.0);
  f[8] = (float)((t.temperature - p.tref) / (p.tmelt - p.tref));
  double over = floor_increment(p, t) / deq;
  over = over > 2.0 ? 2.0 : (over < -2.0 ? -2.0 : over);
  f[9] = (float)over;
}

// Yield stress of the trial state at epInc = 0, as the bisection's first iteration takes it.
__device__ __forceinline__ double jc_yield0(const JcParams &p, const JcTrial &t) {
  const double y = jc_yield_t(p, t.epOld, 0.0, t.thermal);
  return y > t.oldYield ? y : t.oldYield;
}

// Newton on r in u = ln x from x, kept inside (0, xf] (the root's bracket). In u the rate
// term C sigma ln(x / dt), which dominates the curvature of r at the small increments of an
// explicit step, is linear, so the steps x <- x exp(-r / (x r'(x))) converge from guesses
// that an x-space Newton step would not. Returns true with the accepted increment and its
// yield once |r| < tolerance; evaluations counts the residuals formed (at most steps + 1).
__device__ __forceinline__ bool jc_newton(const JcParams &p, double dt, const JcTrial &t, double x, int steps,
                                          double &epInc, double &yield, int &evaluations) {
  const double hi = floor_increment(p, t), lo = 1.0e-12 * hi;
  x = x > lo ? x : lo;  // also maps NaN to lo
  x = x < hi ? x : hi;
  for (int k = 0;; ++k) {
    double slope, y;
    const double r = jc_residual(p, dt, t, x, slope, y);
    ++evaluations;
    if (fabs(r) < p.tolerance) {
      epInc = x, yield = y;
      return true;
    }
    if (k == steps || !(slope < 0.0))
      return false;
    double next = x * exp(-r / (x * slope));
    next = next < hi ? next : hi;
    if (!(next > 0.0))
      return false;
    x = next;
  }
}

}  // namespace vpd
