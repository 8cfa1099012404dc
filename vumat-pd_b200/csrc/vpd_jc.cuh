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

// One evaluation of the bisection (:118-124): the yield stress at epInc, floored at the old
// yield, and the residual qNew - yield.
__device__ __forceinline__ double jc_bisect_residual(const JcParams &p, double dt, const JcTrial &t, double epInc,
                                                     double &yield) {
  const double epRate = epInc / dt;
  yield = jc_yield_t(p, t.epOld + epInc, epRate, t.thermal);
  yield = yield > t.oldYield ? yield : t.oldYield;
  double qNew = t.qTrial - 3.0 * p.mu * epInc;
  qNew = qNew > 0.0 ? qNew : 0.0;
  return qNew - yield;
}

// Bracketed bisection with warm start (:114-136): plastic increment and yield stress; returns
// the iteration count. Every iteration evaluates the flow stress (one pow and one log).
__device__ __forceinline__ int jc_bisection(const JcParams &p, double dt, const JcTrial &t, double warmStart,
                                            double &epIncOut, double &yieldOut) {
  double epInc = 0.0, epLower = 0.0, epUpper = t.qTrial / (2.0 * p.mu), yield = t.oldYield;
  int iteration = 0;
  while (iteration < 50) {
    ++iteration;
    const double residual = jc_bisect_residual(p, dt, t, epInc, yield);
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

// r(x) with its slope. The residual is formed exactly as in the bisection (the same flow
// stress arithmetic, floor at oldYield, qNew clipped at 0) with one pow and one log; the slope
// differentiates the hardening term B n ep^(n-1) = B n ep^n / ep and the rate term C / x (zero
// at x = 0, where the VUMAT uses the reference rate).
__device__ __forceinline__ double jc_residual(const JcParams &p, double dt, const JcTrial &t, double x,
                                              double &slope, double &yield) {
  const double ep = t.epOld + x, rate = x / dt;
  const double hp = pow(ep, p.hardN), rterm = jc_rate_term(p, rate);
  const double y = jc_flow(p, hp, t.thermal, rterm);
  yield = y > t.oldYield ? y : t.oldYield;
  double qNew = t.qTrial - 3.0 * p.mu * x;
  const bool clipped = qNew <= 0.0;
  qNew = clipped ? 0.0 : qNew;
  double dy = 0.0;
  if (y > t.oldYield) {
    const double hard = p.a0 + p.b0 * hp;
    const double dhard = ep > 0.0 ? p.b0 * p.hardN * hp / ep : 0.0;
    const double drate = rate == 0.0 ? 0.0 : p.rateC / x;
    dy = (dhard * rterm + hard * drate) * t.thermal;
  }
  slope = (clipped ? 0.0 : -3.0 * p.mu) - dy;
  return qNew - yield;
}

// ------------------------------------------------------------------ certified bisection
// jc_return_map takes the same decisions as jc_bisection, and so returns the same increment,
// yield stress and iteration count bit for bit, while evaluating the flow stress only where a
// decision cannot be proven without it.
//
// For x > 0 the floored yield Y(x) = max(sigma_y(epOld + x, x / dt, T), oldYield) does not
// decrease with x: the hardening term grows with the plastic strain, the rate term
// 1 + C ln(x / (dt rate0)) grows with x, the thermal factor is fixed during a return, and
// wherever the rate term is negative the product is negative and the floor holds Y at oldYield.
// qNew(x) = max(qTrial - 3 mu x, 0) is known without the flow stress. So an exact evaluation
// of Y at an anchor a bounds Y at every other point: Y(m) <= Y(a) for m <= a, Y(m) >= Y(a)
// for m >= a, and Y(m) >= oldYield everywhere. Where those bounds put the residual
// r(m) = qNew(m) - Y(m) beyond the tolerance by more than a margin (1e-10 of the stresses
// involved, far above the rounding of pow, log and the subtraction), the bisection's branch at
// m is known: no convergence, and the sign of r. Only the remaining midpoints are evaluated,
// with the bisection's own arithmetic (jc_bisect_residual); the yield stress returned is
// always an exact evaluation at the last iteration's point.
//
// The anchors straddle the root closely. From the point the bisection visits after epInc = 0
// (the warm start; the upper end of the root's bracket where there is none), Newton steps on r
// in u = ln x (as jc_newton) move x towards the root until the step starts from |r| <= 256 tol
// (one step from the warm start of steady plastic flow, at most three); then Y is evaluated at
// x -+ 1.125 tol / |r'|, just outside the band |r| < tol where the bisection converges.
// Midpoints outside the pair are decided from them, and midpoints inside it are mostly those
// where the bisection converges. Where the steps fail (a NaN, a non-negative slope) the anchors
// stay NaN and only the oldYield floor is used, which decides nothing wrongly but evaluates
// more midpoints; so do anchors that miss the band.
//
// The lanes of a warp evaluate together: each lane runs its decided iterations up to the next
// one that needs an evaluation, then the lanes that need one evaluate at once, so a warp pays
// for the most evaluations any of its lanes needs rather than for every iteration index at which
// some lane needs one. Newton's steps are shared the same way.
struct JcAnchors {
  double a, ya, b, yb;  // a < b, with the floored yield at each (NaN where absent)
  double margin;
};

// The anchors' bounds as two thresholds on the midpoint m: the bisection's branch is proven
// positive (r(m) >= tol) for mmin < m <= lo and negative (r(m) <= -tol) for m >= hi.
struct JcThresholds {
  double lo, hi, mmin;
};

// Every lane of `lanes` calls it; lanes with active false only take part in the votes.
__device__ __forceinline__ JcAnchors jc_anchors(const JcParams &p, double dt, const JcTrial &t, double x0,
                                                bool active, unsigned lanes) {
  JcAnchors an{NAN, NAN, NAN, NAN, 0.0};
  const double hi = (t.qTrial - t.oldYield) / (3.0 * p.mu);  // r(hi) <= 0: the root lies in (0, hi]
  an.margin = 1.0e-10 * (fabs(t.qTrial) + fabs(t.oldYield));
  // the monotonicity of Y needs non-negative hardening, rate and thermal factors, a positive
  // time step and reference rate, and non-negative old plastic strain and yield stress
  const bool monotone = p.a0 >= 0.0 && p.b0 >= 0.0 && p.hardN >= 0.0 && p.rateC >= 0.0 && p.rate0 > 0.0 &&
                        dt > 0.0 && t.thermal >= 0.0 && t.epOld >= 0.0 && t.oldYield >= 0.0;
  bool go = active && monotone && hi > 0.0, placed = false;
  double x = x0 > 0.0 ? (x0 < hi ? x0 : hi) : hi;
  x = x > 1.0e-12 * hi ? x : 1.0e-12 * hi;  // also maps NaN
  double w = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (go) {
      double slope, y;
      const double r = jc_residual(p, dt, t, x, slope, y);
      double next = x * exp(-r / (x * slope));
      next = next < hi ? next : hi;
      if (!(r == r) || !(slope < 0.0) || !(next > 0.0)) {
        go = false;
      } else {
        x = next, w = 1.125 * p.tolerance / (-slope), placed = true;
        go = fabs(r) > 256.0 * p.tolerance;
      }
    }
    if (!__any_sync(lanes, go))
      break;
  }
  if (placed) {
    const double a = x - w, b = x + w;
    if (a > 0.0 && a > dt * 0x1p-1020) {  // (a / dt must not underflow to the rate-free x = 0 form)
      jc_bisect_residual(p, dt, t, a, an.ya);
      an.a = an.ya == an.ya ? a : NAN;
    }
    jc_bisect_residual(p, dt, t, b, an.yb);
    an.b = an.yb == an.yb ? b : NAN;
    // stresses the rounding scales with: the trial and yield stresses, and the flow stress
    // before the rate factor (where 1 + C ln(rate) nearly cancels)
    const double flow = (p.a0 + p.b0 * (1.0 + t.epOld + b)) * t.thermal * (1.0 + 128.0 * p.rateC);
    an.margin = 1.0e-10 * (fabs(t.qTrial) + fabs(t.oldYield) + (an.a == an.a ? fabs(an.ya) : 0.0) +
                           (an.b == an.b ? fabs(an.yb) : 0.0) + flow);
  }
  return an;
}

// The midpoints whose branch the anchors prove. With an anchor c (floored yield Y(c)):
//   for mmin < m <= c, Y(m) <= Y(c), so r(m) >= qNew(m) - Y(c): positive where
//     qTrial - 3 mu m >= tol + Y(c) + margin, i.e. m <= (qTrial - tol - Y(c) - margin) / (3 mu);
//   for m >= c, Y(m) >= Y(c), so r(m) <= qNew(m) - Y(c): negative where
//     max(qTrial - 3 mu m, 0) <= Y(c) - tol - margin, i.e. (given Y(c) >= tol + margin)
//     m >= (qTrial - Y(c) + tol + margin) / (3 mu);
// and everywhere Y(m) >= oldYield gives the second form with oldYield for Y(c). mmin keeps
// m / dt from underflowing to the rate-free x = 0 form. The margin (1e-10 of the stresses
// involved) covers the rounding of qNew, of these quotients and of the evaluations. NaN anchors
// give NaN thresholds, which prove nothing.
__device__ __forceinline__ JcThresholds jc_thresholds(const JcParams &p, double dt, const JcTrial &t,
                                                      const JcAnchors &an) {
  const double m3 = 3.0 * p.mu, tol = p.tolerance, g = an.margin;
  JcThresholds th;
  th.mmin = dt * 0x1p-1020;
  double lo = -INFINITY, hi = INFINITY;
  // (every bound is taken only where it is a number: a NaN proves nothing)
  const double anchor[2] = {an.a, an.b}, yc[2] = {an.ya, an.yb};
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double c = anchor[k], y = yc[k];
    if (!(c == c))
      continue;
    const double pc = (t.qTrial - tol - y - g) / m3;
    if (pc == pc) {
      const double v = pc < c ? pc : c;
      lo = lo > v ? lo : v;
    }
    if (y >= tol + g) {
      const double nc = (t.qTrial - y + tol + g) / m3;
      if (nc == nc) {
        const double v = nc > c ? nc : c;
        hi = hi < v ? hi : v;
      }
    }
  }
  if (t.oldYield >= tol + g) {
    const double nf = (t.qTrial - t.oldYield + tol + g) / m3;
    if (nf == nf)
      hi = hi < nf ? hi : nf;
  }
  th.lo = lo, th.hi = hi;
  if (!(lo < hi))  // contradictory bounds would mean a broken premise: prove nothing
    th.lo = -INFINITY, th.hi = INFINITY;
  return th;
}

// The bisection of jc_bisection with its branches decided by jc_thresholds where possible (see
// above): the same epInc, yield and iteration count. Every lane of the calling warp that is
// active at the call takes part in its votes.
__device__ __forceinline__ int jc_return_map(const JcParams &p, double dt, const JcTrial &t, double warmStart,
                                             double &epIncOut, double &yieldOut) {
  const unsigned lanes = __activemask();
  double epInc = 0.0, epLower = 0.0, epUpper = t.qTrial / (2.0 * p.mu), yield = t.oldYield;
  JcThresholds th{-INFINITY, INFINITY, 0.0};
  bool done = false, exact = true, anchored = false;
  double lastX = 0.0;
  int iteration = 0;
  for (;;) {
    // the iterations the anchors decide, up to the next one that needs an evaluation
    bool pending = false;
    while (!done) {
      if (iteration >= 50) {
        done = true;
        break;
      }
      const bool up = epInc <= th.lo && epInc > th.mmin, down = epInc >= th.hi;
      if (!(up || down)) {
        pending = true;
        break;
      }
      ++iteration;
      exact = false;
      lastX = epInc;
      if (up)
        epLower = epLower > epInc ? epLower : epInc;
      else
        epUpper = epUpper < epInc ? epUpper : epInc;
      epInc = 0.5 * (epLower + epUpper);  // (iteration > 1 here: the first is never decided)
    }
    if (!__any_sync(lanes, pending))
      break;
    if (pending) {  // one iteration of jc_bisection
      ++iteration;
      const double residual = jc_bisect_residual(p, dt, t, epInc, yield);
      exact = true;
      if (fabs(residual) < p.tolerance || (epInc == 0.0 && residual < 0.0)) {
        done = true;
      } else {
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
    }
    if (!anchored) {  // once, after the first iteration, by the whole warp
      th = jc_thresholds(p, dt, t, jc_anchors(p, dt, t, epInc, !done, lanes));
      anchored = true;
    }
  }
  if (!exact)  // 50 iterations ending on a decided one: its yield stress, evaluated
    jc_bisect_residual(p, dt, t, lastX, yield);
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
// bisection iteration count (0 on the initialising call). CERTIFIED: the return map of
// jc_return_map (same results, fewer flow-stress evaluations), else the literal bisection.
template <bool CERTIFIED = true>
__device__ __forceinline__ int jc_update(const JcParams &p, double dt, const double *inc, JcPoint &pt) {
  JcTrial t;
  if (!jc_trial(p, inc, pt, t))
    return 0;
  double epInc, yield;
  const int iteration = CERTIFIED ? jc_return_map(p, dt, t, pt.state[4], epInc, yield)
                                  : jc_bisection(p, dt, t, pt.state[4], epInc, yield);
  jc_finish(p, inc, t, epInc, yield, (double)iteration, pt);
  return iteration;
}

}  // namespace vpd
