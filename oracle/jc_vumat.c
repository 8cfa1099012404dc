/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- not part of the product path.
 *
 * C restatement of the reference Johnson-Cook VUMAT and its C-ABI bridge, so the
 * reference C++ library (compiled from its own sources into oracle/_ref) can load a
 * material plugin without a Fortran compiler, and so the CPU oracle has the same
 * constitutive update.
 *
 *   materials/examples/JohnsonCook.f90:12-172   (vumat, jc_yield)
 *   materials/bridge/vumat_c_wrapper_jinfo.f90:1-44 (vumat_adapter_call entry)
 *
 * Arithmetic follows the Fortran expression order term by term (left-associative
 * products and sums, x**2 as x*x, SUM as a sequential loop); build with
 * -ffp-contract=off so no FMA contraction changes the roundings.
 *
 * Array layout (the plugin ABI): every per-point array is Fortran column-major
 * [component][nblock], element (k, c) at index k + nblock * c.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define IDX(k, c) ((k) + nb * (c))

/* JohnsonCook.f90:160-170 */
static double jc_yield(double a, double b, double c, double n, double m, double refRate,
                       double refTemp, double meltTemp, double ep, double rate, double temp) {
  double theta = (temp - refTemp) / (meltTemp - refTemp);
  theta = theta > 0.0 ? theta : 0.0; /* max(0, .) */
  theta = theta < 1.0 ? theta : 1.0; /* min(1, .) */
  double effectiveRate = rate;
  if (effectiveRate == 0.0)
    effectiveRate = refRate;
  return (a + b * pow(ep, n)) * (1.0 - pow(theta, m)) * (1.0 + c * log(effectiveRate / refRate));
}

/* Johnson-Cook update of one block, JohnsonCook.f90:43-156. */
static void jc_vumat(int nb, int nstatev, int nfieldv, int nprops, double dt, const double *props,
                     const double *strainInc, const double *tempOld, const double *stretchOld,
                     const double *defgradOld, const double *fieldOld, const double *stressOld,
                     const double *stateOld, const double *enerInternOld,
                     const double *enerInelasOld, double *tempNew, double *stretchNew,
                     double *defgradNew, double *fieldNew, double *stressNew, double *stateNew,
                     double *enerInternNew, double *enerInelasNew) {
  if (nprops < 14 || nstatev < 6) {
    /* JohnsonCook.f90:53 -- Fortran `stop` ends the process. */
    fprintf(stderr, "JohnsonCook VUMAT requires 14 props and 6 states\n");
    exit(1);
  }
  const double young = props[0], poisson = props[1], a0 = props[2], b0 = props[3];
  const double rateC = props[4], hardN = props[5], thermalM = props[6], rate0 = props[7];
  const double tref = props[8], tmelt = props[9], rho = props[10], beta = props[11];
  const double cp = props[12], workToHeat = props[13];
  const double mu = young / (2.0 * (1.0 + poisson));
  const double lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
  const double tolerance = young * 1.0e-9;

  for (int k = 0; k < nb; ++k) {
    double trial[6], deviator[6], updated[6], oldStress[6];
    const double traceInc = strainInc[IDX(k, 0)] + strainInc[IDX(k, 1)] + strainInc[IDX(k, 2)];
    for (int i = 0; i < 3; ++i)
      trial[i] = stressOld[IDX(k, i)] + lambda * traceInc + 2.0 * mu * strainInc[IDX(k, i)];
    for (int i = 3; i < 6; ++i)
      trial[i] = stressOld[IDX(k, i)] + 2.0 * mu * strainInc[IDX(k, i)];
    for (int i = 0; i < 6; ++i)
      updated[i] = trial[i];
    for (int c = 0; c < nstatev; ++c)
      stateNew[IDX(k, c)] = stateOld[IDX(k, c)];
    tempNew[k] = tempOld[k];
    enerInternNew[k] = enerInternOld[k];
    enerInelasNew[k] = enerInelasOld[k];
    for (int c = 0; c < 6; ++c)
      stretchNew[IDX(k, c)] = stretchOld[IDX(k, c)];
    for (int c = 0; c < 9; ++c)
      defgradNew[IDX(k, c)] = defgradOld[IDX(k, c)];
    for (int c = 0; c < nfieldv; ++c)
      fieldNew[IDX(k, c)] = fieldOld[IDX(k, c)];

    if (stateOld[IDX(k, 0)] == 0.0) { /* first-call initialisation, :92-102 */
      stateNew[IDX(k, 0)] = 1.0;
      stateNew[IDX(k, 1)] = 0.0;
      stateNew[IDX(k, 2)] = tref;
      stateNew[IDX(k, 3)] = 0.0;
      stateNew[IDX(k, 4)] = 0.0;
      stateNew[IDX(k, 5)] = 1.0;
      tempNew[k] = tref;
      for (int i = 0; i < 6; ++i)
        stressNew[IDX(k, i)] = updated[i];
      continue;
    }

    for (int i = 0; i < 6; ++i)
      oldStress[i] = stressOld[IDX(k, i)];
    const double epOld = stateOld[IDX(k, 1)];
    const double temperature = stateOld[IDX(k, 2)];
    const double oldYield = stateOld[IDX(k, 3)];
    const double pressure = (trial[0] + trial[1] + trial[2]) / 3.0;
    for (int i = 0; i < 3; ++i)
      deviator[i] = trial[i] - pressure;
    for (int i = 3; i < 6; ++i)
      deviator[i] = trial[i];
    const double qTrial =
        sqrt(1.5 * (deviator[0] * deviator[0] + deviator[1] * deviator[1] +
                    deviator[2] * deviator[2] +
                    2.0 * (deviator[3] * deviator[3] + deviator[4] * deviator[4] +
                           deviator[5] * deviator[5])));

    /* Bracketed bisection return map with warm start, :114-136. */
    double epInc = 0.0, epLower = 0.0, epUpper = qTrial / (2.0 * mu);
    double yield = oldYield;
    int iteration = 0;
    while (iteration < 50) {
      iteration = iteration + 1;
      const double epRate = epInc / dt;
      yield = jc_yield(a0, b0, rateC, hardN, thermalM, rate0, tref, tmelt, epOld + epInc, epRate,
                       temperature);
      yield = yield > oldYield ? yield : oldYield;
      double qNew = qTrial - 3.0 * mu * epInc;
      qNew = qNew > 0.0 ? qNew : 0.0;
      const double residual = qNew - yield;
      if (fabs(residual) < tolerance)
        break;
      if (epInc == 0.0 && residual < 0.0)
        break;
      if (residual >= 0.0)
        epLower = epLower > epInc ? epLower : epInc;
      else
        epUpper = epUpper < epInc ? epUpper : epInc;
      epInc = 0.5 * (epLower + epUpper);
      if (iteration == 1) {
        double warm = stateOld[IDX(k, 4)];
        warm = warm > epLower ? warm : epLower;
        epInc = warm < epUpper ? warm : epUpper;
      }
    }

    if (qTrial > 0.0) { /* radial scaling, :138-142 */
      double scale = 1.0 - 3.0 * mu * epInc / qTrial;
      scale = scale > 0.0 ? scale : 0.0;
      for (int i = 0; i < 3; ++i)
        updated[i] = pressure + scale * deviator[i];
      for (int i = 3; i < 6; ++i)
        updated[i] = scale * deviator[i];
    }
    double qNew = qTrial - 3.0 * mu * epInc;
    qNew = qNew > 0.0 ? qNew : 0.0;
    double work = 0.0; /* SUM((oldStress + updated) * strainInc(k,:)) */
    for (int i = 0; i < 6; ++i)
      work = work + (oldStress[i] + updated[i]) * strainInc[IDX(k, i)];
    const double workInc = 0.5 * work;
    const double plasticWork = 0.5 * epInc * qNew;
    for (int i = 0; i < 6; ++i)
      stressNew[IDX(k, i)] = updated[i];
    enerInternNew[k] = enerInternOld[k] + workInc / rho;
    enerInelasNew[k] = enerInelasOld[k] + plasticWork / rho;
    stateNew[IDX(k, 0)] = 1.0;
    stateNew[IDX(k, 1)] = epOld + epInc;
    stateNew[IDX(k, 2)] = temperature + workToHeat * beta * plasticWork / (rho * cp);
    stateNew[IDX(k, 3)] = yield;
    stateNew[IDX(k, 4)] = epInc;
    stateNew[IDX(k, 5)] = stateOld[IDX(k, 5)] + (double)iteration;
    tempNew[k] = stateNew[IDX(k, 2)];
  }
}

/* C entry with the bridge's signature, vumat_c_wrapper_jinfo.f90:1-44. The bridge's
 * jInfoArray (lanneal, 7, block labels) is not read by this routine; dt is dtArray(1). */
void vumat_adapter_call(int *nblock, int *ndir, int *nshr, int *nstatev, int *nfieldv, int *nprops,
                        int *lanneal, double *stepTime, double *totalTime, double *dt,
                        char *cmname, double *coordMp, double *charLength, double *props,
                        double *density, double *strainInc, double *relSpinInc, double *tempOld,
                        double *stretchOld, double *defgradOld, double *fieldOld,
                        double *stressOld, double *stateOld, double *enerInternOld,
                        double *enerInelasOld, double *tempNew, double *stretchNew,
                        double *defgradNew, double *fieldNew, double *stressNew, double *stateNew,
                        double *enerInternNew, double *enerInelasNew) {
  (void)lanneal, (void)stepTime, (void)totalTime, (void)cmname, (void)coordMp, (void)charLength;
  (void)density, (void)relSpinInc;
  if (*ndir != 3 || *nshr != 3) { /* JohnsonCook.f90:52 */
    fprintf(stderr, "JohnsonCook VUMAT requires ndir=3,nshr=3\n");
    exit(1);
  }
  jc_vumat(*nblock, *nstatev, *nfieldv, *nprops, *dt, props, strainInc, tempOld, stretchOld,
           defgradOld, fieldOld, stressOld, stateOld, enerInternOld, enerInelasOld, tempNew,
           stretchNew, defgradNew, fieldNew, stressNew, stateNew, enerInternNew, enerInelasNew);
}
