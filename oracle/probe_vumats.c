/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- not part of the product path.
 *
 * C restatements of the reference's two non-JC plugins, each exporting the bridge
 * entry `vumat_adapter_call` (materials/bridge/vumat_c_wrapper_jinfo.f90:1-44):
 *   -DVPD_PROBE   tests/fixtures/ContractProbe.f90:1-38 (component-sensitive ABI probe)
 *   -DVPD_ELASTIC materials/examples/Elastic.f:1-58   (linear elastic)
 * Column-major [component][nblock] arrays, element (k, c) at k + nblock * c.
 */
#define IDX(k, c) ((k) + nb * (c))

void vumat_adapter_call(int *nblock, int *ndir, int *nshr, int *nstatev, int *nfieldv, int *nprops,
                        int *lanneal, double *stepTime, double *totalTime, double *dt,
                        char *cmname, double *coordMp, double *charLength, double *props,
                        double *density, double *strainInc, double *relSpinInc, double *tempOld,
                        double *stretchOld, double *defgradOld, double *fieldOld,
                        double *stressOld, double *stateOld, double *enerInternOld,
                        double *enerInelasOld, double *tempNew, double *stretchNew,
                        double *defgradNew, double *fieldNew, double *stressNew, double *stateNew,
                        double *enerInternNew, double *enerInelasNew) {
  const int nb = *nblock;
  (void)lanneal, (void)cmname, (void)coordMp, (void)fieldOld, (void)fieldNew, (void)stretchNew;
  (void)defgradNew, (void)nfieldv, (void)nprops;
#if defined(VPD_PROBE)
  /* ContractProbe.f90:18-36 */
  (void)ndir, (void)nshr, (void)props;
  for (int k = 0; k < nb; ++k) {
    double incSum = 0.0;
    for (int c = 0; c < 6; ++c) {
      stressNew[IDX(k, c)] = stressOld[IDX(k, c)] + (double)(c + 1) * strainInc[IDX(k, c)];
      incSum = incSum + strainInc[IDX(k, c)];
    }
    for (int c = 0; c < 9; ++c) {
      stateNew[IDX(k, c)] = defgradOld[IDX(k, c)];
      stateNew[IDX(k, 9 + c)] = defgradNew[IDX(k, c)];
    }
    for (int c = 0; c < 6; ++c) {
      stateNew[IDX(k, 18 + c)] = stretchOld[IDX(k, c)];
      stateNew[IDX(k, 24 + c)] = stretchNew[IDX(k, c)];
    }
    for (int c = 0; c < 3; ++c)
      stateNew[IDX(k, 30 + c)] = relSpinInc[IDX(k, c)];
    stateNew[IDX(k, 33)] = stateOld[IDX(k, 33)] + 1.0;
    stateNew[IDX(k, 34)] = density[k];
    stateNew[IDX(k, 35)] = charLength[k];
    stateNew[IDX(k, 36)] = (double)nb;
    stateNew[IDX(k, 37)] = *stepTime;
    stateNew[IDX(k, 38)] = *totalTime;
    tempNew[k] = tempOld[k] + stateOld[IDX(k, 33)] + dt[0];
    enerInternNew[k] = enerInternOld[k] + incSum;
    enerInelasNew[k] = enerInelasOld[k] + 2.0 * incSum;
  }
  (void)nstatev;
#elif defined(VPD_ELASTIC)
  /* Elastic.f:24-56 */
  (void)stepTime, (void)totalTime, (void)dt, (void)charLength, (void)density, (void)relSpinInc;
  (void)stretchOld, (void)defgradOld;
  const double e = props[0], anu = props[1];
  const double alam = e * anu / ((1.0 + anu) * (1.0 - 2.0 * anu));
  const double amu = e / (2.0 * (1.0 + anu));
  double cmat[6][6] = {{0}};
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j)
      cmat[i][j] = alam;
    cmat[i][i] = alam + 2.0 * amu;
  }
  for (int i = 3; i < 6; ++i)
    cmat[i][i] = 2.0 * amu;
  const int ntens = *ndir + *nshr;
  for (int k = 0; k < nb; ++k) {
    for (int i = 0; i < ntens; ++i) {
      stressNew[IDX(k, i)] = stressOld[IDX(k, i)];
      for (int j = 0; j < ntens; ++j)
        stressNew[IDX(k, i)] = stressNew[IDX(k, i)] + cmat[i][j] * strainInc[IDX(k, j)];
    }
    tempNew[k] = tempOld[k];
    enerInternNew[k] = enerInternOld[k];
    enerInelasNew[k] = enerInelasOld[k];
    for (int i = 0; i < *nstatev; ++i)
      stateNew[IDX(k, i)] = stateOld[IDX(k, i)];
  }
#else
#error "define VPD_PROBE or VPD_ELASTIC"
#endif
}
