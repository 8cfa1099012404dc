/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- the checker for libvpd_gpu.so, never shipped or timed
 * as the product. Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline.
 *
 * CPU restatement (C11 + OpenMP) of the reference's correspondence-peridynamics increment,
 * 1998yu/vumat-pd. Each function cites the reference lines it follows and keeps their
 * floating-point operation order (products and sums left to right, no FMA contraction:
 * build with -ffp-contract=off), so a run matches the reference library bit for bit on
 * the reference's own cases. The Johnson-Cook VUMAT comes from jc_vumat.c.
 *
 * Layout follows the reference: point-major arrays, Tensor3 row-major (9 doubles), Vec3
 * (3 doubles), neighbour lists as CSR (row_ptr int64, col int32), bond damage one double
 * per CSR entry (include/PdTypes.hpp:9-47, include/PdSimpleDamage.hpp:11-21).
 *
 * Extensions beyond the reference, shared with the GPU path and defined here once:
 *   - seeded lattice jitter (counter-based splitmix64, vo_jitter_value);
 *   - the regional_velocity_ramp boundary condition (vo_ramp, mode VPD_BC_VELOCITY_RAMP);
 *   - boundary bands, pins and the observation window taken from the un-jittered lattice.
 */
#include "../include/vpd_gpu.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void vumat_adapter_call(int *nblock, int *ndir, int *nshr, int *nstatev, int *nfieldv, int *nprops,
                        int *lanneal, double *stepTime, double *totalTime, double *dt,
                        char *cmname, double *coordMp, double *charLength, double *props,
                        double *density, double *strainInc, double *relSpinInc, double *tempOld,
                        double *stretchOld, double *defgradOld, double *fieldOld,
                        double *stressOld, double *stateOld, double *enerInternOld,
                        double *enerInelasOld, double *tempNew, double *stretchNew,
                        double *defgradNew, double *fieldNew, double *stressNew, double *stateNew,
                        double *enerInternNew, double *enerInelasNew);

/* case_ext.c: extensions shared with the GPU path */
double vo_jitter_value(uint64_t seed, int64_t p, int c, double amp);
void vo_ramp(const vpd_case *c, double t, double *out);

/* ------------------------------------------------------------------ 3x3 algebra */
/* PdCorrespondenceSkeleton.cpp:52-91 and CorotationalKinematics.cpp:13-57 */
static void m_mul(const double *a, const double *b, double *out) {
  double t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k)
        s += a[3 * i + k] * b[3 * k + j];
      t[3 * i + j] = s;
    }
  memcpy(out, t, sizeof t);
}
static void m_vec(const double *a, const double *x, double *out) {
  double t0 = a[0] * x[0] + a[1] * x[1] + a[2] * x[2];
  double t1 = a[3] * x[0] + a[4] * x[1] + a[5] * x[2];
  double t2 = a[6] * x[0] + a[7] * x[1] + a[8] * x[2];
  out[0] = t0, out[1] = t1, out[2] = t2;
}
static void m_tr(const double *a, double *out) {
  double t[9] = {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]};
  memcpy(out, t, sizeof t);
}
static double m_det(const double *a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}
/* Cofactor inverse; returns 0 (and leaves out untouched) when |det| < 1e-14. The two
   reference variants (:67-76 and CorotationalKinematics.cpp:45-54) round identically. */
static int m_inv(const double *a, double *out) {
  const double det = m_det(a);
  if (fabs(det) < 1.0e-14)
    return 0;
  double t[9] = {(a[4] * a[8] - a[5] * a[7]) / det, -(a[1] * a[8] - a[2] * a[7]) / det,
                 (a[1] * a[5] - a[2] * a[4]) / det, -(a[3] * a[8] - a[5] * a[6]) / det,
                 (a[0] * a[8] - a[2] * a[6]) / det, -(a[0] * a[5] - a[2] * a[3]) / det,
                 (a[3] * a[7] - a[4] * a[6]) / det, -(a[0] * a[7] - a[1] * a[6]) / det,
                 (a[0] * a[4] - a[1] * a[3]) / det};
  memcpy(out, t, sizeof t);
  return 1;
}
static const double I9[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

/* ------------------------------------------------------------------ neighbours */
typedef struct {
  long long cx, cy, cz;
  int64_t idx;
} vo_cell_entry;
static int cmp_cell(const void *pa, const void *pb) {
  const vo_cell_entry *a = pa, *b = pb;
  if (a->cx != b->cx) return a->cx < b->cx ? -1 : 1;
  if (a->cy != b->cy) return a->cy < b->cy ? -1 : 1;
  if (a->cz != b->cz) return a->cz < b->cz ? -1 : 1;
  return a->idx < b->idx ? -1 : (a->idx > b->idx);
}
static int cmp_int(const void *pa, const void *pb) {
  int a = *(const int *)pa, b = *(const int *)pb;
  return (a > b) - (a < b);
}
static int64_t lower_cell(const vo_cell_entry *e, int64_t n, long long cx, long long cy,
                          long long cz) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    const vo_cell_entry *m = &e[mid];
    int less = m->cx != cx ? m->cx < cx : (m->cy != cy ? m->cy < cy : m->cz < cz);
    if (less) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* horizonTolerance, PdCorrespondenceSkeleton.cpp:30-39. Returns <0 for non-finite input. */
double vo_horizon_tolerance(const double *pos, int64_t n, double horizon) {
  double scale = horizon;
  for (int64_t i = 0; i < 3 * n; ++i) {
    if (!isfinite(pos[i]))
      return -1.0;
    double v = fabs(pos[i]);
    scale = scale > v ? scale : v;
  }
  return 64.0 * 2.220446049250313080847e-16 * scale;
}

/* buildNeighborList, PdCorrespondenceSkeleton.cpp:95-129: candidates from the 27 cells of
   width delta+2tol, kept when |Xj - Xi| <= delta + tol, each row sorted ascending.
   col == NULL: fill row_ptr and return the total; else fill col using row_ptr. */
static int64_t neighbor_pass(const double *pos, int64_t n, double horizon, int64_t *row_ptr,
                             int32_t *col) {
  if (horizon <= 0.0 || n <= 0)
    return -VPD_ERR_INVALID;
  const double tolerance = vo_horizon_tolerance(pos, n, horizon);
  if (tolerance < 0.0)
    return -VPD_ERR_NONFINITE;
  const double radius = horizon + tolerance;
  const double cellWidth = horizon + 2.0 * tolerance;
  vo_cell_entry *cells = malloc(sizeof(vo_cell_entry) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    cells[i].cx = (long long)floor(pos[3 * i] / cellWidth);
    cells[i].cy = (long long)floor(pos[3 * i + 1] / cellWidth);
    cells[i].cz = (long long)floor(pos[3 * i + 2] / cellWidth);
    cells[i].idx = i;
  }
  vo_cell_entry *sorted = malloc(sizeof(vo_cell_entry) * (size_t)n);
  memcpy(sorted, cells, sizeof(vo_cell_entry) * (size_t)n);
  qsort(sorted, (size_t)n, sizeof(vo_cell_entry), cmp_cell);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    const double *pi = pos + 3 * i;
    int64_t count = 0;
    int32_t *row = col ? col + row_ptr[i] : NULL;
    for (long long dx = -1; dx <= 1; ++dx)
      for (long long dy = -1; dy <= 1; ++dy)
        for (long long dz = -1; dz <= 1; ++dz) {
          const long long cx = cells[i].cx + dx, cy = cells[i].cy + dy, cz = cells[i].cz + dz;
          for (int64_t s = lower_cell(sorted, n, cx, cy, cz);
               s < n && sorted[s].cx == cx && sorted[s].cy == cy && sorted[s].cz == cz; ++s) {
            const int64_t j = sorted[s].idx;
            if (j == i)
              continue;
            const double *pj = pos + 3 * j;
            const double a0 = pj[0] - pi[0], a1 = pj[1] - pi[1], a2 = pj[2] - pi[2];
            if (sqrt(a0 * a0 + a1 * a1 + a2 * a2) <= radius) {
              if (row)
                row[count] = (int32_t)j;
              ++count;
            }
          }
        }
    if (row)
      qsort(row, (size_t)count, sizeof(int32_t), cmp_int);
    else
      row_ptr[i + 1] = count;
  }
  free(cells);
  free(sorted);
  if (!col) {
    row_ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i)
      row_ptr[i + 1] += row_ptr[i];
    return row_ptr[n];
  }
  return row_ptr[n];
}
int64_t vo_neighbor_count(const double *pos, int64_t n, double horizon, int64_t *row_ptr) {
  return neighbor_pass(pos, n, horizon, row_ptr, NULL);
}
int vo_neighbor_fill(const double *pos, int64_t n, double horizon, const int64_t *row_ptr,
                     int32_t *col) {
  int64_t r = neighbor_pass(pos, n, horizon, (int64_t *)row_ptr, col);
  return r < 0 ? (int)-r : VPD_OK;
}

/* ------------------------------------------------------------------ skeleton */
/* PdCorrespondenceSkeleton::initialize, :149-170 */
int vo_shape_inverse(int64_t n, const double *pos, const double *vol, const int64_t *row_ptr,
                     const int32_t *col, double *kinv) {
  int status = VPD_OK;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double shape[9] = {0};
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
      const int64_t j = col[p];
      const double xi[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                            pos[3 * j + 2] - pos[3 * i + 2]};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          shape[3 * a + b] += vol[j] * xi[a] * xi[b];
    }
    if (!m_inv(shape, kinv + 9 * i)) {
#pragma omp atomic write
      status = VPD_ERR_SINGULAR;
    }
  }
  return status;
}

/* A planted rounding change for the sensitivity test (tests/test_oracle.py): when every > 0,
   the first component of the deformation sum of each point i with i % every == 3 is moved up
   by one unit in the last place before F is formed. 0 (the default) leaves the reference's
   arithmetic untouched. */
static int g_perturb_every = 0;
void vo_set_perturbation(int every) { g_perturb_every = every; }

/* computeDeformationGradients, :172-197 */
int vo_deformation(int64_t n, const double *pos, const double *disp, const double *vol,
                   const int64_t *row_ptr, const int32_t *col, const double *kinv, double *F) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double num[9] = {0};
    const double yi[3] = {pos[3 * i] + disp[3 * i], pos[3 * i + 1] + disp[3 * i + 1],
                          pos[3 * i + 2] + disp[3 * i + 2]};
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
      const int64_t j = col[p];
      double xi[3], yij[3];
      for (int d = 0; d < 3; ++d) {
        xi[d] = pos[3 * j + d] - pos[3 * i + d];
        yij[d] = (pos[3 * j + d] + disp[3 * j + d]) - yi[d];
      }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          num[3 * a + b] += vol[j] * yij[a] * xi[b];
    }
    if (g_perturb_every > 0 && i % g_perturb_every == 3)
      num[0] = nextafter(num[0], INFINITY);
    m_mul(num, kinv + 9 * i, F + 9 * i);
  }
  return VPD_OK;
}

/* cauchyToFirstPiola :83-91 then forceMap = P K^-1 (:209-211). 0 on a singular F. */
static int force_map(const double *sigma, const double *F, const double *kinv, double *M) {
  const double j = m_det(F);
  double finv[9], finvT[9], p[9];
  if (fabs(j) < 1.0e-14 || !m_inv(F, finv))
    return 0;
  m_tr(finv, finvT);
  m_mul(sigma, finvT, p);
  for (int c = 0; c < 9; ++c)
    p[c] *= j;
  m_mul(p, kinv, M);
  return 1;
}

/* computeForceDensity, :199-230 */
int vo_force(int64_t n, const double *pos, const double *vol, const int64_t *row_ptr,
             const int32_t *col, const double *kinv, const double *F, const double *sigma,
             const double *bond_damage, double *force) {
  double *M = malloc(sizeof(double) * 9 * (size_t)n);
  int status = VPD_OK;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    if (!force_map(sigma + 9 * i, F + 9 * i, kinv + 9 * i, M + 9 * i)) {
#pragma omp atomic write
      status = VPD_ERR_SINGULAR;
    }
  if (status == VPD_OK) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double f[3] = {0.0, 0.0, 0.0};
      for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        const int64_t j = col[p];
        const double xi[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                              pos[3 * j + 2] - pos[3 * i + 2]};
        const double nxi[3] = {-xi[0], -xi[1], -xi[2]};
        double ti[3], tj[3];
        m_vec(M + 9 * i, xi, ti);
        m_vec(M + 9 * j, nxi, tj);
        double dmg = bond_damage ? bond_damage[p] : 0.0;
        dmg = dmg < 0.0 ? 0.0 : (dmg > 1.0 ? 1.0 : dmg);
        const double intact = 1.0 - dmg;
        for (int d = 0; d < 3; ++d)
          f[d] += intact * (ti[d] - tj[d]) * vol[j];
      }
      force[3 * i] = f[0], force[3 * i + 1] = f[1], force[3 * i + 2] = f[2];
    }
  }
  free(M);
  return status;
}

/* ------------------------------------------------------------------ kinematics */
/* updateCorotationalKinematics, CorotationalKinematics.cpp:61-135. Outputs D-bar
   (unrotated rate of deformation), relative spin increment, R_n+1, V_n+1. */
static int corotational(const double *fN, const double *fNP1, const double *vN, const double *rN,
                        double dt, double *dbar, double *spin, double *rNew, double *vNew) {
  double fDot[9], fNinv[9], L[9], lt[9], d[9], w[9];
  for (int i = 0; i < 9; ++i)
    fDot[i] = (fNP1[i] - fN[i]) / dt;
  if (!m_inv(fN, fNinv))
    return 0;
  m_mul(fDot, fNinv, L);
  m_tr(L, lt);
  for (int i = 0; i < 9; ++i) {
    d[i] = 0.5 * (L[i] + lt[i]);
    w[i] = 0.5 * (L[i] - lt[i]);
  }
  const double zX =
      -vN[2] * d[3] - vN[5] * d[4] - vN[8] * d[5] + vN[1] * d[6] + vN[4] * d[7] + vN[7] * d[8];
  const double zY =
      vN[2] * d[0] + vN[5] * d[1] + vN[8] * d[2] - vN[0] * d[6] - vN[3] * d[7] - vN[6] * d[8];
  const double zZ =
      -vN[1] * d[0] - vN[4] * d[1] - vN[7] * d[2] + vN[0] * d[3] + vN[3] * d[4] + vN[6] * d[5];
  const double wX = 0.5 * (w[7] - w[5]);
  const double wY = 0.5 * (w[2] - w[6]);
  const double wZ = 0.5 * (w[3] - w[1]);
  const double trV = vN[0] + vN[4] + vN[8];
  double tiv[9], corr[9];
  for (int i = 0; i < 9; ++i)
    tiv[i] = I9[i] * trV - vN[i];
  if (!m_inv(tiv, corr))
    return 0;
  const double oX = wX + corr[0] * zX + corr[1] * zY + corr[2] * zZ;
  const double oY = wY + corr[3] * zX + corr[4] * zY + corr[5] * zZ;
  const double oZ = wZ + corr[6] * zX + corr[7] * zY + corr[8] * zZ;
  const double omega[9] = {0.0, -oZ, oY, oZ, 0.0, -oX, -oY, oX, 0.0};
  const double oSq = oX * oX + oY * oY + oZ * oZ;
  double q[9];
  memcpy(q, I9, sizeof q);
  if (oSq > 1.0e-30) {
    const double mag = sqrt(oSq);
    const double s1 = sin(dt * mag) / mag;
    const double hs = sin(0.5 * dt * mag);
    const double s2 = 2.0 * hs * hs / oSq;
    double o2[9];
    m_mul(omega, omega, o2);
    for (int i = 0; i < 9; ++i)
      q[i] += s1 * omega[i] + s2 * o2[i];
  }
  m_mul(q, rN, rNew);
  double ra[9], rb[9];
  m_mul(L, vN, ra);
  m_mul(vN, omega, rb);
  for (int i = 0; i < 9; ++i)
    vNew[i] = vN[i] + dt * (ra[i] - rb[i]);
  double rt[9], tmp[9];
  m_tr(rNew, rt);
  m_mul(d, rNew, tmp);
  m_mul(rt, tmp, dbar);
  double rel[9];
  for (int i = 0; i < 9; ++i)
    rel[i] = w[i] - omega[i];
  m_mul(rel, rNew, tmp);
  m_mul(rt, tmp, spin);
  for (int i = 0; i < 9; ++i)
    spin[i] *= dt;
  return 1;
}
/* greenLagrangeStrain :141-149 */
static void green_lagrange(const double *f, double *e) {
  double ft[9];
  m_tr(f, ft);
  m_mul(ft, f, e);
  e[0] -= 1.0, e[4] -= 1.0, e[8] -= 1.0;
  for (int i = 0; i < 9; ++i)
    e[i] *= 0.5;
}
/* rotateCorotationalStressToSpatial :137-139 */
static void rotate_to_spatial(const double *s, const double *r, double *out) {
  double rt[9], tmp[9];
  m_tr(r, rt);
  m_mul(s, rt, tmp);
  m_mul(r, tmp, out);
}

int vo_corotational(int64_t n, const double *fN, const double *fNP1, const double *vN,
                    const double *rN, double dt, double *dbar, double *spin, double *rNew,
                    double *vNew, double *strain) {
  int status = VPD_OK;
  if (!(dt > 0.0))
    return VPD_ERR_INVALID;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (!corotational(fN + 9 * i, fNP1 + 9 * i, vN + 9 * i, rN + 9 * i, dt, dbar + 9 * i,
                      spin + 9 * i, rNew + 9 * i, vNew + 9 * i)) {
#pragma omp atomic write
      status = VPD_ERR_SINGULAR;
    }
    green_lagrange(fNP1 + 9 * i, strain + 9 * i);
  }
  return status;
}

/* ------------------------------------------------------------------ material bridge */
/* One point of VumatPdCorrespondenceMaterial::update (:83-170): kinematics, legacy_vumat_pd
   packing (TensorVoigtMap.cpp:9-25, VumatMaterialAdapter.cpp:265-330), the VUMAT, and the
   history commit. State arrays are updated in place; sigmaSpatial/strainOut are outputs. */
static int material_point(const double *props, int nstatev, double dt, double stepTime,
                          double totalTime, double charLength, double densityKg,
                          const double *F, double *Fn, double *Vn, double *Rn, double *En,
                          double *sig, double *state, double *temp, double *eI, double *eP,
                          double *sigmaSpatial) {
  double dbar[9], spin[9], rNew[9], vNew[9], strain[9];
  if (!corotational(Fn, F, Vn, Rn, dt, dbar, spin, rNew, vNew))
    return 0;
  green_lagrange(F, strain);
  int nb = 1, ndir = 3, nshr = 3, nsv = nstatev, nfv = 1, np = 14, lanneal = 0;
  double st = stepTime, tt = totalTime, dtv = dt, cl = charLength, dens = densityKg;
  char cmname[80];
  memset(cmname, ' ', sizeof cmname);
  double coord[3] = {0, 0, 0}, fieldOld[1] = {0}, fieldNew[1] = {0};
  double strainInc[6] = {dbar[0], dbar[4], dbar[8], 0.5 * (dbar[5] + dbar[7]),
                         0.5 * (dbar[2] + dbar[6]), 0.5 * (dbar[1] + dbar[3])};
  for (int c = 0; c < 6; ++c)
    strainInc[c] *= dt;
  double relSpin[3] = {spin[5], spin[6], spin[1]};
  double stretchOld[6] = {Vn[0], Vn[4], Vn[8], 0.5 * (Vn[5] + Vn[7]), 0.5 * (Vn[2] + Vn[6]),
                          0.5 * (Vn[1] + Vn[3])};
  double stretchNewIn[6] = {vNew[0], vNew[4], vNew[8], 0.5 * (vNew[5] + vNew[7]),
                            0.5 * (vNew[2] + vNew[6]), 0.5 * (vNew[1] + vNew[3])};
  double stressOld[6] = {sig[0], sig[4], sig[8], 0.5 * (sig[5] + sig[7]),
                         0.5 * (sig[2] + sig[6]), 0.5 * (sig[1] + sig[3])};
  double defOld[9] = {Fn[0], Fn[4], Fn[8], Fn[1], Fn[5], Fn[6], Fn[3], Fn[7], Fn[2]};
  double defNew[9] = {F[0], F[4], F[8], F[1], F[5], F[6], F[3], F[7], F[2]};
  double stateOld[64], stateNew[64];
  for (int c = 0; c < nstatev; ++c)
    stateOld[c] = state[c], stateNew[c] = 0.0;
  double tempOld = *temp, tempNew = *temp, eIo = *eI, ePo = *eP, eIn = *eI, ePn = *eP;
  double stressNew[6] = {0}, stretchNewOut[6] = {0}, defNewOut[9] = {0};
  (void)stretchNewIn;
  vumat_adapter_call(&nb, &ndir, &nshr, &nsv, &nfv, &np, &lanneal, &st, &tt, &dtv, cmname, coord,
                     &cl, (double *)props, &dens, strainInc, relSpin, &tempOld, stretchOld,
                     defOld, fieldOld, stressOld, stateOld, &eIo, &ePo, &tempNew, stretchNewOut,
                     defNewOut, fieldNew, stressNew, stateNew, &eIn, &ePn);
  const double full[9] = {stressNew[0], stressNew[5], stressNew[4], stressNew[5], stressNew[1],
                          stressNew[3], stressNew[4], stressNew[3], stressNew[2]};
  rotate_to_spatial(full, rNew, sigmaSpatial);
  memcpy(Fn, F, sizeof(double) * 9);
  memcpy(Vn, vNew, sizeof(double) * 9);
  memcpy(Rn, rNew, sizeof(double) * 9);
  memcpy(En, strain, sizeof(double) * 9);
  memcpy(sig, full, sizeof(double) * 9);
  for (int c = 0; c < nstatev; ++c)
    state[c] = stateNew[c];
  *temp = tempNew, *eI = eIn, *eP = ePn;
  return 1;
}

int vo_material_update(int64_t n, const double *props, int32_t nstatev, double dt,
                       const double *F, double *Fn, double *Vn, double *Rn, double *En,
                       double *sig, double *state, double *temp, double *eI, double *eP,
                       double *sigmaSpatial) {
  int status = VPD_OK;
  if (nstatev > 64 || nstatev < 6 || !(dt > 0.0))
    return VPD_ERR_INVALID;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    if (!material_point(props, nstatev, dt, 0.0, 0.0, 1.0, props[10], F + 9 * i, Fn + 9 * i,
                        Vn + 9 * i, Rn + 9 * i, En + 9 * i, sig + 9 * i, state + nstatev * i,
                        temp + i, eI + i, eP + i, sigmaSpatial + 9 * i)) {
#pragma omp atomic write
      status = VPD_ERR_SINGULAR;
    }
  return status;
}

/* ------------------------------------------------------------------ damage */
/* PdSimpleDamage::update (critical_stretch) :51-82 and damageIndex :23-36 */
int vo_damage(int64_t n, const double *pos, const double *disp, const double *vol,
              const int64_t *row_ptr, const int32_t *col, double initiation, double failure,
              double *bond_damage, double *damage_index) {
  if (!(initiation > 0.0))
    return VPD_ERR_INVALID;
  const int useCompression = failure > 0.0 && isfinite(failure);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double yi[3] = {pos[3 * i] + disp[3 * i], pos[3 * i + 1] + disp[3 * i + 1],
                          pos[3 * i + 2] + disp[3 * i + 2]};
    for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
      const int64_t j = col[p];
      double xi[3], y[3];
      for (int d = 0; d < 3; ++d) {
        xi[d] = pos[3 * j + d] - pos[3 * i + d];
        y[d] = (pos[3 * j + d] + disp[3 * j + d]) - yi[d];
      }
      const double initial = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
      const double stretch = (sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]) - initial) / initial;
      if (stretch > initiation || (useCompression && stretch < -failure))
        bond_damage[p] = 1.0;
    }
  }
  if (damage_index) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double damaged = 0.0, total = 0.0;
      for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
        damaged += bond_damage[p] * vol[col[p]];
        total += vol[col[p]];
      }
      damage_index[i] = total > 0.0 ? damaged / total : 0.0;
    }
  }
  return VPD_OK;
}

/* ------------------------------------------------------------------ lattice and bands */
/* makeParticlePatch, Geometry.cpp:10-34 (nominal lattice) plus jitter on the positions. */
void vo_lattice(const vpd_case *c, double *nominal, double *pos, double *vol) {
  const double h = c->spacing;
  const double yOffset = 0.5 * (double)(c->ny - 1) * h;
  const double zOffset = 0.5 * (double)(c->nz - 1) * h;
  const double volume = h * h * h;
  const double amp = c->jitter * h;
  int64_t p = 0;
  for (int i = 0; i < c->nx; ++i)
    for (int j = 0; j < c->ny; ++j)
      for (int k = 0; k < c->nz; ++k, ++p) {
        const double x[3] = {(double)i * h, (double)j * h - yOffset, (double)k * h - zOffset};
        for (int d = 0; d < 3; ++d) {
          nominal[3 * p + d] = x[d];
          pos[3 * p + d] = c->jitter != 0.0 ? x[d] + vo_jitter_value(c->jitter_seed, p, d, amp)
                                            : x[d];
        }
        vol[p] = volume * ((i == 0 || i == c->nx - 1) ? 0.5 : 1.0) *
                 ((j == 0 || j == c->ny - 1) ? 0.5 : 1.0) *
                 ((k == 0 || k == c->nz - 1) ? 0.5 : 1.0);
      }
}

/* selectBoundaryRegion, ParticleSets.cpp:12-50: flags[i] |= bit for the selected points. */
static int select_region(const double *x, int64_t n, int component, int selectMinimum,
                         double width, unsigned char *flags, unsigned char bit) {
  double extreme = selectMinimum ? INFINITY : -INFINITY;
  for (int64_t i = 0; i < n; ++i) {
    const double v = x[3 * i + component];
    extreme = selectMinimum ? (extreme < v ? extreme : v) : (extreme > v ? extreme : v);
  }
  const double tol = 1.0e-10 * (1.0 > fabs(extreme) ? 1.0 : fabs(extreme));
  int any = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double v = x[3 * i + component];
    const double dist = selectMinimum ? v - extreme : extreme - v;
    if (dist <= width + tol) {
      flags[i] |= bit;
      any = 1;
    }
  }
  return any;
}

/* Boundary and diagnostic sets: RegionalConstraintSystem ctor (BoundaryConditions.cpp:54-68),
   rotation pin (:96-110), runMaterial set-up (BoundaryValueCaseRunner.cpp:145-167),
   observationBounds / observationWeights (include/ObservationWindow.hpp:13-56). */
typedef struct {
  unsigned char *flags; /* bit0 support, bit1 loaded, bit2 lateral negative, bit3 lateral positive */
  int64_t anchor, rotationPin;
  double gaugeLength, lateralGauge, crossSectionArea, observationMin, observationMax;
  double *obsWeight;
  int axis, lateral;
} vo_sets;

enum { VO_SUPPORT = 1, VO_LOADED = 2, VO_LATNEG = 4, VO_LATPOS = 8 };

static int build_sets(const vpd_case *c, const double *x, const double *vol, int64_t n,
                      vo_sets *s) {
  const double h = c->spacing;
  s->axis = c->load_axis;
  s->lateral = s->axis == 0 ? 1 : 0;
  s->flags = calloc((size_t)n, 1);
  s->obsWeight = calloc((size_t)n, sizeof(double));
  const double width = (double)(c->region_layers - 1) * h + 1.0e-9 * h;
  if (!select_region(x, n, s->axis, 1, width, s->flags, VO_SUPPORT) ||
      !select_region(x, n, s->axis, 0, width, s->flags, VO_LOADED))
    return 0;
  double centre[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d)
      centre[d] += x[3 * i + d];
  for (int d = 0; d < 3; ++d)
    centre[d] /= (double)n;
  double best = INFINITY;
  s->anchor = -1;
  for (int64_t i = 0; i < n; ++i)
    if (s->flags[i] & VO_SUPPORT) {
      double dist = 0.0;
      for (int d = 0; d < 3; ++d) {
        const double delta = x[3 * i + d] - centre[d];
        dist += delta * delta;
      }
      if (dist < best)
        best = dist, s->anchor = i;
    }
  s->rotationPin = s->anchor;
  double greatestY = -1.0e100;
  const double *ctr = x + 3 * s->anchor;
  for (int64_t i = 0; i < n; ++i)
    if (s->flags[i] & VO_SUPPORT) {
      const double *xi = x + 3 * i;
      if (fabs(xi[0] - ctr[0]) < 1e-8 && fabs(xi[2] - ctr[2]) < 1e-8 && xi[1] > greatestY)
        greatestY = xi[1], s->rotationPin = i;
    }
  /* gauge lengths (meanCoordinate, BoundaryValueCaseRunner.cpp:84-91,148-157) */
  double sl = 0, ss = 0, nl = 0, ns = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (s->flags[i] & VO_LOADED) sl += x[3 * i + s->axis], nl += 1;
    if (s->flags[i] & VO_SUPPORT) ss += x[3 * i + s->axis], ns += 1;
  }
  s->gaugeLength = fabs(sl / nl - ss / ns);
  const double tiny = 1.0e-9 * h;
  select_region(x, n, s->lateral, 1, tiny, s->flags, VO_LATNEG);
  select_region(x, n, s->lateral, 0, tiny, s->flags, VO_LATPOS);
  double sp = 0, sn = 0, np_ = 0, nn = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (s->flags[i] & VO_LATPOS) sp += x[3 * i + s->lateral], np_ += 1;
    if (s->flags[i] & VO_LATNEG) sn += x[3 * i + s->lateral], nn += 1;
  }
  s->lateralGauge = fabs(sp / np_ - sn / nn);
  /* observation window */
  double lo = x[s->axis], hi = lo;
  for (int64_t i = 0; i < n; ++i) {
    const double v = x[3 * i + s->axis];
    lo = lo < v ? lo : v;
    hi = hi > v ? hi : v;
  }
  const double band = (double)(c->region_layers - 1) * h;
  const double a = isnan(c->observation_min) ? lo + band : c->observation_min;
  const double b = isnan(c->observation_max) ? hi - band : c->observation_max;
  if (!isfinite(a) || !isfinite(b) || a < lo || b > hi || a >= b)
    return 0;
  s->observationMin = a, s->observationMax = b;
  const double tol = 1e-8 * h;
  int foundA = 0, foundB = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double v = x[3 * i + s->axis];
    const int atA = fabs(v - a) < tol, atB = fabs(v - b) < tol;
    foundA = foundA || atA;
    foundB = foundB || atB;
    if (v < a - tol || v > b + tol)
      continue;
    const int interiorEnd = (atA && a > lo + tol) || (atB && b < hi - tol);
    s->obsWeight[i] = vol[i] * (interiorEnd ? 0.5 : 1.0);
  }
  if (!foundA || !foundB)
    return 0;
  const int crossCount = s->axis == 0 ? c->ny : c->nx;
  s->crossSectionArea = (double)((crossCount - 1) * (c->nz - 1)) * h * h;
  return 1;
}

/* ------------------------------------------------------------------ full increment */
typedef struct vo_sim {
  vpd_case c;
  int64_t n, nbonds;
  double *nominal, *X, *V, *u, *v, *a, *kinv, *Fn, *Vn, *Rn, *En, *sig, *state, *temp, *eI, *eP;
  double *sigSpatial, *F, *force, *bondDamage, *damageIndex;
  double *pointDamage, *sigEffective; /* point damage modes */
  int64_t *row_ptr;
  int32_t *col;
  vo_sets sets;
  int64_t step;
  double internalEnergy, externalWork, previousPower;
  int finite;
} vo_sim;

static void set_component(vo_sim *s, int64_t i, int d, double u, double v, double a) {
  s->u[3 * i + d] = u, s->v[3 * i + d] = v, s->a[3 * i + d] = a;
}
/* RegionalConstraintSystem::apply, BoundaryConditions.cpp:81-115 (+ moving support band). */
static void apply_constraints(vo_sim *s, double t) {
  double r[6];
  vo_ramp(&s->c, t, r);
  const int ax = s->sets.axis;
  for (int64_t i = 0; i < s->n; ++i)
    if (s->sets.flags[i] & VO_SUPPORT)
      set_component(s, i, ax, r[3], r[4], r[5]);
  for (int64_t i = 0; i < s->n; ++i)
    if (s->sets.flags[i] & VO_LOADED)
      set_component(s, i, ax, r[0], r[1], r[2]);
  set_component(s, s->sets.anchor, s->sets.lateral, 0.0, 0.0, 0.0);
  if (!s->c.plane_strain) {
    set_component(s, s->sets.anchor, 2, 0.0, 0.0, 0.0);
    set_component(s, s->sets.rotationPin, 2, 0.0, 0.0, 0.0);
  } else {
    for (int64_t i = 0; i < s->n; ++i)
      set_component(s, i, 2, 0.0, 0.0, 0.0);
  }
}

void vo_destroy(vo_sim *s) {
  if (!s)
    return;
  double *arrs[] = {s->nominal, s->X, s->V, s->u, s->v, s->a, s->kinv, s->Fn, s->Vn, s->Rn,
                    s->En, s->sig, s->state, s->temp, s->eI, s->eP, s->sigSpatial, s->F,
                    s->force, s->bondDamage, s->damageIndex, s->sets.obsWeight,
                    s->pointDamage, s->sigEffective};
  for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; ++k)
    free(arrs[k]);
  free(s->row_ptr), free(s->col), free(s->sets.flags), free(s);
}

/* runMaterial set-up, BoundaryValueCaseRunner.cpp:142-190. positions/volumes optional. */
vo_sim *vo_create(const vpd_case *c, const double *positions, const double *volumes,
                  int *status) {
  *status = VPD_ERR_INVALID;
  if (c->nx < 2 || c->ny < 2 || c->nz < 2 || !(c->spacing > 0) || !(c->horizon > 0) ||
      !(c->dt > 0) || !(c->density > 0) || c->nstatev < 6 || c->nstatev > 64 ||
      c->region_layers < 1 || (c->load_axis != 0 && c->load_axis != 1))
    return NULL;
  vo_sim *s = calloc(1, sizeof(vo_sim));
  s->c = *c;
  const int64_t n = (int64_t)c->nx * c->ny * c->nz;
  s->n = n;
#define ALLOC(p, cnt) p = calloc((size_t)(cnt), sizeof(double))
  ALLOC(s->nominal, 3 * n), ALLOC(s->X, 3 * n), ALLOC(s->V, n), ALLOC(s->u, 3 * n);
  ALLOC(s->v, 3 * n), ALLOC(s->a, 3 * n), ALLOC(s->kinv, 9 * n), ALLOC(s->Fn, 9 * n);
  ALLOC(s->Vn, 9 * n), ALLOC(s->Rn, 9 * n), ALLOC(s->En, 9 * n), ALLOC(s->sig, 9 * n);
  ALLOC(s->state, (int64_t)c->nstatev * n), ALLOC(s->temp, n), ALLOC(s->eI, n), ALLOC(s->eP, n);
  ALLOC(s->sigSpatial, 9 * n), ALLOC(s->F, 9 * n), ALLOC(s->force, 3 * n);
  ALLOC(s->damageIndex, n), ALLOC(s->pointDamage, n), ALLOC(s->sigEffective, 9 * n);
  vo_lattice(c, s->nominal, s->X, s->V);
  if (positions)
    memcpy(s->X, positions, sizeof(double) * 3 * (size_t)n);
  if (volumes)
    memcpy(s->V, volumes, sizeof(double) * (size_t)n);
  s->row_ptr = calloc((size_t)n + 1, sizeof(int64_t));
  int64_t total = vo_neighbor_count(s->X, n, c->horizon, s->row_ptr);
  if (total < 0) {
    *status = (int)-total;
    vo_destroy(s);
    return NULL;
  }
  s->nbonds = total;
  s->col = malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  vo_neighbor_fill(s->X, n, c->horizon, s->row_ptr, s->col);
  ALLOC(s->bondDamage, total > 0 ? total : 1);
  if (!build_sets(c, s->nominal, s->V, n, &s->sets)) {
    vo_destroy(s);
    return NULL;
  }
  if ((*status = vo_shape_inverse(n, s->X, s->V, s->row_ptr, s->col, s->kinv)) != VPD_OK) {
    vo_destroy(s);
    return NULL;
  }
  /* bridge.initialize(F_0) (VumatPdCorrespondenceMaterial.cpp:48-70) */
  vo_deformation(n, s->X, s->u, s->V, s->row_ptr, s->col, s->kinv, s->Fn);
  for (int64_t i = 0; i < n; ++i) {
    memcpy(s->Vn + 9 * i, I9, sizeof I9);
    memcpy(s->Rn + 9 * i, I9, sizeof I9);
    green_lagrange(s->Fn + 9 * i, s->En + 9 * i);
    s->temp[i] = c->reference_temperature;
  }
  apply_constraints(s, 0.0);
  s->finite = 1;
  *status = VPD_OK;
  return s;
#undef ALLOC
}

static double contraction(const double *s, const double *e) {
  return s[0] * e[0] + s[4] * e[4] + s[8] * e[8] + 2.0 * (s[1] * e[1] + s[2] * e[2] + s[5] * e[5]);
}
static int finite9(const double *x) {
  for (int i = 0; i < 9; ++i)
    if (!isfinite(x[i]))
      return 0;
  return 1;
}

/* maxPrincipalStrainSymmetric3x3 (TensorVoigtMap.cpp:35-71): the largest eigenvalue of the
   symmetric part of a row-major 3x3 tensor, by the trigonometric solution of the cubic. */
static double max_principal(const double *t) {
  const double a = t[0], b = 0.5 * (t[1] + t[3]), c = 0.5 * (t[2] + t[6]);
  const double d = t[4], e = 0.5 * (t[5] + t[7]), f = t[8];
  const double p1 = b * b + c * c + e * e;
  if (p1 == 0.0)
    return fmax(fmax(a, d), f);
  const double q = (a + d + f) / 3.0;
  const double a11 = a - q, a22 = d - q, a33 = f - q;
  const double p = sqrt((a11 * a11 + a22 * a22 + a33 * a33 + 2.0 * p1) / 6.0);
  const double inv = 1.0 / p;
  const double b11 = a11 * inv, b12 = b * inv, b13 = c * inv;
  const double b22 = a22 * inv, b23 = e * inv, b33 = a33 * inv;
  const double det = b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) +
                     b13 * (b12 * b23 - b22 * b13);
  const double h = det / 2.0;
  const double r = h < -1.0 ? -1.0 : (1.0 < h ? 1.0 : h);
  const double pi = 3.141592653589793238462643383279502884;
  const double phi = acos(r) / 3.0;
  const double e1 = q + 2.0 * p * cos(phi);
  const double e3 = q + 2.0 * p * cos(phi + 2.0 * pi / 3.0);
  const double e2 = 3.0 * q - e1 - e3;
  return fmax(fmax(e1, e2), e3);
}

/* The point damage modes: SimpleDamageModel::update and degradeStress (SimpleDamageModel.cpp:14-50)
   as PdSimpleDamage::update runs them (PdSimpleDamage.cpp:84-92). The damage follows the new eqps
   (state variable 2) or the largest principal Green-Lagrange strain, never decreases, and scales
   the spatial stress the force density uses; a deleted point (deletionEnabled, damage 1) drops
   out of it. The diagnostics keep the undegraded stress. */
static void point_damage(vo_sim *s) {
  const vpd_case *c = &s->c;
  for (int64_t i = 0; i < s->n; ++i) {
    const double metric = c->damage_mode == VPD_DAMAGE_EQPS_THRESHOLD ? s->state[c->nstatev * i + 1]
                                                                      : max_principal(s->En + 9 * i);
    const double t = (metric - c->damage_initiation) / (c->damage_failure - c->damage_initiation);
    const double clamped = t < 0.0 ? 0.0 : (1.0 < t ? 1.0 : t);
    const double dmg = s->pointDamage[i] < clamped ? clamped : s->pointDamage[i];
    s->pointDamage[i] = dmg;
    const double factor = (c->damage_deletion && dmg >= 1.0) ? 0.0 : 1.0 - (dmg < 0.0 ? 0.0 : (1.0 < dmg ? 1.0 : dmg));
    for (int k = 0; k < 9; ++k)
      s->sigEffective[9 * i + k] = s->sigSpatial[9 * i + k] * factor;
  }
}

/* The step loop body of runMaterial, BoundaryValueCaseRunner.cpp:207-306. diag: nsteps rows
   of VPD_DIAG_COLS doubles (may be NULL). */
int vo_step(vo_sim *s, int32_t nsteps, double *diag) {
  const vpd_case *c = &s->c;
  const int64_t n = s->n;
  const double dt = c->dt, rho = c->density;
  double *prevSig = malloc(sizeof(double) * 9 * (size_t)n);
  double *prevStrain = malloc(sizeof(double) * 9 * (size_t)n);
  int status = VPD_OK;
  for (int32_t it = 0; it < nsteps && status == VPD_OK; ++it) {
    const int64_t step = ++s->step;
    const double time = (double)step * dt;
    /* predictDisplacement, ExplicitTimeIntegrator.cpp:23-34 */
    for (int64_t q = 0; q < 3 * n; ++q)
      s->u[q] += dt * s->v[q] + 0.5 * dt * dt * s->a[q];
    apply_constraints(s, time);
    memcpy(prevSig, s->sig, sizeof(double) * 9 * (size_t)n);
    memcpy(prevStrain, s->En, sizeof(double) * 9 * (size_t)n);
    vo_deformation(n, s->X, s->u, s->V, s->row_ptr, s->col, s->kinv, s->F);
    const double stepTime = (double)(step - 1) * dt;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
      if (!material_point(c->props, c->nstatev, dt, stepTime, stepTime, c->spacing, c->props[10],
                          s->F + 9 * i, s->Fn + 9 * i, s->Vn + 9 * i, s->Rn + 9 * i,
                          s->En + 9 * i, s->sig + 9 * i, s->state + c->nstatev * i, s->temp + i,
                          s->eI + i, s->eP + i, s->sigSpatial + 9 * i)) {
#pragma omp atomic write
        status = VPD_ERR_SINGULAR;
      }
    if (status != VPD_OK)
      break;
    if (c->damage_mode == VPD_DAMAGE_CRITICAL_STRETCH)
      vo_damage(n, s->X, s->u, s->V, s->row_ptr, s->col, c->damage_initiation, c->damage_failure,
                s->bondDamage, s->damageIndex);
    const double *sigForce = s->sigSpatial;
    if (c->damage_mode >= VPD_DAMAGE_EQPS_THRESHOLD) {
      point_damage(s);
      sigForce = s->sigEffective;
    }
    if ((status = vo_force(n, s->X, s->V, s->row_ptr, s->col, s->kinv, s->F, sigForce,
                           s->bondDamage, s->force)) != VPD_OK)
      break;
    /* correctVelocity, ExplicitTimeIntegrator.cpp:36-52 */
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) {
        const double next = s->force[3 * i + d] / rho;
        s->v[3 * i + d] += 0.5 * dt * (s->a[3 * i + d] + next);
        s->a[3 * i + d] = next;
      }
    apply_constraints(s, time);
    /* diagnostics, BoundaryValueCaseRunner.cpp:231-306 */
    for (int64_t i = 0; i < n; ++i) {
      double avg[9], inc[9];
      for (int k = 0; k < 9; ++k) {
        avg[k] = 0.5 * (prevSig[9 * i + k] + s->sigSpatial[9 * i + k]);
        inc[k] = s->En[9 * i + k] - prevStrain[9 * i + k];
      }
      s->internalEnergy += contraction(avg, inc) * s->V[i];
    }
    const int ax = s->sets.axis, lat = s->sets.lateral;
    const double sign = (c->bc_mode == VPD_BC_SMOOTH_DISPLACEMENT ? c->amplitude : c->grip_velocity)
                                > 0.0 ? 1.0 : -1.0;
    double r[6];
    vo_ramp(c, time, r);
    double net[3] = {0, 0, 0}, reaction = 0.0, supportReaction = 0.0, avgS = 0.0, avgE = 0.0;
    double maxEqps = 0.0, interior = 0.0, plastic = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      if (c->nstatev > 4 && s->state[c->nstatev * i + 4] > 0.0)
        plastic += 1.0;
      for (int d = 0; d < 3; ++d)
        net[d] += s->force[3 * i + d] * s->V[i];
      if (s->sets.obsWeight[i] > 0.0) {
        const double w = s->sets.obsWeight[i];
        avgS += sign * s->sigSpatial[9 * i + 4 * ax] * w;
        avgE += sign * s->En[9 * i + 4 * ax] * w;
        interior += w;
      }
      const double eq = s->state[c->nstatev * i + 1];
      maxEqps = maxEqps > eq ? maxEqps : eq;
      s->finite = s->finite && finite9(s->sigSpatial + 9 * i) && finite9(s->En + 9 * i) &&
                  isfinite(s->force[3 * i]) && isfinite(s->force[3 * i + 1]) &&
                  isfinite(s->force[3 * i + 2]);
      for (int k = 0; k < c->nstatev; ++k)
        s->finite = s->finite && isfinite(s->state[c->nstatev * i + k]);
    }
    for (int64_t i = 0; i < n; ++i) {
      if (s->sets.flags[i] & VO_LOADED)
        reaction += (rho * r[2] - s->force[3 * i + ax]) * s->V[i];
      if (s->sets.flags[i] & VO_SUPPORT)
        supportReaction += (rho * r[5] - s->force[3 * i + ax]) * s->V[i];
    }
    avgS /= interior;
    avgE /= interior;
    const double power = reaction * r[1] + (c->bc_mode == VPD_BC_VELOCITY_RAMP ?
                                            supportReaction * r[4] : 0.0);
    s->externalWork += 0.5 * dt * (s->previousPower + power);
    s->previousPower = power;
    double kinetic = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double *vv = s->v + 3 * i;
      kinetic += 0.5 * rho * s->V[i] * (vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]);
    }
    double scale = fabs(s->externalWork);
    const double alt = fabs(s->internalEnergy) + kinetic;
    scale = scale > alt ? scale : alt;
    scale = scale > 1.0e-12 ? scale : 1.0e-12;
    const double energyError = fabs(kinetic + s->internalEnergy - s->externalWork) / scale;
    const double relDisp = r[0] - r[3];
    const double engineering = sign * relDisp / s->sets.gaugeLength;
    double sp = 0, sn = 0, np_ = 0, nn = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (s->sets.flags[i] & VO_LATPOS) sp += s->u[3 * i + lat], np_ += 1;
      if (s->sets.flags[i] & VO_LATNEG) sn += s->u[3 * i + lat], nn += 1;
    }
    const double lateralStrain = (sp / np_ - sn / nn) / s->sets.lateralGauge;
    const double nominal = sign * reaction / s->sets.crossSectionArea;
    s->finite = s->finite && isfinite(kinetic) && isfinite(s->internalEnergy) &&
                isfinite(s->externalWork) && isfinite(energyError);
    if (diag) {
      double *row = diag + (size_t)it * VPD_DIAG_COLS;
      row[VPD_DIAG_STEP] = (double)step;
      row[VPD_DIAG_TIME] = time;
      row[VPD_DIAG_LOAD_DISPLACEMENT] = r[0];
      row[VPD_DIAG_LOAD_VELOCITY] = r[1];
      row[VPD_DIAG_REACTION] = reaction;
      row[VPD_DIAG_ENGINEERING_STRAIN] = engineering;
      row[VPD_DIAG_LATERAL_STRAIN] = lateralStrain;
      row[VPD_DIAG_NOMINAL_STRESS] = nominal;
      row[VPD_DIAG_AVERAGE_AXIAL_STRAIN] = avgE;
      row[VPD_DIAG_AVERAGE_AXIAL_STRESS] = avgS;
      row[VPD_DIAG_MAX_EQPS] = maxEqps;
      row[VPD_DIAG_MAX_INTERNAL_INDICATOR] = 0.0;
      row[VPD_DIAG_KINETIC_ENERGY] = kinetic;
      row[VPD_DIAG_INTERNAL_ENERGY] = s->internalEnergy;
      row[VPD_DIAG_EXTERNAL_WORK] = s->externalWork;
      row[VPD_DIAG_ENERGY_ERROR] = energyError;
      row[VPD_DIAG_NET_INTERNAL_FORCE] = sqrt(net[0] * net[0] + net[1] * net[1] + net[2] * net[2]);
      row[VPD_DIAG_FINITE] = s->finite ? 1.0 : 0.0;
      row[VPD_DIAG_PLASTIC_POINTS] = plastic;
      row[VPD_DIAG_FALLBACK_POINTS] = 0.0;
    }
  }
  free(prevSig);
  free(prevStrain);
  return status;
}

int64_t vo_num_points(const vo_sim *s) { return s->n; }
int64_t vo_num_bonds(const vo_sim *s) { return s->nbonds; }
int vo_neighbors(const vo_sim *s, int64_t *row_ptr, int32_t *col) {
  memcpy(row_ptr, s->row_ptr, sizeof(int64_t) * (size_t)(s->n + 1));
  memcpy(col, s->col, sizeof(int32_t) * (size_t)s->nbonds);
  return VPD_OK;
}

/* Field export in the layout of vpd_download. */
int vo_get(vo_sim *s, int32_t field, double *out) {
  const int64_t n = s->n;
  const size_t b3 = sizeof(double) * 3 * (size_t)n, b9 = sizeof(double) * 9 * (size_t)n;
  const size_t b1 = sizeof(double) * (size_t)n;
  switch (field) {
  case VPD_FIELD_POSITION: memcpy(out, s->X, b3); return VPD_OK;
  case VPD_FIELD_VOLUME: memcpy(out, s->V, b1); return VPD_OK;
  case VPD_FIELD_DISPLACEMENT: memcpy(out, s->u, b3); return VPD_OK;
  case VPD_FIELD_VELOCITY: memcpy(out, s->v, b3); return VPD_OK;
  case VPD_FIELD_ACCELERATION: memcpy(out, s->a, b3); return VPD_OK;
  case VPD_FIELD_DEFGRAD: memcpy(out, s->Fn, b9); return VPD_OK;
  case VPD_FIELD_STRESS_COROTATIONAL: memcpy(out, s->sig, b9); return VPD_OK;
  case VPD_FIELD_STRESS_SPATIAL:
    for (int64_t i = 0; i < n; ++i)
      rotate_to_spatial(s->sig + 9 * i, s->Rn + 9 * i, out + 9 * i);
    return VPD_OK;
  case VPD_FIELD_STRAIN: memcpy(out, s->En, b9); return VPD_OK;
  case VPD_FIELD_ROTATION: memcpy(out, s->Rn, b9); return VPD_OK;
  case VPD_FIELD_LEFT_STRETCH: memcpy(out, s->Vn, b9); return VPD_OK;
  case VPD_FIELD_STATE: memcpy(out, s->state, b1 * (size_t)s->c.nstatev); return VPD_OK;
  case VPD_FIELD_TEMPERATURE: memcpy(out, s->temp, b1); return VPD_OK;
  case VPD_FIELD_ENERGY_INTERNAL: memcpy(out, s->eI, b1); return VPD_OK;
  case VPD_FIELD_ENERGY_INELASTIC: memcpy(out, s->eP, b1); return VPD_OK;
  case VPD_FIELD_DAMAGE_INDEX:
    if (s->c.damage_mode >= VPD_DAMAGE_EQPS_THRESHOLD) {
      memcpy(out, s->pointDamage, b1);
      return VPD_OK;
    }
    for (int64_t i = 0; i < n; ++i) {
      double damaged = 0.0, total = 0.0;
      for (int64_t p = s->row_ptr[i]; p < s->row_ptr[i + 1]; ++p) {
        damaged += s->bondDamage[p] * s->V[s->col[p]];
        total += s->V[s->col[p]];
      }
      out[i] = total > 0.0 ? damaged / total : 0.0;
    }
    return VPD_OK;
  case VPD_FIELD_FORCE_DENSITY: memcpy(out, s->force, b3); return VPD_OK;
  case VPD_FIELD_SHAPE_INVERSE: memcpy(out, s->kinv, b9); return VPD_OK;
  default: return VPD_ERR_INVALID;
  }
}
