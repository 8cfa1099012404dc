// Device FP64 3x3 algebra and the corotational (Flanagan-Taylor) kinematic update.
//
// Tensors are row-major double[9] held in registers. The kinematics follow
// updateCorotationalKinematics (src/pd/CorotationalKinematics.cpp:61-135): L = Fdot F_n^-1,
// D/W split, spin correction, Rodrigues rotation increment in half-angle form, left-stretch
// rate, unrotated rate of deformation and the relative spin increment.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace vpd {

// 32-byte global load through the read-only path and 32-byte store (sm_100 vector width);
// the address must be 32-byte aligned (every double4 array here is). A warp reading
// consecutive double4 elements then touches each 32-byte sector once, where two 16-byte
// halves would touch every sector twice.
__device__ __forceinline__ double4 ldg256(const double4 *p) {
  double4 r;
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
  return r;
}
__device__ __forceinline__ void st256(double4 *p, double4 v) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v.x), "d"(v.y), "d"(v.z), "d"(v.w)
               : "memory");
}

__device__ __forceinline__ void m_mul(const double *a, const double *b, double *o) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      o[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

// o = a * b^T
__device__ __forceinline__ void m_mul_bt(const double *a, const double *b, double *o) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      o[3 * i + j] = a[3 * i] * b[3 * j] + a[3 * i + 1] * b[3 * j + 1] + a[3 * i + 2] * b[3 * j + 2];
}

// o = a^T * b
__device__ __forceinline__ void m_mul_at(const double *a, const double *b, double *o) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      o[3 * i + j] = a[i] * b[j] + a[3 + i] * b[3 + j] + a[6 + i] * b[6 + j];
}

__device__ __forceinline__ double m_det(const double *a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
         a[2] * (a[3] * a[7] - a[4] * a[6]);
}

// Cofactor inverse (PdCorrespondenceSkeleton.cpp:67-76); false when |det| < 1e-14.
__device__ __forceinline__ bool m_inv(const double *a, double *o) {
  const double det = m_det(a);
  if (fabs(det) < 1.0e-14)  // NaN passes, as in the reference, and surfaces as non-finite
    return false;
  const double r = 1.0 / det;
  o[0] = (a[4] * a[8] - a[5] * a[7]) * r;
  o[1] = (a[2] * a[7] - a[1] * a[8]) * r;
  o[2] = (a[1] * a[5] - a[2] * a[4]) * r;
  o[3] = (a[5] * a[6] - a[3] * a[8]) * r;
  o[4] = (a[0] * a[8] - a[2] * a[6]) * r;
  o[5] = (a[2] * a[3] - a[0] * a[5]) * r;
  o[6] = (a[3] * a[7] - a[4] * a[6]) * r;
  o[7] = (a[1] * a[6] - a[0] * a[7]) * r;
  o[8] = (a[0] * a[4] - a[1] * a[3]) * r;
  return true;
}

// Green-Lagrange strain 0.5 (F^T F - I) (CorotationalKinematics.cpp:141-149), as the six
// independent components in legacy Voigt order 11,22,33,23,13,12.
__device__ __forceinline__ void green_lagrange6(const double *f, double *e6) {
  double c[9];
  m_mul_at(f, f, c);
  e6[0] = 0.5 * (c[0] - 1.0);
  e6[1] = 0.5 * (c[4] - 1.0);
  e6[2] = 0.5 * (c[8] - 1.0);
  e6[3] = 0.5 * c[5];
  e6[4] = 0.5 * c[2];
  e6[5] = 0.5 * c[1];
}

// Largest eigenvalue of a symmetric tensor given in legacy Voigt order (11,22,33,23,13,12):
// the trigonometric solution of the characteristic cubic, in the reference's order of
// operations with every rounding spelled out (maxPrincipalStrainSymmetric3x3,
// TensorVoigtMap.cpp:35-71). Only acos and cos may differ from the host's by an ulp.
__device__ inline double max_principal6(const double *v) {
  const double a = v[0], b = v[5], c = v[4], d = v[1], e = v[3], f = v[2];
  const double p1 = __dadd_rn(__dadd_rn(__dmul_rn(b, b), __dmul_rn(c, c)), __dmul_rn(e, e));
  if (p1 == 0.0)
    return fmax(fmax(a, d), f);
  const double q = __dadd_rn(__dadd_rn(a, d), f) / 3.0;
  const double a11 = a - q, a22 = d - q, a33 = f - q;
  const double p2 = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a11, a11), __dmul_rn(a22, a22)), __dmul_rn(a33, a33)),
                              2.0 * p1);
  const double pp = sqrt(p2 / 6.0);
  const double invP = 1.0 / pp;
  const double b11 = a11 * invP, b12 = b * invP, b13 = c * invP;
  const double b22 = a22 * invP, b23 = e * invP, b33 = a33 * invP;
  const double m1 = __dsub_rn(__dmul_rn(b22, b33), __dmul_rn(b23, b23));
  const double m2 = __dsub_rn(__dmul_rn(b12, b33), __dmul_rn(b23, b13));
  const double m3 = __dsub_rn(__dmul_rn(b12, b23), __dmul_rn(b22, b13));
  const double detB = __dadd_rn(__dsub_rn(__dmul_rn(b11, m1), __dmul_rn(b12, m2)), __dmul_rn(b13, m3));
  const double half = detB / 2.0;
  const double r = half < -1.0 ? -1.0 : (1.0 < half ? 1.0 : half);
  const double pi = 3.141592653589793238462643383279502884;
  const double phi = acos(r) / 3.0;
  const double eig1 = __dadd_rn(q, __dmul_rn(2.0 * pp, cos(phi)));
  const double eig3 = __dadd_rn(q, __dmul_rn(2.0 * pp, cos(phi + 2.0 * pi / 3.0)));
  const double eig2 = __dsub_rn(__dsub_rn(__dmul_rn(3.0, q), eig1), eig3);
  return fmax(fmax(eig1, eig2), eig3);
}

// Symmetric tensor <-> legacy Voigt 11,22,33,23,13,12 (TensorVoigtMap.cpp:9-20).
__device__ __forceinline__ void voigt_to_full(const double *v, double *f) {
  f[0] = v[0], f[1] = v[5], f[2] = v[4];
  f[3] = v[5], f[4] = v[1], f[5] = v[3];
  f[6] = v[4], f[7] = v[3], f[8] = v[2];
}
__device__ __forceinline__ void full_to_voigt(const double *f, double *v) {
  v[0] = f[0], v[1] = f[4], v[2] = f[8];
  v[3] = 0.5 * (f[5] + f[7]), v[4] = 0.5 * (f[2] + f[6]), v[5] = 0.5 * (f[1] + f[3]);
}

struct Corotational {
  double dbar[9];  // unrotated rate of deformation R^T D R
  double spin[9];  // relative spin increment dt R^T (W - Omega) R
  double r[9];     // R_{n+1}
  double v[9];     // V_{n+1}
};

// updateCorotationalKinematics (CorotationalKinematics.cpp:61-135). false on a singular
// F_n or (tr V) I - V.
__device__ __forceinline__ bool corotational_update(const double *fN, const double *fNP1,
                                                    const double *vN, const double *rN,
                                                    double dt, Corotational &out) {
  double fDot[9], fNinv[9], L[9], d[9], w[9];
#pragma unroll
  for (int i = 0; i < 9; ++i)
    fDot[i] = (fNP1[i] - fN[i]) / dt;
  if (!m_inv(fN, fNinv))
    return false;
  m_mul(fDot, fNinv, L);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      d[3 * i + j] = 0.5 * (L[3 * i + j] + L[3 * j + i]);
      w[3 * i + j] = 0.5 * (L[3 * i + j] - L[3 * j + i]);
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
#pragma unroll
  for (int i = 0; i < 9; ++i)
    tiv[i] = ((i % 4 == 0) ? trV : 0.0) - vN[i];
  if (!m_inv(tiv, corr))
    return false;
  const double oX = wX + corr[0] * zX + corr[1] * zY + corr[2] * zZ;
  const double oY = wY + corr[3] * zX + corr[4] * zY + corr[5] * zZ;
  const double oZ = wZ + corr[6] * zX + corr[7] * zY + corr[8] * zZ;
  const double omega[9] = {0.0, -oZ, oY, oZ, 0.0, -oX, -oY, oX, 0.0};
  const double oSq = oX * oX + oY * oY + oZ * oZ;
  double q[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (oSq > 1.0e-30) {
    const double mag = sqrt(oSq);
    const double s1 = sin(dt * mag) / mag;
    const double hs = sin(0.5 * dt * mag);
    const double s2 = 2.0 * hs * hs / oSq;
    double o2[9];
    m_mul(omega, omega, o2);
#pragma unroll
    for (int i = 0; i < 9; ++i)
      q[i] += s1 * omega[i] + s2 * o2[i];
  }
  m_mul(q, rN, out.r);
  double ra[9], rb[9];
  m_mul(L, vN, ra);
  m_mul(vN, omega, rb);
#pragma unroll
  for (int i = 0; i < 9; ++i)
    out.v[i] = vN[i] + dt * (ra[i] - rb[i]);
  double tmp[9];
  m_mul(d, out.r, tmp);
  m_mul_at(out.r, tmp, out.dbar);
  double rel[9];
#pragma unroll
  for (int i = 0; i < 9; ++i)
    rel[i] = w[i] - omega[i];
  m_mul(rel, out.r, tmp);
  m_mul_at(out.r, tmp, out.spin);
#pragma unroll
  for (int i = 0; i < 9; ++i)
    out.spin[i] *= dt;
  return true;
}

// sigma_spatial = R sigma R^T (rotateCorotationalStressToSpatial, :137-139).
__device__ __forceinline__ void rotate_to_spatial(const double *s, const double *r, double *o) {
  double tmp[9];
  m_mul_bt(s, r, tmp);
  m_mul(r, tmp, o);
}

// Force map M = (det F) sigma F^-T K^-1 (cauchyToFirstPiola :83-91 then :209-211).
__device__ __forceinline__ bool force_map(const double *sigma, const double *f,
                                          const double *kinv, double *m) {
  double finv[9], p[9];
  const double j = m_det(f);
  if (fabs(j) < 1.0e-14 || !m_inv(f, finv))
    return false;
  m_mul_bt(sigma, finv, p);  // sigma * (F^-1)^T
#pragma unroll
  for (int i = 0; i < 9; ++i)
    p[i] *= j;
  m_mul(p, kinv, m);
  return true;
}

}  // namespace vpd
