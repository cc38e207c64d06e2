// Device functions for the sp NDDO two-centre integrals and Slater overlaps.
//
// These evaluate the Dewar-Sabelli-Klopman multipole model with PM7 feathering
// (pm7-rs src/integrals.rs:32-538) and the analytic n<=3 Slater overlaps
// (pm7-rs src/overlap.rs:16-462) for one atom pair in FP64. Every output
// follows the reference's orientation: the first atom is the one with more
// orbitals, the displacement points from the first atom to the second.
#pragma once

#include "device_params.hpp"

namespace pm7 {

__device__ __forceinline__ int dpack(int a, int b) {
  int h = a >= b ? a : b, l = a >= b ? b : a;
  return h * (h + 1) / 2 + l;
}

__device__ __forceinline__ double dinvsqrt(double x) { return 1.0 / sqrt(x); }

// PM7 feathering (integrals.rs:32-41): cfrac -> 0 beyond 7 Angstrom, point = EV/r.
__device__ __forceinline__ void d_feather(double r, double &cfrac, double &point) {
  point = (1.0 / r) * kEv;
  const double ra = r * kA0;
  if (ra < 7.0) {
    const double t = ra - 7.0;
    cfrac = 1.0 - exp(-(t * t) * 0.22);
  } else {
    cfrac = 0.0;
  }
}

// Quaternion rotation taking (vx,vy,vz) onto +x (integrals.rs:73-105); rows r0,r1,r2.
__device__ __forceinline__ void d_rotation_to_x(double vx, double vy, double vz, double r[3][3]) {
  double qy = vz, qz = -vy, qw = vx + 1.0;
  if (fabs(qw) < 1.0e-13) {
    qy = 0.0;
    qz = 1.0;
    qw = 0.0;
  }
  const double inv = 1.0 / sqrt(qy * qy + qz * qz + qw * qw);
  qy *= inv;
  qz *= inv;
  qw *= inv;
  r[0][0] = (qy * qy + qz * qz) * (-2.0) + 1.0;
  r[0][1] = qz * qw * (-2.0);
  r[0][2] = qy * qw * 2.0;
  r[1][0] = qz * qw * 2.0;
  r[1][1] = qz * qz * (-2.0) + 1.0;
  r[1][2] = qy * qz * 2.0;
  r[2][0] = qy * qw * (-2.0);
  r[2][1] = qy * qz * 2.0;
  r[2][2] = qy * qy * (-2.0) + 1.0;
}

// Heavy atom i (s,p) with hydrogen j: the four local integrals, feathered (integrals.rs:273-294).
__device__ __forceinline__ void d_local_xh(const ElementRec &ei, const ElementRec &ej, double r, double ri[4]) {
  const double ev1 = kEv / 2.0, ev2 = kEv / 4.0;
  const double da = ei.dd, qa = ei.qq * 2.0;
  const double aee = (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0);
  const double ade = (ei.rho1 + ej.rho0) * (ei.rho1 + ej.rho0);
  const double aqe = (ei.rho2 + ej.rho0) * (ei.rho2 + ej.rho0);
  const double ee = dinvsqrt(r * r + aee) * kEv;
  const double q6 = dinvsqrt(r * r + aqe) * ev1;
  ri[0] = ee;
  ri[1] = dinvsqrt((r + da) * (r + da) + ade) * ev1 - dinvsqrt((r - da) * (r - da) + ade) * ev1;
  ri[2] = ee + dinvsqrt((r + qa) * (r + qa) + aqe) * ev2 + dinvsqrt((r - qa) * (r - qa) + aqe) * ev2 - q6;
  ri[3] = ee + dinvsqrt(r * r + qa * qa + aqe) * ev1 - q6;
  double cf, pt;
  d_feather(r, cf, pt);
  const double add = pt * (1.0 - cf);
  for (int k = 0; k < 4; ++k) ri[k] *= cf;
  ri[0] += add;
  ri[2] += add;
  ri[3] += add;
}

// Two heavy atoms: the 22 local integrals, feathered (integrals.rs:296-450).
__device__ __forceinline__ void d_local_xx(const ElementRec &ei, const ElementRec &ej, double r, double ri[22]) {
  const double ev1 = kEv / 2.0, ev2 = kEv / 4.0, ev3 = kEv / 8.0, ev4 = kEv / 16.0;
  const double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0, qa1 = ei.qq, qb1 = ej.qq;
#define SQ_(x) ((x) * (x))
  const double aee = SQ_(ei.rho0 + ej.rho0), ade = SQ_(ei.rho1 + ej.rho0), aqe = SQ_(ei.rho2 + ej.rho0),
               aed = SQ_(ei.rho0 + ej.rho1), aeq = SQ_(ei.rho0 + ej.rho2), axx = SQ_(ei.rho1 + ej.rho1),
               adq = SQ_(ei.rho1 + ej.rho2), aqd = SQ_(ei.rho2 + ej.rho1), aqq = SQ_(ei.rho2 + ej.rho2);
  const double r2 = r * r;
  const double ee = dinvsqrt(r2 + aee) * kEv;
  const double dze = dinvsqrt(SQ_(r - da) + ade) * ev1 - dinvsqrt(SQ_(r + da) + ade) * ev1;
  const double q6 = dinvsqrt(r2 + aqe) * ev1;
  const double qzze = dinvsqrt(SQ_(r - qa) + aqe) * ev2 + dinvsqrt(SQ_(r + qa) + aqe) * ev2 - q6;
  const double qxxe = dinvsqrt(r2 + qa * qa + aqe) * ev1 - q6;
  const double edz = dinvsqrt(SQ_(r + db) + aed) * ev1 - dinvsqrt(SQ_(r - db) + aed) * ev1;
  const double q12 = dinvsqrt(r2 + aeq) * ev1;
  const double eqzz = dinvsqrt(SQ_(r - qb) + aeq) * ev2 + dinvsqrt(SQ_(r + qb) + aeq) * ev2 - q12;
  const double eqxx = dinvsqrt(r2 + qb * qb + aeq) * ev1 - q12;
  const double t20 = dinvsqrt(SQ_(r + da) + adq) * ev2;
  const double t22 = dinvsqrt(SQ_(r - da) + adq) * ev2;
  const double t24 = dinvsqrt(SQ_(r - db) + aqd) * ev2;
  const double t26 = dinvsqrt(SQ_(r + db) + aqd) * ev2;
  const double t36 = dinvsqrt(r2 + aqq) * ev2;
  const double t39 = dinvsqrt(r2 + qa * qa + aqq) * ev2;
  const double t40 = dinvsqrt(r2 + qb * qb + aqq) * ev2;
  const double t42 = dinvsqrt(SQ_(r - qb) + aqq) * ev3;
  const double t44 = dinvsqrt(SQ_(r + qb) + aqq) * ev3;
  const double t46 = dinvsqrt(SQ_(r + qa) + aqq) * ev3;
  const double t48 = dinvsqrt(SQ_(r - qa) + aqq) * ev3;
  ri[0] = ee;
  ri[1] = -dze;
  ri[2] = ee + qzze;
  ri[3] = ee + qxxe;
  ri[4] = -edz;
  ri[5] = dinvsqrt(SQ_(r + da - db) + axx) * ev2 + dinvsqrt(SQ_(r - da + db) + axx) * ev2 -
          dinvsqrt(SQ_(r - da - db) + axx) * ev2 - dinvsqrt(SQ_(r + da + db) + axx) * ev2;
  ri[6] = dinvsqrt(r2 + SQ_(da - db) + axx) * ev1 - dinvsqrt(r2 + SQ_(da + db) + axx) * ev1;
  ri[7] = -edz + dinvsqrt(SQ_(r + qa - db) + aqd) * ev3 - dinvsqrt(SQ_(r + qa + db) + aqd) * ev3 +
          dinvsqrt(SQ_(r - qa - db) + aqd) * ev3 - dinvsqrt(SQ_(r - qa + db) + aqd) * ev3 - t24 + t26;
  ri[8] = -edz - t24 + dinvsqrt(SQ_(r - db) + qa * qa + aqd) * ev2 + t26 - dinvsqrt(SQ_(r + db) + qa * qa + aqd) * ev2;
  ri[9] = dinvsqrt(SQ_(qa1 - db) + SQ_(r + qa1) + aqd) * ev2 - dinvsqrt(SQ_(qa1 - db) + SQ_(r - qa1) + aqd) * ev2 -
          dinvsqrt(SQ_(qa1 + db) + SQ_(r + qa1) + aqd) * ev2 + dinvsqrt(SQ_(qa1 + db) + SQ_(r - qa1) + aqd) * ev2;
  ri[10] = ee + eqzz;
  ri[11] = ee + eqxx;
  ri[12] = -dze + dinvsqrt(SQ_(r + da - qb) + adq) * ev3 - dinvsqrt(SQ_(r - da - qb) + adq) * ev3 +
           dinvsqrt(SQ_(r + da + qb) + adq) * ev3 - dinvsqrt(SQ_(r - da + qb) + adq) * ev3 + t22 - t20;
  ri[13] = -dze - t20 + dinvsqrt(SQ_(r + da) + qb * qb + adq) * ev2 + t22 - dinvsqrt(SQ_(r - da) + qb * qb + adq) * ev2;
  ri[14] = dinvsqrt(SQ_(da - qb1) + SQ_(r - qb1) + adq) * ev2 - dinvsqrt(SQ_(da - qb1) + SQ_(r + qb1) + adq) * ev2 -
           dinvsqrt(SQ_(da + qb1) + SQ_(r - qb1) + adq) * ev2 + dinvsqrt(SQ_(da + qb1) + SQ_(r + qb1) + adq) * ev2;
  ri[15] = ee + eqzz + qzze + dinvsqrt(SQ_(r + qa - qb) + aqq) * ev4 + dinvsqrt(SQ_(r + qa + qb) + aqq) * ev4 +
           dinvsqrt(SQ_(r - qa - qb) + aqq) * ev4 + dinvsqrt(SQ_(r - qa + qb) + aqq) * ev4 - t48 - t46 - t42 - t44 + t36;
  ri[16] = ee + eqzz + qxxe + dinvsqrt(SQ_(r - qb) + qa * qa + aqq) * ev3 + dinvsqrt(SQ_(r + qb) + qa * qa + aqq) * ev3 -
           t42 - t44 - t39 + t36;
  ri[17] = ee + eqxx + qzze + dinvsqrt(SQ_(r + qa) + qb * qb + aqq) * ev3 + dinvsqrt(SQ_(r - qa) + qb * qb + aqq) * ev3 -
           t46 - t48 - t40 + t36;
  const double qxxqxx =
      dinvsqrt(r2 + SQ_(qa - qb) + aqq) * ev3 + dinvsqrt(r2 + SQ_(qa + qb) + aqq) * ev3 - t39 - t40 + t36;
  ri[18] = ee + eqxx + qxxe + qxxqxx;
  const double dm = SQ_(qa1 - qb1), dp = SQ_(qa1 + qb1);
  ri[19] = dinvsqrt(SQ_(r + qa1 - qb1) + dm + aqq) * ev3 - dinvsqrt(SQ_(r + qa1 + qb1) + dm + aqq) * ev3 -
           dinvsqrt(SQ_(r - qa1 - qb1) + dm + aqq) * ev3 + dinvsqrt(SQ_(r - qa1 + qb1) + dm + aqq) * ev3 -
           dinvsqrt(SQ_(r + qa1 - qb1) + dp + aqq) * ev3 + dinvsqrt(SQ_(r + qa1 + qb1) + dp + aqq) * ev3 +
           dinvsqrt(SQ_(r - qa1 - qb1) + dp + aqq) * ev3 - dinvsqrt(SQ_(r - qa1 + qb1) + dp + aqq) * ev3;
  const double qxxqyy = dinvsqrt(r2 + qa * qa + qb * qb + aqq) * ev2 - t39 - t40 + t36;
  ri[20] = ee + eqxx + qxxe + qxxqyy;
  ri[21] = (qxxqxx - qxxqyy) * 0.5;
#undef SQ_
  double cf, pt;
  d_feather(r, cf, pt);
  const double add = pt * (1.0 - cf);
  for (int k = 0; k < 22; ++k) ri[k] *= cf;
  ri[0] += add;
  ri[2] += add;
  ri[3] += add;
  ri[10] += add;
  ri[11] += add;
  ri[15] += add;
  ri[16] += add;
  ri[17] += add;
  ri[18] += add;
  ri[20] += add;
}

// One element of the rotated 10x10 sp-sp block (integrals.rs:466-538): bra pair (kk,ll),
// ket pair (mm,nn), kk>=ll, mm>=nn, orbital 0 = s, 1..3 = p.
__device__ __forceinline__ double d_rotate_xx_elem(const double ri[22], const double r[3][3], int kk, int ll, int mm,
                                                   int nn) {
  const double *r0 = r[0], *r1 = r[1], *r2 = r[2];
  const int k = kk - 1, l = ll - 1, m = mm - 1, n = nn - 1;
  if (kk == 0) {
    if (mm == 0) return ri[0];
    if (nn == 0) return ri[4] * r0[m];
    return ri[10] * (r0[m] * r0[n]) + ri[11] * (r1[m] * r1[n] + r2[m] * r2[n]);
  }
  if (ll == 0) {
    if (mm == 0) return ri[1] * r0[k];
    if (nn == 0) return ri[5] * (r0[k] * r0[m]) + ri[6] * (r1[k] * r1[m] + r2[k] * r2[m]);
    const double t0 = r0[k] * r0[m] * r0[n];
    const double t1 = (r1[m] * r1[n] + r2[m] * r2[n]) * r0[k];
    const double mix = r1[k] * (r1[n] * r0[m] + r1[m] * r0[n]) + r2[k] * (r2[m] * r0[n] + r2[n] * r0[m]);
    return ri[12] * t0 + ri[13] * t1 + ri[14] * mix;
  }
  if (mm == 0) return ri[2] * (r0[k] * r0[l]) + ri[3] * (r1[k] * r1[l] + r2[k] * r2[l]);
  if (nn == 0) {
    const double t0 = r0[k] * r0[l] * r0[m];
    const double t1 = (r1[k] * r1[l] + r2[k] * r2[l]) * r0[m];
    const double t2 = r1[l] * r1[m] + r2[l] * r2[m];
    return ri[7] * t0 + ri[8] * t1 + ri[9] * (r0[k] * t2 + r0[l] * (r1[k] * r1[m] + r2[k] * r2[m]));
  }
  double v = ri[15] * (r0[k] * r0[l] * r0[m] * r0[n]);
  v += ri[16] * ((r1[k] * r1[l] + r2[k] * r2[l]) * r0[m] * r0[n]);
  v += ri[17] * ((r1[m] * r1[n] + r2[m] * r2[n]) * (r0[k] * r0[l]));
  v += ri[18] * (r1[k] * r1[l] * r1[m] * r1[n] + r2[k] * r2[l] * r2[m] * r2[n]);
  const double mix1 = r0[m] * (r1[l] * r1[n] + r2[l] * r2[n]);
  const double mix2 = r0[n] * (r1[l] * r1[m] + r2[l] * r2[m]);
  v += ri[19] * (r0[k] * (mix1 + mix2) + r0[l] * (r0[m] * (r1[k] * r1[n] + r2[k] * r2[n]) +
                                                  r0[n] * (r1[k] * r1[m] + r2[k] * r2[m])));
  v += ri[20] * (r1[k] * r1[l] * r2[m] * r2[n] + r2[k] * r2[l] * r1[m] * r1[n]);
  v += ri[21] * ((r1[k] * r2[l] + r2[k] * r1[l]) * (r1[m] * r2[n] + r2[m] * r1[n]));
  return v;
}

// ---- Slater overlaps, n <= 3 (overlap.rs) ---------------------------------

__device__ __forceinline__ void d_aint(double x, double a[13]) {
  for (int i = 0; i < 13; ++i) a[i] = 0.0;
  if (fabs(x) < 1.0e-12) return;
  const double inv = 1.0 / x;
  a[0] = exp(-x) * inv;
  for (int i = 1; i < 13; ++i) a[i] = a[0] + a[i - 1] * inv * (double)i;
}

__device__ __forceinline__ void d_bint(double x, double b[13]) {
  const double ax = fabs(x);
  if (ax > 0.5) {
    const double inv = 1.0 / x;
    const double tx = exp(x) * inv, tmx = -exp(-x) * inv;
    b[0] = tx + tmx;
    for (int i = 1; i < 13; ++i) b[i] = ((i & 1) ? -tx : tx) + tmx + b[i - 1] * inv * (double)i;
  } else if (ax > 1.0e-6) {
    const double x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x, x6 = x4 * x2;
    b[0] = x2 * (1.0 / 3.0) + x4 * (1.0 / 60.0) + x6 * (1.0 / 2520.0) + 2.0;
    b[2] = x2 * (1.0 / 5.0) + x4 * (1.0 / 84.0) + x6 * (1.0 / 3240.0) + 2.0 / 3.0;
    b[4] = x2 * (1.0 / 7.0) + x4 * (1.0 / 108.0) + x6 * (1.0 / 3960.0) + 2.0 / 5.0;
    b[6] = x2 * (1.0 / 9.0) + x4 * (1.0 / 132.0) + x6 * (1.0 / 4680.0) + 2.0 / 7.0;
    b[8] = x2 * (1.0 / 11.0) + x4 * (1.0 / 156.0) + x6 * (1.0 / 5400.0) + 2.0 / 9.0;
    b[10] = x2 * (1.0 / 13.0) + x4 * (1.0 / 180.0) + x6 * (1.0 / 6120.0) + 2.0 / 11.0;
    b[12] = x2 * (1.0 / 15.0) + x4 * (1.0 / 204.0) + x6 * (1.0 / 6840.0) + 2.0 / 13.0;
    b[1] = x * (-2.0 / 3.0) - x3 * (1.0 / 15.0) - x5 * (1.0 / 420.0);
    b[3] = x * (-2.0 / 5.0) - x3 * (1.0 / 21.0) - x5 * (1.0 / 540.0);
    b[5] = x * (-2.0 / 7.0) - x3 * (1.0 / 27.0) - x5 * (1.0 / 660.0);
    b[7] = x * (-2.0 / 9.0) - x3 * (1.0 / 33.0) - x5 * (1.0 / 780.0);
    b[9] = x * (-2.0 / 11.0) - x3 * (1.0 / 39.0) - x5 * (1.0 / 900.0);
    b[11] = x * (-2.0 / 13.0) - x3 * (1.0 / 45.0) - x5 * (1.0 / 1020.0);
  } else {
    for (int i = 0; i < 13; ++i) b[i] = (i & 1) ? 0.0 : 2.0 / (i + 1.0);
  }
}

// a^b for integer b by binary exponentiation (the evaluation Rust's f64::powi lowers to).
__device__ __forceinline__ double d_powi(double a, int b) {
  const bool recip = b < 0;
  double r = 1.0;
  while (true) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

// Radial normalisation (2 zeta)^(n+1/2) / sqrt((2n)!) of a Slater orbital.
__device__ __forceinline__ double d_slater_norm(int n, double zeta) {
  double f = 1.0;
  for (int k = 1; k <= 2 * n; ++k) f *= (double)k;
  return pow(2.0 * zeta, n + 0.5) / sqrt(fmax(f, 1.0));
}

// <chi(na, la, m) on a | chi(nb, lb, m) on b> for Slater orbitals in the local frame, by
// Gauss-Legendre quadrature in prolate spheroidal coordinates: 48 points in xi on
// [1, 1 + 60/max(p, 0.05)] and 40 in eta on [-1, 1] (overlap_numeric.rs:48-113).
__device__ inline double d_overlap_sto(const DTables *T, int na, double za, int la, int ma, int nb, double zb, int lb,
                                       double r) {
  double c;
  if (la == 0 && lb == 0) c = 0.5;
  else if ((la == 1 && lb == 0 && ma == 0) || (la == 0 && lb == 1 && ma == 0)) c = 0.8660254037844386;
  else if (la == 1 && lb == 1 && ma == 0) c = 1.5;
  else if (la == 1 && lb == 1 && ma == 1) c = 0.75;
  else return 0.0;
  const double norm = d_slater_norm(na, za) * d_slater_norm(nb, zb);
  const double half_r = r * 0.5;
  const double p = (za + zb) * half_r;
  const double xi_max = 1.0 + 60.0 / fmax(p, 0.05);
  const double mid = 0.5 * (1.0 + xi_max), half = 0.5 * (xi_max - 1.0);
  double sum = 0.0;
  for (int i = 0; i < 48; ++i) {
    const double xi = mid + half * T->gl48_t[i], wx = half * T->gl48_w[i];
    for (int j = 0; j < 40; ++j) {
      const double eta = T->gl40_t[j];
      const double ra = half_r * (xi + eta), rb = half_r * (xi - eta);
      if (ra <= 0.0 || rb <= 0.0) continue;
      const double cos_a = (1.0 + xi * eta) / (xi + eta), cos_b = (xi * eta - 1.0) / (xi - eta);
      const double ang_a = la == 0 ? 1.0 : (ma == 0 ? cos_a : sqrt(fmax(1.0 - cos_a * cos_a, 0.0)));
      const double ang_b = lb == 0 ? 1.0 : (ma == 0 ? cos_b : sqrt(fmax(1.0 - cos_b * cos_b, 0.0)));
      const double radial = d_powi(ra, na - 1) * d_powi(rb, nb - 1) * exp(ra * (-za) - rb * zb);
      sum = sum + radial * (wx * T->gl40_w[j] * ang_a * ang_b * (xi * xi - eta * eta));
    }
  }
  return d_powi(half_r, 3) * sum * (norm * c);
}

// Local overlaps (s111, s211, s121, s221, s222) with ea.n >= eb.n >= 1 (overlap.rs:120-296):
// the closed forms for valence shells n <= 3 and the numerical quadrature of
// overlap_numeric.rs:25-43 above (Zn, Ge, As, Se, ... as sp elements).
__device__ inline bool d_overlap_locals(const ElementRec &ea, const ElementRec &eb, double r, double s[5],
                                        const DTables *T) {
  const double za0 = ea.zeta_s, za1 = ea.zeta_p, zb0 = eb.zeta_s, zb1 = eb.zeta_p;
  s[0] = s[1] = s[2] = s[3] = s[4] = 0.0;
  const int na = ea.n, nb = eb.n;
  if (na > 3) {
    s[0] = d_overlap_sto(T, na, za0, 0, 0, nb, zb0, 0, r);
    s[1] = d_overlap_sto(T, na, za1, 1, 0, nb, zb0, 0, r);
    s[2] = -d_overlap_sto(T, na, za0, 0, 0, nb, zb1, 1, r);
    s[3] = -d_overlap_sto(T, na, za1, 1, 0, nb, zb1, 1, r);
    s[4] = d_overlap_sto(T, na, za1, 1, 1, nb, zb1, 1, r);
    return true;
  }
  double A[13], B[13];
  const double sq3 = 1.7320508075688772;
  // s111 (s-s)
  d_aint(r * (0.5 * (za0 + zb0)), A);
  d_bint(r * (0.5 * (za0 - zb0)), B);
  if (na == 1 && nb == 1) {
    s[0] = pow(r * r * (za0 * zb0), 1.5) * (A[2] * B[0] - B[2] * A[0]) / 4.0;
    return true;
  }
  const double r4 = r * r * r * r, r5 = r4 * r, r6 = r5 * r, r7 = r6 * r;
  if (na == 2 && nb == 1) {
    s[0] = r4 * (pow(zb0, 1.5) * pow(za0, 2.5)) * (A[3] * B[0] - B[3] * A[0] + A[2] * B[1] - B[2] * A[1]) / (sq3 * 8.0);
    d_aint(r * (0.5 * (za1 + zb0)), A);
    d_bint(r * (0.5 * (za1 - zb0)), B);
    s[1] = r4 * (pow(zb0, 1.5) * pow(za1, 2.5)) * (A[2] * B[0] - B[2] * A[0] + A[3] * B[1] - B[3] * A[1]) / 8.0;
    return true;
  }
  if (na == 2 && nb == 2) {
    s[0] = r5 * pow(zb0 * za0, 2.5) * (A[4] * B[0] + B[4] * A[0] - A[2] * B[2] * 2.0) / 48.0;
    d_aint(r * (0.5 * (za1 + zb0)), A);
    d_bint(r * (0.5 * (za1 - zb0)), B);
    s[1] = r5 * pow(zb0 * za1, 2.5) *
           (A[3] * (B[0] - B[2]) - A[1] * (B[2] - B[4]) + B[3] * (A[0] - A[2]) - B[1] * (A[2] - A[4])) / (16.0 * sq3);
    d_aint(r * (0.5 * (za0 + zb1)), A);
    d_bint(r * (0.5 * (za0 - zb1)), B);
    s[2] = r5 * pow(zb1 * za0, 2.5) *
           (A[3] * (B[0] - B[2]) - A[1] * (B[2] - B[4]) - B[3] * (A[0] - A[2]) + B[1] * (A[2] - A[4])) / (16.0 * sq3);
    d_aint(r * (0.5 * (za1 + zb1)), A);
    d_bint(r * (0.5 * (za1 - zb1)), B);
    const double w = r5 * pow(zb1 * za1, 2.5) / 16.0;
    s[3] = -(w * (B[2] * (A[4] + A[0]) - A[2] * (B[4] + B[0])));
    s[4] = w * (A[4] * (B[0] - B[2]) - B[4] * (A[0] - A[2]) - A[2] * B[0] + B[2] * A[0]) * 0.5;
    return true;
  }
  if (na == 3 && nb == 1) {
    s[0] = r5 * (pow(zb0, 1.5) * pow(za0, 3.5)) * (A[4] * B[0] + B[1] * A[3] * 2.0 - A[1] * B[3] * 2.0 - B[4] * A[0]) /
           (sqrt(10.0) * 24.0);
    d_aint(r * (0.5 * (za1 + zb0)), A);
    d_bint(r * (0.5 * (za1 - zb0)), B);
    s[1] = r5 * (pow(zb0, 1.5) * pow(za1, 3.5)) *
           (A[3] * (B[0] + B[2]) - A[1] * (B[4] + B[2]) + B[1] * (A[2] + A[4]) - B[3] * (A[2] + A[0])) /
           (8.0 * sqrt(30.0));
    return true;
  }
  if (na == 3 && nb == 2) {
    s[0] = r6 * (pow(zb0, 2.5) * pow(za0, 3.5)) *
           (A[5] * B[0] + B[1] * A[4] - B[2] * A[3] * 2.0 - A[2] * B[3] * 2.0 + B[4] * A[1] + B[5] * A[0]) /
           (sqrt(30.0) * 48.0);
    d_aint(r * (0.5 * (za1 + zb0)), A);
    d_bint(r * (0.5 * (za1 - zb0)), B);
    s[1] = r6 * (pow(zb0, 2.5) * pow(za1, 3.5)) *
           (A[4] * B[0] + B[1] * A[5] - B[3] * A[3] * 2.0 - A[2] * B[2] * 2.0 + A[1] * B[5] + A[0] * B[4]) /
           (48.0 * sqrt(10.0));
    d_aint(r * (0.5 * (za0 + zb1)), A);
    d_bint(r * (0.5 * (za0 - zb1)), B);
    s[2] = r6 * (pow(zb1, 2.5) * pow(za0, 3.5)) *
           ((A[4] * B[0] - A[5] * B[1]) + (A[3] * B[1] - A[4] * B[2]) * 2.0 - (A[1] * B[3] - A[2] * B[4]) * 2.0 -
            (A[0] * B[4] - A[1] * B[5])) /
           (48.0 * sqrt(10.0));
    d_aint(r * (0.5 * (za1 + zb1)), A);
    d_bint(r * (0.5 * (za1 - zb1)), B);
    const double pre = r6 * (pow(zb1, 2.5) * pow(za1, 3.5));
    s[3] = pre *
           ((A[3] * B[0] - A[5] * B[2]) + (A[2] * B[1] - A[4] * B[3]) - (A[1] * B[2] - A[3] * B[4]) -
            (A[0] * B[3] - A[2] * B[5])) /
           (16.0 * sqrt(30.0));
    s[4] = pre *
           ((A[5] - A[3]) * (B[0] - B[2]) + (A[4] - A[2]) * (B[1] - B[3]) - (A[3] - A[1]) * (B[2] - B[4]) -
            (A[2] - A[0]) * (B[3] - B[5])) /
           (32.0 * sqrt(30.0));
    return true;
  }
  if (na == 3 && nb == 3) {
    s[0] = r7 * pow(zb0 * za0, 3.5) * (A[6] * B[0] - B[2] * A[4] * 3.0 + A[2] * B[4] * 3.0 - A[0] * B[6]) / 1440.0;
    d_aint(r * (0.5 * (za1 + zb0)), A);
    d_bint(r * (0.5 * (za1 - zb0)), B);
    s[1] = r7 * pow(zb0 * za1, 3.5) *
           ((A[5] * B[0] + A[6] * B[1]) + (-A[4] * B[1] - A[5] * B[2]) - (A[3] * B[2] + A[4] * B[3]) * 2.0 -
            (-A[2] * B[3] - A[3] * B[4]) * 2.0 + (A[1] * B[4] + A[2] * B[5]) + (-A[0] * B[5] - A[1] * B[6])) /
           (480.0 * sq3);
    d_aint(r * (0.5 * (za0 + zb1)), A);
    d_bint(r * (0.5 * (za0 - zb1)), B);
    s[2] = r7 * pow(zb1 * za0, 3.5) *
           ((A[5] * B[0] - A[6] * B[1]) + (A[4] * B[1] - A[5] * B[2]) - (A[3] * B[2] - A[4] * B[3]) * 2.0 -
            (A[2] * B[3] - A[3] * B[4]) * 2.0 + (A[1] * B[4] - A[2] * B[5]) + (A[0] * B[5] - A[1] * B[6])) /
           (480.0 * sq3);
    d_aint(r * (0.5 * (za1 + zb1)), A);
    d_bint(r * (0.5 * (za1 - zb1)), B);
    const double pre = r7 * (pow(zb1, 3.5) * pow(za1, 3.5));
    s[3] = pre * ((A[4] * B[0] - A[6] * B[2]) - (A[2] * B[2] - A[4] * B[4]) * 2.0 + (A[0] * B[4] - A[2] * B[6])) / 480.0;
    s[4] = pre *
           ((A[6] - A[4]) * (B[0] - B[2]) - (A[4] - A[2]) * (B[2] - B[4]) * 2.0 + (A[2] - A[0]) * (B[4] - B[6])) /
           960.0;
    return true;
  }
  return false;
}

// 4x4 overlap block S[a_i][b_j] for atoms i, j with displacement d = R_j - R_i
// (overlap.rs:16-40,301-328). Returns false for a shell pair no formula covers.
__device__ inline bool d_overlap_sp(const ElementRec &ei, const ElementRec &ej, double dx, double dy, double dz,
                                    double S[4][4], const DTables *T) {
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) S[a][b] = 0.0;
  if (r < 1.0e-8) {
    for (int k = 0; k < 4; ++k) S[k][k] = 1.0;
    return true;
  }
  const bool swap = ei.n < ej.n;
  const ElementRec &ea = swap ? ej : ei;
  const ElementRec &eb = swap ? ei : ej;
  double loc[5];
  if (!d_overlap_locals(ea, eb, r, loc, T)) return false;
  const double sgn = swap ? -1.0 : 1.0;
  double rr[3][3];
  d_rotation_to_x(sgn * dx / r, sgn * dy / r, sgn * dz / r, rr);
  double di[4][4];
  di[0][0] = loc[0];
  for (int a = 0; a < 3; ++a) {
    di[1 + a][0] = loc[1] * rr[0][a];
    di[0][1 + a] = -loc[2] * rr[0][a];
  }
  const double mm[3] = {-loc[3], loc[4], loc[4]};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v = v + rr[k][a] * mm[k] * rr[k][b];
      di[1 + a][1 + b] = v;
    }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) S[a][b] = swap ? di[b][a] : di[a][b];
  return true;
}

}  // namespace pm7
