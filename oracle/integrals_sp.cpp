// Oracle (test infrastructure): sp two-centre integrals and sp overlaps.
// Restates pm7-rs src/integrals.rs and src/overlap.rs (f64 instantiation).
#include <cmath>

#include "oracle_internal.hpp"

namespace oracle {

// PM7 feathering, src/integrals.rs:32-41.
void feather_to_point(double r, double &cfrac, double &point) {
  point = (1.0 / r) * EV;
  double r_ang = r * A0;
  cfrac = r_ang < 7.0 ? 1.0 - std::exp(-std::pow(r_ang - 7.0, 2) * 0.22) : 0.0;
}

static void feather_ri(double *ri, int n, double r, const int *mono, int nmono) {
  double cfrac, point;
  feather_to_point(r, cfrac, point);
  double add = point * (1.0 - cfrac);
  for (int k = 0; k < n; ++k) ri[k] = ri[k] * cfrac;
  for (int k = 0; k < nmono; ++k) ri[mono[k]] = ri[mono[k]] + add;
}

static const int XX_MONOPOLE[10] = {0, 2, 3, 10, 11, 15, 16, 17, 18, 20};
static const int XH_MONOPOLE[3] = {0, 2, 3};

// Shortest-arc quaternion rotation taking v onto +x, src/integrals.rs:73-105.
void rotation_to_x(double vx, double vy, double vz, double r[3][3]) {
  double qy = vz, qz = -vy, qw = vx + 1.0;
  if (std::fabs(qw) < 1.0e-13) {
    qy = 0.0;
    qz = 1.0;
    qw = 0.0;
  }
  double inv = 1.0 / std::sqrt(qy * qy + qz * qz + qw * qw);
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

// src/integrals.rs:273-294
static void local_xh(const Element &ei, const Element &ej, double r, double ri[4]) {
  const double ev1 = EV / 2.0, ev2 = EV / 4.0;
  double da = ei.dd, qa = ei.qq * 2.0;
  double aee = std::pow(ei.rho0 + ej.rho0, 2), ade = std::pow(ei.rho1 + ej.rho0, 2),
         aqe = std::pow(ei.rho2 + ej.rho0, 2);
  double ee = (1.0 / std::sqrt(r * r + aee)) * EV;
  double ev1dsqr6 = (1.0 / std::sqrt(r * r + aqe)) * ev1;
  ri[0] = ee;
  ri[1] = (1.0 / std::sqrt((r + da) * (r + da) + ade)) * ev1 - (1.0 / std::sqrt((r - da) * (r - da) + ade)) * ev1;
  ri[2] = ee + (1.0 / std::sqrt((r + qa) * (r + qa) + aqe)) * ev2 +
          (1.0 / std::sqrt((r - qa) * (r - qa) + aqe)) * ev2 - ev1dsqr6;
  ri[3] = ee + (1.0 / std::sqrt(r * r + qa * qa + aqe)) * ev1 - ev1dsqr6;
  feather_ri(ri, 4, r, XH_MONOPOLE, 3);
}

// src/integrals.rs:296-450 (Dewar-Sabelli-Klopman multipole interactions).
static void local_xx(const Element &ei, const Element &ej, double r, double ri[22]) {
  const double ev1 = EV / 2.0, ev2 = EV / 4.0, ev3 = EV / 8.0, ev4 = EV / 16.0;
  double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0, qa1 = ei.qq, qb1 = ej.qq;
  double aee = std::pow(ei.rho0 + ej.rho0, 2), ade = std::pow(ei.rho1 + ej.rho0, 2),
         aqe = std::pow(ei.rho2 + ej.rho0, 2), aed = std::pow(ei.rho0 + ej.rho1, 2),
         aeq = std::pow(ei.rho0 + ej.rho2, 2), axx = std::pow(ei.rho1 + ej.rho1, 2),
         adq = std::pow(ei.rho1 + ej.rho2, 2), aqd = std::pow(ei.rho2 + ej.rho1, 2),
         aqq = std::pow(ei.rho2 + ej.rho2, 2);
  auto g = [](double x, double c) { return 1.0 / std::sqrt(x + c); };
  auto sq2 = [](double a, double c) { return 1.0 / std::sqrt(a * a + c); };
  double ee = (1.0 / std::sqrt(r * r + aee)) * EV;
  double dze = sq2(r - da, ade) * ev1 - sq2(r + da, ade) * ev1;
  double ev1dsqr6 = (1.0 / std::sqrt(r * r + aqe)) * ev1;
  double qzze = sq2(r - qa, aqe) * ev2 + sq2(r + qa, aqe) * ev2 - ev1dsqr6;
  double qxxe = g(r * r + qa * qa, aqe) * ev1 - ev1dsqr6;
  double edz = sq2(r + db, aed) * ev1 - sq2(r - db, aed) * ev1;
  double ev1dsqr12 = (1.0 / std::sqrt(r * r + aeq)) * ev1;
  double eqzz = sq2(r - qb, aeq) * ev2 + sq2(r + qb, aeq) * ev2 - ev1dsqr12;
  double eqxx = g(r * r + qb * qb, aeq) * ev1 - ev1dsqr12;
  double ev2dsqr20 = sq2(r + da, adq) * ev2;
  double ev2dsqr22 = sq2(r - da, adq) * ev2;
  double ev2dsqr24 = sq2(r - db, aqd) * ev2;
  double ev2dsqr26 = sq2(r + db, aqd) * ev2;
  double ev2dsqr36 = (1.0 / std::sqrt(r * r + aqq)) * ev2;
  double ev2dsqr39 = g(r * r + qa * qa, aqq) * ev2;
  double ev2dsqr40 = g(r * r + qb * qb, aqq) * ev2;
  double ev3dsqr42 = sq2(r - qb, aqq) * ev3;
  double ev3dsqr44 = sq2(r + qb, aqq) * ev3;
  double ev3dsqr46 = sq2(r + qa, aqq) * ev3;
  double ev3dsqr48 = sq2(r - qa, aqq) * ev3;
  ri[0] = ee;
  ri[1] = -dze;
  ri[2] = ee + qzze;
  ri[3] = ee + qxxe;
  ri[4] = -edz;
  ri[5] = sq2(r + da - db, axx) * ev2 + sq2(r - da + db, axx) * ev2 - sq2(r - da - db, axx) * ev2 -
          sq2(r + da + db, axx) * ev2;
  ri[6] = g(r * r + (da - db) * (da - db), axx) * ev1 - g(r * r + (da + db) * (da + db), axx) * ev1;
  ri[7] = -edz + sq2(r + qa - db, aqd) * ev3 - sq2(r + qa + db, aqd) * ev3 + sq2(r - qa - db, aqd) * ev3 -
          sq2(r - qa + db, aqd) * ev3 - ev2dsqr24 + ev2dsqr26;
  ri[8] = -edz - ev2dsqr24 + g((r - db) * (r - db) + qa * qa, aqd) * ev2 + ev2dsqr26 -
          g((r + db) * (r + db) + qa * qa, aqd) * ev2;
  ri[9] = g((qa1 - db) * (qa1 - db) + (r + qa1) * (r + qa1), aqd) * ev2 -
          g((qa1 - db) * (qa1 - db) + (r - qa1) * (r - qa1), aqd) * ev2 -
          g((qa1 + db) * (qa1 + db) + (r + qa1) * (r + qa1), aqd) * ev2 +
          g((qa1 + db) * (qa1 + db) + (r - qa1) * (r - qa1), aqd) * ev2;
  ri[10] = ee + eqzz;
  ri[11] = ee + eqxx;
  ri[12] = -dze + sq2(r + da - qb, adq) * ev3 - sq2(r - da - qb, adq) * ev3 + sq2(r + da + qb, adq) * ev3 -
           sq2(r - da + qb, adq) * ev3 + ev2dsqr22 - ev2dsqr20;
  ri[13] = -dze - ev2dsqr20 + g((r + da) * (r + da) + qb * qb, adq) * ev2 + ev2dsqr22 -
           g((r - da) * (r - da) + qb * qb, adq) * ev2;
  ri[14] = g((da - qb1) * (da - qb1) + (r - qb1) * (r - qb1), adq) * ev2 -
           g((da - qb1) * (da - qb1) + (r + qb1) * (r + qb1), adq) * ev2 -
           g((da + qb1) * (da + qb1) + (r - qb1) * (r - qb1), adq) * ev2 +
           g((da + qb1) * (da + qb1) + (r + qb1) * (r + qb1), adq) * ev2;
  ri[15] = ee + eqzz + qzze + sq2(r + qa - qb, aqq) * ev4 + sq2(r + qa + qb, aqq) * ev4 +
           sq2(r - qa - qb, aqq) * ev4 + sq2(r - qa + qb, aqq) * ev4 - ev3dsqr48 - ev3dsqr46 - ev3dsqr42 -
           ev3dsqr44 + ev2dsqr36;
  ri[16] = ee + eqzz + qxxe + g((r - qb) * (r - qb) + qa * qa, aqq) * ev3 +
           g((r + qb) * (r + qb) + qa * qa, aqq) * ev3 - ev3dsqr42 - ev3dsqr44 - ev2dsqr39 + ev2dsqr36;
  ri[17] = ee + eqxx + qzze + g((r + qa) * (r + qa) + qb * qb, aqq) * ev3 +
           g((r - qa) * (r - qa) + qb * qb, aqq) * ev3 - ev3dsqr46 - ev3dsqr48 - ev2dsqr40 + ev2dsqr36;
  double qxxqxx = g(r * r + (qa - qb) * (qa - qb), aqq) * ev3 + g(r * r + (qa + qb) * (qa + qb), aqq) * ev3 -
                  ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
  ri[18] = ee + eqxx + qxxe + qxxqxx;
  double dm = (qa1 - qb1) * (qa1 - qb1), dp = (qa1 + qb1) * (qa1 + qb1);
  ri[19] = g((r + qa1 - qb1) * (r + qa1 - qb1) + dm, aqq) * ev3 - g((r + qa1 + qb1) * (r + qa1 + qb1) + dm, aqq) * ev3 -
           g((r - qa1 - qb1) * (r - qa1 - qb1) + dm, aqq) * ev3 + g((r - qa1 + qb1) * (r - qa1 + qb1) + dm, aqq) * ev3 -
           g((r + qa1 - qb1) * (r + qa1 - qb1) + dp, aqq) * ev3 + g((r + qa1 + qb1) * (r + qa1 + qb1) + dp, aqq) * ev3 +
           g((r - qa1 - qb1) * (r - qa1 - qb1) + dp, aqq) * ev3 - g((r - qa1 + qb1) * (r - qa1 + qb1) + dp, aqq) * ev3;
  double qxxqyy = g(r * r + qa * qa + qb * qb, aqq) * ev2 - ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
  ri[20] = ee + eqxx + qxxe + qxxqyy;
  ri[21] = (qxxqxx - qxxqyy) * 0.5;
  feather_ri(ri, 22, r, XX_MONOPOLE, 10);
}

// src/integrals.rs:466-538: rotate the 22 local integrals into the 10x10 block.
static void rotate_xx(const double ri[22], const double r0[3], const double r1[3], const double r2[3],
                      double *w) {
  int idx = 0;
  for (int kk = 0; kk < 4; ++kk)
    for (int ll = 0; ll <= kk; ++ll)
      for (int mm = 0; mm < 4; ++mm)
        for (int nn = 0; nn <= mm; ++nn) {
          int k = kk - 1, l = ll - 1, m = mm - 1, n = nn - 1;
          double val;
          if (kk == 0) {
            if (mm == 0) val = ri[0];
            else if (nn == 0) val = ri[4] * r0[m];
            else val = ri[10] * (r0[m] * r0[n]) + ri[11] * (r1[m] * r1[n] + r2[m] * r2[n]);
          } else if (ll == 0) {
            if (mm == 0) val = ri[1] * r0[k];
            else if (nn == 0) val = ri[5] * (r0[k] * r0[m]) + ri[6] * (r1[k] * r1[m] + r2[k] * r2[m]);
            else {
              double t0 = r0[k] * r0[m] * r0[n];
              double t1 = (r1[m] * r1[n] + r2[m] * r2[n]) * r0[k];
              double mix = r1[k] * (r1[n] * r0[m] + r1[m] * r0[n]) + r2[k] * (r2[m] * r0[n] + r2[n] * r0[m]);
              val = ri[12] * t0 + ri[13] * t1 + ri[14] * mix;
            }
          } else if (mm == 0) {
            double t0 = r0[k] * r0[l];
            double t1 = r1[k] * r1[l] + r2[k] * r2[l];
            val = ri[2] * t0 + ri[3] * t1;
          } else if (nn == 0) {
            double t0 = r0[k] * r0[l] * r0[m];
            double t1 = (r1[k] * r1[l] + r2[k] * r2[l]) * r0[m];
            double t2 = r1[l] * r1[m] + r2[l] * r2[m];
            val = ri[7] * t0 + ri[8] * t1 + ri[9] * (r0[k] * t2 + r0[l] * (r1[k] * r1[m] + r2[k] * r2[m]));
          } else {
            double t0 = r0[k] * r0[l] * r0[m] * r0[n];
            double v = ri[15] * t0;
            v = v + ri[16] * ((r1[k] * r1[l] + r2[k] * r2[l]) * r0[m] * r0[n]);
            v = v + ri[17] * ((r1[m] * r1[n] + r2[m] * r2[n]) * (r0[k] * r0[l]));
            v = v + ri[18] * (r1[k] * r1[l] * r1[m] * r1[n] + r2[k] * r2[l] * r2[m] * r2[n]);
            double mix1 = r0[m] * (r1[l] * r1[n] + r2[l] * r2[n]);
            double mix2 = r0[n] * (r1[l] * r1[m] + r2[l] * r2[m]);
            double val5 = r0[k] * (mix1 + mix2) +
                          r0[l] * (r0[m] * (r1[k] * r1[n] + r2[k] * r2[n]) + r0[n] * (r1[k] * r1[m] + r2[k] * r2[m]));
            v = v + ri[19] * val5;
            v = v + ri[20] * (r1[k] * r1[l] * r2[m] * r2[n] + r2[k] * r2[l] * r1[m] * r1[n]);
            double cross = (r1[k] * r2[l] + r2[k] * r1[l]) * (r1[m] * r2[n] + r2[m] * r1[n]);
            v = v + ri[21] * cross;
            val = v;
          }
          w[idx++] = val;
        }
}

// pair_two_electron_g, sp branch (src/integrals.rs:186-271).
PairBlock pair_two_electron_sp(const Element &ei, const Element &ej, const double d[3]) {
  double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  double inv = 1.0 / r;
  double x[3] = {d[0] * inv, d[1] * inv, d[2] * inv};
  bool heavy_i = ei.has_p(), heavy_j = ej.has_p();
  PairBlock out;
  double rot[3][3];
  rotation_to_x(-x[0], -x[1], -x[2], rot);
  if (!heavy_i && !heavy_j) {
    double aee = std::pow(ei.rho0 + ej.rho0, 2);
    double ee_nddo = (1.0 / std::sqrt(r * r + aee)) * EV;
    double cfrac, point;
    feather_to_point(r, cfrac, point);
    double ee = ee_nddo * cfrac + point * (1.0 - cfrac);
    out.norb_i = out.norb_j = out.npair_i = out.npair_j = 1;
    out.w = {ee};
    out.e1b[0][0] = ee * (-ej.core_charge);
    out.e2a[0][0] = ee * (-ei.core_charge);
    return out;
  }
  if (heavy_i && !heavy_j) {
    double ri[4];
    local_xh(ei, ej, r, ri);
    double wxh[10];
    wxh[pack(0, 0)] = ri[0];
    for (int k = 0; k < 3; ++k) wxh[pack(k + 1, 0)] = ri[1] * rot[0][k];
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l <= k; ++l) {
        double t0 = rot[0][k] * rot[0][l];
        double t1 = rot[1][k] * rot[1][l] + rot[2][k] * rot[2][l];
        wxh[pack(k + 1, l + 1)] = ri[2] * t0 + ri[3] * t1;
      }
    out.norb_i = 4;
    out.norb_j = 1;
    out.npair_i = 10;
    out.npair_j = 1;
    out.w.assign(wxh, wxh + 10);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) out.e1b[a][b] = wxh[pack(a, b)] * (-ej.core_charge);
    out.e2a[0][0] = wxh[0] * (-ei.core_charge);
    return out;
  }
  double ri[22];
  local_xx(ei, ej, r, ri);
  out.norb_i = out.norb_j = 4;
  out.npair_i = out.npair_j = 10;
  out.w.assign(100, 0.0);
  rotate_xx(ri, rot[0], rot[1], rot[2], out.w.data());
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      out.e1b[a][b] = out.w[pack(a, b) * 10] * (-ej.core_charge);
      out.e2a[a][b] = out.w[pack(a, b)] * (-ei.core_charge);
    }
  return out;
}

PairBlock pair_two_electron(const Element &ei, const Element &ej, const double d[3]) {
  if (ei.n_orb == 9 || ej.n_orb == 9) return pair_two_electron_d(ei, ej, d);
  return pair_two_electron_sp(ei, ej, d);
}

// ---- sp overlaps (src/overlap.rs) ------------------------------------

// A_k(x) = int_1^inf t^k e^{-xt} dt, src/overlap.rs:403-414.
static void aintgs(double x, double a[13]) {
  for (int i = 0; i < 13; ++i) a[i] = 0.0;
  if (std::fabs(x) < 1.0e-12) return;
  double inv = 1.0 / x;
  a[0] = std::exp(-x) * inv;
  for (int i = 1; i < 13; ++i) a[i] = a[0] + a[i - 1] * inv * (double)i;
}

// B_k(x) = int_-1^1 t^k e^{-xt} dt, src/overlap.rs:418-462.
static void bintgs(double x, double b[13]) {
  for (int i = 0; i < 13; ++i) b[i] = 0.0;
  double absx = std::fabs(x);
  if (absx > 0.5) {
    double inv = 1.0 / x;
    double tx = std::exp(x) * inv;
    double tmx = std::exp(-x) * inv * (-1.0);
    b[0] = tx + tmx;
    for (int i = 1; i < 13; ++i) {
      double sign = (i % 2 == 0) ? 1.0 : -1.0;
      b[i] = tx * sign + tmx + b[i - 1] * inv * (double)i;
    }
  } else if (absx > 1.0e-6) {
    double x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x, x6 = x4 * x2;
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
    for (int i = 0; i < 13; ++i) b[i] = (i % 2 == 0) ? 2.0 / (i + 1.0) : 0.0;
  }
}

// src/overlap.rs:120-296: local overlaps (s111, s211, s121, s221, s222), ea.n >= eb.n.
static void overlap_locals(const Element &ea, const Element &eb, double r, double s[5]) {
  int jcall = 0;
  if (ea.n == 1 && eb.n == 1) jcall = 2;
  else if (ea.n == 2 && eb.n == 1) jcall = 3;
  else if (ea.n == 2 && eb.n == 2) jcall = 4;
  else if (ea.n == 3 && eb.n == 1) jcall = 431;
  else if (ea.n == 3 && eb.n == 2) jcall = 5;
  else if (ea.n == 3 && eb.n == 3) jcall = 6;
  double za[2] = {ea.zeta_s, ea.zeta_p}, zb[2] = {eb.zeta_s, eb.zeta_p};
  double a111[13], b111[13], a211[13], b211[13], a121[13], b121[13], a22[13], b22[13];
  aintgs(r * (0.5 * (za[0] + zb[0])), a111);
  bintgs(r * (0.5 * (za[0] - zb[0])), b111);
  aintgs(r * (0.5 * (za[1] + zb[0])), a211);
  bintgs(r * (0.5 * (za[1] - zb[0])), b211);
  aintgs(r * (0.5 * (za[0] + zb[1])), a121);
  bintgs(r * (0.5 * (za[0] - zb[1])), b121);
  aintgs(r * (0.5 * (za[1] + zb[1])), a22);
  bintgs(r * (0.5 * (za[1] - zb[1])), b22);
  double s111 = 0, s211 = 0, s121 = 0, s221 = 0, s222 = 0;
  const double sq3 = std::sqrt(3.0);
  switch (jcall) {
    case 0:
      slater_locals_numeric(ea.n, ea.zeta_s, ea.zeta_p, eb.n, eb.zeta_s, eb.zeta_p, r, s);
      return;
    case 2:
      s111 = std::pow(r * r * (za[0] * zb[0]), 1.5) * (a111[2] * b111[0] - b111[2] * a111[0]) / 4.0;
      break;
    case 3:
      s111 = std::pow(r, 4) * (std::pow(zb[0], 1.5) * std::pow(za[0], 2.5)) *
             (a111[3] * b111[0] - b111[3] * a111[0] + a111[2] * b111[1] - b111[2] * a111[1]) / (sq3 * 8.0);
      s211 = std::pow(r, 4) * (std::pow(zb[0], 1.5) * std::pow(za[1], 2.5)) *
             (a211[2] * b211[0] - b211[2] * a211[0] + a211[3] * b211[1] - b211[3] * a211[1]) / 8.0;
      break;
    case 4: {
      s111 = std::pow(r, 5) * std::pow(zb[0] * za[0], 2.5) *
             (a111[4] * b111[0] + b111[4] * a111[0] - a111[2] * b111[2] * 2.0) / 48.0;
      s211 = std::pow(r, 5) * std::pow(zb[0] * za[1], 2.5) *
             (a211[3] * (b211[0] - b211[2]) - a211[1] * (b211[2] - b211[4]) + b211[3] * (a211[0] - a211[2]) -
              b211[1] * (a211[2] - a211[4])) /
             (16.0 * sq3);
      s121 = std::pow(r, 5) * std::pow(zb[1] * za[0], 2.5) *
             (a121[3] * (b121[0] - b121[2]) - a121[1] * (b121[2] - b121[4]) - b121[3] * (a121[0] - a121[2]) +
              b121[1] * (a121[2] - a121[4])) /
             (16.0 * sq3);
      double w = std::pow(r, 5) * std::pow(zb[1] * za[1], 2.5) / 16.0;
      s221 = -(w * (b22[2] * (a22[4] + a22[0]) - a22[2] * (b22[4] + b22[0])));
      s222 = w * (a22[4] * (b22[0] - b22[2]) - b22[4] * (a22[0] - a22[2]) - a22[2] * b22[0] + b22[2] * a22[0]) * 0.5;
      break;
    }
    case 431:
      s111 = std::pow(r, 5) * (std::pow(zb[0], 1.5) * std::pow(za[0], 3.5)) *
             (a111[4] * b111[0] + b111[1] * a111[3] * 2.0 - a111[1] * b111[3] * 2.0 - b111[4] * a111[0]) /
             (std::sqrt(10.0) * 24.0);
      s211 = std::pow(r, 5) * (std::pow(zb[0], 1.5) * std::pow(za[1], 3.5)) *
             (a211[3] * (b211[0] + b211[2]) - a211[1] * (b211[4] + b211[2]) + b211[1] * (a211[2] + a211[4]) -
              b211[3] * (a211[2] + a211[0])) /
             (8.0 * std::sqrt(30.0));
      break;
    case 5:
      s111 = std::pow(r, 6) * (std::pow(zb[0], 2.5) * std::pow(za[0], 3.5)) *
             (a111[5] * b111[0] + b111[1] * a111[4] - b111[2] * a111[3] * 2.0 - a111[2] * b111[3] * 2.0 +
              b111[4] * a111[1] + b111[5] * a111[0]) /
             (std::sqrt(30.0) * 48.0);
      s211 = std::pow(r, 6) * (std::pow(zb[0], 2.5) * std::pow(za[1], 3.5)) *
             (a211[4] * b211[0] + b211[1] * a211[5] - b211[3] * a211[3] * 2.0 - a211[2] * b211[2] * 2.0 +
              a211[1] * b211[5] + a211[0] * b211[4]) /
             (48.0 * std::sqrt(10.0));
      s121 = std::pow(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[0], 3.5)) *
             ((a121[4] * b121[0] - a121[5] * b121[1]) + (a121[3] * b121[1] - a121[4] * b121[2]) * 2.0 -
              (a121[1] * b121[3] - a121[2] * b121[4]) * 2.0 - (a121[0] * b121[4] - a121[1] * b121[5])) /
             (48.0 * std::sqrt(10.0));
      s221 = std::pow(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[1], 3.5)) *
             ((a22[3] * b22[0] - a22[5] * b22[2]) + (a22[2] * b22[1] - a22[4] * b22[3]) -
              (a22[1] * b22[2] - a22[3] * b22[4]) - (a22[0] * b22[3] - a22[2] * b22[5])) /
             (16.0 * std::sqrt(30.0));
      s222 = std::pow(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[1], 3.5)) *
             ((a22[5] - a22[3]) * (b22[0] - b22[2]) + (a22[4] - a22[2]) * (b22[1] - b22[3]) -
              (a22[3] - a22[1]) * (b22[2] - b22[4]) - (a22[2] - a22[0]) * (b22[3] - b22[5])) /
             (32.0 * std::sqrt(30.0));
      break;
    case 6:
      s111 = std::pow(r, 7) * std::pow(zb[0] * za[0], 3.5) *
             (a111[6] * b111[0] - b111[2] * a111[4] * 3.0 + a111[2] * b111[4] * 3.0 - a111[0] * b111[6]) / 1440.0;
      s211 = std::pow(r, 7) * std::pow(zb[0] * za[1], 3.5) *
             ((a211[5] * b211[0] + a211[6] * b211[1]) + (-a211[4] * b211[1] - a211[5] * b211[2]) -
              (a211[3] * b211[2] + a211[4] * b211[3]) * 2.0 - (-a211[2] * b211[3] - a211[3] * b211[4]) * 2.0 +
              (a211[1] * b211[4] + a211[2] * b211[5]) + (-a211[0] * b211[5] - a211[1] * b211[6])) /
             (480.0 * sq3);
      s121 = std::pow(r, 7) * std::pow(zb[1] * za[0], 3.5) *
             ((a121[5] * b121[0] - a121[6] * b121[1]) + (a121[4] * b121[1] - a121[5] * b121[2]) -
              (a121[3] * b121[2] - a121[4] * b121[3]) * 2.0 - (a121[2] * b121[3] - a121[3] * b121[4]) * 2.0 +
              (a121[1] * b121[4] - a121[2] * b121[5]) + (a121[0] * b121[5] - a121[1] * b121[6])) /
             (480.0 * sq3);
      s221 = std::pow(r, 7) * (std::pow(zb[1], 3.5) * std::pow(za[1], 3.5)) *
             ((a22[4] * b22[0] - a22[6] * b22[2]) - (a22[2] * b22[2] - a22[4] * b22[4]) * 2.0 +
              (a22[0] * b22[4] - a22[2] * b22[6])) /
             480.0;
      s222 = std::pow(r, 7) * (std::pow(zb[1], 3.5) * std::pow(za[1], 3.5)) *
             ((a22[6] - a22[4]) * (b22[0] - b22[2]) - (a22[4] - a22[2]) * (b22[2] - b22[4]) * 2.0 +
              (a22[2] - a22[0]) * (b22[4] - b22[6])) /
             960.0;
      break;
    default:
      break;
  }
  s[0] = s111;
  s[1] = s211;
  s[2] = s121;
  s[3] = s221;
  s[4] = s222;
}

// src/overlap.rs:301-328
static void build_di(const double s[5], const double dir[3], double di[4][4]) {
  double rr[3][3];
  rotation_to_x(dir[0], dir[1], dir[2], rr);
  double rot[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) rot[a][b] = rr[b][a];
  di[0][0] = s[0];
  for (int a = 0; a < 3; ++a) {
    di[1 + a][0] = s[1] * rot[a][0];
    di[0][1 + a] = -s[2] * rot[a][0];
  }
  double mm[3] = {-s[3], s[4], s[4]};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v = v + rot[a][k] * mm[k] * rot[b][k];
      di[1 + a][1 + b] = v;
    }
}

// diatom_overlap (src/overlap.rs:16-40), embedded in a 9x9 block.
void diatom_overlap_sp(const Element &ei, const Element &ej, const Vec3 &d, double s9[9][9]) {
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) s9[i][j] = 0.0;
  double r = d.norm();
  double di[4][4];
  if (r < 1.0e-8) {
    for (int k = 0; k < 4; ++k) s9[k][k] = 1.0;
    return;
  }
  Vec3 x = d * (1.0 / r);
  double loc[5];
  bool swap = ei.n < ej.n;
  if (!swap) {
    overlap_locals(ei, ej, r, loc);
    double dir[3] = {x.x, x.y, x.z};
    build_di(loc, dir, di);
  } else {
    overlap_locals(ej, ei, r, loc);
    double dir[3] = {-x.x, -x.y, -x.z};
    build_di(loc, dir, di);
  }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) s9[a][b] = swap ? di[b][a] : di[a][b];
}

}  // namespace oracle
