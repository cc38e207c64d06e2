// Oracle (test infrastructure): MNDO/d two-centre integrals, general Slater overlaps
// and the numerical Slater overlaps of n >= 4 shells. Restates pm7-rs
// src/mndod_twocenter.rs, src/mndod.rs::charg, src/overlap_d.rs and
// src/overlap_numeric.rs (f64 instantiation). Arrays keep MOPAC's 1-based slots.
#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle_internal.hpp"
#include "pm7_param_data.h"

namespace oracle {
namespace {

// Charge-distribution class of the 45 local pairs (MOPAC met), 1-based.
const int MET[46] = {0, 1, 2, 3, 2, 3, 3, 2, 3, 3, 3, 4, 5, 5, 5, 6, 4, 5, 5, 5, 6, 6, 4,
                     5, 5, 5, 6, 6, 6, 4, 5, 5, 5, 6, 6, 6, 6, 4, 5, 5, 5, 6, 6, 6, 6, 6};
// rep(1..34) = ri(IPOS) (MOPAC reppd2), 1-based.
const int IPOS[35] = {0,  1,  5,  11, 12, 12, 2,  6,  13, 14, 14, 3,  8,  16, 18, 18, 7, 15,
                      10, 20, 4,  9,  17, 19, 21, 7,  15, 10, 20, 22, 4,  9,  17, 21, 19};
// Sign convention on the 22 sp local integrals (MOPAC nri), 1-based.
const double NRI[23] = {0.0, 1.0,  -1.0, 1.0,  1.0,  -1.0, 1.0, 1.0, -1.0, -1.0, -1.0, 1.0,
                        1.0, -1.0, -1.0, -1.0, 1.0,  1.0,  1.0, 1.0, 1.0,  1.0,  1.0};

int indexd(int i, int j) {  // MOPAC indexd, 1-based
  if (i < j) std::swap(i, j);
  return (i + 9 * (j - 1)) - (j * (j - 1)) / 2;
}
int indx(int i, int j) {  // MOPAC indx, 1-based lower-triangle
  if (i < j) std::swap(i, j);
  return (i * (i - 1)) / 2 + j;
}
double chv(int i, int l, int m) { return MNDOD_CH[((i - 1) * 3 + l) * 5 + (m + 2)]; }
double po(const Element &e, int i) { return e.dshell.po[i]; }
double ddp(const Element &e, int i) { return e.dshell.ddp[i]; }

// Rotation tensors of MOPAC rotmat (src/mndod_twocenter.rs:75-230), 1-based.
struct Rot {
  double sp[4][4] = {{0}};
  double pp[7][4][4] = {{{0}}};
  double sd[6][6] = {{0}};
  double dp[16][6][4] = {{{0}}};
  double dd[16][6][6] = {{{0}}};
};

double rotmat(const double v[3], bool has_d, Rot &R) {
  const double SMALL = 1.0e-7, PT5SQ3 = 0.8660254037841;
  double x11 = v[0], x22 = v[1], x33 = v[2];
  double b = x11 * x11 + x22 * x22;
  double r = std::sqrt(b + x33 * x33);
  double sqb = std::sqrt(b);
  double sb = sqb * (1.0 / r);
  double ca, sa, cb;
  if (sb > SMALL) {
    ca = x11 * (1.0 / sqb);
    sa = x22 * (1.0 / sqb);
    cb = x33 * (1.0 / r);
  } else {
    sa = 0.0;
    sb = 0.0;
    if (x33 < 0.0) {
      ca = -1.0;
      cb = -1.0;
    } else if (x33 > 0.0) {
      ca = 1.0;
      cb = 1.0;
    } else {
      ca = 0.0;
      cb = 0.0;
    }
  }
  double p[4][4] = {{0}};
  p[1][1] = ca * sb;
  p[2][1] = ca * cb;
  p[3][1] = -sa;
  p[1][2] = sa * sb;
  p[2][2] = sa * cb;
  p[3][2] = ca;
  p[1][3] = cb;
  p[2][3] = -sb;
  p[3][3] = 0.0;
  double d[6][6] = {{0}};
  if (has_d) {
    double c2a = ca * ca * 2.0 - 1.0, c2b = cb * cb * 2.0 - 1.0, s2a = sa * ca * 2.0, s2b = sb * cb * 2.0;
    d[1][1] = c2a * sb * sb * PT5SQ3;
    d[2][1] = c2a * s2b * 0.5;
    d[3][1] = -(s2a * sb);
    d[4][1] = c2a * (cb * cb + sb * sb * 0.5);
    d[5][1] = -(s2a * cb);
    d[1][2] = ca * s2b * PT5SQ3;
    d[2][2] = ca * c2b;
    d[3][2] = -(sa * cb);
    d[4][2] = ca * s2b * (-0.5);
    d[5][2] = sa * sb;
    d[1][3] = cb * cb - sb * sb * 0.5;
    d[2][3] = -(s2b * PT5SQ3);
    d[3][3] = 0.0;
    d[4][3] = sb * sb * PT5SQ3;
    d[5][3] = 0.0;
    d[1][4] = sa * s2b * PT5SQ3;
    d[2][4] = sa * c2b;
    d[3][4] = ca * cb;
    d[4][4] = sa * s2b * (-0.5);
    d[5][4] = -(ca * sb);
    d[1][5] = s2a * sb * sb * PT5SQ3;
    d[2][5] = s2a * s2b * 0.5;
    d[3][5] = c2a * sb;
    d[4][5] = s2a * (cb * cb + sb * sb * 0.5);
    d[5][5] = c2a * cb;
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) R.sp[i][j] = p[i][j];
  for (int k = 1; k <= 3; ++k) {
    R.pp[1][k][k] = p[k][1] * p[k][1];
    R.pp[2][k][k] = p[k][2] * p[k][2];
    R.pp[3][k][k] = p[k][3] * p[k][3];
    R.pp[4][k][k] = p[k][1] * p[k][2];
    R.pp[5][k][k] = p[k][1] * p[k][3];
    R.pp[6][k][k] = p[k][2] * p[k][3];
    for (int j = 1; j < k; ++j) {
      R.pp[1][k][j] = p[k][1] * p[j][1] * 2.0;
      R.pp[2][k][j] = p[k][2] * p[j][2] * 2.0;
      R.pp[3][k][j] = p[k][3] * p[j][3] * 2.0;
      R.pp[4][k][j] = p[k][1] * p[j][2] + p[k][2] * p[j][1];
      R.pp[5][k][j] = p[k][1] * p[j][3] + p[k][3] * p[j][1];
      R.pp[6][k][j] = p[k][2] * p[j][3] + p[k][3] * p[j][2];
    }
  }
  if (has_d) {
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) R.sd[i][j] = d[i][j];
    for (int k = 1; k <= 5; ++k)
      for (int col = 1; col <= 3; ++col) {
        for (int a = 1; a <= 5; ++a)
          for (int bb = 1; bb <= 3; ++bb) {
            // dp[3(a-1)+bb][k][col] = d[k][a] * p[col][bb]
            R.dp[3 * (a - 1) + bb][k][col] = d[k][a] * p[col][bb];
          }
      }
    for (int k = 1; k <= 5; ++k) {
      for (int a = 1; a <= 5; ++a) R.dd[a][k][k] = d[k][a] * d[k][a];
      R.dd[6][k][k] = d[k][1] * d[k][2];
      R.dd[7][k][k] = d[k][1] * d[k][3];
      R.dd[8][k][k] = d[k][2] * d[k][3];
      R.dd[9][k][k] = d[k][1] * d[k][4];
      R.dd[10][k][k] = d[k][2] * d[k][4];
      R.dd[11][k][k] = d[k][3] * d[k][4];
      R.dd[12][k][k] = d[k][1] * d[k][5];
      R.dd[13][k][k] = d[k][2] * d[k][5];
      R.dd[14][k][k] = d[k][3] * d[k][5];
      R.dd[15][k][k] = d[k][4] * d[k][5];
      for (int j = 1; j < k; ++j) {
        for (int a = 1; a <= 5; ++a) R.dd[a][k][j] = d[k][a] * d[j][a] * 2.0;
        R.dd[6][k][j] = d[k][1] * d[j][2] + d[k][2] * d[j][1];
        R.dd[7][k][j] = d[k][1] * d[j][3] + d[k][3] * d[j][1];
        R.dd[8][k][j] = d[k][2] * d[j][3] + d[k][3] * d[j][2];
        R.dd[9][k][j] = d[k][1] * d[j][4] + d[k][4] * d[j][1];
        R.dd[10][k][j] = d[k][2] * d[j][4] + d[k][4] * d[j][2];
        R.dd[11][k][j] = d[k][3] * d[j][4] + d[k][4] * d[j][3];
        R.dd[12][k][j] = d[k][1] * d[j][5] + d[k][5] * d[j][1];
        R.dd[13][k][j] = d[k][2] * d[j][5] + d[k][5] * d[j][2];
        R.dd[14][k][j] = d[k][3] * d[j][5] + d[k][5] * d[j][3];
        R.dd[15][k][j] = d[k][4] * d[j][5] + d[k][5] * d[j][4];
      }
    }
  }
  return r;
}

// MOPAC charg, src/mndod.rs:30-187.
double charg(double r, int l1, int l2, int m, double da, double db, double add) {
  auto inv = [add](double x) { return 1.0 / std::sqrt(x * x + add); };
  auto q = [](double x) { return 1.0 / std::sqrt(x); };
  if (l1 == 0 && l2 == 0) return 1.0 / std::sqrt(r * r + add);
  if (l1 == 1 && l2 == 0) return (inv(r - da) - inv(r + da)) * 0.5;
  if (l1 == 0 && l2 == 1) return (inv(r + db) - inv(r - db)) * 0.5;
  if (l1 == 1 && l2 == 1 && m == 0)
    return (inv(r + da - db) + inv(r - da + db) - inv(r - da - db) - inv(r + da + db)) * 0.25;
  if (l1 == 1 && l2 == 1)
    return (q(r * r + (da - db) * (da - db) + add) - q(r * r + (da + db) * (da + db) + add)) * 0.5;
  if (l1 == 0 && l2 == 2) return (inv(r - db) - q(r * r + (db * db + add)) * 2.0 + inv(r + db)) * 0.25;
  if (l1 == 2 && l2 == 0) return (inv(r - da) - q(r * r + (da * da + add)) * 2.0 + inv(r + da)) * 0.25;
  if (l1 == 1 && l2 == 2 && m == 0)
    return (inv(r - da - db) - q((r - da) * (r - da) + (db * db + add)) * 2.0 + inv(r + db - da) - inv(r - db + da) +
            q((r + da) * (r + da) + (db * db + add)) * 2.0 - inv(r + da + db)) *
           0.125;
  if (l1 == 2 && l2 == 1 && m == 0)
    return (-inv(r - da - db) + q((r - db) * (r - db) + (da * da + add)) * 2.0 - inv(r + da - db) + inv(r - da + db) -
            q((r + db) * (r + db) + (da * da + add)) * 2.0 + inv(r + da + db)) *
           0.125;
  if (l1 == 2 && l2 == 2 && m == 0) {
    double zzzz = inv(r - da - db) + inv(r + da + db) + inv(r - da + db) + inv(r + da - db) -
                  q((r - da) * (r - da) + (db * db + add)) * 2.0 - q((r - db) * (r - db) + (da * da + add)) * 2.0 -
                  q((r + da) * (r + da) + (db * db + add)) * 2.0 - q((r + db) * (r + db) + (da * da + add)) * 2.0 +
                  q(r * r + ((da - db) * (da - db) + add)) * 2.0 + q(r * r + ((da + db) * (da + db) + add)) * 2.0;
    double xyxy = q(r * r + ((da - db) * (da - db) + add)) * 4.0 + q(r * r + ((da + db) * (da + db) + add)) * 4.0 -
                  q(r * r + (da * da + db * db + add)) * 8.0;
    return zzzz * (1.0 / 16.0) - xyxy * (1.0 / 64.0);
  }
  if (l1 == 1 && l2 == 2) {
    double ab = db / std::sqrt(2.0);
    return (q((r - ab) * (r - ab) + ((da - ab) * (da - ab) + add)) * (-2.0) +
            q((r + ab) * (r + ab) + ((da - ab) * (da - ab) + add)) * 2.0 +
            q((r - ab) * (r - ab) + ((da + ab) * (da + ab) + add)) * 2.0 -
            q((r + ab) * (r + ab) + ((da + ab) * (da + ab) + add)) * 2.0) *
           0.125;
  }
  if (l1 == 2 && l2 == 1) {
    double aa = da / std::sqrt(2.0);
    return (q((r + aa) * (r + aa) + ((aa - db) * (aa - db) + add)) * (-2.0) +
            q((r - aa) * (r - aa) + ((aa - db) * (aa - db) + add)) * 2.0 +
            q((r + aa) * (r + aa) + ((aa + db) * (aa + db) + add)) * 2.0 -
            q((r - aa) * (r - aa) + ((aa + db) * (aa + db) + add)) * 2.0) *
           0.125;
  }
  if (l1 == 2 && l2 == 2 && m == 1) {
    double aa = da / std::sqrt(2.0), ab = db / std::sqrt(2.0);
    double m1 = (aa - ab) * (aa - ab) + add, p1 = (aa + ab) * (aa + ab) + add;
    return (q((r + aa - ab) * (r + aa - ab) + m1) * 2.0 - q((r + aa + ab) * (r + aa + ab) + m1) * 2.0 -
            q((r - aa - ab) * (r - aa - ab) + m1) * 2.0 + q((r - aa + ab) * (r - aa + ab) + m1) * 2.0 -
            q((r + aa - ab) * (r + aa - ab) + p1) * 2.0 + q((r + aa + ab) * (r + aa + ab) + p1) * 2.0 +
            q((r - aa - ab) * (r - aa - ab) + p1) * 2.0 - q((r - aa + ab) * (r - aa + ab) + p1) * 2.0) *
           (1.0 / 16.0);
  }
  if (l1 == 2 && l2 == 2) {
    double xyxy = q(r * r + ((da - db) * (da - db) + add)) * 4.0 + q(r * r + ((da + db) * (da + db) + add)) * 4.0 -
                  q(r * r + (da * da + db * db + add)) * 8.0;
    return xyxy * (1.0 / 16.0);
  }
  return 0.0;
}

// MOPAC reppd: 22 sp local integrals with the po additive terms (mndod_twocenter.rs:244-482).
void reppd(const Element &ei, const Element &ej, double r, double ri[23]) {
  const double ev = EV, ev1 = ev / 2.0, ev2 = ev1 / 2.0, ev3 = ev2 / 2.0, ev4 = ev3 / 2.0;
  for (int k = 0; k < 23; ++k) ri[k] = 0.0;
  bool si = ei.n_orb >= 4, sj = ej.n_orb >= 4;
  auto sq = [](double x, double off) { return 1.0 / std::sqrt(x * x + off); };
  auto sqp = [](double a, double b) { return (a + b) * (a + b); };
  double aee = sqp(po(ei, 1), po(ej, 1));
  if (!si && !sj) {
    ri[1] = sq(r, aee) * ev;
  } else if (si && !sj) {
    double da = ei.dd, qa = ei.qq * 2.0;
    double ade = sqp(po(ei, 2), po(ej, 1)), aqe = sqp(po(ei, 3), po(ej, 1));
    double ee = sq(r, aee) * ev;
    ri[1] = ee;
    ri[2] = sq(r + da, ade) * ev1 - sq(r - da, ade) * ev1;
    ri[3] = ee + sq(r + qa, aqe) * ev2 + sq(r - qa, aqe) * ev2 - sq(r, aqe) * ev1;
    ri[4] = ee + (1.0 / std::sqrt(r * r + (qa * qa + aqe))) * ev1 - sq(r, aqe) * ev1;
  } else if (!si && sj) {
    double db = ej.dd, qb = ej.qq * 2.0;
    double aed = sqp(po(ei, 1), po(ej, 2)), aeq = sqp(po(ei, 1), po(ej, 3));
    double ee = sq(r, aee) * ev;
    ri[1] = ee;
    ri[5] = sq(r - db, aed) * ev1 - sq(r + db, aed) * ev1;
    ri[11] = ee + sq(r - qb, aeq) * ev2 + sq(r + qb, aeq) * ev2 - sq(r, aeq) * ev1;
    ri[12] = ee + (1.0 / std::sqrt(r * r + (qb * qb + aeq))) * ev1 - sq(r, aeq) * ev1;
  } else {
    double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0;
    double ade = sqp(po(ei, 2), po(ej, 1)), aqe = sqp(po(ei, 3), po(ej, 1)), aed = sqp(po(ei, 1), po(ej, 2)),
           aeq = sqp(po(ei, 1), po(ej, 3)), axx = sqp(po(ei, 2), po(ej, 2)), adq = sqp(po(ei, 2), po(ej, 3)),
           aqd = sqp(po(ei, 3), po(ej, 2)), aqq = sqp(po(ei, 3), po(ej, 3));
    auto g = [](double x, double off) { return 1.0 / std::sqrt(x * x + off); };
    auto q = [](double x) { return 1.0 / std::sqrt(x); };
    double ee = g(r, aee) * ev;
    double dze = -(sq(r + da, ade)) * ev1 + sq(r - da, ade) * ev1;
    double qzze = sq(r - qa, aqe) * ev2 + sq(r + qa, aqe) * ev2 - g(r, aqe) * ev1;
    double qxxe = q(r * r + (qa * qa + aqe)) * ev1 - g(r, aqe) * ev1;
    double edz = -(sq(r - db, aed)) * ev1 + sq(r + db, aed) * ev1;
    double eqzz = sq(r - qb, aeq) * ev2 + sq(r + qb, aeq) * ev2 - g(r, aeq) * ev1;
    double eqxx = q(r * r + (qb * qb + aeq)) * ev1 - g(r, aeq) * ev1;
    double dxdx = q(r * r + ((da - db) * (da - db) + axx)) * ev1 - q(r * r + ((da + db) * (da + db) + axx)) * ev1;
    double dzdz = sq(r + da - db, axx) * ev2 + sq(r - da + db, axx) * ev2 - sq(r - da - db, axx) * ev2 -
                  sq(r + da + db, axx) * ev2;
    double qa1 = ei.qq, qb1 = ej.qq;
    double dzqxx = sq(r + da, adq) * ev2 - q((r + da) * (r + da) + (qb * qb + adq)) * ev2 - sq(r - da, adq) * ev2 +
                   q((r - da) * (r - da) + (qb * qb + adq)) * ev2;
    double qxxdz = sq(r - db, aqd) * ev2 - q((r - db) * (r - db) + (qa * qa + aqd)) * ev2 - sq(r + db, aqd) * ev2 +
                   q((r + db) * (r + db) + (qa * qa + aqd)) * ev2;
    double dzqzz = -(sq(r + da - qb, adq)) * ev3 + sq(r - da - qb, adq) * ev3 - sq(r + da + qb, adq) * ev3 +
                   sq(r - da + qb, adq) * ev3 - sq(r - da, adq) * ev2 + sq(r + da, adq) * ev2;
    double qzzdz = -(sq(r + qa - db, aqd)) * ev3 + sq(r + qa + db, aqd) * ev3 - sq(r - qa - db, aqd) * ev3 +
                   sq(r - qa + db, aqd) * ev3 + sq(r - db, aqd) * ev2 - sq(r + db, aqd) * ev2;
    double qxxqxx = q(r * r + ((qa - qb) * (qa - qb) + aqq)) * ev3 + q(r * r + ((qa + qb) * (qa + qb) + aqq)) * ev3 -
                    q(r * r + (qa * qa + aqq)) * ev2 - q(r * r + (qb * qb + aqq)) * ev2 + g(r, aqq) * ev2;
    double qxxqyy = q(r * r + (qa * qa + qb * qb + aqq)) * ev2 - q(r * r + (qa * qa + aqq)) * ev2 -
                    q(r * r + (qb * qb + aqq)) * ev2 + g(r, aqq) * ev2;
    double qxxqzz = q((r - qb) * (r - qb) + (qa * qa + aqq)) * ev3 + q((r + qb) * (r + qb) + (qa * qa + aqq)) * ev3 -
                    sq(r - qb, aqq) * ev3 - sq(r + qb, aqq) * ev3 - q(r * r + (qa * qa + aqq)) * ev2 + g(r, aqq) * ev2;
    double qzzqxx = q((r + qa) * (r + qa) + (qb * qb + aqq)) * ev3 + q((r - qa) * (r - qa) + (qb * qb + aqq)) * ev3 -
                    sq(r + qa, aqq) * ev3 - sq(r - qa, aqq) * ev3 - q(r * r + (qb * qb + aqq)) * ev2 + g(r, aqq) * ev2;
    double qzzqzz = sq(r + qa - qb, aqq) * ev4 + sq(r + qa + qb, aqq) * ev4 + sq(r - qa - qb, aqq) * ev4 +
                    sq(r - qa + qb, aqq) * ev4 - sq(r - qa, aqq) * ev3 - sq(r + qa, aqq) * ev3 - sq(r - qb, aqq) * ev3 -
                    sq(r + qb, aqq) * ev3 + g(r, aqq) * ev2;
    double dxqxz = -q((r - qb1) * (r - qb1) + ((da - qb1) * (da - qb1) + adq)) * ev2 +
                   q((r + qb1) * (r + qb1) + ((da - qb1) * (da - qb1) + adq)) * ev2 +
                   q((r - qb1) * (r - qb1) + ((da + qb1) * (da + qb1) + adq)) * ev2 -
                   q((r + qb1) * (r + qb1) + ((da + qb1) * (da + qb1) + adq)) * ev2;
    double qxzdx = -q((r + qa1) * (r + qa1) + ((qa1 - db) * (qa1 - db) + aqd)) * ev2 +
                   q((r - qa1) * (r - qa1) + ((qa1 - db) * (qa1 - db) + aqd)) * ev2 +
                   q((r + qa1) * (r + qa1) + ((qa1 + db) * (qa1 + db) + aqd)) * ev2 -
                   q((r - qa1) * (r - qa1) + ((qa1 + db) * (qa1 + db) + aqd)) * ev2;
    double m1 = (qa1 - qb1) * (qa1 - qb1) + aqq, p1 = (qa1 + qb1) * (qa1 + qb1) + aqq;
    double qxzqxz = q((r + qa1 - qb1) * (r + qa1 - qb1) + m1) * ev3 - q((r + qa1 + qb1) * (r + qa1 + qb1) + m1) * ev3 -
                    q((r - qa1 - qb1) * (r - qa1 - qb1) + m1) * ev3 + q((r - qa1 + qb1) * (r - qa1 + qb1) + m1) * ev3 -
                    q((r + qa1 - qb1) * (r + qa1 - qb1) + p1) * ev3 + q((r + qa1 + qb1) * (r + qa1 + qb1) + p1) * ev3 +
                    q((r - qa1 - qb1) * (r - qa1 - qb1) + p1) * ev3 - q((r - qa1 + qb1) * (r - qa1 + qb1) + p1) * ev3;
    ri[1] = ee;
    ri[2] = -dze;
    ri[3] = ee + qzze;
    ri[4] = ee + qxxe;
    ri[5] = -edz;
    ri[6] = dzdz;
    ri[7] = dxdx;
    ri[8] = -edz - qzzdz;
    ri[9] = -edz - qxxdz;
    ri[10] = -qxzdx;
    ri[11] = ee + eqzz;
    ri[12] = ee + eqxx;
    ri[13] = -dze - dzqzz;
    ri[14] = -dze - dzqxx;
    ri[15] = -dxqxz;
    ri[16] = ee + eqzz + qzze + qzzqzz;
    ri[17] = ee + eqzz + qxxe + qxxqzz;
    ri[18] = ee + eqxx + qzze + qzzqxx;
    ri[19] = ee + eqxx + qxxe + qxxqxx;
    ri[20] = qxzqxz;
    ri[21] = ee + eqxx + qxxe + qxxqyy;
    ri[22] = (qxxqxx - qxxqyy) * 0.5;
  }
  for (int k = 1; k <= 22; ++k) ri[k] = ri[k] * NRI[k];
  double cfrac, point;
  feather_to_point(r, cfrac, point);
  double add = point * (1.0 - cfrac);
  for (int k = 1; k <= 22; ++k) ri[k] *= cfrac;
  for (int k : {1, 3, 4, 11, 12, 16, 17, 18, 19, 21}) ri[k] += add;
}

// MOPAC spcore (mndod_twocenter.rs:492-572): core[1..4][1..2].
void spcore(const Element &ei, const Element &ej, double r, double core[11][3]) {
  const double ev = EV;
  const double pxy[8] = {0.0, 1.0, -0.5, -0.5, 0.5, 0.25, 0.25, 0.5};
  for (int i = 0; i < 11; ++i) core[i][0] = core[i][1] = core[i][2] = 0.0;
  double r2 = r * r, aci = po(ei, 9), acj = po(ej, 9);
  double ssj = (acj + po(ei, 1)) * (acj + po(ei, 1)), ssi = (aci + po(ej, 1)) * (aci + po(ej, 1));
  core[1][1] = -(1.0 / std::sqrt(r2 + ssj)) * (ej.core_charge * ev);
  core[1][2] = -(1.0 / std::sqrt(r2 + ssi)) * (ei.core_charge * ev);
  if (ei.n_orb >= 4 || ej.n_orb >= 4) {
    if (ei.n_orb >= 4) {
      double ppj = (acj + po(ei, 7)) * (acj + po(ei, 7));
      double da = ddp(ei, 2), qa = ddp(ei, 3) / std::sqrt(2.0), tq = qa + qa;
      double adj = (po(ei, 2) + acj) * (po(ei, 2) + acj), aqj = (po(ei, 3) + acj) * (po(ei, 3) + acj);
      double x1 = (1.0 / std::sqrt(r2 + ppj)) * pxy[1], x2 = (1.0 / std::sqrt(r2 + aqj)) * pxy[2];
      double x3 = (1.0 / std::sqrt((r + da) * (r + da) + adj)) * pxy[3];
      double x4 = (1.0 / std::sqrt((r - da) * (r - da) + adj)) * pxy[4];
      double x5 = (1.0 / std::sqrt((r - tq) * (r - tq) + aqj)) * pxy[5];
      double x6 = (1.0 / std::sqrt((r + tq) * (r + tq) + aqj)) * pxy[6];
      double x7 = (1.0 / std::sqrt(r2 + (tq * tq + aqj))) * pxy[7];
      core[2][1] = -((x3 + x4) * ev) * ej.core_charge;
      core[3][1] = -((x1 + x2 + x5 + x6) * ev) * ej.core_charge;
      core[4][1] = -((x1 + x2 + x7) * ev) * ej.core_charge;
    }
    if (ej.n_orb >= 4) {
      double ppi = (aci + po(ej, 7)) * (aci + po(ej, 7));
      double db = ddp(ej, 2), qb = ddp(ej, 3) / std::sqrt(2.0), tq = qb + qb;
      double adi = (po(ej, 2) + aci) * (po(ej, 2) + aci), aqi = (po(ej, 3) + aci) * (po(ej, 3) + aci);
      double x1 = (1.0 / std::sqrt(r2 + ppi)) * pxy[1], x2 = (1.0 / std::sqrt(r2 + aqi)) * pxy[2];
      double x3 = (1.0 / std::sqrt((r + db) * (r + db) + adi)) * pxy[3];
      double x4 = (1.0 / std::sqrt((r - db) * (r - db) + adi)) * pxy[4];
      double x5 = (1.0 / std::sqrt((r - tq) * (r - tq) + aqi)) * pxy[5];
      double x6 = (1.0 / std::sqrt((r + tq) * (r + tq) + aqi)) * pxy[6];
      double x7 = (1.0 / std::sqrt(r2 + (tq * tq + aqi))) * pxy[7];
      double ai2 = -(x3 + x4) * ev;
      core[2][2] = -(ai2)*ei.core_charge;
      core[3][2] = -((x1 + x2 + x5 + x6) * ev) * ei.core_charge;
      core[4][2] = -((x1 + x2 + x7) * ev) * ei.core_charge;
    }
  }
}

// MOPAC rijkl (mndod_twocenter.rs:583-655).
double rijkl(const Element &ei, const Element &ej, int ij, int kl, int li, int lj, int lk, int ll, int ic, double r) {
  int lij = indx(li + 1, lj + 1), lkl = indx(lk + 1, ll + 1);
  int l1min = std::min(std::abs(li - lj), 2), l1max = std::min(li + lj, 2);
  int l2min = std::min(std::abs(lk - ll), 2), l2max = std::min(lk + ll, 2);
  double sum = 0.0;
  for (int l1 = l1min; l1 <= l1max; ++l1) {
    double dij, pij;
    if (l1 == 0) {
      dij = 0.0;
      pij = lij == 1 ? (ic == 1 ? po(ei, 9) : po(ei, 1)) : lij == 3 ? po(ei, 7) : lij == 6 ? po(ei, 8) : po(ei, 1);
    } else {
      dij = ddp(ei, lij);
      pij = po(ei, lij);
    }
    for (int l2 = l2min; l2 <= l2max; ++l2) {
      double dkl, pkl;
      if (l2 == 0) {
        dkl = 0.0;
        pkl = lkl == 1 ? (ic == 2 ? po(ej, 9) : po(ej, 1)) : lkl == 3 ? po(ej, 7) : lkl == 6 ? po(ej, 8) : po(ej, 1);
      } else {
        dkl = ddp(ej, lkl);
        pkl = po(ej, lkl);
      }
      double add = (pij + pkl) * (pij + pkl);
      int lmin = std::min(l1, l2);
      for (int m = -lmin; m <= lmin; ++m) {
        double ccc = chv(ij, l1, m) * chv(kl, l2, m);
        if (ccc == 0.0) continue;
        sum = sum + charg(r, l1, l2, std::abs(m), dij, dkl, add) * ccc;
      }
    }
  }
  return sum;
}

// MOPAC reppd2 (mndod_twocenter.rs:658-751): rep[1..491] and the d core terms.
void reppd2(const Element &ei, const Element &ej, double r, const double ri[23], double core[11][3],
            std::vector<double> &rep) {
  const double ev = EV;
  bool di = ei.n_orb == 9, dj = ej.n_orb == 9;
  const int lorb[10] = {0, 0, 1, 1, 1, 2, 2, 2, 2, 2};
  rep.assign(492, 0.0);
  for (int k = 1; k <= 34; ++k) rep[k] = ri[IPOS[k]];
  if (!(di || dj)) return;
  double cfrac, point;
  feather_to_point(r, cfrac, point);
  double point_add = point * (1.0 - cfrac);
  int lasti = di ? 9 : (ei.n_orb == 1 ? 1 : 4), lastk = dj ? 9 : (ej.n_orb == 1 ? 1 : 4);
  for (int i = 1; i <= lasti; ++i)
    for (int j = 1; j <= i; ++j) {
      int ij = indexd(i, j);
      for (int k = 1; k <= lastk; ++k)
        for (int l = 1; l <= k; ++l) {
          int kl = indexd(k, l);
          int numb = MNDOD_IND2[(ij - 1) * 45 + (kl - 1)];
          if (numb <= 34) continue;
          int nold = MNDOD_ISYM[numb];
          if (nold >= 35) rep[numb] = rep[nold];
          else if (nold <= -35) rep[numb] = -rep[-nold];
          else if (nold == 0) {
            double v = rijkl(ei, ej, ij, kl, lorb[i], lorb[j], lorb[k], lorb[l], 0, r) * ev;
            rep[numb] = (i == j && k == l) ? v * cfrac + point_add : v * cfrac;
          }
        }
    }
  for (int n = 5; n <= 10; ++n) core[n][1] = core[n][2] = 0.0;
  if (dj) {
    double t = ei.core_charge;
    core[5][2] = -rijkl(ei, ej, 1, indexd(5, 1), 0, 0, 2, 0, 1, r) * (ev * t);
    core[6][2] = -rijkl(ei, ej, 1, indexd(5, 2), 0, 0, 2, 1, 1, r) * (ev * t);
    core[7][2] = -rijkl(ei, ej, 1, indexd(5, 5), 0, 0, 2, 2, 1, r) * (ev * t);
    core[8][2] = -rijkl(ei, ej, 1, indexd(6, 3), 0, 0, 2, 1, 1, r) * (ev * t);
    core[9][2] = -rijkl(ei, ej, 1, indexd(6, 6), 0, 0, 2, 2, 1, r) * (ev * t);
    core[10][2] = -rijkl(ei, ej, 1, indexd(8, 8), 0, 0, 2, 2, 1, r) * (ev * t);
  }
  if (di) {
    double t = ej.core_charge;
    core[5][1] = -rijkl(ei, ej, indexd(5, 1), 1, 2, 0, 0, 0, 2, r) * (ev * t);
    core[6][1] = -rijkl(ei, ej, indexd(5, 2), 1, 2, 1, 0, 0, 2, r) * (ev * t);
    core[7][1] = -rijkl(ei, ej, indexd(5, 5), 1, 2, 2, 0, 0, 2, r) * (ev * t);
    core[8][1] = -rijkl(ei, ej, indexd(6, 3), 1, 2, 1, 0, 0, 2, r) * (ev * t);
    core[9][1] = -rijkl(ei, ej, indexd(6, 6), 1, 2, 2, 0, 0, 2, r) * (ev * t);
    core[10][1] = -rijkl(ei, ej, indexd(8, 8), 1, 2, 2, 0, 0, 2, r) * (ev * t);
  }
}

// MOPAC tx (mndod_twocenter.rs:754-834): first rotation step, v[ij][1..limkl].
void tx(int ii, int kk, const std::vector<double> &rep, const Rot &R, std::vector<std::vector<double>> &v) {
  int limkl = indx(kk, kk);
  v.assign(46, std::vector<double>(limkl + 1, 0.0));
  static const int cols5[15] = {12, 13, 14, 17, 18, 19, 23, 24, 25, 30, 31, 32, 38, 39, 40};
  static const int diag6[5][2] = {{15, 1}, {21, 2}, {28, 3}, {36, 4}, {45, 5}};
  static const int offd6[10][2] = {{20, 6},  {26, 7},  {27, 8},  {33, 9},  {34, 10},
                                   {35, 11}, {41, 12}, {42, 13}, {43, 14}, {44, 15}};
  for (int i1 = 1; i1 <= ii; ++i1)
    for (int j1 = 1; j1 <= i1; ++j1) {
      int ij = indexd(i1, j1);
      for (int k1 = 1; k1 <= kk; ++k1)
        for (int l1 = 1; l1 <= k1; ++l1) {
          int kl = indexd(k1, l1);
          int nd = MNDOD_IND2[(ij - 1) * 45 + (kl - 1)];
          if (nd == 0) continue;
          double w = rep[nd];
          int ll = indx(k1, l1);
          switch (MET[ll]) {
            case 1: v[ij][1] = w; break;
            case 2: {
              int k = k1 - 1;
              v[ij][2] += R.sp[k][1] * w;
              v[ij][4] += R.sp[k][2] * w;
              v[ij][7] += R.sp[k][3] * w;
              break;
            }
            case 3: {
              int k = k1 - 1, l = l1 - 1;
              v[ij][3] += R.pp[1][k][l] * w;
              v[ij][6] += R.pp[2][k][l] * w;
              v[ij][10] += R.pp[3][k][l] * w;
              v[ij][5] += R.pp[4][k][l] * w;
              v[ij][8] += R.pp[5][k][l] * w;
              v[ij][9] += R.pp[6][k][l] * w;
              break;
            }
            case 4: {
              int k = k1 - 4;
              v[ij][11] += R.sd[k][1] * w;
              v[ij][16] += R.sd[k][2] * w;
              v[ij][22] += R.sd[k][3] * w;
              v[ij][29] += R.sd[k][4] * w;
              v[ij][37] += R.sd[k][5] * w;
              break;
            }
            case 5: {
              int k = k1 - 4, l = l1 - 1;
              for (int t = 0; t < 15; ++t) v[ij][cols5[t]] += R.dp[t + 1][k][l] * w;
              break;
            }
            case 6: {
              int k = k1 - 4, l = l1 - 4;
              for (auto &c : diag6) v[ij][c[0]] += R.dd[c[1]][k][l] * w;
              for (auto &c : offd6) v[ij][c[0]] += R.dd[c[1]][k][l] * w;
              break;
            }
            default: break;
          }
        }
    }
}

// MOPAC rotatd second step (mndod_twocenter.rs:838-915): ww[1..limij*limkl].
void rotate_left(int ii, int kk, const std::vector<std::vector<double>> &v, const Rot &R, std::vector<double> &ww) {
  int limij = indx(ii, ii), limkl = indx(kk, kk);
  ww.assign((size_t)limij * limkl + 1, 0.0);
  auto indw = [limkl](int i, int j, int kl) { return (indx(i, j) - 1) * limkl + kl; };
  for (int i1 = 1; i1 <= ii; ++i1)
    for (int j1 = 1; j1 <= i1; ++j1) {
      int ij = indexd(i1, j1), jj = indx(i1, j1), mm = MET[jj];
      for (int k = 1; k <= kk; ++k)
        for (int l = 1; l <= k; ++l) {
          int kl = indx(k, l);
          double w = v[ij][kl];
          switch (mm) {
            case 1: ww[indw(1, 1, kl)] = w; break;
            case 2:
              for (int i = 1; i <= 3; ++i) ww[indw(i + 1, 1, kl)] += R.sp[i1 - 1][i] * w;
              break;
            case 3:
              for (int i = 1; i <= 3; ++i) {
                ww[indw(i + 1, i + 1, kl)] += R.pp[i][i1 - 1][j1 - 1] * w;
                for (int j = 1; j < i; ++j) ww[indw(i + 1, j + 1, kl)] += R.pp[1 + i + j][i1 - 1][j1 - 1] * w;
              }
              break;
            case 4:
              for (int i = 1; i <= 5; ++i) ww[indw(i + 4, 1, kl)] += R.sd[i1 - 4][i] * w;
              break;
            case 5:
              for (int i = 1; i <= 5; ++i)
                for (int j = 1; j <= 3; ++j) ww[indw(i + 4, j + 1, kl)] += R.dp[3 * (i - 1) + j][i1 - 4][j1 - 1] * w;
              break;
            case 6:
              for (int i = 1; i <= 5; ++i) {
                ww[indw(i + 4, i + 4, kl)] += R.dd[i][i1 - 4][j1 - 4] * w;
                for (int j = 1; j < i; ++j)
                  ww[indw(i + 4, j + 4, kl)] += R.dd[MNDOD_INDDD[(i - 1) * 5 + (j - 1)]][i1 - 4][j1 - 4] * w;
              }
              break;
            default: break;
          }
        }
    }
}

// PM7 d-imbalance correction (mndod_twocenter.rs:919-1004).
void pm7_balance(std::vector<double> &ww, double core[11][3], const Element &ei, const Element &ej) {
  int ni = ei.n_orb, nj = ej.n_orb;
  if (ei.iod > 0) {
    int k = nj == 9 ? 45 : (nj == 4 ? 10 : 1);
    if (nj > 1) {
      double sum = 0.0;
      for (int i = 5; i <= 9; ++i) {
        int j = k * ((i * (i + 1)) / 2 - 1);
        sum = sum + ww[j + 3] + ww[j + 6] + ww[j + 10];
      }
      sum = ww[1] - sum * (1.0 / 15.0);
      for (int i = 5; i <= 9; ++i) {
        int j = k * ((i * (i + 1)) / 2 - 1);
        for (int l = 2; l <= 4; ++l) ww[(l * (l + 1)) / 2 + j] += sum;
      }
      double s = core[1][1] - (core[3][1] + core[4][1] * 2.0) * (1.0 / 3.0);
      core[3][1] += s;
      core[4][1] += s;
    }
    double sum = 0.0;
    for (int i = 5; i <= 9; ++i) sum = sum + ww[k * ((i * (i + 1)) / 2 - 1) + 1];
    sum = ww[1] - sum * (1.0 / 5.0);
    for (int i = 5; i <= 9; ++i) ww[k * ((i * (i + 1)) / 2 - 1) + 1] += sum;
    double s = core[1][1] - (core[7][1] + core[9][1] * 2.0 + core[10][1] * 2.0) * (1.0 / 5.0);
    core[7][1] += s;
    core[9][1] += s;
    core[10][1] += s;
  }
  if (ej.iod > 0) {
    if (ei.iod > 0) {
      double sum = 0.0;
      for (int i = 5; i <= 9; ++i) {
        int j = 45 * ((i * (i + 1)) / 2 - 1);
        sum = sum + ww[j + 15] + ww[j + 21] + ww[j + 28] + ww[j + 36] + ww[j + 45];
      }
      sum = ww[1] - sum * (1.0 / 25.0);
      for (int i = 5; i <= 9; ++i) {
        int j = 45 * ((i * (i + 1)) / 2 - 1);
        for (int kk = 5; kk <= 9; ++kk) ww[(kk * (kk + 1)) / 2 + j] += sum;
      }
    }
    if (ni > 1) {
      double sum = 0.0;
      for (int i = 2; i <= 4; ++i) {
        int j = 45 * ((i * (i + 1)) / 2 - 1);
        sum = sum + ww[j + 15] + ww[j + 21] + ww[j + 28] + ww[j + 36] + ww[j + 45];
      }
      sum = ww[1] - sum * (1.0 / 15.0);
      for (int i = 2; i <= 4; ++i) {
        int j = 45 * ((i * (i + 1)) / 2 - 1);
        for (int kk = 5; kk <= 9; ++kk) ww[(kk * (kk + 1)) / 2 + j] += sum;
      }
      double s = core[1][2] - (core[3][2] + core[4][2] * 2.0) * (1.0 / 3.0);
      core[3][2] += s;
      core[4][2] += s;
    }
    double sum = ww[1] - (ww[15] + ww[21] + ww[28] + ww[36] + ww[45]) * (1.0 / 5.0);
    for (int kk = 5; kk <= 9; ++kk) ww[(kk * (kk + 1)) / 2] += sum;
    double s = core[1][2] - (core[7][2] + core[9][2] * 2.0 + core[10][2] * 2.0) * (1.0 / 5.0);
    core[7][2] += s;
    core[9][2] += s;
    core[10][2] += s;
  }
}

// MOPAC elenuc (mndod_twocenter.rs:1008-1047): electron-core block of atom n.
void elenuc_block(const double core[11][3], const Rot &R, int n, int norb, double blk[9][9]) {
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) blk[i][j] = 0.0;
  for (int i = 1; i <= norb; ++i) {
    int ind1 = i - 1;
    for (int j = 1; j <= i; ++j) {
      int ind2 = j - 1;
      double val;
      if (ind1 == 0) val = core[1][n];
      else if (ind1 < 4) {
        if (ind2 == 0) val = R.sp[1][ind1] * core[2][n];
        else {
          int ipp = MNDOD_INDPP[(ind1 - 1) * 3 + (ind2 - 1)];
          val = core[3][n] * R.pp[ipp][1][1] + core[4][n] * (R.pp[ipp][2][2] + R.pp[ipp][3][3]);
        }
      } else if (ind2 == 0) {
        val = R.sd[1][ind1 - 3] * core[5][n];
      } else if (ind2 < 4) {
        int idp = MNDOD_INDDP[(ind1 - 4) * 3 + (ind2 - 1)];
        val = core[6][n] * R.dp[idp][1][1] + core[8][n] * (R.dp[idp][2][2] + R.dp[idp][3][3]);
      } else {
        int idd = MNDOD_INDDD[(ind1 - 4) * 5 + (ind2 - 4)];
        val = core[7][n] * R.dd[idd][1][1] + core[9][n] * (R.dd[idd][2][2] + R.dd[idd][3][3]) +
              core[10][n] * (R.dd[idd][4][4] + R.dd[idd][5][5]);
      }
      blk[i - 1][j - 1] = val;
      blk[j - 1][i - 1] = val;
    }
  }
}

// ---- general Slater overlaps (src/overlap_d.rs) ----------------------------

// Integer power by binary exponentiation: the lowering of Rust's f64::powi.
double powi(double a, int b) {
  bool recip = b < 0;
  double r = 1.0;
  while (true) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

double fact(int n) {
  static double F[25];
  static bool init = false;
  if (!init) {
    F[0] = 1.0;
    for (int i = 1; i < 25; ++i) F[i] = F[i - 1] * i;
    init = true;
  }
  return F[n];
}

void bfn(double x, double bf[13]) {
  double absx = std::fabs(x);
  if (absx > 3.0) {
    double expx = std::exp(x), expmx = 1.0 / expx, inv = 1.0 / x;
    bf[0] = (expx - expmx) * inv;
    for (int i = 1; i <= 12; ++i) {
      double sign = (i % 2 == 0) ? 1.0 : -1.0;
      bf[i] = (bf[i - 1] * i + expx * sign - expmx) * inv;
    }
  } else if (absx <= 1.0e-6) {
    for (int i = 0; i <= 12; ++i) bf[i] = (2 * ((i + 1) % 2)) / (i + 1.0);
  } else {
    int last = absx > 2.0 ? 15 : absx > 1.0 ? 12 : absx > 0.5 ? 7 : 6;
    for (int i = 0; i <= 12; ++i) {
      double y = 0.0;
      for (int m = 0; m <= last; ++m) {
        double xf = m != 0 ? fact(m) : 1.0;
        double coeff = (2 * ((m + i + 1) % 2)) / (xf * (m + i + 1));
        double xm = 1.0;
        for (int t = 0; t < m; ++t) xm = xm * (-x);
        y = y + xm * coeff;
      }
      bf[i] = y;
    }
  }
}

double aff(int la, int m, int i) {
  if (la == 0 && m == 0 && i == 0) return 1.0;
  if (la == 1 && m == 0 && i == 0) return 1.0;
  if (la == 1 && m == 1 && i == 0) return std::sqrt(0.5);
  if (la == 2 && m == 0 && i == 0) return 1.5;
  if (la == 2 && m == 1 && i == 0) return std::sqrt(1.5);
  if (la == 2 && m == 2 && i == 0) return std::sqrt(0.375);
  if (la == 2 && m == 0 && i == 2) return -0.5;
  return 0.0;
}

double bi(int i, int j) {
  if (j < 0 || j > i) return 0.0;
  return fact(i) / (fact(j) * fact(i - j));
}

// Slater overlap radial integral (src/overlap_d.rs ss).
double ss(int na, int nb, int la1, int lb1, int m1, double ua, double ub, double r) {
  int m = m1 - 1, lb = lb1 - 1, la = la1 - 1;
  double p = r * ((ua + ub) * 0.5), bb = r * ((ua - ub) * 0.5);
  double af[20];
  double quo = 1.0 / p;
  af[0] = quo * std::exp(-p);
  for (int n = 1; n < 20; ++n) af[n] = af[n - 1] * n * quo + af[0];
  double bf[13];
  bfn(bb, bf);
  double sum = 0.0;
  int lam1 = la - m, lbm1 = lb - m;
  for (int i = 0; i <= lam1; i += 2) {
    int ia = na + i - la, ic = la - i - m;
    for (int j = 0; j <= lbm1; j += 2) {
      int ib = nb + j - lb, id = lb - j - m;
      double sum1 = 0.0;
      int iab = ia + ib;
      for (int k1 = 0; k1 <= ia; ++k1)
        for (int k2 = 0; k2 <= ib; ++k2)
          for (int k3 = 0; k3 <= ic; ++k3)
            for (int k4 = 0; k4 <= id; ++k4)
              for (int k5 = 0; k5 <= m; ++k5) {
                int iaf = iab - k1 - k2 + k3 + k4 + 2 * k5;
                for (int k6 = 0; k6 <= m; ++k6) {
                  int ibf = k1 + k2 + k3 + k4 + 2 * k6;
                  double sign = 1 - 2 * ((m + k2 + k4 + k5 + k6) % 2);
                  double coeff = bi(id, k4) * bi(ic, k3) * bi(ib, k2) * bi(ia, k1) * bi(m, k5) * bi(m, k6) * sign;
                  sum1 = sum1 + af[iaf] * bf[ibf] * coeff;
                }
              }
      sum = sum + sum1 * (aff(la, m, i) * aff(lb, m, j));
    }
  }
  double rpow = 1.0;
  for (int t = 0; t < na + nb + 1; ++t) rpow = rpow * r;
  double norm = std::sqrt(ua * ub / (fact(na + na) * fact(nb + nb)) * ((la + la + 1) * (lb + lb + 1)));
  return sum * rpow * (powi(ua, na) * powi(ub, nb) / 2.0 * norm);
}

double coe(const double v[3], int nij, double c[76]) {
  const double RT34 = 0.86602540378444, RT13 = 0.57735026918963;
  double x2 = v[0], y2 = v[1], z2 = v[2];
  double xy2 = x2 * x2 + y2 * y2;
  double r = std::sqrt(xy2 + z2 * z2), xy = std::sqrt(xy2);
  double ca, cb, sa, sb;
  if (xy >= 1.0e-10) {
    ca = x2 * (1.0 / xy);
    cb = z2 * (1.0 / r);
    sa = y2 * (1.0 / xy);
    sb = xy * (1.0 / r);
  } else if (z2 < 0.0) {
    ca = -1.0;
    cb = -1.0;
    sa = 0.0;
    sb = 0.0;
  } else if (z2 == 0.0) {
    ca = cb = sa = sb = 0.0;
  } else {
    ca = 1.0;
    cb = 1.0;
    sa = 0.0;
    sb = 0.0;
  }
  for (int i = 0; i < 76; ++i) c[i] = 0.0;
  c[37] = 1.0;
  if (nij >= 2) {
    c[56] = ca * cb;
    c[41] = ca * sb;
    c[26] = -sa;
    c[53] = -sb;
    c[38] = cb;
    c[23] = 0.0;
    c[50] = sa * cb;
    c[35] = sa * sb;
    c[20] = ca;
    if (nij >= 5) {
      double c2a = ca * ca * 2.0 - 1.0, c2b = cb * cb * 2.0 - 1.0, s2a = sa * ca * 2.0, s2b = sb * cb * 2.0;
      c[75] = c2a * cb * cb + c2a * sb * sb * 0.5;
      c[60] = c2a * s2b * 0.5;
      c[45] = c2a * sb * sb * RT34;
      c[30] = -(s2a * sb);
      c[15] = -(s2a * cb);
      c[72] = ca * s2b * (-0.5);
      c[57] = ca * c2b;
      c[42] = ca * s2b * RT34;
      c[27] = -(sa * cb);
      c[12] = sa * sb;
      c[69] = sb * sb * (RT13 * 1.5);
      c[54] = -(s2b * RT34);
      c[39] = cb * cb - sb * sb * 0.5;
      c[66] = sa * s2b * (-0.5);
      c[51] = sa * c2b;
      c[36] = sa * s2b * RT34;
      c[21] = ca * cb;
      c[6] = -(ca * sb);
      c[63] = s2a * cb * cb + s2a * sb * sb * 0.5;
      c[48] = s2a * s2b * 0.5;
      c[33] = s2a * sb * sb * RT34;
      c[18] = c2a * sb;
      c[3] = c2a * cb;
    }
  }
  return r;
}

const int IVAL[4][6] = {{0, 0, 0, 0, 0, 0}, {0, 1, 1, 1, 1, 0}, {0, 0, 3, 4, 2, 0}, {0, 9, 8, 7, 6, 5}};

int shells(int norb) { return norb == 1 ? 1 : (norb == 4 ? 2 : 3); }

int n_sp(int z) {
  return (z >= 1 && z <= 2) ? 1 : z <= 10 ? 2 : z <= 18 ? 3 : z <= 36 ? 4 : z <= 54 ? 5 : z <= 86 ? 6 : 0;
}
int n_d(int z) { return (z >= 1 && z <= 30) ? 3 : z <= 48 ? 4 : z <= 80 ? 5 : z <= 86 ? 6 : 0; }

// ---- numerical Slater overlaps for n >= 4 (src/overlap_numeric.rs) --------------

void legendre_p_dp(int n, double x, double &p, double &dp) {
  double p0 = 1.0, p1 = x;
  if (n == 0) {
    p = 1.0;
    dp = 0.0;
    return;
  }
  for (int k = 2; k <= n; ++k) {
    double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  p = p1;
  dp = n * (x * p1 - p0) / (x * x - 1.0);
}

void gauss_legendre(int n, double a, double b, std::vector<double> &x, std::vector<double> &w) {
  std::vector<double> nodes(n), weights(n);
  int m = (n + 1) / 2;
  for (int i = 0; i < m; ++i) {
    double xx = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p, dp;
      legendre_p_dp(n, xx, p, dp);
      double dx = -p / dp;
      xx += dx;
      if (std::fabs(dx) < 1.0e-15) break;
    }
    double p, dp;
    legendre_p_dp(n, xx, p, dp);
    double wt = 2.0 / ((1.0 - xx * xx) * dp * dp);
    nodes[i] = -xx;
    nodes[n - 1 - i] = xx;
    weights[i] = wt;
    weights[n - 1 - i] = wt;
  }
  double mid = 0.5 * (a + b), half = 0.5 * (b - a);
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    x[i] = mid + half * nodes[i];
    w[i] = half * weights[i];
  }
}

double slater_norm(int n, double zeta) {
  double f = 1.0;
  for (int k = 1; k <= 2 * n; ++k) f *= k;
  return std::pow(2.0 * zeta, n + 0.5) / std::sqrt(std::max(f, 1.0));
}

double overlap_sto(int na, double za, int la, int ma, int nb, double zb, int lb, double r) {
  double norm_a = slater_norm(na, za), norm_b = slater_norm(nb, zb);
  double c;
  if (la == 0 && lb == 0) c = 0.5;
  else if ((la == 1 && lb == 0 && ma == 0) || (la == 0 && lb == 1 && ma == 0)) c = std::sqrt(3.0) / 2.0;
  else if (la == 1 && lb == 1 && ma == 0) c = 1.5;
  else if (la == 1 && lb == 1 && ma == 1) c = 0.75;
  else return 0.0;
  double half_r = r * 0.5;
  double p = (za + zb) * half_r;
  double xi_max = 1.0 + 60.0 / std::max(p, 0.05);
  std::vector<double> xn, xw, en, ew;
  gauss_legendre(48, 1.0, xi_max, xn, xw);
  gauss_legendre(40, -1.0, 1.0, en, ew);
  double sum = 0.0;
  for (size_t i = 0; i < xn.size(); ++i)
    for (size_t j = 0; j < en.size(); ++j) {
      double xi = xn[i], eta = en[j];
      double ra = half_r * (xi + eta), rb = half_r * (xi - eta);
      if (ra <= 0.0 || rb <= 0.0) continue;
      double cos_a = (1.0 + xi * eta) / (xi + eta), cos_b = (xi * eta - 1.0) / (xi - eta);
      double ang_a = la == 0 ? 1.0 : (ma == 0 ? cos_a : std::sqrt(std::max(1.0 - cos_a * cos_a, 0.0)));
      double ang_b = lb == 0 ? 1.0 : (ma == 0 ? cos_b : std::sqrt(std::max(1.0 - cos_b * cos_b, 0.0)));
      double radial = powi(ra, na - 1) * powi(rb, nb - 1) * std::exp(ra * (-za) - rb * zb);
      double jac = xi * xi - eta * eta;
      sum = sum + radial * (xw[i] * ew[j] * ang_a * ang_b * jac);
    }
  return powi(half_r, 3) * sum * (norm_a * norm_b * c);
}

}  // namespace

// pair_two_electron_d_g (src/mndod_twocenter.rs:1053-1108).
PairBlock pair_two_electron_d(const Element &ei, const Element &ej, const double dvec[3]) {
  bool has_d = ei.n_orb == 9 || ej.n_orb == 9;
  Rot R;
  double r = rotmat(dvec, has_d, R);
  double ri[23];
  reppd(ei, ej, r, ri);
  double core[11][3];
  spcore(ei, ej, r, core);
  std::vector<double> rep;
  reppd2(ei, ej, r, ri, core, rep);
  {
    double cfrac, point;
    feather_to_point(r, cfrac, point);
    double one_minus = 1.0 - cfrac;
    double point1 = (1.0 / r) * (-EV * ej.core_charge), point2 = (1.0 / r) * (-EV * ei.core_charge);
    for (int k = 1; k <= 10; ++k) {
      core[k][1] *= cfrac;
      core[k][2] *= cfrac;
    }
    for (int k : {1, 3, 4, 7, 9, 10}) {
      core[k][1] += point1 * one_minus;
      core[k][2] += point2 * one_minus;
    }
  }
  int ii = ei.n_orb, kk = ej.n_orb;
  std::vector<std::vector<double>> v;
  tx(ii, kk, rep, R, v);
  std::vector<double> ww;
  rotate_left(ii, kk, v, R, ww);
  pm7_balance(ww, core, ei, ej);
  int limij = indx(ii, ii), limkl = indx(kk, kk);
  PairBlock out;
  out.norb_i = ii;
  out.norb_j = kk;
  out.npair_i = limij;
  out.npair_j = limkl;
  out.w.assign((size_t)limij * limkl, 0.0);
  for (int pi = 0; pi < limij; ++pi)
    for (int pj = 0; pj < limkl; ++pj) out.w[(size_t)pi * limkl + pj] = ww[(size_t)pi * limkl + pj + 1];
  elenuc_block(core, R, 1, ii, out.e1b);
  elenuc_block(core, R, 2, kk, out.e2a);
  return out;
}

// diat_overlap (src/overlap_d.rs:264-340).
void diat_overlap_d(const Element &ei, const Element &ej, const double dvec[3], double di[9][9]) {
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) di[i][j] = 0.0;
  int norbi = ei.n_orb, norbj = ej.n_orb;
  if (norbi == 0 || norbj == 0) return;
  int nij = std::max(norbi, norbj);
  double c[76];
  double r = coe(dvec, nij, c);
  auto cc = [&c](int i, int k, int orb) { return c[i + 3 * (k - 1) + 15 * (orb - 1)]; };
  int ia = shells(norbi), ib = shells(norbj);
  double ex_i[3] = {ei.zeta_s, ei.zeta_p, std::max(ei.zeta_d, 0.3)};
  double ex_j[3] = {ej.zeta_s, ej.zeta_p, std::max(ej.zeta_d, 0.3)};
  double s[4][4][4] = {{{0}}};
  int newk = std::min(ia - 1, ib - 1);
  for (int i = 1; i <= ia; ++i) {
    int pq1 = i == 3 ? n_d(ei.z) : n_sp(ei.z);
    for (int j = 1; j <= ib; ++j) {
      int pq2 = j == 3 ? n_d(ej.z) : n_sp(ej.z);
      for (int k = 1; k <= newk + 1; ++k) {
        if (k > i || k > j) continue;
        int pi = std::max(pq1, i), pj = std::max(pq2, j);
        s[i][j][k] = ss(pi, pj, i, j, k, ex_i[i - 1], ex_j[j - 1], r);
      }
    }
  }
  for (int i = 1; i <= ia; ++i) {
    int kmin = 4 - i, kmax = 2 + i;
    for (int j = 1; j <= ib; ++j) {
      double aa = 1.0, bb = 1.0;
      if (j == 2) {
        aa = -1.0;
        bb = 1.0;
      } else if (j == 3) {
        aa = 1.0;
        bb = -1.0;
      }
      int lmin = 4 - j, lmax = 2 + j;
      for (int k = kmin; k <= kmax; ++k)
        for (int l = lmin; l <= lmax; ++l) {
          int ii = IVAL[i][k], jj = IVAL[j][l];
          if (ii == 0 || jj == 0) continue;
          double s1 = s[i][j][1], s2 = s[i][j][2], s3 = s[i][j][3];
          double val = s1 * (cc(i, k, 3) * cc(j, l, 3)) * aa +
                       s2 * (cc(i, k, 4) * cc(j, l, 4) + cc(i, k, 2) * cc(j, l, 2)) * bb +
                       s3 * (cc(i, k, 5) * cc(j, l, 5) + cc(i, k, 1) * cc(j, l, 1));
          di[ii - 1][jj - 1] = val;
        }
    }
  }
}

// slater_locals_numeric (src/overlap_numeric.rs).
void slater_locals_numeric(int na, double zsa, double zpa, int nb, double zsb, double zpb, double r, double out[5]) {
  out[0] = overlap_sto(na, zsa, 0, 0, nb, zsb, 0, r);
  double i_pss = overlap_sto(na, zpa, 1, 0, nb, zsb, 0, r);
  double i_sps = overlap_sto(na, zsa, 0, 0, nb, zpb, 1, r);
  double i_pps = overlap_sto(na, zpa, 1, 0, nb, zpb, 1, r);
  double i_ppp = overlap_sto(na, zpa, 1, 1, nb, zpb, 1, r);
  out[1] = i_pss;
  out[2] = -i_sps;
  out[3] = -i_pps;
  out[4] = i_ppp;
}

}  // namespace oracle
