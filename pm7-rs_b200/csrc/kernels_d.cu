// MNDO/d frame of the core Hamiltonian on the device: the two-centre two-electron and
// electron-core integrals of pm7-rs src/mndod_twocenter.rs (MOPAC rotmat, reppd, spcore,
// reppd2/rijkl/charg, the two-step rotation tx + rotatd, the PM7 d balance and elenuc)
// and the general Slater overlaps of src/overlap_d.rs (MOPAC coe, bfn, ss, diat).
//
// A molecule with any d-shell atom is evaluated entirely in this frame (hamiltonian.rs:
// 346-355, 424-428), so every near pair goes through the warp-per-pair integral kernel
// and every pair through the d-frame overlap.
//
// Warp-per-pair layout: one warp owns one atom pair and a 34 KB slice of shared memory
// holding the rotation matrices, the local integrals rep(1..491) and the half-rotated
// v(ij, kl). Work is split so that every output value is accumulated by a single lane in
// the reference's order: lanes over local integrals, then over the rows of the first
// rotation, then over the columns of the second. No atomics; the bits repeat run to run.
#include <cuda_runtime.h>

#include "common.cuh"
#include "core_repulsion.cuh"
#include "batch.hpp"
#include "gradient.cuh"
#include "kernels.hpp"
#include "nddo_sp.cuh"

#include <mutex>
#include <set>
#include <utility>

namespace pm7 {
namespace {

// Charge-distribution class of a pair index indx(k, l) (MOPAC met): 1 ss, 2 ps, 3 pp,
// 4 ds, 5 dp, 6 dd.
__constant__ int c_met[46] = {0, 1, 2, 3, 2, 3, 3, 2, 3, 3, 3, 4, 5, 5, 5, 6, 4, 5, 5, 5, 6, 6, 4,
                              5, 5, 5, 6, 6, 6, 4, 5, 5, 5, 6, 6, 6, 6, 4, 5, 5, 5, 6, 6, 6, 6, 6};
// rep(k) = ri(ipos(k)), k = 1..34 (MOPAC reppd2).
__constant__ int c_ipos[35] = {0,  1,  5,  11, 12, 12, 2,  6,  13, 14, 14, 3,  8,  16, 18, 18, 7, 15,
                               10, 20, 4,  9,  17, 19, 21, 7,  15, 10, 20, 22, 4,  9,  17, 21, 19};
// Signs of the 22 sp local integrals (MOPAC nri).
__constant__ double c_nri[23] = {0.0, 1.0,  -1.0, 1.0,  1.0,  -1.0, 1.0, 1.0, -1.0, -1.0, -1.0, 1.0,
                                 1.0, -1.0, -1.0, -1.0, 1.0,  1.0,  1.0, 1.0, 1.0,  1.0,  1.0};

__device__ __forceinline__ int indexd(int i, int j) {  // MOPAC indexd, 1-based
  if (i < j) {
    const int t = i;
    i = j;
    j = t;
  }
  return (i + 9 * (j - 1)) - (j * (j - 1)) / 2;
}
__device__ __forceinline__ int indx(int i, int j) {  // lower-triangle pair index, 1-based
  if (i < j) {
    const int t = i;
    i = j;
    j = t;
  }
  return (i * (i - 1)) / 2 + j;
}
// q = indx(i, j) - 1 -> (i, j), i >= j, 1-based; the order of the loops i = 1.., j = 1..i.
__device__ __forceinline__ void pair_of(int q, int &i, int &j) {
  int a = 1;
  while ((a * (a + 1)) / 2 <= q) ++a;
  i = a;
  j = q - (a * (a - 1)) / 2 + 1;
}

// ---- rotation tensors (MOPAC rotmat), evaluated from p (3x3) and d (5x5) -----------

struct RotPD {
  double p[4][4];  // 1-based
  double d[6][6];
};

__device__ inline double rotmat(double x11, double x22, double x33, bool has_d, RotPD &R) {
  const double SMALL = 1.0e-7, PT5SQ3 = 0.8660254037841;
  const double b = x11 * x11 + x22 * x22;
  const double r = sqrt(b + x33 * x33);
  const double sqb = sqrt(b);
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
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) R.p[i][j] = 0.0;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) R.d[i][j] = 0.0;
  R.p[1][1] = ca * sb;
  R.p[2][1] = ca * cb;
  R.p[3][1] = -sa;
  R.p[1][2] = sa * sb;
  R.p[2][2] = sa * cb;
  R.p[3][2] = ca;
  R.p[1][3] = cb;
  R.p[2][3] = -sb;
  if (has_d) {
    const double c2a = ca * ca * 2.0 - 1.0, c2b = cb * cb * 2.0 - 1.0, s2a = sa * ca * 2.0, s2b = sb * cb * 2.0;
    R.d[1][1] = c2a * sb * sb * PT5SQ3;
    R.d[2][1] = c2a * s2b * 0.5;
    R.d[3][1] = -(s2a * sb);
    R.d[4][1] = c2a * (cb * cb + sb * sb * 0.5);
    R.d[5][1] = -(s2a * cb);
    R.d[1][2] = ca * s2b * PT5SQ3;
    R.d[2][2] = ca * c2b;
    R.d[3][2] = -(sa * cb);
    R.d[4][2] = ca * s2b * (-0.5);
    R.d[5][2] = sa * sb;
    R.d[1][3] = cb * cb - sb * sb * 0.5;
    R.d[2][3] = -(s2b * PT5SQ3);
    R.d[4][3] = sb * sb * PT5SQ3;
    R.d[1][4] = sa * s2b * PT5SQ3;
    R.d[2][4] = sa * c2b;
    R.d[3][4] = ca * cb;
    R.d[4][4] = sa * s2b * (-0.5);
    R.d[5][4] = -(ca * sb);
    R.d[1][5] = s2a * sb * sb * PT5SQ3;
    R.d[2][5] = s2a * s2b * 0.5;
    R.d[3][5] = c2a * sb;
    R.d[4][5] = s2a * (cb * cb + sb * sb * 0.5);
    R.d[5][5] = c2a * cb;
  }
  return r;
}

// Pair components of the product tensors dd(6..15): (1,2) (1,3) (2,3) (1,4) (2,4) (3,4)
// (1,5) (2,5) (3,5) (4,5).
__constant__ int c_dd_a[16] = {0, 0, 0, 0, 0, 0, 1, 1, 2, 1, 2, 3, 1, 2, 3, 4};
__constant__ int c_dd_b[16] = {0, 0, 0, 0, 0, 0, 2, 3, 3, 4, 4, 4, 5, 5, 5, 5};

// pp(t, k, l), t = 1..6, 1 <= l <= k <= 3 (zero above the diagonal).
__device__ __forceinline__ double rot_pp(const RotPD &R, int t, int k, int l) {
  if (l > k) return 0.0;
  const double(*p)[4] = R.p;
  if (k == l) {
    switch (t) {
      case 1: return p[k][1] * p[k][1];
      case 2: return p[k][2] * p[k][2];
      case 3: return p[k][3] * p[k][3];
      case 4: return p[k][1] * p[k][2];
      case 5: return p[k][1] * p[k][3];
      default: return p[k][2] * p[k][3];
    }
  }
  switch (t) {
    case 1: return p[k][1] * p[l][1] * 2.0;
    case 2: return p[k][2] * p[l][2] * 2.0;
    case 3: return p[k][3] * p[l][3] * 2.0;
    case 4: return p[k][1] * p[l][2] + p[k][2] * p[l][1];
    case 5: return p[k][1] * p[l][3] + p[k][3] * p[l][1];
    default: return p[k][2] * p[l][3] + p[k][3] * p[l][2];
  }
}
// dp(t, k, col) = d(k, a) p(col, b), t = 3(a-1) + b.
__device__ __forceinline__ double rot_dp(const RotPD &R, int t, int k, int col) {
  const int a = (t - 1) / 3 + 1, b = (t - 1) % 3 + 1;
  return R.d[k][a] * R.p[col][b];
}
// dd(t, k, l), t = 1..15, 1 <= l <= k <= 5 (zero above the diagonal).
__device__ __forceinline__ double rot_dd(const RotPD &R, int t, int k, int l) {
  if (l > k) return 0.0;
  const double(*d)[6] = R.d;
  if (k == l) {
    if (t <= 5) return d[k][t] * d[k][t];
    return d[k][c_dd_a[t]] * d[k][c_dd_b[t]];
  }
  if (t <= 5) return d[k][t] * d[l][t] * 2.0;
  const int a = c_dd_a[t], b = c_dd_b[t];
  return d[k][a] * d[l][b] + d[k][b] * d[l][a];
}

// ---- local integrals --------------------------------------------------------------

// MOPAC reppd (mndod_twocenter.rs:244-482): the 22 sp local integrals, signed and feathered.
__device__ void reppd(const ElementRec &ei, const ElementRec &ej, double r, double ri[23]) {
  const double ev = kEv, ev1 = ev / 2.0, ev2 = ev1 / 2.0, ev3 = ev2 / 2.0, ev4 = ev3 / 2.0;
  for (int k = 0; k < 23; ++k) ri[k] = 0.0;
  const bool si = ei.n_orb >= 4, sj = ej.n_orb >= 4;
  auto sq = [](double x, double off) { return 1.0 / sqrt(x * x + off); };
  auto q = [](double x) { return 1.0 / sqrt(x); };
  auto sqp = [](double a, double b) { return (a + b) * (a + b); };
  const double aee = sqp(ei.po[1], ej.po[1]);
  if (!si && !sj) {
    ri[1] = sq(r, aee) * ev;
  } else if (si && !sj) {
    const double da = ei.dd, qa = ei.qq * 2.0;
    const double ade = sqp(ei.po[2], ej.po[1]), aqe = sqp(ei.po[3], ej.po[1]);
    const double ee = sq(r, aee) * ev;
    ri[1] = ee;
    ri[2] = sq(r + da, ade) * ev1 - sq(r - da, ade) * ev1;
    ri[3] = ee + sq(r + qa, aqe) * ev2 + sq(r - qa, aqe) * ev2 - sq(r, aqe) * ev1;
    ri[4] = ee + q(r * r + (qa * qa + aqe)) * ev1 - sq(r, aqe) * ev1;
  } else if (!si && sj) {
    const double db = ej.dd, qb = ej.qq * 2.0;
    const double aed = sqp(ei.po[1], ej.po[2]), aeq = sqp(ei.po[1], ej.po[3]);
    const double ee = sq(r, aee) * ev;
    ri[1] = ee;
    ri[5] = sq(r - db, aed) * ev1 - sq(r + db, aed) * ev1;
    ri[11] = ee + sq(r - qb, aeq) * ev2 + sq(r + qb, aeq) * ev2 - sq(r, aeq) * ev1;
    ri[12] = ee + q(r * r + (qb * qb + aeq)) * ev1 - sq(r, aeq) * ev1;
  } else {
    const double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0;
    const double ade = sqp(ei.po[2], ej.po[1]), aqe = sqp(ei.po[3], ej.po[1]), aed = sqp(ei.po[1], ej.po[2]),
                 aeq = sqp(ei.po[1], ej.po[3]), axx = sqp(ei.po[2], ej.po[2]), adq = sqp(ei.po[2], ej.po[3]),
                 aqd = sqp(ei.po[3], ej.po[2]), aqq = sqp(ei.po[3], ej.po[3]);
    const double ee = sq(r, aee) * ev;
    const double dze = -(sq(r + da, ade)) * ev1 + sq(r - da, ade) * ev1;
    const double qzze = sq(r - qa, aqe) * ev2 + sq(r + qa, aqe) * ev2 - sq(r, aqe) * ev1;
    const double qxxe = q(r * r + (qa * qa + aqe)) * ev1 - sq(r, aqe) * ev1;
    const double edz = -(sq(r - db, aed)) * ev1 + sq(r + db, aed) * ev1;
    const double eqzz = sq(r - qb, aeq) * ev2 + sq(r + qb, aeq) * ev2 - sq(r, aeq) * ev1;
    const double eqxx = q(r * r + (qb * qb + aeq)) * ev1 - sq(r, aeq) * ev1;
    const double dxdx = q(r * r + ((da - db) * (da - db) + axx)) * ev1 - q(r * r + ((da + db) * (da + db) + axx)) * ev1;
    const double dzdz = sq(r + da - db, axx) * ev2 + sq(r - da + db, axx) * ev2 - sq(r - da - db, axx) * ev2 -
                        sq(r + da + db, axx) * ev2;
    const double qa1 = ei.qq, qb1 = ej.qq;
    const double dzqxx = sq(r + da, adq) * ev2 - q((r + da) * (r + da) + (qb * qb + adq)) * ev2 -
                         sq(r - da, adq) * ev2 + q((r - da) * (r - da) + (qb * qb + adq)) * ev2;
    const double qxxdz = sq(r - db, aqd) * ev2 - q((r - db) * (r - db) + (qa * qa + aqd)) * ev2 -
                         sq(r + db, aqd) * ev2 + q((r + db) * (r + db) + (qa * qa + aqd)) * ev2;
    const double dzqzz = -(sq(r + da - qb, adq)) * ev3 + sq(r - da - qb, adq) * ev3 - sq(r + da + qb, adq) * ev3 +
                         sq(r - da + qb, adq) * ev3 - sq(r - da, adq) * ev2 + sq(r + da, adq) * ev2;
    const double qzzdz = -(sq(r + qa - db, aqd)) * ev3 + sq(r + qa + db, aqd) * ev3 - sq(r - qa - db, aqd) * ev3 +
                         sq(r - qa + db, aqd) * ev3 + sq(r - db, aqd) * ev2 - sq(r + db, aqd) * ev2;
    const double qxxqxx = q(r * r + ((qa - qb) * (qa - qb) + aqq)) * ev3 +
                          q(r * r + ((qa + qb) * (qa + qb) + aqq)) * ev3 - q(r * r + (qa * qa + aqq)) * ev2 -
                          q(r * r + (qb * qb + aqq)) * ev2 + sq(r, aqq) * ev2;
    const double qxxqyy = q(r * r + (qa * qa + qb * qb + aqq)) * ev2 - q(r * r + (qa * qa + aqq)) * ev2 -
                          q(r * r + (qb * qb + aqq)) * ev2 + sq(r, aqq) * ev2;
    const double qxxqzz = q((r - qb) * (r - qb) + (qa * qa + aqq)) * ev3 +
                          q((r + qb) * (r + qb) + (qa * qa + aqq)) * ev3 - sq(r - qb, aqq) * ev3 -
                          sq(r + qb, aqq) * ev3 - q(r * r + (qa * qa + aqq)) * ev2 + sq(r, aqq) * ev2;
    const double qzzqxx = q((r + qa) * (r + qa) + (qb * qb + aqq)) * ev3 +
                          q((r - qa) * (r - qa) + (qb * qb + aqq)) * ev3 - sq(r + qa, aqq) * ev3 -
                          sq(r - qa, aqq) * ev3 - q(r * r + (qb * qb + aqq)) * ev2 + sq(r, aqq) * ev2;
    const double qzzqzz = sq(r + qa - qb, aqq) * ev4 + sq(r + qa + qb, aqq) * ev4 + sq(r - qa - qb, aqq) * ev4 +
                          sq(r - qa + qb, aqq) * ev4 - sq(r - qa, aqq) * ev3 - sq(r + qa, aqq) * ev3 -
                          sq(r - qb, aqq) * ev3 - sq(r + qb, aqq) * ev3 + sq(r, aqq) * ev2;
    const double dxqxz = -q((r - qb1) * (r - qb1) + ((da - qb1) * (da - qb1) + adq)) * ev2 +
                         q((r + qb1) * (r + qb1) + ((da - qb1) * (da - qb1) + adq)) * ev2 +
                         q((r - qb1) * (r - qb1) + ((da + qb1) * (da + qb1) + adq)) * ev2 -
                         q((r + qb1) * (r + qb1) + ((da + qb1) * (da + qb1) + adq)) * ev2;
    const double qxzdx = -q((r + qa1) * (r + qa1) + ((qa1 - db) * (qa1 - db) + aqd)) * ev2 +
                         q((r - qa1) * (r - qa1) + ((qa1 - db) * (qa1 - db) + aqd)) * ev2 +
                         q((r + qa1) * (r + qa1) + ((qa1 + db) * (qa1 + db) + aqd)) * ev2 -
                         q((r - qa1) * (r - qa1) + ((qa1 + db) * (qa1 + db) + aqd)) * ev2;
    const double m1 = (qa1 - qb1) * (qa1 - qb1) + aqq, p1 = (qa1 + qb1) * (qa1 + qb1) + aqq;
    const double qxzqxz =
        q((r + qa1 - qb1) * (r + qa1 - qb1) + m1) * ev3 - q((r + qa1 + qb1) * (r + qa1 + qb1) + m1) * ev3 -
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
  for (int k = 1; k <= 22; ++k) ri[k] = ri[k] * c_nri[k];
  double cf, pt;
  d_feather(r, cf, pt);
  const double add = pt * (1.0 - cf);
  for (int k = 1; k <= 22; ++k) ri[k] *= cf;
  // charge-charge integrals decay to the point charge: 1, 3, 4, 11, 12, 16..19, 21
  ri[1] += add;
  ri[3] += add;
  ri[4] += add;
  ri[11] += add;
  ri[12] += add;
  ri[16] += add;
  ri[17] += add;
  ri[18] += add;
  ri[19] += add;
  ri[21] += add;
}

// MOPAC spcore (mndod_twocenter.rs:492-572): core[1..4][1..2]; core[k][1] = electrons of
// i in the field of core j, core[k][2] the reverse. core[5..10] start at zero.
__device__ void spcore(const ElementRec &ei, const ElementRec &ej, double r, double core[11][3]) {
  const double ev = kEv;
  for (int i = 0; i < 11; ++i) core[i][0] = core[i][1] = core[i][2] = 0.0;
  const double r2 = r * r, aci = ei.po[9], acj = ej.po[9];
  const double ssj = (acj + ei.po[1]) * (acj + ei.po[1]), ssi = (aci + ej.po[1]) * (aci + ej.po[1]);
  core[1][1] = -(1.0 / sqrt(r2 + ssj)) * (ej.core * ev);
  core[1][2] = -(1.0 / sqrt(r2 + ssi)) * (ei.core * ev);
  // multipole weights of the sp charge distributions: 1, -1/2, -1/2, 1/2, 1/4, 1/4, 1/2
  auto terms = [&](const ElementRec &e, double ac, double &a2, double &a3, double &a4) {
    const double pp = (ac + e.po[7]) * (ac + e.po[7]);
    const double da = e.ddp[2], qa = e.ddp[3] / sqrt(2.0), tq = qa + qa;
    const double ad = (e.po[2] + ac) * (e.po[2] + ac), aq = (e.po[3] + ac) * (e.po[3] + ac);
    const double x1 = (1.0 / sqrt(r2 + pp)) * 1.0, x2 = (1.0 / sqrt(r2 + aq)) * -0.5;
    const double x3 = (1.0 / sqrt((r + da) * (r + da) + ad)) * -0.5;
    const double x4 = (1.0 / sqrt((r - da) * (r - da) + ad)) * 0.5;
    const double x5 = (1.0 / sqrt((r - tq) * (r - tq) + aq)) * 0.25;
    const double x6 = (1.0 / sqrt((r + tq) * (r + tq) + aq)) * 0.25;
    const double x7 = (1.0 / sqrt(r2 + (tq * tq + aq))) * 0.5;
    a2 = (x3 + x4) * ev;
    a3 = (x1 + x2 + x5 + x6) * ev;
    a4 = (x1 + x2 + x7) * ev;
  };
  if (ei.n_orb >= 4) {
    double a2, a3, a4;
    terms(ei, acj, a2, a3, a4);
    core[2][1] = -(a2)*ej.core;
    core[3][1] = -(a3)*ej.core;
    core[4][1] = -(a4)*ej.core;
  }
  if (ej.n_orb >= 4) {
    double a2, a3, a4;
    terms(ej, aci, a2, a3, a4);
    // the dipole term of atom j enters with the opposite sign (its axis points back to i)
    core[2][2] = (a2)*ei.core;
    core[3][2] = -(a3)*ei.core;
    core[4][2] = -(a4)*ei.core;
  }
}

// MOPAC charg (src/mndod.rs:30-187): interaction of two multipoles of orders l1, l2 with
// shared component m, charge separations da, db and additive term add.
__device__ double charg(double r, int l1, int l2, int m, double da, double db, double add) {
  auto inv = [add](double x) { return 1.0 / sqrt(x * x + add); };
  auto q = [](double x) { return 1.0 / sqrt(x); };
  if (l1 == 0 && l2 == 0) return 1.0 / sqrt(r * r + add);
  if (l1 == 1 && l2 == 0) return (inv(r - da) - inv(r + da)) * 0.5;
  if (l1 == 0 && l2 == 1) return (inv(r + db) - inv(r - db)) * 0.5;
  if (l1 == 1 && l2 == 1) {
    if (m == 0) return (inv(r + da - db) + inv(r - da + db) - inv(r - da - db) - inv(r + da + db)) * 0.25;
    return (q(r * r + (da - db) * (da - db) + add) - q(r * r + (da + db) * (da + db) + add)) * 0.5;
  }
  if (l1 == 0 && l2 == 2) return (inv(r - db) - q(r * r + (db * db + add)) * 2.0 + inv(r + db)) * 0.25;
  if (l1 == 2 && l2 == 0) return (inv(r - da) - q(r * r + (da * da + add)) * 2.0 + inv(r + da)) * 0.25;
  if (l1 == 1 && l2 == 2) {
    if (m == 0)
      return (inv(r - da - db) - q((r - da) * (r - da) + (db * db + add)) * 2.0 + inv(r + db - da) -
              inv(r - db + da) + q((r + da) * (r + da) + (db * db + add)) * 2.0 - inv(r + da + db)) *
             0.125;
    const double ab = db / sqrt(2.0);
    return (q((r - ab) * (r - ab) + ((da - ab) * (da - ab) + add)) * (-2.0) +
            q((r + ab) * (r + ab) + ((da - ab) * (da - ab) + add)) * 2.0 +
            q((r - ab) * (r - ab) + ((da + ab) * (da + ab) + add)) * 2.0 -
            q((r + ab) * (r + ab) + ((da + ab) * (da + ab) + add)) * 2.0) *
           0.125;
  }
  if (l1 == 2 && l2 == 1) {
    if (m == 0)
      return (-inv(r - da - db) + q((r - db) * (r - db) + (da * da + add)) * 2.0 - inv(r + da - db) +
              inv(r - da + db) - q((r + db) * (r + db) + (da * da + add)) * 2.0 + inv(r + da + db)) *
             0.125;
    const double aa = da / sqrt(2.0);
    return (q((r + aa) * (r + aa) + ((aa - db) * (aa - db) + add)) * (-2.0) +
            q((r - aa) * (r - aa) + ((aa - db) * (aa - db) + add)) * 2.0 +
            q((r + aa) * (r + aa) + ((aa + db) * (aa + db) + add)) * 2.0 -
            q((r - aa) * (r - aa) + ((aa + db) * (aa + db) + add)) * 2.0) *
           0.125;
  }
  if (l1 == 2 && l2 == 2) {
    const double xyxy = q(r * r + ((da - db) * (da - db) + add)) * 4.0 +
                        q(r * r + ((da + db) * (da + db) + add)) * 4.0 - q(r * r + (da * da + db * db + add)) * 8.0;
    if (m == 0) {
      const double zzzz = inv(r - da - db) + inv(r + da + db) + inv(r - da + db) + inv(r + da - db) -
                          q((r - da) * (r - da) + (db * db + add)) * 2.0 -
                          q((r - db) * (r - db) + (da * da + add)) * 2.0 -
                          q((r + da) * (r + da) + (db * db + add)) * 2.0 -
                          q((r + db) * (r + db) + (da * da + add)) * 2.0 +
                          q(r * r + ((da - db) * (da - db) + add)) * 2.0 +
                          q(r * r + ((da + db) * (da + db) + add)) * 2.0;
      return zzzz * (1.0 / 16.0) - xyxy * (1.0 / 64.0);
    }
    if (m == 1) {
      const double aa = da / sqrt(2.0), ab = db / sqrt(2.0);
      const double m1 = (aa - ab) * (aa - ab) + add, p1 = (aa + ab) * (aa + ab) + add;
      return (q((r + aa - ab) * (r + aa - ab) + m1) * 2.0 - q((r + aa + ab) * (r + aa + ab) + m1) * 2.0 -
              q((r - aa - ab) * (r - aa - ab) + m1) * 2.0 + q((r - aa + ab) * (r - aa + ab) + m1) * 2.0 -
              q((r + aa - ab) * (r + aa - ab) + p1) * 2.0 + q((r + aa + ab) * (r + aa + ab) + p1) * 2.0 +
              q((r - aa - ab) * (r - aa - ab) + p1) * 2.0 - q((r - aa + ab) * (r - aa + ab) + p1) * 2.0) *
             (1.0 / 16.0);
    }
    return xyxy * (1.0 / 16.0);
  }
  return 0.0;
}

// MOPAC rijkl (mndod_twocenter.rs:583-655), without the EV factor.
__device__ double rijkl(const DTables *T, const ElementRec &ei, const ElementRec &ej, int ij, int kl, int li, int lj,
                        int lk, int ll, int ic, double r) {
  const int lij = indx(li + 1, lj + 1), lkl = indx(lk + 1, ll + 1);
  const int l1min = min(abs(li - lj), 2), l1max = min(li + lj, 2);
  const int l2min = min(abs(lk - ll), 2), l2max = min(lk + ll, 2);
  double sum = 0.0;
  for (int l1 = l1min; l1 <= l1max; ++l1) {
    double dij, pij;
    if (l1 == 0) {
      dij = 0.0;
      pij = lij == 1 ? (ic == 1 ? ei.po[9] : ei.po[1]) : lij == 3 ? ei.po[7] : lij == 6 ? ei.po[8] : ei.po[1];
    } else {
      dij = ei.ddp[lij];
      pij = ei.po[lij];
    }
    for (int l2 = l2min; l2 <= l2max; ++l2) {
      double dkl, pkl;
      if (l2 == 0) {
        dkl = 0.0;
        pkl = lkl == 1 ? (ic == 2 ? ej.po[9] : ej.po[1]) : lkl == 3 ? ej.po[7] : lkl == 6 ? ej.po[8] : ej.po[1];
      } else {
        dkl = ej.ddp[lkl];
        pkl = ej.po[lkl];
      }
      const double add = (pij + pkl) * (pij + pkl);
      const int lmin = min(l1, l2);
      for (int m = -lmin; m <= lmin; ++m) {
        const double ccc = T->ch[((ij - 1) * 3 + l1) * 5 + (m + 2)] * T->ch[((kl - 1) * 3 + l2) * 5 + (m + 2)];
        if (ccc == 0.0) continue;
        sum = sum + charg(r, l1, l2, abs(m), dij, dkl, add) * ccc;
      }
    }
  }
  return sum;
}

__device__ __forceinline__ int lorb(int i) { return i == 1 ? 0 : (i <= 4 ? 1 : 2); }

// ---- one pair, one warp ------------------------------------------------------------

constexpr int kVStride = 46;
struct DPairShared {
  RotPD R;
  double ri[23];
  double core[11][3];
  double v[46 * kVStride];  // v[ij][kl], ij = indexd 1..45, kl = 1..limkl
  double ww[2026];          // rep(1..491) during the first rotation, then ww(1..limij*limkl)
};

// Computes the pair's molecular-frame w (left in S.ww, 1-based, row-major limij x limkl)
// and the electron-core terms (S.core) for the ordered pair (ea, eb), displacement d = R_b - R_a.
__device__ void warp_pair_d(DPairShared &S, const DTables *T, const ElementRec &ea, const ElementRec &eb, double dx,
                            double dy, double dz, int lane) {
  const bool has_d = ea.n_orb == 9 || eb.n_orb == 9;
  const double r = sqrt((dx * dx + dy * dy) + dz * dz);
  if (lane == 0) rotmat(dx, dy, dz, has_d, S.R);
  if (lane == 1) reppd(ea, eb, r, S.ri);
  if (lane == 2) spcore(ea, eb, r, S.core);
  double *rep = S.ww;
  for (int k = lane; k < 492; k += 32) rep[k] = 0.0;
  __syncwarp();
  for (int k = lane + 1; k <= 34; k += 32) rep[k] = S.ri[c_ipos[k]];
  double cf, pt;
  d_feather(r, cf, pt);
  if (has_d) {
    // MOPAC reppd2 (mndod_twocenter.rs:658-751): the independent d integrals, then copies.
    const double padd = pt * (1.0 - cf);
    const int lasti = ea.n_orb == 9 ? 9 : (ea.n_orb == 1 ? 1 : 4);
    const int lastk = eb.n_orb == 9 ? 9 : (eb.n_orb == 1 ? 1 : 4);
    const int ni = lasti * (lasti + 1) / 2, nk = lastk * (lastk + 1) / 2;
    for (int t = lane; t < ni * nk; t += 32) {
      const int qi = t / nk, qk = t - qi * nk;
      int i, j, k, l;
      pair_of(qi, i, j);
      pair_of(qk, k, l);
      const int ij = indexd(i, j), kl = indexd(k, l);
      const int numb = T->ind2[(ij - 1) * 45 + (kl - 1)];
      if (numb <= 34 || T->isym[numb] != 0) continue;
      const double v = rijkl(T, ea, eb, ij, kl, lorb(i), lorb(j), lorb(k), lorb(l), 0, r) * kEv;
      rep[numb] = (i == j && k == l) ? v * cf + padd : v * cf;
    }
    // the d electron-core terms core[5..10] (lanes 0-5: electrons of b, 6-11: of a)
    if (lane < 6 && eb.n_orb == 9) {
      const int kd[6] = {indexd(5, 1), indexd(5, 2), indexd(5, 5), indexd(6, 3), indexd(6, 6), indexd(8, 8)};
      const int l1[6] = {0, 1, 2, 1, 2, 2};
      S.core[5 + lane][2] = -rijkl(T, ea, eb, 1, kd[lane], 0, 0, 2, l1[lane], 1, r) * (kEv * ea.core);
    }
    if (lane >= 6 && lane < 12 && ea.n_orb == 9) {
      const int t = lane - 6;
      const int kd[6] = {indexd(5, 1), indexd(5, 2), indexd(5, 5), indexd(6, 3), indexd(6, 6), indexd(8, 8)};
      const int l1[6] = {0, 1, 2, 1, 2, 2};
      S.core[5 + t][1] = -rijkl(T, ea, eb, kd[t], 1, 2, l1[t], 0, 0, 2, r) * (kEv * eb.core);
    }
    __syncwarp();
    for (int t = lane; t < ni * nk; t += 32) {
      const int qi = t / nk, qk = t - qi * nk;
      int i, j, k, l;
      pair_of(qi, i, j);
      pair_of(qk, k, l);
      const int numb = T->ind2[(indexd(i, j) - 1) * 45 + (indexd(k, l) - 1)];
      if (numb <= 34) continue;
      const int nold = T->isym[numb];
      if (nold >= 35) rep[numb] = rep[nold];
      else if (nold <= -35) rep[numb] = -rep[-nold];
    }
  }
  __syncwarp();
  // Feather the electron-core terms toward the point charge (rotatd.F90:1160-1181):
  // all ten scale by cfrac, the charge-charge ones {1,3,4,7,9,10} add the point charge.
  if (lane < 10) {
    const int k = lane + 1;
    const double one_minus = 1.0 - cf;
    const double point1 = (1.0 / r) * (-kEv * eb.core), point2 = (1.0 / r) * (-kEv * ea.core);
    const bool mono = k == 1 || k == 3 || k == 4 || k == 7 || k == 9 || k == 10;
    S.core[k][1] = S.core[k][1] * cf;
    S.core[k][2] = S.core[k][2] * cf;
    if (mono) {
      S.core[k][1] = S.core[k][1] + point1 * one_minus;
      S.core[k][2] = S.core[k][2] + point2 * one_minus;
    }
  }
  // First rotation (MOPAC tx): each lane owns rows ij of v.
  const int ii = ea.n_orb, kk = eb.n_orb;
  const int limij = ii * (ii + 1) / 2, limkl = kk * (kk + 1) / 2;
  for (int q = lane; q < limij; q += 32) {
    int i1, j1;
    pair_of(q, i1, j1);
    const int ij = indexd(i1, j1);
    double *v = S.v + ij * kVStride;
    for (int c = 0; c <= limkl; ++c) v[c] = 0.0;
    for (int k1 = 1; k1 <= kk; ++k1)
      for (int l1 = 1; l1 <= k1; ++l1) {
        const int nd = T->ind2[(ij - 1) * 45 + (indexd(k1, l1) - 1)];
        if (nd == 0) continue;
        const double w = rep[nd];
        switch (c_met[indx(k1, l1)]) {
          case 1: v[1] = w; break;
          case 2: {
            const int k = k1 - 1;
            v[2] = v[2] + S.R.p[k][1] * w;
            v[4] = v[4] + S.R.p[k][2] * w;
            v[7] = v[7] + S.R.p[k][3] * w;
            break;
          }
          case 3: {
            const int k = k1 - 1, l = l1 - 1;
            v[3] = v[3] + rot_pp(S.R, 1, k, l) * w;
            v[6] = v[6] + rot_pp(S.R, 2, k, l) * w;
            v[10] = v[10] + rot_pp(S.R, 3, k, l) * w;
            v[5] = v[5] + rot_pp(S.R, 4, k, l) * w;
            v[8] = v[8] + rot_pp(S.R, 5, k, l) * w;
            v[9] = v[9] + rot_pp(S.R, 6, k, l) * w;
            break;
          }
          case 4: {
            const int k = k1 - 4;
            v[11] = v[11] + S.R.d[k][1] * w;
            v[16] = v[16] + S.R.d[k][2] * w;
            v[22] = v[22] + S.R.d[k][3] * w;
            v[29] = v[29] + S.R.d[k][4] * w;
            v[37] = v[37] + S.R.d[k][5] * w;
            break;
          }
          case 5: {
            const int k = k1 - 4, l = l1 - 1;
            const int cols[15] = {12, 13, 14, 17, 18, 19, 23, 24, 25, 30, 31, 32, 38, 39, 40};
#pragma unroll
            for (int t = 0; t < 15; ++t) v[cols[t]] = v[cols[t]] + rot_dp(S.R, t + 1, k, l) * w;
            break;
          }
          default: {
            const int k = k1 - 4, l = l1 - 4;
            const int diag[5] = {15, 21, 28, 36, 45};
#pragma unroll
            for (int t = 0; t < 5; ++t) v[diag[t]] = v[diag[t]] + rot_dd(S.R, t + 1, k, l) * w;
            const int offd[10] = {20, 26, 27, 33, 34, 35, 41, 42, 43, 44};
#pragma unroll
            for (int t = 0; t < 10; ++t) v[offd[t]] = v[offd[t]] + rot_dd(S.R, t + 6, k, l) * w;
            break;
          }
        }
      }
  }
  __syncwarp();
  // Second rotation (MOPAC rotatd): each lane owns columns kl of ww.
  double *ww = S.ww;
  for (int kl = lane + 1; kl <= limkl; kl += 32) {
    for (int p = 0; p < limij; ++p) ww[p * limkl + kl] = 0.0;
    auto at = [&](int i, int j) -> double & { return ww[(indx(i, j) - 1) * limkl + kl]; };
    for (int i1 = 1; i1 <= ii; ++i1)
      for (int j1 = 1; j1 <= i1; ++j1) {
        const double w = S.v[indexd(i1, j1) * kVStride + kl];
        switch (c_met[indx(i1, j1)]) {
          case 1: at(1, 1) = w; break;
          case 2:
            for (int i = 1; i <= 3; ++i) at(i + 1, 1) += S.R.p[i1 - 1][i] * w;
            break;
          case 3:
            for (int i = 1; i <= 3; ++i) {
              at(i + 1, i + 1) += rot_pp(S.R, i, i1 - 1, j1 - 1) * w;
              for (int j = 1; j < i; ++j) at(i + 1, j + 1) += rot_pp(S.R, 1 + i + j, i1 - 1, j1 - 1) * w;
            }
            break;
          case 4:
            for (int i = 1; i <= 5; ++i) at(i + 4, 1) += S.R.d[i1 - 4][i] * w;
            break;
          case 5:
            for (int i = 1; i <= 5; ++i)
              for (int j = 1; j <= 3; ++j) at(i + 4, j + 1) += rot_dp(S.R, 3 * (i - 1) + j, i1 - 4, j1 - 1) * w;
            break;
          default:
            for (int i = 1; i <= 5; ++i) {
              at(i + 4, i + 4) += rot_dd(S.R, i, i1 - 4, j1 - 4) * w;
              for (int j = 1; j < i; ++j)
                at(i + 4, j + 4) += rot_dd(S.R, T->inddd[(i - 1) * 5 + (j - 1)], i1 - 4, j1 - 4) * w;
            }
            break;
        }
      }
  }
  __syncwarp();
  // PM7 d balance (mndod_twocenter.rs:919-1004): the mean of the two-centre d Coulomb
  // integrals is set to <ss|ss>. Small and sequential: lane 0.
  if (lane == 0 && (ea.iod > 0 || eb.iod > 0)) {
    double(*core)[3] = S.core;
    if (ea.iod > 0) {
      const int k = kk == 9 ? 45 : (kk == 4 ? 10 : 1);
      if (kk > 1) {
        double sum = 0.0;
        for (int i = 5; i <= 9; ++i) {
          const int j = k * ((i * (i + 1)) / 2 - 1);
          sum = sum + ww[j + 3] + ww[j + 6] + ww[j + 10];
        }
        sum = ww[1] - sum * (1.0 / 15.0);
        for (int i = 5; i <= 9; ++i) {
          const int j = k * ((i * (i + 1)) / 2 - 1);
          for (int l = 2; l <= 4; ++l) ww[(l * (l + 1)) / 2 + j] += sum;
        }
        const double s = core[1][1] - (core[3][1] + core[4][1] * 2.0) * (1.0 / 3.0);
        core[3][1] += s;
        core[4][1] += s;
      }
      double sum = 0.0;
      for (int i = 5; i <= 9; ++i) sum = sum + ww[k * ((i * (i + 1)) / 2 - 1) + 1];
      sum = ww[1] - sum * (1.0 / 5.0);
      for (int i = 5; i <= 9; ++i) ww[k * ((i * (i + 1)) / 2 - 1) + 1] += sum;
      const double s = core[1][1] - (core[7][1] + core[9][1] * 2.0 + core[10][1] * 2.0) * (1.0 / 5.0);
      core[7][1] += s;
      core[9][1] += s;
      core[10][1] += s;
    }
    if (eb.iod > 0) {
      if (ea.iod > 0) {
        double sum = 0.0;
        for (int i = 5; i <= 9; ++i) {
          const int j = 45 * ((i * (i + 1)) / 2 - 1);
          sum = sum + ww[j + 15] + ww[j + 21] + ww[j + 28] + ww[j + 36] + ww[j + 45];
        }
        sum = ww[1] - sum * (1.0 / 25.0);
        for (int i = 5; i <= 9; ++i) {
          const int j = 45 * ((i * (i + 1)) / 2 - 1);
          for (int m = 5; m <= 9; ++m) ww[(m * (m + 1)) / 2 + j] += sum;
        }
      }
      if (ii > 1) {
        double sum = 0.0;
        for (int i = 2; i <= 4; ++i) {
          const int j = 45 * ((i * (i + 1)) / 2 - 1);
          sum = sum + ww[j + 15] + ww[j + 21] + ww[j + 28] + ww[j + 36] + ww[j + 45];
        }
        sum = ww[1] - sum * (1.0 / 15.0);
        for (int i = 2; i <= 4; ++i) {
          const int j = 45 * ((i * (i + 1)) / 2 - 1);
          for (int m = 5; m <= 9; ++m) ww[(m * (m + 1)) / 2 + j] += sum;
        }
        const double s = core[1][2] - (core[3][2] + core[4][2] * 2.0) * (1.0 / 3.0);
        core[3][2] += s;
        core[4][2] += s;
      }
      const double sum = ww[1] - (ww[15] + ww[21] + ww[28] + ww[36] + ww[45]) * (1.0 / 5.0);
      for (int m = 5; m <= 9; ++m) ww[(m * (m + 1)) / 2] += sum;
      const double s = core[1][2] - (core[7][2] + core[9][2] * 2.0 + core[10][2] * 2.0) * (1.0 / 5.0);
      core[7][2] += s;
      core[9][2] += s;
      core[10][2] += s;
    }
  }
  __syncwarp();
}

// One element (i >= j, 1-based) of the electron-core block of atom n (1 = a, 2 = b),
// MOPAC elenuc (mndod_twocenter.rs:1008-1047).
__device__ double elenuc(const DPairShared &S, const DTables *T, int n, int i, int j) {
  const int ind1 = i - 1, ind2 = j - 1;
  const double(*core)[3] = S.core;
  if (ind1 == 0) return core[1][n];
  if (ind1 < 4) {
    if (ind2 == 0) return S.R.p[1][ind1] * core[2][n];
    const int ipp = T->indpp[(ind1 - 1) * 3 + (ind2 - 1)];
    return core[3][n] * rot_pp(S.R, ipp, 1, 1) + core[4][n] * (rot_pp(S.R, ipp, 2, 2) + rot_pp(S.R, ipp, 3, 3));
  }
  if (ind2 == 0) return S.R.d[1][ind1 - 3] * core[5][n];
  if (ind2 < 4) {
    const int idp = T->inddp[(ind1 - 4) * 3 + (ind2 - 1)];
    return core[6][n] * rot_dp(S.R, idp, 1, 1) + core[8][n] * (rot_dp(S.R, idp, 2, 2) + rot_dp(S.R, idp, 3, 3));
  }
  const int idd = T->inddd[(ind1 - 4) * 5 + (ind2 - 4)];
  return core[7][n] * rot_dd(S.R, idd, 1, 1) + core[9][n] * (rot_dd(S.R, idd, 2, 2) + rot_dd(S.R, idd, 3, 3)) +
         core[10][n] * (rot_dd(S.R, idd, 4, 4) + rot_dd(S.R, idd, 5, 5));
}

// Unpacks a packed lower-triangle index k -> (mu, nu), mu >= nu, 0-based.
__device__ __forceinline__ void unpack(int k, int &mu, int &nu) {
  int m = 0;
  while ((m + 1) * (m + 2) / 2 <= k) ++m;
  mu = m;
  nu = k - m * (m + 1) / 2;
}

constexpr int kDWarps = kDPairsPerBlock;  // pairs (warps) per block

// One near pair in the MNDO/d frame by one warp: w in (u, v) orientation and the packed
// electron-core blocks of both atoms.
__device__ __forceinline__ void near_d_pair(DPairShared &S, const DeviceParams &P, const int *__restrict__ z,
                                            const double *__restrict__ xyz, const NearPair q,
                                            double *__restrict__ w, double *__restrict__ ecore, int lane) {
  const ElementRec &eu = P.elements[z[q.u]];
  const ElementRec &ev = P.elements[z[q.v]];
  const bool keep = eu.n_orb >= ev.n_orb;  // heavier-first ordering (hamiltonian.rs:388-392)
  const int a = keep ? q.u : q.v, b = keep ? q.v : q.u;
  const ElementRec &ea = keep ? eu : ev;
  const ElementRec &eb = keep ? ev : eu;
  const double dx = xyz[3 * b] - xyz[3 * a], dy = xyz[3 * b + 1] - xyz[3 * a + 1], dz = xyz[3 * b + 2] - xyz[3 * a + 2];
  warp_pair_d(S, P.tab, ea, eb, dx, dy, dz, lane);
  const int limij = ea.n_orb * (ea.n_orb + 1) / 2, limkl = eb.n_orb * (eb.n_orb + 1) / 2;
  double *wp = w + q.woff;
  for (int t = lane; t < limij * limkl; t += 32) {
    const int pi = t / limkl, pj = t - pi * limkl;
    wp[keep ? t : pj * limij + pi] = S.ww[t + 1];
  }
  double *e_a = ecore + (keep ? q.eoff_u : q.eoff_v);
  double *e_b = ecore + (keep ? q.eoff_v : q.eoff_u);
  for (int t = lane; t < limij + limkl; t += 32) {
    int mu, nu;
    if (t < limij) {
      unpack(t, mu, nu);
      e_a[t] = elenuc(S, P.tab, 1, mu + 1, nu + 1);
    } else {
      unpack(t - limij, mu, nu);
      e_b[t - limij] = elenuc(S, P.tab, 2, mu + 1, nu + 1);
    }
  }
  __syncwarp();
}

// Near pairs in the MNDO/d frame, one warp per pair.
__global__ void __launch_bounds__(32 * kDWarps) k_near_integrals_d(int n_near, const int *__restrict__ z,
                                                                   const double *__restrict__ xyz,
                                                                   const NearPair *__restrict__ np, DeviceParams P,
                                                                   double *__restrict__ w, double *__restrict__ ecore) {
  extern __shared__ double smem_d[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * kDWarps + warp;
  if (p >= n_near) return;
  near_d_pair(reinterpret_cast<DPairShared *>(smem_d)[warp], P, z, xyz, np[p], w, ecore, lane);
}

// Batched: item = kDWarps consecutive near pairs of one molecule.
__global__ void __launch_bounds__(32 * kDWarps) k_b_near_integrals_d(BatchList L, const MolDesc *__restrict__ D,
                                                                     DeviceParams P) {
  extern __shared__ double smem_d[];
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const MolDesc &d = D[L.slot[m]];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = (item - L.prefix[m]) * kDWarps + warp;
  if (p >= d.g.n_near) return;
  near_d_pair(reinterpret_cast<DPairShared *>(smem_d)[warp], P, d.g.z, d.g.xyz, d.g.np[p], d.w, d.ecore, lane);
}

// ---- general Slater overlaps (src/overlap_d.rs) -------------------------------------

__device__ __forceinline__ double fact(int n) {
  double f = 1.0;
  for (int i = 1; i <= n; ++i) f = f * (double)i;
  return f;
}

// MOPAC bfn: B integrals bf[0..12] of x = (ua - ub) r / 2.
__device__ void bfn(double x, double bf[13]) {
  const double absx = fabs(x);
  if (absx > 3.0) {
    const double expx = exp(x), expmx = 1.0 / expx, inv = 1.0 / x;
    bf[0] = (expx - expmx) * inv;
    for (int i = 1; i <= 12; ++i) {
      const double sign = (i % 2 == 0) ? 1.0 : -1.0;
      bf[i] = (bf[i - 1] * (double)i + expx * sign - expmx) * inv;
    }
  } else if (absx <= 1.0e-6) {
    for (int i = 0; i <= 12; ++i) bf[i] = (double)(2 * ((i + 1) % 2)) / ((double)i + 1.0);
  } else {
    const int last = absx > 2.0 ? 15 : absx > 1.0 ? 12 : absx > 0.5 ? 7 : 6;
    for (int i = 0; i <= 12; ++i) {
      double y = 0.0, xf = 1.0, xm = 1.0;
      for (int m = 0; m <= last; ++m) {
        if (m != 0) {
          xf = xf * (double)m;  // m!
          xm = xm * (-x);       // (-x)^m
        }
        const double coeff = (double)(2 * ((m + i + 1) % 2)) / (xf * (double)(m + i + 1));
        y = y + xm * coeff;
      }
      bf[i] = y;
    }
  }
}

__device__ __forceinline__ double aff(int la, int m, int i) {
  if (i == 0) {
    if (la == 0 && m == 0) return 1.0;
    if (la == 1) return m == 0 ? 1.0 : (m == 1 ? 0.7071067811865476 : 0.0);
    if (la == 2) return m == 0 ? 1.5 : (m == 1 ? 1.224744871391589 : (m == 2 ? 0.6123724356957945 : 0.0));
    return 0.0;
  }
  return (la == 2 && m == 0 && i == 2) ? -0.5 : 0.0;
}

__device__ __forceinline__ double binom(int i, int j) {
  if (j < 0 || j > i) return 0.0;
  return fact(i) / (fact(j) * fact(i - j));
}

// MOPAC ss: Slater overlap of shells la1, lb1 (1 s, 2 p, 3 d), component m1 (1 sigma,
// 2 pi, 3 delta); af/bf are the A and B integrals of the shell pair at this distance.
__device__ double ss(int na, int nb, int la1, int lb1, int m1, double ua, double ub, double r, const double af[20],
                     const double bf[13]) {
  const int m = m1 - 1, lb = lb1 - 1, la = la1 - 1;
  double sum = 0.0;
  const int lam1 = la - m, lbm1 = lb - m;
  for (int i = 0; i <= lam1; i += 2) {
    const int ia = na + i - la, ic = la - i - m;
    for (int j = 0; j <= lbm1; j += 2) {
      const int ib = nb + j - lb, id = lb - j - m;
      double sum1 = 0.0;
      const int iab = ia + ib;
      for (int k1 = 0; k1 <= ia; ++k1)
        for (int k2 = 0; k2 <= ib; ++k2)
          for (int k3 = 0; k3 <= ic; ++k3)
            for (int k4 = 0; k4 <= id; ++k4)
              for (int k5 = 0; k5 <= m; ++k5) {
                const int iaf = iab - k1 - k2 + k3 + k4 + 2 * k5;
                for (int k6 = 0; k6 <= m; ++k6) {
                  const int ibf = k1 + k2 + k3 + k4 + 2 * k6;
                  const double sign = (double)(1 - 2 * ((m + k2 + k4 + k5 + k6) % 2));
                  const double coeff =
                      binom(id, k4) * binom(ic, k3) * binom(ib, k2) * binom(ia, k1) * binom(m, k5) * binom(m, k6) * sign;
                  sum1 = sum1 + af[iaf] * bf[ibf] * coeff;
                }
              }
      sum = sum + sum1 * (aff(la, m, i) * aff(lb, m, j));
    }
  }
  double rpow = 1.0;
  for (int t = 0; t < na + nb + 1; ++t) rpow = rpow * r;
  const double norm = sqrt(ua * ub / (fact(na + na) * fact(nb + nb)) * (double)((la + la + 1) * (lb + lb + 1)));
  return sum * rpow * (d_powi(ua, na) * d_powi(ub, nb) / 2.0 * norm);
}

// Orbital of shell i (1 s, 2 p, 3 d) and M_L component k (1..5): s -> 1; p: 2 py, 3 pz,
// 4 px; d: 1..5 -> 9, 8, 7, 6, 5 (1-based orbitals, 0 = none).
__device__ __forceinline__ int ival(int i, int k) {
  if (i == 1) return (k >= 1 && k <= 4) ? 1 : 0;
  if (i == 2) return k == 2 ? 3 : (k == 3 ? 4 : (k == 4 ? 2 : 0));
  return (k >= 1 && k <= 5) ? 10 - k : 0;
}

__device__ __forceinline__ int n_sp_shell(int z) {
  return (z >= 1 && z <= 2) ? 1 : z <= 10 ? 2 : z <= 18 ? 3 : z <= 36 ? 4 : z <= 54 ? 5 : z <= 86 ? 6 : 0;
}
__device__ __forceinline__ int n_d_shell(int z) {
  return (z >= 1 && z <= 30) ? 3 : z <= 48 ? 4 : z <= 80 ? 5 : z <= 86 ? 6 : 0;
}

// MOPAC coe: rotation coefficients c[1..75], c(i, k, orb) = c[i + 3(k-1) + 15(orb-1)].
__device__ double coe(double x2, double y2, double z2, int nij, double c[76]) {
  const double RT34 = 0.86602540378444, RT13 = 0.57735026918963;
  const double xy2 = x2 * x2 + y2 * y2;
  const double r = sqrt(xy2 + z2 * z2), xy = sqrt(xy2);
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
    c[50] = sa * cb;
    c[35] = sa * sb;
    c[20] = ca;
    if (nij >= 5) {
      const double c2a = ca * ca * 2.0 - 1.0, c2b = cb * cb * 2.0 - 1.0, s2a = sa * ca * 2.0, s2b = sb * cb * 2.0;
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

__device__ __forceinline__ int shells(int norb) { return norb == 1 ? 1 : (norb == 4 ? 2 : 3); }

// MOPAC diat (overlap_d.rs:264-340): the overlap of the ordered pair (ea, eb), d = R_b - R_a,
// handed element by element (1-based orbitals a, b and the value) to `emit`.
template <class Emit>
__device__ void diat_overlap(const ElementRec &ea, const ElementRec &eb, double dx, double dy, double dz, Emit emit) {
  const int norbi = ea.n_orb, norbj = eb.n_orb;
  if (norbi == 0 || norbj == 0) return;
  double c[76];
  const double r = coe(dx, dy, dz, norbi > norbj ? norbi : norbj, c);
  auto cc = [&c](int i, int k, int orb) { return c[i + 3 * (k - 1) + 15 * (orb - 1)]; };
  const int ia = shells(norbi), ib = shells(norbj);
  const double ex_i[3] = {ea.zeta_s, ea.zeta_p, fmax(ea.zeta_d, 0.3)};
  const double ex_j[3] = {eb.zeta_s, eb.zeta_p, fmax(eb.zeta_d, 0.3)};
  for (int i = 1; i <= ia; ++i) {
    const int pq1 = i == 3 ? n_d_shell(ea.z) : n_sp_shell(ea.z);
    for (int j = 1; j <= ib; ++j) {
      const int pq2 = j == 3 ? n_d_shell(eb.z) : n_sp_shell(eb.z);
      const int pi = pq1 > i ? pq1 : i, pj = pq2 > j ? pq2 : j;
      const double ua = ex_i[i - 1], ub = ex_j[j - 1];
      // A and B integrals shared by the sigma, pi and delta components of this shell pair
      double af[20], bf[13];
      const double p = r * ((ua + ub) * 0.5);
      const double quo = 1.0 / p;
      af[0] = quo * exp(-p);
      for (int n = 1; n < 20; ++n) af[n] = af[n - 1] * (double)n * quo + af[0];
      bfn(r * ((ua - ub) * 0.5), bf);
      double s[4] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 1; k <= (i < j ? i : j); ++k) s[k] = ss(pi, pj, i, j, k, ua, ub, r, af, bf);
      double aa = 1.0, bb = 1.0;
      if (j == 2) {
        aa = -1.0;
        bb = 1.0;
      } else if (j == 3) {
        aa = 1.0;
        bb = -1.0;
      }
      for (int k = 4 - i; k <= 2 + i; ++k)
        for (int l = 4 - j; l <= 2 + j; ++l) {
          const int oa = ival(i, k), ob = ival(j, l);
          if (oa == 0 || ob == 0) continue;
          const double val = s[1] * (cc(i, k, 3) * cc(j, l, 3)) * aa +
                             s[2] * (cc(i, k, 4) * cc(j, l, 4) + cc(i, k, 2) * cc(j, l, 2)) * bb +
                             s[3] * (cc(i, k, 5) * cc(j, l, 5) + cc(i, k, 1) * cc(j, l, 1));
          emit(oa, ob, val);
        }
    }
  }
}

__device__ __forceinline__ double beta_of(const ElementRec &e, int orb) {
  return orb == 0 ? e.beta_s : (orb <= 3 ? e.beta_p : e.beta_d);
}

// One pair u < v in the MNDO/d frame (v may be out of range): beta*S blocks of H from the
// d-frame overlap; returns the pair's core-core energy.
__device__ __forceinline__ double pair_d_elem(int n_atoms, const int *__restrict__ z, const double *__restrict__ xyz,
                                              const int *__restrict__ aoff, int nao, const DeviceParams &P,
                                              double *__restrict__ H, int u, int v) {
  if (!(v > u && v < n_atoms)) return 0.0;
  const ElementRec &eu = P.elements[z[u]];
  const ElementRec &ev = P.elements[z[v]];
  const bool keep = eu.n_orb >= ev.n_orb;
  const int a = keep ? u : v, b = keep ? v : u;
  const ElementRec &ea = keep ? eu : ev;
  const ElementRec &eb = keep ? ev : eu;
  const double dx = xyz[3 * b] - xyz[3 * a], dy = xyz[3 * b + 1] - xyz[3 * a + 1], dz = xyz[3 * b + 2] - xyz[3 * a + 2];
  const int oa = aoff[a], ob = aoff[b];
  diat_overlap(ea, eb, dx, dy, dz, [&](int i, int j, double s) {
    const double val = 0.5 * (beta_of(ea, i - 1) + beta_of(eb, j - 1)) * s;
    H[(size_t)(oa + i - 1) * nao + ob + j - 1] = val;
    H[(size_t)(ob + j - 1) * nao + oa + i - 1] = val;
  });
  const double ex = xyz[3 * v] - xyz[3 * u], ey = xyz[3 * v + 1] - xyz[3 * u + 1], ez = xyz[3 * v + 2] - xyz[3 * u + 2];
  return pair_core_energy(P, eu, ev, sqrt(ex * ex + ey * ey + ez * ez));
}

// The partner atoms v0 .. v0 + 127 of a block (128 threads), dealt to the threads grouped by
// orbital count (1, 4, 9; the pairs without work last), so that a warp mostly runs one shell
// structure of the overlap. Each pair writes only its own outputs, so the dealing order does not
// change any result.
__device__ __forceinline__ int deal_partner(int n_atoms, const int *__restrict__ z, const DeviceParams &P, int u,
                                            int v0) {
  __shared__ int count[4], sorted[128];
  if (threadIdx.x < 4) count[threadIdx.x] = 0;
  __syncthreads();
  const int v = v0 + threadIdx.x;
  int cls = 3;
  if (v > u && v < n_atoms) {
    const int no = P.elements[z[v]].n_orb;
    cls = no <= 1 ? 0 : (no <= 4 ? 1 : 2);
  }
  const int rank = atomicAdd(&count[cls], 1);
  __syncthreads();
  int base = 0;
  for (int c = 0; c < cls; ++c) base += count[c];
  sorted[base + rank] = v;
  __syncthreads();
  return sorted[threadIdx.x];
}

// All pairs u < v in the MNDO/d frame: beta*S blocks of H and each pair's core-core
// energy in pair order. Grid (ceil(N/128), N), block 128, blockIdx.y = u.
__global__ void k_pairs_all_d(int n_atoms, const int *__restrict__ z,
                                                     const double *__restrict__ xyz, const int *__restrict__ aoff,
                                                     int nao, DeviceParams P, double *__restrict__ H,
                                                     double *__restrict__ cc_terms) {
  const int u = blockIdx.y;
  const int v = deal_partner(n_atoms, z, P, u, blockIdx.x * 128);
  const double ecc = pair_d_elem(n_atoms, z, xyz, aoff, nao, P, H, u, v);
  if (v > u && v < n_atoms) cc_terms[pair_index(n_atoms, u, v)] = ecc;
}

// Batched: item = (atom u, column block) of one molecule; pair energies to cc_terms.
__global__ void k_b_pairs_all_d(BatchList L, const MolDesc *__restrict__ D, DeviceParams P) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const MolDesc &d = D[L.slot[m]];
  const int local = item - L.prefix[m];
  const int u = local / d.cc_nx, bx = local - u * d.cc_nx;
  const int v = deal_partner(d.g.n_atoms, d.g.z, P, u, bx * 128);
  const double ecc = pair_d_elem(d.g.n_atoms, d.g.z, d.g.xyz, d.g.aoff, d.g.nao, P, d.H, u, v);
  if (v > u && v < d.g.n_atoms) d.cc_terms[pair_index(d.g.n_atoms, u, v)] = ecc;
}

// One pair for the stage entry point: w (npair_a x npair_b), e1b/e2a and S (9x9 each).
__global__ void __launch_bounds__(32) k_stage_pair_d(DeviceParams P, int zi, int zj, double dx, double dy, double dz,
                                                     double *w, double *e1b, double *e2a, double *s, int *np_out) {
  extern __shared__ double smem_d[];
  DPairShared &S = *reinterpret_cast<DPairShared *>(smem_d);
  const int lane = threadIdx.x;
  const ElementRec &ea = P.elements[zi];
  const ElementRec &eb = P.elements[zj];
  for (int k = lane; k < 81; k += 32) e1b[k] = e2a[k] = s[k] = 0.0;
  warp_pair_d(S, P.tab, ea, eb, dx, dy, dz, lane);
  const int limij = ea.n_orb * (ea.n_orb + 1) / 2, limkl = eb.n_orb * (eb.n_orb + 1) / 2;
  for (int t = lane; t < limij * limkl; t += 32) w[t] = S.ww[t + 1];
  for (int t = lane; t < 81; t += 32) {
    const int i = t / 9, j = t % 9;
    const int hi = i > j ? i : j, lo = i > j ? j : i;
    if (hi < ea.n_orb) e1b[t] = elenuc(S, P.tab, 1, hi + 1, lo + 1);
    if (hi < eb.n_orb) e2a[t] = elenuc(S, P.tab, 2, hi + 1, lo + 1);
  }
  if (lane == 0) {
    diat_overlap(ea, eb, dx, dy, dz, [&](int i, int j, double v) { s[(i - 1) * 9 + (j - 1)] = v; });
    np_out[0] = limij;
    np_out[1] = limkl;
  }
}

// ---- nuclear gradient at a fixed density, MNDO/d frame (gradient.cuh) ----------------

// Every pair u < v and stencil point s: core-core, beta*S from the d-frame overlap and the
// point-charge terms beyond the feather range. Grid (ceil((N - 1) * 12 / 128), N), blockIdx.y = u.
__global__ void k_grad_pairs_d(GradGeometry g, DeviceParams P) {
  const int u = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = u + 1 + t / kStencil, s = t % kStencil;
  if (v >= g.n_atoms) return;
  const StencilPair q = stencil_pair(g, P, u, v, s);
  const ElementRec &ea = P.elements[g.z[q.a]];
  const ElementRec &eb = P.elements[g.z[q.b]];
  double E = pair_core_energy(P, ea, eb, q.r);
  const int oa = g.aoff[q.a], ob = g.aoff[q.b];
  diat_overlap(ea, eb, q.d[0], q.d[1], q.d[2], [&](int i, int j, double sv) {
    E += g.Pt[(size_t)(oa + i - 1) * g.nao + ob + j - 1] * (beta_of(ea, i - 1) + beta_of(eb, j - 1)) * sv;
  });
  if (!g.near_mask[(size_t)u * g.n_atoms + v])
    E += ((1.0 / q.r) * kEv) * far_bracket(g, oa, ea.n_orb, ob, eb.n_orb, ea.core, eb.core);
  g.E[tri_index(g.n_atoms, u, v) * kStencil + s] = E;
}

// Near pair p and stencil point s, a warp per item: w and the electron-core blocks of the
// warp-per-pair kernel at the displaced separation, contracted with the density (lanes over
// elements, fixed xor tree), added to the pair's stencil energy.
__global__ void __launch_bounds__(32 * kDWarps) k_grad_near_d(GradGeometry g, DeviceParams P) {
  extern __shared__ double smem_d[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long item = (long long)blockIdx.x * kDWarps + warp;
  const int p = (int)(item / kStencil), s = (int)(item % kStencil);
  if (p >= g.n_near) return;
  DPairShared &S = reinterpret_cast<DPairShared *>(smem_d)[warp];
  const NearPair np = g.np[p];
  const int u = np.u < np.v ? np.u : np.v, v = np.u < np.v ? np.v : np.u;
  const StencilPair q = stencil_pair(g, P, u, v, s);
  const ElementRec &ea = P.elements[g.z[q.a]];
  const ElementRec &eb = P.elements[g.z[q.b]];
  warp_pair_d(S, P.tab, ea, eb, q.d[0], q.d[1], q.d[2], lane);
  const int oa = g.aoff[q.a], ob = g.aoff[q.b];
  const int limij = ea.n_orb * (ea.n_orb + 1) / 2, limkl = eb.n_orb * (eb.n_orb + 1) / 2;
  double E = 0.0;
  for (int t = lane; t < limij * limkl; t += 32) {
    const int pi = t / limkl, pj = t - pi * limkl;
    int mu, nu, la, si;
    unpack(pi, mu, nu);
    unpack(pj, la, si);
    E += two_e_coef(g, oa, ob, mu, nu, la, si) * S.ww[t + 1];
  }
  for (int t = lane; t < limij + limkl; t += 32) {
    int mu, nu;
    if (t < limij) {
      unpack(t, mu, nu);
      E += ecore_coef(g, oa, mu, nu) * elenuc(S, P.tab, 1, mu + 1, nu + 1);
    } else {
      unpack(t - limij, mu, nu);
      E += ecore_coef(g, ob, mu, nu) * elenuc(S, P.tab, 2, mu + 1, nu + 1);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) E += __shfl_xor_sync(0xffffffffu, E, o);
  if (lane == 0) g.E[tri_index(g.n_atoms, u, v) * kStencil + s] += E;
}

// Sets a kernel's dynamic shared-memory limit once per (kernel, device).
void ensure_smem(const void *fn, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void *, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.insert({fn, dev}).second) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

// ---- host launchers ------------------------------------------------------

void launch_pairs_all_d(cudaStream_t st, int n_atoms, const int *z, const double *xyz, const int *aoff, int nao,
                        const DeviceParams &P, double *H, double *cc_terms) {
  if (n_atoms < 2) return;
  dim3 grid((n_atoms + 127) / 128, n_atoms);
  k_pairs_all_d<<<grid, 128, 0, st>>>(n_atoms, z, xyz, aoff, nao, P, H, cc_terms);
  note_launch();
}

void launch_near_integrals_d(cudaStream_t st, int n_near, const int *z, const double *xyz, const NearPair *np,
                             const DeviceParams &P, double *w, double *ecore) {
  if (n_near == 0) return;
  const size_t smem = sizeof(DPairShared) * kDWarps;
  ensure_smem((const void *)k_near_integrals_d, smem);
  k_near_integrals_d<<<(n_near + kDWarps - 1) / kDWarps, 32 * kDWarps, smem, st>>>(n_near, z, xyz, np, P, w, ecore);
  note_launch();
}

void launch_b_pairs_all_d(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P) {
  if (L.total <= 0) return;
  k_b_pairs_all_d<<<L.total, 128, 0, st>>>(L, D, P);
  note_launch();
}

void launch_b_near_integrals_d(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P) {
  if (L.total <= 0) return;
  const size_t smem = sizeof(DPairShared) * kDWarps;
  ensure_smem((const void *)k_b_near_integrals_d, smem);
  k_b_near_integrals_d<<<L.total, 32 * kDWarps, smem, st>>>(L, D, P);
  note_launch();
}

void launch_grad_pairs_d(cudaStream_t st, const GradGeometry &g, const DeviceParams &P) {
  if (g.n_atoms < 2) return;
  const dim3 grid((unsigned)(((size_t)(g.n_atoms - 1) * kStencil + 127) / 128), (unsigned)g.n_atoms);
  k_grad_pairs_d<<<grid, 128, 0, st>>>(g, P);
  note_launch();
}

void launch_grad_near_d(cudaStream_t st, const GradGeometry &g, const DeviceParams &P) {
  if (g.n_near <= 0) return;
  const size_t smem = sizeof(DPairShared) * kDWarps;
  ensure_smem((const void *)k_grad_near_d, smem);
  const size_t items = (size_t)g.n_near * kStencil;
  k_grad_near_d<<<(unsigned)((items + kDWarps - 1) / kDWarps), 32 * kDWarps, smem, st>>>(g, P);
  note_launch();
}

void launch_stage_pair_d(cudaStream_t st, const DeviceParams &P, int zi, int zj, const double d[3], double *w,
                         double *e1b, double *e2a, double *s, int *np_out) {
  k_stage_pair_d<<<1, 32, sizeof(DPairShared), st>>>(P, zi, zj, d[0], d[1], d[2], w, e1b, e2a, s, np_out);
  note_launch();
}

}  // namespace pm7
