// Oracle (test infrastructure): PM7 parameter load and derived quantities.
// Restates pm7-rs src/params.rs and the one-centre parts of src/mndod.rs.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "oracle_internal.hpp"
#include "pm7_param_data.h"

namespace oracle {
namespace {

enum Col {
  C_Z, C_N, C_IOS, C_IOP, C_IOD, C_CORE, C_EHEAT, C_USS, C_UPP, C_UDD, C_ZS, C_ZP, C_ZD, C_BS, C_BP,
  C_BD, C_GSS, C_GSP, C_GPP, C_GP2, C_HSP, C_ZSN, C_ZPN, C_ZDN, C_F0SD, C_G2SD, C_ALPHA, C_POC,
  C_POLVOL, C_G1_1, C_G1_2, C_G1_3, C_G1_4, C_G2_1, C_G2_2, C_G2_3, C_G2_4, C_G3_1, C_G3_2, C_G3_3,
  C_G3_4
};

// MOPAC ddpo.F90 via src/params.rs:492-503.
double dd_charge_sep(int n, double zs, double zp) {
  double nn = n;
  return (2.0 * nn + 1.0) * std::pow(4.0 * zs * zp, nn + 0.5) / std::pow(zs + zp, 2.0 * nn + 2.0) /
         std::sqrt(3.0);
}
double qq_charge_sep(int n, double zp) {
  double nn = n;
  return std::sqrt((4.0 * nn * nn + 6.0 * nn + 2.0) / 20.0) / zp;
}

// Fixed five-step secant of MOPAC calpar.F90 (src/params.rs:512-525).
template <class F>
double calpar_secant(double target, double guess, F f) {
  double d1 = guess, d2 = guess + 0.04;
  for (int it = 0; it < 5; ++it) {
    double f1 = f(d1), f2 = f(d2);
    if (std::fabs(f2 - f1) < 1.0e-25) break;
    double d3 = d1 + (d2 - d1) * (target - f1) / (f2 - f1);
    d1 = d2;
    d2 = d3;
  }
  return d2;
}

double signum(double x) { return std::signbit(x) ? -1.0 : 1.0; }

// src/params.rs:527-533
double additive_rho1(double hsp_ev, double dd) {
  double hsp = hsp_ev / EV;
  auto f = [dd](double d) { return 0.5 * d - 0.5 / std::sqrt(4.0 * dd * dd + 1.0 / (d * d)); };
  double guess = std::pow(std::fabs(hsp) / (dd * dd), 1.0 / 3.0) * signum(hsp);
  return 0.5 / calpar_secant(hsp, guess, f);
}

// src/params.rs:535-545
double additive_rho2(double hpp_ev, double qq) {
  double hpp = hpp_ev / EV;
  auto f = [qq](double q) {
    return 0.25 * q - 0.5 / std::sqrt(4.0 * qq * qq + 1.0 / (q * q)) +
           0.25 / std::sqrt(8.0 * qq * qq + 1.0 / (q * q));
  };
  double guess = std::pow(std::fabs(hpp) / (3.0 * std::pow(qq, 4)), 0.2) * signum(hpp);
  return 0.5 / calpar_secant(hpp, guess, f);
}

// ---- MNDO/d one-centre machinery (src/mndod.rs:214-736) ----------------

int iii(int z) {  // src/mndod.rs:215-225
  if (z >= 1 && z <= 2) return 1;
  if (z <= 10) return 2;
  if (z <= 18) return 3;
  if (z <= 36) return 4;
  if (z <= 54) return 5;
  if (z <= 86) return 6;
  return 0;
}
int iiid(int z) {  // src/mndod.rs:228-236
  if (z >= 1 && z <= 30) return 3;
  if (z <= 48) return 4;
  if (z <= 80) return 5;
  if (z <= 86) return 6;
  return 0;
}
bool main_group(int z) {  // src/mndod.rs:239-241
  return !((z >= 21 && z <= 29) || (z >= 39 && z <= 47) || (z >= 57 && z <= 79));
}

// Factorials fx(i) = (i-1)! and binomials b(i,j) = C(i-1, j-1) (MOPAC fbx).
struct Fb {
  double fx[31];
  double b[31][31];
  Fb() {
    for (int i = 0; i < 31; ++i) {
      fx[i] = 0.0;
      for (int j = 0; j < 31; ++j) b[i][j] = 0.0;
    }
    fx[1] = 1.0;
    for (int i = 2; i <= 30; ++i) fx[i] = fx[i - 1] * (double)(i - 1);
    for (int i = 0; i < 31; ++i) b[i][1] = 1.0;
    for (int i = 2; i <= 30; ++i)
      for (int j = 2; j <= i; ++j) b[i][j] = b[i - 1][j - 1] + b[i - 1][j];
  }
  // Radial Slater-Condon integral, MOPAC rsc (src/mndod.rs:271-331).
  double rsc(int k, int na, double ea, int nb, double eb, int nc, double ec, int nd, double ed) const {
    double aea = std::log(ea), aeb = std::log(eb), aec = std::log(ec), aed = std::log(ed);
    int nab = na + nb, ncd = nc + nd;
    double ecd = ec + ed, eab = ea + eb, e = ecd + eab;
    int n = nab + ncd;
    double ae = std::log(e), a2 = std::log(2.0), acd = std::log(ecd), aab = std::log(eab);
    double ff = fx[n] / std::sqrt(fx[2 * na + 1] * fx[2 * nb + 1] * fx[2 * nc + 1] * fx[2 * nd + 1]);
    double c = EV * ff *
               std::exp(na * aea + nb * aeb + nc * aec + nd * aed + 0.5 * (aea + aeb + aec + aed) +
                        a2 * (n + 2.0) - ae * n);
    double s0 = 1.0 / e, s1 = 0.0, s2 = 0.0;
    int m = ncd - k;
    for (int i = 1; i <= m; ++i) {
      s0 *= e / ecd;
      s1 += s0 * (b[ncd - k][i] - b[ncd + k + 1][i]) / b[n][i];
    }
    int m1 = m + 1, m2 = ncd + k + 1;
    for (int i = m1; i <= m2; ++i) {
      s0 *= e / ecd;
      s2 += s0 * b[m2][i] / b[n][i];
    }
    double s3 = std::exp(ae * n - acd * m2 - aab * (nab - k)) / b[n][m2];
    return c * (s1 - s2 + s3);
  }
};

// MOPAC eiscor (src/mndod.rs:463-499).
double eiscor(int z, double r016, double r066, double r244, double r266, double r466) {
  int a[5] = {0, 0, 0, 0, 0};
  auto set = [&](int x0, int x1, int x2, int x3, int x4) {
    a[0] = x0; a[1] = x1; a[2] = x2; a[3] = x3; a[4] = x4;
  };
  switch (z) {
    case 21: set(2, 0, 1, 0, 0); break;
    case 22: set(4, 1, 2, 8, 1); break;
    case 23: set(6, 3, 3, 15, 8); break;
    case 24: set(5, 10, 5, 35, 35); break;
    case 25: set(10, 10, 5, 35, 35); break;
    case 26: set(12, 15, 6, 35, 35); break;
    case 27: set(14, 21, 7, 43, 36); break;
    case 28: set(16, 28, 8, 50, 43); break;
    case 29: set(10, 45, 5, 70, 70); break;
    case 39: set(2, 0, 1, 0, 0); break;
    case 40: set(4, 1, 2, 8, 1); break;
    case 41: set(4, 6, 4, 21, 21); break;
    case 42: set(5, 10, 5, 35, 35); break;
    case 43: set(10, 10, 5, 35, 35); break;
    case 44: set(7, 21, 5, 43, 36); break;
    case 45: set(8, 28, 5, 50, 43); break;
    case 46: set(0, 45, 0, 70, 70); break;
    case 47: set(10, 45, 5, 70, 70); break;
    case 57: case 71: set(2, 0, 1, 0, 0); break;
    case 72: set(4, 1, 2, 8, 1); break;
    case 73: set(6, 3, 3, 15, 8); break;
    case 74: set(5, 10, 5, 35, 35); break;
    case 75: set(10, 10, 5, 35, 35); break;
    case 76: set(12, 15, 6, 35, 35); break;
    case 77: set(14, 21, 7, 43, 36); break;
    case 78: set(9, 36, 5, 56, 56); break;
    case 79: set(10, 45, 5, 70, 70); break;
    default: break;
  }
  return a[0] * r016 + a[1] * r066 - a[2] * r244 / 5.0 - a[3] * r266 / 49.0 - a[4] * r466 / 49.0;
}

// MOPAC scprm + inighd (src/mndod.rs:350-460): repd(1..52) and eiscor.
void inighd(const Fb &fb, int z, double zsn, double zpn, double zdn, double f0sd, double g2sd,
            double repd[53], double &eis) {
  const double s3 = 1.7320508, s5 = 2.23606797, s15 = 3.87298334;
  int ns = iii(z), nd = iiid(z);
  double es = zsn, ep = zpn, ed = zdn;
  double r016 = fb.rsc(0, ns, es, ns, es, nd, ed, nd, ed);
  double r036 = fb.rsc(0, ns, ep, ns, ep, nd, ed, nd, ed);
  double r066 = fb.rsc(0, nd, ed, nd, ed, nd, ed, nd, ed);
  double r155 = fb.rsc(1, ns, ep, nd, ed, ns, ep, nd, ed);
  double r125 = fb.rsc(1, ns, es, ns, ep, ns, ep, nd, ed);
  double r244 = fb.rsc(2, ns, es, nd, ed, ns, es, nd, ed);
  double r236 = fb.rsc(2, ns, ep, ns, ep, nd, ed, nd, ed);
  double r266 = fb.rsc(2, nd, ed, nd, ed, nd, ed, nd, ed);
  double r234 = fb.rsc(2, ns, ep, ns, ep, ns, es, nd, ed);
  double r246 = fb.rsc(2, ns, es, nd, ed, nd, ed, nd, ed);
  double r355 = fb.rsc(3, ns, ep, nd, ed, ns, ep, nd, ed);
  double r466 = fb.rsc(4, nd, ed, nd, ed, nd, ed, nd, ed);
  if (f0sd > 0.001) r016 = f0sd;
  if (g2sd > 0.001) r244 = g2sd;
  eis = eiscor(z, r016, r066, r244, r266, r466);
  for (int i = 0; i < 53; ++i) repd[i] = 0.0;
  repd[1] = r016;
  repd[2] = 2.0 / (3.0 * s5) * r125;
  repd[3] = 1.0 / s15 * r125;
  repd[4] = 2.0 / (5.0 * s5) * r234;
  repd[5] = r036 + 4.0 / 35.0 * r236;
  repd[6] = r036 + 2.0 / 35.0 * r236;
  repd[7] = r036 - 4.0 / 35.0 * r236;
  repd[8] = -1.0 / (3.0 * s5) * r125;
  repd[9] = std::sqrt(3.0 / 125.0) * r234;
  repd[10] = s3 / 35.0 * r236;
  repd[11] = 3.0 / 35.0 * r236;
  repd[12] = -1.0 / (5.0 * s5) * r234;
  repd[13] = r036 - 2.0 / 35.0 * r236;
  repd[14] = -2.0 * s3 / 35.0 * r236;
  repd[15] = -repd[3];
  repd[16] = -repd[11];
  repd[17] = -repd[9];
  repd[18] = -repd[14];
  repd[19] = 1.0 / 5.0 * r244;
  repd[20] = 2.0 / (7.0 * s5) * r246;
  repd[21] = repd[20] / 2.0;
  repd[22] = -repd[20];
  repd[23] = 4.0 / 15.0 * r155 + 27.0 / 245.0 * r355;
  repd[24] = 2.0 * s3 / 15.0 * r155 - 9.0 * s3 / 245.0 * r355;
  repd[25] = 1.0 / 15.0 * r155 + 18.0 / 245.0 * r355;
  repd[26] = -s3 / 15.0 * r155 + 12.0 * s3 / 245.0 * r355;
  repd[27] = -s3 / 15.0 * r155 - 3.0 * s3 / 245.0 * r355;
  repd[28] = -repd[27];
  repd[29] = r066 + 4.0 / 49.0 * r266 + 4.0 / 49.0 * r466;
  repd[30] = r066 + 2.0 / 49.0 * r266 - 24.0 / 441.0 * r466;
  repd[31] = r066 - 4.0 / 49.0 * r266 + 6.0 / 441.0 * r466;
  repd[32] = std::sqrt(3.0 / 245.0) * r246;
  repd[33] = 1.0 / 5.0 * r155 + 24.0 / 245.0 * r355;
  repd[34] = 1.0 / 5.0 * r155 - 6.0 / 245.0 * r355;
  repd[35] = 3.0 / 49.0 * r355;
  repd[36] = 1.0 / 49.0 * r266 + 30.0 / 441.0 * r466;
  repd[37] = s3 / 49.0 * r266 - 5.0 * s3 / 441.0 * r466;
  repd[38] = r066 - 2.0 / 49.0 * r266 - 4.0 / 441.0 * r466;
  repd[39] = -2.0 * s3 / 49.0 * r266 + 10.0 * s3 / 441.0 * r466;
  repd[40] = -repd[32];
  repd[41] = -repd[34];
  repd[42] = -repd[35];
  repd[43] = -repd[37];
  repd[44] = 3.0 / 49.0 * r266 + 20.0 / 441.0 * r466;
  repd[45] = -repd[39];
  repd[46] = 1.0 / 5.0 * r155 - 3.0 / 35.0 * r355;
  repd[47] = -repd[46];
  repd[48] = 4.0 / 49.0 * r266 + 15.0 / 441.0 * r466;
  repd[49] = 3.0 / 49.0 * r266 - 5.0 / 147.0 * r466;
  repd[50] = -repd[49];
  repd[51] = r066 + 4.0 / 49.0 * r266 - 34.0 / 441.0 * r466;
  repd[52] = 35.0 / 441.0 * r466;
}

// Thiel-Voityuk aijl (src/mndod.rs:502-512).
double aijl(const Fb &fb, double z1, double z2, int n1, int n2, int l) {
  double zz = z1 + z2 + 1.0e-20;
  return fb.fx[n1 + n2 + l + 1] / std::sqrt(fb.fx[2 * n1 + 1] * fb.fx[2 * n2 + 1]) *
         std::pow(2.0 * z1 / zz, n1) * std::sqrt(2.0 * z1 / zz) * std::pow(2.0 * z2 / zz, n2) *
         std::sqrt(2.0 * z2 / zz) * std::pow(2.0, l) / std::pow(zz, l);
}

// MOPAC poij golden-section search (src/mndod.rs:536-580).
double poij(int l, double d, double fg) {
  const double eps = 1.0e-8, g1 = 0.382, g2 = 0.618;
  if (l == 0) return 0.5 * EV / fg;
  double dsq = d * d, ev4 = EV * 0.25, ev8 = EV / 8.0;
  double a1 = 0.1, a2 = 5.0, f1 = 0.0, f2 = 0.0;
  for (int it = 0; it < 100; ++it) {
    double delta = a2 - a1;
    if (delta < eps) break;
    double y1 = a1 + delta * g1, y2 = a1 + delta * g2;
    if (l == 1) {
      double t1 = ev4 * (1.0 / y1 - 1.0 / std::sqrt(y1 * y1 + dsq)) - fg;
      double t2 = ev4 * (1.0 / y2 - 1.0 / std::sqrt(y2 * y2 + dsq)) - fg;
      f1 = t1 * t1;
      f2 = t2 * t2;
    } else {
      double t1 = ev8 * (1.0 / y1 - 2.0 / std::sqrt(y1 * y1 + dsq * 0.5) + 1.0 / std::sqrt(y1 * y1 + dsq)) - fg;
      double t2 = ev8 * (1.0 / y2 - 2.0 / std::sqrt(y2 * y2 + dsq * 0.5) + 1.0 / std::sqrt(y2 * y2 + dsq)) - fg;
      f1 = t1 * t1;
      f2 = t2 * t2;
    }
    if (f1 < f2) a2 = y2;
    else a1 = y1;
  }
  return f1 >= f2 ? a2 : a1;
}

// MOPAC wstore one-centre matrix (src/mndod.rs:704-735).
void build_onecenter(const Element &e, const double repd[53], std::vector<double> &w) {
  w.assign(45 * 45, 0.0);
  auto set = [&](int ij, int kl, double v) { w[(ij - 1) * 45 + (kl - 1)] = v; };
  set(1, 1, e.g_ss);
  for (int ip : {3, 6, 10}) {
    set(ip, 1, e.g_sp);
    set(1, ip, e.g_sp);
    set(ip, ip, e.g_pp);
  }
  const int off[6][2] = {{6, 3}, {10, 3}, {10, 6}, {3, 6}, {3, 10}, {6, 10}};
  for (auto &ab : off) set(ab[0], ab[1], e.g_p2);
  for (int p : {2, 4, 7}) set(p, p, e.h_sp);
  for (int p : {5, 8, 9}) set(p, p, 0.5 * (e.g_pp - e.g_p2));
  for (int i = 0; i < 243; ++i) set(MNDOD_INTIJ[i], MNDOD_INTKL[i], repd[MNDOD_INTREP[i]]);
}

// derive_dshell (src/mndod.rs:610-699).
DShell derive_dshell(const Element &e) {
  static const Fb fb;
  DShell d;
  bool has_d = e.zeta_d > 1.0e-20;
  // aijm (src/mndod.rs:515-533)
  if (e.z >= 3 && !(e.zeta_s * e.zeta_p < 0.01)) {
    int nsp = iii(e.z);
    d.aij[2] = aijl(fb, e.zeta_s, e.zeta_p, nsp, nsp, 1);
    d.aij[3] = aijl(fb, e.zeta_p, e.zeta_p, nsp, nsp, 2);
    if (has_d) {
      int nd = iiid(e.z);
      d.aij[4] = aijl(fb, e.zeta_s, e.zeta_d, nsp, nd, 2);
      d.aij[5] = aijl(fb, e.zeta_p, e.zeta_d, nsp, nd, 1);
      d.aij[6] = aijl(fb, e.zeta_d, e.zeta_d, nd, nd, 2);
    }
  }
  if (has_d && e.zdn > 1.0e-4) inighd(fb, e.z, e.zsn, e.zpn, e.zdn, e.f0sd, e.g2sd, d.repd, d.eiscor);
  if (e.g_ss > 0.1) d.po[1] = poij(0, 1.0, e.g_ss);
  if (e.z >= 3) {
    double dd = d.aij[2] / std::sqrt(12.0);
    d.ddp[2] = dd;
    d.po[2] = poij(1, dd, e.h_sp);
    d.po[7] = d.po[1];
    dd = std::sqrt(d.aij[3] * 0.1);
    d.ddp[3] = dd;
    d.po[3] = poij(2, dd, 0.5 * (e.g_pp - e.g_p2));
    if (has_d) {
      double da = std::sqrt(1.0 / 60.0);
      dd = std::sqrt(d.aij[4] * da);
      d.ddp[4] = dd;
      d.po[4] = poij(2, dd, d.repd[19]);
      dd = d.aij[5] / std::sqrt(20.0);
      d.ddp[5] = dd;
      d.po[5] = poij(1, dd, d.repd[23] - 1.8 * d.repd[35]);
      double fg = 0.2 * (d.repd[29] + 2.0 * d.repd[30] + 2.0 * d.repd[31]);
      d.po[8] = fg > 1.0e-5 ? poij(0, 1.0, fg) : 1.0e5;
      dd = std::sqrt(d.aij[6] / 14.0);
      d.ddp[6] = dd;
      d.po[6] = poij(2, dd, d.repd[44] - (20.0 / 35.0) * d.repd[52]);
    }
  }
  if (main_group(e.z) || !has_d) {
    d.po[1] = e.rho0;
    if (e.rho1 > 1.0e-5) d.po[2] = e.rho1;
    if (e.rho2 > 1.0e-5) d.po[3] = e.rho2;
    d.po[7] = d.po[1];
    d.ddp[2] = e.dd;
    d.ddp[3] = e.qq * std::sqrt(2.0);
  }
  d.po[9] = e.poc > 1.0e-5 ? e.poc : d.po[1];
  d.has_d = has_d;
  if (has_d) build_onecenter(e, d.repd, d.onecenter);
  return d;
}

// `from_tables` element rows (src/params.rs:229-411).
Element element_from_row(const double *r) {
  Element e;
  e.z = (int)r[C_Z];
  e.n = (int)r[C_N];
  e.ios = (int)r[C_IOS];
  e.iop = (int)r[C_IOP];
  e.iod = (int)r[C_IOD];
  e.zeta_s = r[C_ZS];
  e.zeta_p = r[C_ZP];
  e.zeta_d = r[C_ZD];
  e.n_orb = e.zeta_d > 1.0e-20 ? 9 : (e.zeta_p > 1.0e-20 ? 4 : 1);
  e.g_ss = r[C_GSS];
  e.g_sp = r[C_GSP];
  e.g_pp = r[C_GPP];
  e.g_p2 = r[C_GP2];
  e.h_sp = r[C_HSP];
  if (e.n_orb >= 4) {
    e.dd = dd_charge_sep(e.n, e.zeta_s, std::max(e.zeta_p, 0.3));
    e.qq = qq_charge_sep(e.n, std::max(e.zeta_p, 0.3));
    e.rho1 = additive_rho1(std::max(e.h_sp, 1.0e-7), e.dd);
    e.rho2 = additive_rho2(std::max(0.5 * (e.g_pp - e.g_p2), 0.1), e.qq);
  }
  for (int slot = 0; slot < 4; ++slot) {
    double k = r[C_G1_1 + slot], l = r[C_G2_1 + slot], m = r[C_G3_1 + slot];
    if (k != 0.0 || l != 0.0 || m != 0.0) e.gauss.push_back({k, l, m});
  }
  double gssc = (double)std::max(e.ios - 1, 0);
  double p = e.iop;
  double l = std::min(p, 6.0 - p);
  double gspc = e.ios * p;
  double gp2c = p * (p - 1.0) / 2.0 + 0.5 * l * (l - 1.0) / 2.0;
  double gppc = -0.5 * l * (l - 1.0) / 2.0;
  double hspc = -p * e.ios * 0.5;
  e.u_ss = r[C_USS];
  e.u_pp = r[C_UPP];
  e.u_dd = r[C_UDD];
  e.e_isol = e.u_ss * e.ios + e.u_pp * p + e.u_dd * e.iod + e.g_ss * gssc + e.g_pp * gppc +
             e.g_sp * gspc + e.g_p2 * gp2c + e.h_sp * hspc;
  e.beta_s = r[C_BS];
  e.beta_p = r[C_BP];
  e.beta_d = r[C_BD];
  e.zsn = r[C_ZSN];
  e.zpn = r[C_ZPN];
  e.zdn = r[C_ZDN];
  e.f0sd = r[C_F0SD];
  e.g2sd = r[C_G2SD];
  e.poc = r[C_POC];
  e.alpha = r[C_ALPHA];
  e.polvol = r[C_POLVOL];
  e.core_charge = r[C_CORE];
  e.eheat_ev = r[C_EHEAT] * KCAL_TO_EV;
  e.rho0 = e.g_ss != 0.0 ? EV / (2.0 * e.g_ss) : 0.0;
  e.dshell = derive_dshell(e);
  e.has_dshell = true;
  e.e_isol += e.dshell.eiscor;
  return e;
}

std::pair<int, int> ordered(int a, int b) { return {std::max(a, b), std::min(a, b)}; }

Params parse(int method) {
  Params p;
  p.method = method;
  const double(*el)[PM7_ELEMENT_NCOL] = method == PM7_METHOD_PM7_TS ? PM7TS_ELEMENTS : PM7_ELEMENTS;
  int nel = method == PM7_METHOD_PM7_TS ? PM7TS_ELEMENTS_ROWS : PM7_ELEMENTS_ROWS;
  for (int i = 0; i < nel; ++i) {
    const double *r = el[i];
    if (r[C_ZS] == 0.0 && r[C_BS] == 0.0) continue;
    Element e = element_from_row(r);
    p.elements[e.z] = e;
  }
  const double(*pr)[4] = method == PM7_METHOD_PM7_TS ? PM7TS_PAIRS : PM7_PAIRS;
  int npr = method == PM7_METHOD_PM7_TS ? PM7TS_PAIRS_ROWS : PM7_PAIRS_ROWS;
  for (int i = 0; i < npr; ++i)
    p.pairs[ordered((int)pr[i][0], (int)pr[i][1])] = PairParam{pr[i][2], pr[i][3]};
  const double(*vp)[2] = method == PM7_METHOD_PM7_TS ? PM7TS_VPAR : PM7_VPAR;
  int nvp = method == PM7_METHOD_PM7_TS ? PM7TS_VPAR_ROWS : PM7_VPAR_ROWS;
  for (int i = 0; i < nvp; ++i) {
    int idx = (int)vp[i][0];
    if (idx >= 1 && idx <= 60) p.vpar_table[idx - 1] = vp[i][1];
  }
  if (method == PM7_METHOD_PM7_SPARKLE) {
    // install_sparkles (src/params.rs:339-438)
    static const double eheat_sparkle[15] = {928.9, 944.7, 952.9, 962.8, 976.9, 974.4, 1006.6, 991.37,
                                             999.0, 1001.3, 1009.6, 1016.15, 1022.06, 1039.03, 1031.2};
    for (int i = 0; i < PM7_SPARKLES_ROWS; ++i) {
      const double *r = PM7_SPARKLES[i];
      int z = (int)r[0];
      if (z < 57 || z > 71) continue;
      Element e;
      e.z = z;
      e.n = 6;
      e.n_orb = 0;
      e.core_charge = 3.0;
      e.alpha = r[1];
      e.g_ss = r[2];
      e.gauss.push_back({r[3], r[4], r[5]});
      e.gauss.push_back({r[6], r[7], r[8]});
      e.rho0 = EV / (2.0 * e.g_ss);
      e.eheat_ev = eheat_sparkle[z - 57] * KCAL_TO_EV;
      e.is_sparkle = true;
      e.has_dshell = false;
      p.elements[z] = e;
    }
    for (auto it = p.pairs.begin(); it != p.pairs.end();) {
      int a = it->first.first, b = it->first.second;
      if ((a >= 57 && a <= 71) || (b >= 57 && b <= 71)) it = p.pairs.erase(it);
      else ++it;
    }
  }
  return p;
}

}  // namespace

const Element &Params::element(int z) const {
  auto it = elements.find(z);
  if (it == elements.end())
    throw Error(PM7_ERR_MISSING_ELEMENT, "missing PM7 parameter block for Z=" + std::to_string(z));
  return it->second;
}

// src/params.rs:168-192
PairParam Params::pair(int zi, int zj) const {
  auto it = pairs.find(ordered(zi, zj));
  if (it != pairs.end()) return it->second;
  PairParam ii, jj;
  auto a = pairs.find(ordered(zi, zi));
  if (a != pairs.end()) ii = a->second;
  auto b = pairs.find(ordered(zj, zj));
  if (b != pairs.end()) jj = b->second;
  return PairParam{0.5 * (ii.alpb + jj.alpb), 0.5 * (ii.xfac + jj.xfac)};
}

const Params &params_for(int method) {
  static std::mutex mu;
  static std::map<int, Params> cache;
  std::lock_guard<std::mutex> g(mu);
  int table = method;
  auto it = cache.find(table);
  if (it == cache.end()) it = cache.emplace(table, parse(method)).first;
  return it->second;
}

Basis build_basis(const Molecule &mol, const Params &p) {
  Basis b;
  for (int ia = 0; ia < mol.size(); ++ia) {
    const Element &e = p.element(mol.z[ia]);
    b.atom_offset.push_back(b.nao);
    b.atom_norb.push_back(e.n_orb);
    for (int o = 0; o < e.n_orb; ++o) {
      b.ao_atom.push_back(ia);
      b.ao_orb.push_back(o);
    }
    b.nao += e.n_orb;
  }
  return b;
}

}  // namespace oracle
