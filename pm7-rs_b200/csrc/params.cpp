// Host-side parameter set: parses the PM7 tables and derives the NDDO multipole
// quantities once per method, then mirrors them to the device.
//
// Follows pm7-rs src/params.rs (`from_tables`, `calpar` secant, `ddpo`) and the
// geometry-independent part of src/mndod.rs (`derive_dshell`: aijm, inighd/rsc,
// eiscor, poij, wstore).
#include "params.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "pm7_param_data.h"

namespace pm7 {
namespace {

// Column positions of the element table (gen_param_data.py ELEMENT_COLUMNS).
struct Cols {
  enum {
    z, n, ios, iop, iod, core, eheat, uss, upp, udd, zs, zp, zd, bs, bp, bd, gss, gsp, gpp, gp2, hsp, zsn, zpn,
    zdn, f0sd, g2sd, alpha, poc, polvol, g1, g2 = g1 + 4, g3 = g2 + 4
  };
};

double powi(double x, int k) {
  double r = 1.0;
  for (int i = 0; i < k; ++i) r *= x;
  return r;
}

// Five fixed secant steps from `x0` (pm7-rs src/params.rs:512-525, MOPAC calpar).
template <class Fn>
double secant5(double target, double x0, Fn fn) {
  double a = x0, b = x0 + 0.04;
  for (int step = 0; step < 5; ++step) {
    double fa = fn(a), fb = fn(b);
    if (std::fabs(fb - fa) < 1.0e-25) break;
    double c = a + (b - a) * (target - fa) / (fb - fa);
    a = b;
    b = c;
  }
  return b;
}

double sgn(double x) { return std::signbit(x) ? -1.0 : 1.0; }

struct Radial {
  double fact[31];      // fact[i] = (i-1)!
  double binom[31][31]; // binom[i][j] = C(i-1, j-1)
  Radial() {
    std::memset(fact, 0, sizeof fact);
    std::memset(binom, 0, sizeof binom);
    fact[1] = 1.0;
    for (int i = 2; i <= 30; ++i) fact[i] = fact[i - 1] * (i - 1);
    for (int i = 0; i <= 30; ++i) binom[i][1] = 1.0;
    for (int i = 2; i <= 30; ++i)
      for (int j = 2; j <= i; ++j) binom[i][j] = binom[i - 1][j - 1] + binom[i - 1][j];
  }
  // One-centre radial integral of multipole order k over four Slater functions (MOPAC rsc).
  double rsc(int k, int na, double ea, int nb, double eb, int nc, double ec, int nd, double ed) const {
    const int nab = na + nb, ncd = nc + nd, n = nab + ncd;
    const double eab = ea + eb, ecd = ec + ed, e = eab + ecd;
    const double lea = std::log(ea), leb = std::log(eb), lec = std::log(ec), led = std::log(ed);
    const double le = std::log(e), lecd = std::log(ecd), leab = std::log(eab);
    const double norm = fact[n] / std::sqrt(fact[2 * na + 1] * fact[2 * nb + 1] * fact[2 * nc + 1] * fact[2 * nd + 1]);
    const double pre = kEv * norm *
                       std::exp(na * lea + nb * leb + nc * lec + nd * led + 0.5 * (lea + leb + lec + led) +
                                std::log(2.0) * (n + 2.0) - le * n);
    double t = 1.0 / e, s1 = 0.0, s2 = 0.0;
    const int m = ncd - k;
    for (int i = 1; i <= m; ++i) {
      t *= e / ecd;
      s1 += t * (binom[ncd - k][i] - binom[ncd + k + 1][i]) / binom[n][i];
    }
    const int top = ncd + k + 1;
    for (int i = m + 1; i <= top; ++i) {
      t *= e / ecd;
      s2 += t * binom[top][i] / binom[n][i];
    }
    const double s3 = std::exp(le * n - lecd * top - leab * (nab - k)) / binom[n][top];
    return pre * (s1 - s2 + s3);
  }
  double aij(double z1, double z2, int n1, int n2, int l) const {
    const double zz = z1 + z2 + 1.0e-20;
    return fact[n1 + n2 + l + 1] / std::sqrt(fact[2 * n1 + 1] * fact[2 * n2 + 1]) * std::pow(2.0 * z1 / zz, n1) *
           std::sqrt(2.0 * z1 / zz) * std::pow(2.0 * z2 / zz, n2) * std::sqrt(2.0 * z2 / zz) * std::pow(2.0, l) /
           std::pow(zz, l);
  }
};

int shell_n_sp(int z) { return z <= 0 ? 0 : z <= 2 ? 1 : z <= 10 ? 2 : z <= 18 ? 3 : z <= 36 ? 4 : z <= 54 ? 5 : z <= 86 ? 6 : 0; }
int shell_n_d(int z) { return z <= 0 ? 0 : z <= 30 ? 3 : z <= 48 ? 4 : z <= 80 ? 5 : z <= 86 ? 6 : 0; }
bool is_transition_metal(int z) { return (z >= 21 && z <= 29) || (z >= 39 && z <= 47) || (z >= 57 && z <= 79); }

// Golden-section Klopman-Ohno additive term for multipole order l (MOPAC poij).
double additive_term(int l, double d, double fg) {
  if (l == 0) return 0.5 * kEv / fg;
  const double d2 = d * d;
  auto err = [&](double y) {
    double v = (l == 1) ? (kEv * 0.25) * (1.0 / y - 1.0 / std::sqrt(y * y + d2))
                        : (kEv / 8.0) * (1.0 / y - 2.0 / std::sqrt(y * y + d2 * 0.5) + 1.0 / std::sqrt(y * y + d2));
    v -= fg;
    return v * v;
  };
  double lo = 0.1, hi = 5.0, flo = 0.0, fhi = 0.0;
  for (int it = 0; it < 100; ++it) {
    double span = hi - lo;
    if (span < 1.0e-8) break;
    double y1 = lo + span * 0.382, y2 = lo + span * 0.618;
    flo = err(y1);
    fhi = err(y2);
    if (flo < fhi) hi = y2;
    else lo = y1;
  }
  return flo >= fhi ? hi : lo;
}

// Reference-configuration d-shell occupation weights of MOPAC eiscor.
const int kEiscorTable[][6] = {
    {21, 2, 0, 1, 0, 0},   {22, 4, 1, 2, 8, 1},    {23, 6, 3, 3, 15, 8},   {24, 5, 10, 5, 35, 35},
    {25, 10, 10, 5, 35, 35}, {26, 12, 15, 6, 35, 35}, {27, 14, 21, 7, 43, 36}, {28, 16, 28, 8, 50, 43},
    {29, 10, 45, 5, 70, 70}, {39, 2, 0, 1, 0, 0},    {40, 4, 1, 2, 8, 1},    {41, 4, 6, 4, 21, 21},
    {42, 5, 10, 5, 35, 35}, {43, 10, 10, 5, 35, 35}, {44, 7, 21, 5, 43, 36}, {45, 8, 28, 5, 50, 43},
    {46, 0, 45, 0, 70, 70}, {47, 10, 45, 5, 70, 70}, {57, 2, 0, 1, 0, 0},    {71, 2, 0, 1, 0, 0},
    {72, 4, 1, 2, 8, 1},    {73, 6, 3, 3, 15, 8},   {74, 5, 10, 5, 35, 35}, {75, 10, 10, 5, 35, 35},
    {76, 12, 15, 6, 35, 35}, {77, 14, 21, 7, 43, 36}, {78, 9, 36, 5, 56, 56}, {79, 10, 45, 5, 70, 70}};

// repd(1..52) from the radial Slater-Condon parameters (MOPAC inighd), and eiscor.
void one_centre_d(const Radial &R, ElementRec &e, double zsn, double zpn, double zdn, double f0sd, double g2sd,
                  double &eis) {
  const int ns = shell_n_sp(e.z), nd = shell_n_d(e.z);
  const double s3 = 1.7320508, s5 = 2.23606797, s15 = 3.87298334;
  double F0sd = R.rsc(0, ns, zsn, ns, zsn, nd, zdn, nd, zdn);
  const double F0pd = R.rsc(0, ns, zpn, ns, zpn, nd, zdn, nd, zdn);
  const double F0dd = R.rsc(0, nd, zdn, nd, zdn, nd, zdn, nd, zdn);
  const double G1pd = R.rsc(1, ns, zpn, nd, zdn, ns, zpn, nd, zdn);
  const double R1sppd = R.rsc(1, ns, zsn, ns, zpn, ns, zpn, nd, zdn);
  double G2sd = R.rsc(2, ns, zsn, nd, zdn, ns, zsn, nd, zdn);
  const double F2pd = R.rsc(2, ns, zpn, ns, zpn, nd, zdn, nd, zdn);
  const double F2dd = R.rsc(2, nd, zdn, nd, zdn, nd, zdn, nd, zdn);
  const double R2sdpp = R.rsc(2, ns, zpn, ns, zpn, ns, zsn, nd, zdn);
  const double R2sddd = R.rsc(2, ns, zsn, nd, zdn, nd, zdn, nd, zdn);
  const double G3pd = R.rsc(3, ns, zpn, nd, zdn, ns, zpn, nd, zdn);
  const double F4dd = R.rsc(4, nd, zdn, nd, zdn, nd, zdn, nd, zdn);
  if (f0sd > 0.001) F0sd = f0sd;
  if (g2sd > 0.001) G2sd = g2sd;
  int w[5] = {0, 0, 0, 0, 0};
  for (const auto &row : kEiscorTable)
    if (row[0] == e.z)
      for (int k = 0; k < 5; ++k) w[k] = row[k + 1];
  eis = w[0] * F0sd + w[1] * F0dd - w[2] * G2sd / 5.0 - w[3] * F2dd / 49.0 - w[4] * F4dd / 49.0;
  double *r = e.repd;
  for (int i = 0; i < 53; ++i) r[i] = 0.0;
  r[1] = F0sd;
  r[2] = 2.0 / (3.0 * s5) * R1sppd;
  r[3] = 1.0 / s15 * R1sppd;
  r[4] = 2.0 / (5.0 * s5) * R2sdpp;
  r[5] = F0pd + 4.0 / 35.0 * F2pd;
  r[6] = F0pd + 2.0 / 35.0 * F2pd;
  r[7] = F0pd - 4.0 / 35.0 * F2pd;
  r[8] = -1.0 / (3.0 * s5) * R1sppd;
  r[9] = std::sqrt(3.0 / 125.0) * R2sdpp;
  r[10] = s3 / 35.0 * F2pd;
  r[11] = 3.0 / 35.0 * F2pd;
  r[12] = -1.0 / (5.0 * s5) * R2sdpp;
  r[13] = F0pd - 2.0 / 35.0 * F2pd;
  r[14] = -2.0 * s3 / 35.0 * F2pd;
  r[15] = -r[3];
  r[16] = -r[11];
  r[17] = -r[9];
  r[18] = -r[14];
  r[19] = 1.0 / 5.0 * G2sd;
  r[20] = 2.0 / (7.0 * s5) * R2sddd;
  r[21] = r[20] / 2.0;
  r[22] = -r[20];
  r[23] = 4.0 / 15.0 * G1pd + 27.0 / 245.0 * G3pd;
  r[24] = 2.0 * s3 / 15.0 * G1pd - 9.0 * s3 / 245.0 * G3pd;
  r[25] = 1.0 / 15.0 * G1pd + 18.0 / 245.0 * G3pd;
  r[26] = -s3 / 15.0 * G1pd + 12.0 * s3 / 245.0 * G3pd;
  r[27] = -s3 / 15.0 * G1pd - 3.0 * s3 / 245.0 * G3pd;
  r[28] = -r[27];
  r[29] = F0dd + 4.0 / 49.0 * F2dd + 4.0 / 49.0 * F4dd;
  r[30] = F0dd + 2.0 / 49.0 * F2dd - 24.0 / 441.0 * F4dd;
  r[31] = F0dd - 4.0 / 49.0 * F2dd + 6.0 / 441.0 * F4dd;
  r[32] = std::sqrt(3.0 / 245.0) * R2sddd;
  r[33] = 1.0 / 5.0 * G1pd + 24.0 / 245.0 * G3pd;
  r[34] = 1.0 / 5.0 * G1pd - 6.0 / 245.0 * G3pd;
  r[35] = 3.0 / 49.0 * G3pd;
  r[36] = 1.0 / 49.0 * F2dd + 30.0 / 441.0 * F4dd;
  r[37] = s3 / 49.0 * F2dd - 5.0 * s3 / 441.0 * F4dd;
  r[38] = F0dd - 2.0 / 49.0 * F2dd - 4.0 / 441.0 * F4dd;
  r[39] = -2.0 * s3 / 49.0 * F2dd + 10.0 * s3 / 441.0 * F4dd;
  r[40] = -r[32];
  r[41] = -r[34];
  r[42] = -r[35];
  r[43] = -r[37];
  r[44] = 3.0 / 49.0 * F2dd + 20.0 / 441.0 * F4dd;
  r[45] = -r[39];
  r[46] = 1.0 / 5.0 * G1pd - 3.0 / 35.0 * G3pd;
  r[47] = -r[46];
  r[48] = 4.0 / 49.0 * F2dd + 15.0 / 441.0 * F4dd;
  r[49] = 3.0 / 49.0 * F2dd - 5.0 / 147.0 * F4dd;
  r[50] = -r[49];
  r[51] = F0dd + 4.0 / 49.0 * F2dd - 34.0 / 441.0 * F4dd;
  r[52] = 35.0 / 441.0 * F4dd;
}

// MNDO/d additive terms and charge separations of one element (MOPAC inid).
void derive_multipoles(const Radial &R, ElementRec &e, const double *row, std::vector<double> &onecenter_store) {
  const bool has_d = e.zeta_d > 1.0e-20;
  double aij[7] = {0, 0, 0, 0, 0, 0, 0};
  if (e.z >= 3 && e.zeta_s * e.zeta_p >= 0.01) {
    const int nsp = shell_n_sp(e.z);
    aij[2] = R.aij(e.zeta_s, e.zeta_p, nsp, nsp, 1);
    aij[3] = R.aij(e.zeta_p, e.zeta_p, nsp, nsp, 2);
    if (has_d) {
      const int nd = shell_n_d(e.z);
      aij[4] = R.aij(e.zeta_s, e.zeta_d, nsp, nd, 2);
      aij[5] = R.aij(e.zeta_p, e.zeta_d, nsp, nd, 1);
      aij[6] = R.aij(e.zeta_d, e.zeta_d, nd, nd, 2);
    }
  }
  double eis = 0.0;
  for (double &v : e.repd) v = 0.0;
  if (has_d && row[Cols::zdn] > 1.0e-4)
    one_centre_d(R, e, row[Cols::zsn], row[Cols::zpn], row[Cols::zdn], row[Cols::f0sd], row[Cols::g2sd], eis);
  for (double &v : e.po) v = 0.0;
  for (double &v : e.ddp) v = 0.0;
  if (e.g_ss > 0.1) e.po[1] = additive_term(0, 1.0, e.g_ss);
  if (e.z >= 3) {
    e.ddp[2] = aij[2] / std::sqrt(12.0);
    e.po[2] = additive_term(1, e.ddp[2], e.h_sp);
    e.po[7] = e.po[1];
    e.ddp[3] = std::sqrt(aij[3] * 0.1);
    e.po[3] = additive_term(2, e.ddp[3], 0.5 * (e.g_pp - e.g_p2));
    if (has_d) {
      e.ddp[4] = std::sqrt(aij[4] * std::sqrt(1.0 / 60.0));
      e.po[4] = additive_term(2, e.ddp[4], e.repd[19]);
      e.ddp[5] = aij[5] / std::sqrt(20.0);
      e.po[5] = additive_term(1, e.ddp[5], e.repd[23] - 1.8 * e.repd[35]);
      const double fg = 0.2 * (e.repd[29] + 2.0 * e.repd[30] + 2.0 * e.repd[31]);
      e.po[8] = fg > 1.0e-5 ? additive_term(0, 1.0, fg) : 1.0e5;
      e.ddp[6] = std::sqrt(aij[6] / 14.0);
      e.po[6] = additive_term(2, e.ddp[6], e.repd[44] - (20.0 / 35.0) * e.repd[52]);
    }
  }
  if (!is_transition_metal(e.z) || !has_d) {
    e.po[1] = e.rho0;
    if (e.rho1 > 1.0e-5) e.po[2] = e.rho1;
    if (e.rho2 > 1.0e-5) e.po[3] = e.rho2;
    e.po[7] = e.po[1];
    e.ddp[2] = e.dd;
    e.ddp[3] = e.qq * std::sqrt(2.0);
  }
  e.po[9] = e.poc > 1.0e-5 ? e.poc : e.po[1];
  e.e_isol += eis;
  e.onecenter_slot = -1;
  if (has_d) {
    // 45x45 one-centre integral matrix (MOPAC wstore), indexed by 1-based pair indices.
    const size_t base = onecenter_store.size();
    onecenter_store.resize(base + 2025, 0.0);
    double *w = &onecenter_store[base];
    auto put = [w](int ij, int kl, double v) { w[(ij - 1) * 45 + (kl - 1)] = v; };
    put(1, 1, e.g_ss);
    for (int p : {3, 6, 10}) {
      put(p, 1, e.g_sp);
      put(1, p, e.g_sp);
      put(p, p, e.g_pp);
    }
    for (int a : {3, 6, 10})
      for (int b : {3, 6, 10})
        if (a != b) put(a, b, e.g_p2);
    for (int p : {2, 4, 7}) put(p, p, e.h_sp);
    for (int p : {5, 8, 9}) put(p, p, 0.5 * (e.g_pp - e.g_p2));
    for (int i = 0; i < 243; ++i) put(MNDOD_INTIJ[i], MNDOD_INTKL[i], e.repd[MNDOD_INTREP[i]]);
    e.onecenter_slot = (int32_t)(base / 2025);
  }
}

ElementRec element_from_row(const double *row, const Radial &R, std::vector<double> &onecenter_store) {
  ElementRec e;
  std::memset(&e, 0, sizeof e);
  e.present = 1;
  e.z = (int)row[Cols::z];
  e.n = (int)row[Cols::n];
  e.ios = (int)row[Cols::ios];
  e.iop = (int)row[Cols::iop];
  const int iod = (int)row[Cols::iod];
  e.iod = iod;
  e.core = row[Cols::core];
  e.u_ss = row[Cols::uss];
  e.u_pp = row[Cols::upp];
  e.u_dd = row[Cols::udd];
  e.zeta_s = row[Cols::zs];
  e.zeta_p = row[Cols::zp];
  e.zeta_d = row[Cols::zd];
  e.beta_s = row[Cols::bs];
  e.beta_p = row[Cols::bp];
  e.beta_d = row[Cols::bd];
  e.g_ss = row[Cols::gss];
  e.g_sp = row[Cols::gsp];
  e.g_pp = row[Cols::gpp];
  e.g_p2 = row[Cols::gp2];
  e.h_sp = row[Cols::hsp];
  e.poc = row[Cols::poc];
  e.n_orb = e.zeta_d > 1.0e-20 ? 9 : e.zeta_p > 1.0e-20 ? 4 : 1;
  if (e.n_orb >= 4) {
    // Dipole and quadrupole charge separations (MOPAC ddpo) and their additive terms (calpar).
    const double zp = std::max(e.zeta_p, 0.3), nn = e.n;
    e.dd = (2.0 * nn + 1.0) * std::pow(4.0 * e.zeta_s * zp, nn + 0.5) / std::pow(e.zeta_s + zp, 2.0 * nn + 2.0) /
           std::sqrt(3.0);
    e.qq = std::sqrt((4.0 * nn * nn + 6.0 * nn + 2.0) / 20.0) / zp;
    const double dd = e.dd, qq = e.qq;
    const double hsp = std::max(e.h_sp, 1.0e-7) / kEv;
    const double d1 = secant5(hsp, std::pow(std::fabs(hsp) / (dd * dd), 1.0 / 3.0) * sgn(hsp), [dd](double x) {
      return 0.5 * x - 0.5 / std::sqrt(4.0 * dd * dd + 1.0 / (x * x));
    });
    e.rho1 = 0.5 / d1;
    const double hpp = std::max(0.5 * (e.g_pp - e.g_p2), 0.1) / kEv;
    const double d2 = secant5(hpp, std::pow(std::fabs(hpp) / (3.0 * powi(qq, 4)), 0.2) * sgn(hpp), [qq](double x) {
      return 0.25 * x - 0.5 / std::sqrt(4.0 * qq * qq + 1.0 / (x * x)) + 0.25 / std::sqrt(8.0 * qq * qq + 1.0 / (x * x));
    });
    e.rho2 = 0.5 / d2;
  }
  e.rho0 = e.g_ss != 0.0 ? kEv / (2.0 * e.g_ss) : 0.0;
  e.n_gauss = 0;
  for (int s = 0; s < 4; ++s) {
    const double k = row[Cols::g1 + s], l = row[Cols::g2 + s], m = row[Cols::g3 + s];
    if (k != 0.0 || l != 0.0 || m != 0.0) {
      e.gauss[e.n_gauss][0] = k;
      e.gauss[e.n_gauss][1] = l;
      e.gauss[e.n_gauss][2] = m;
      ++e.n_gauss;
    }
  }
  // Isolated-atom energy from the ground-state occupations (MOPAC calpar).
  const double p = e.iop, l = std::min(p, 6.0 - p);
  e.e_isol = e.u_ss * e.ios + e.u_pp * p + e.u_dd * iod + e.g_ss * std::max(e.ios - 1, 0) +
             e.g_pp * (-0.5 * l * (l - 1.0) / 2.0) + e.g_sp * (e.ios * p) +
             e.g_p2 * (p * (p - 1.0) / 2.0 + 0.5 * l * (l - 1.0) / 2.0) + e.h_sp * (-p * e.ios * 0.5);
  e.eheat_ev = row[Cols::eheat] * kKcalToEv;
  derive_multipoles(R, e, row, onecenter_store);
  return e;
}

}  // namespace

ParamSet::ParamSet(int method) : method_(method) {
  const Radial R;
  elements_.assign(kMaxZ, ElementRec{});
  for (auto &e : elements_) std::memset(&e, 0, sizeof e);
  const bool ts = method == 1;
  const double(*rows)[PM7_ELEMENT_NCOL] = ts ? PM7TS_ELEMENTS : PM7_ELEMENTS;
  const int nrows = ts ? PM7TS_ELEMENTS_ROWS : PM7_ELEMENTS_ROWS;
  for (int i = 0; i < nrows; ++i) {
    const double *row = rows[i];
    if (row[Cols::zs] == 0.0 && row[Cols::bs] == 0.0) continue;  // no PM7 parameters
    ElementRec e = element_from_row(row, R, onecenter_);
    if (e.z > 0 && e.z < kMaxZ) elements_[e.z] = e;
  }
  // Pair core-core parameters; missing pairs take the average of the two diagonal entries.
  std::vector<PairParamRec> explicit_pairs((size_t)kMaxZ * kMaxZ, PairParamRec{0.0, 0.0});
  std::vector<char> have((size_t)kMaxZ * kMaxZ, 0);
  const double(*prs)[4] = ts ? PM7TS_PAIRS : PM7_PAIRS;
  const int nprs = ts ? PM7TS_PAIRS_ROWS : PM7_PAIRS_ROWS;
  for (int i = 0; i < nprs; ++i) {
    const int a = (int)prs[i][0], b = (int)prs[i][1];
    if (a <= 0 || b <= 0 || a >= kMaxZ || b >= kMaxZ) continue;
    const int hi = std::max(a, b), lo = std::min(a, b);
    explicit_pairs[(size_t)hi * kMaxZ + lo] = PairParamRec{prs[i][2], prs[i][3]};
    have[(size_t)hi * kMaxZ + lo] = 1;
  }
  if (method == 2) {
    // PM7 SPARKLE: La..Lu become +3 point cores without orbitals, and lose their pair entries.
    static const double sparkle_heat_kcal[15] = {928.9, 944.7, 952.9, 962.8, 976.9, 974.4, 1006.6, 991.37,
                                                 999.0, 1001.3, 1009.6, 1016.15, 1022.06, 1039.03, 1031.2};
    for (int i = 0; i < PM7_SPARKLES_ROWS; ++i) {
      const double *r = PM7_SPARKLES[i];
      const int z = (int)r[0];
      if (z < 57 || z > 71) continue;
      ElementRec e;
      std::memset(&e, 0, sizeof e);
      e.present = 1;
      e.z = z;
      e.n = 6;
      e.n_orb = 0;
      e.is_sparkle = 1;
      e.core = 3.0;
      e.g_ss = r[2];
      e.rho0 = kEv / (2.0 * e.g_ss);
      e.n_gauss = 2;
      for (int k = 0; k < 3; ++k) {
        e.gauss[0][k] = r[3 + k];
        e.gauss[1][k] = r[6 + k];
      }
      e.eheat_ev = sparkle_heat_kcal[z - 57] * kKcalToEv;
      e.onecenter_slot = -1;
      elements_[z] = e;
    }
    for (int a = 0; a < kMaxZ; ++a)
      for (int b = 0; b <= a; ++b)
        if ((a >= 57 && a <= 71) || (b >= 57 && b <= 71)) have[(size_t)a * kMaxZ + b] = 0;
  }
  pairs_.assign((size_t)kMaxZ * kMaxZ, PairParamRec{0.0, 0.0});
  for (int a = 0; a < kMaxZ; ++a)
    for (int b = 0; b < kMaxZ; ++b) {
      const int hi = std::max(a, b), lo = std::min(a, b);
      PairParamRec v{0.0, 0.0};
      if (have[(size_t)hi * kMaxZ + lo]) {
        v = explicit_pairs[(size_t)hi * kMaxZ + lo];
      } else {
        PairParamRec aa = have[(size_t)a * kMaxZ + a] ? explicit_pairs[(size_t)a * kMaxZ + a] : PairParamRec{0, 0};
        PairParamRec bb = have[(size_t)b * kMaxZ + b] ? explicit_pairs[(size_t)b * kMaxZ + b] : PairParamRec{0, 0};
        v = PairParamRec{0.5 * (aa.alpb + bb.alpb), 0.5 * (aa.xfac + bb.xfac)};
      }
      pairs_[(size_t)a * kMaxZ + b] = v;
    }
  for (double &v : vpar_) v = 0.0;
  const double(*vp)[2] = ts ? PM7TS_VPAR : PM7_VPAR;
  const int nvp = ts ? PM7TS_VPAR_ROWS : PM7_VPAR_ROWS;
  for (int i = 0; i < nvp; ++i) {
    const int idx = (int)vp[i][0];
    if (idx >= 1 && idx <= 60) vpar_[idx] = vp[i][1];
  }
}

const ElementRec *ParamSet::element(int z) const {
  if (z <= 0 || z >= kMaxZ || !elements_[z].present) return nullptr;
  return &elements_[z];
}

namespace {

// Legendre polynomial P_n and its derivative by the three-term recurrence.
void legendre(int n, double x, double &p, double &dp) {
  double p0 = 1.0, p1 = x;
  for (int k = 2; k <= n; ++k) {
    const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  p = p1;
  dp = n * (x * p1 - p0) / (x * x - 1.0);
}

// n-point Gauss-Legendre rule on [-1, 1]: Newton iteration from the Chebyshev guess
// (the rule pm7-rs src/overlap_numeric.rs:134-159 uses for the heavy-shell overlaps).
void gauss_legendre(int n, double *t, double *w) {
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p, dp;
      legendre(n, x, p, dp);
      const double dx = -p / dp;
      x += dx;
      if (std::fabs(dx) < 1.0e-15) break;
    }
    double p, dp;
    legendre(n, x, p, dp);
    const double wt = 2.0 / ((1.0 - x * x) * dp * dp);
    t[i] = -x;
    t[n - 1 - i] = x;
    w[i] = wt;
    w[n - 1 - i] = wt;
  }
}

}  // namespace

const DTables &mndod_tables() {
  static const DTables *tab = [] {
    auto *t = new DTables;
    std::memset(t, 0, sizeof *t);
    for (int i = 0; i < 2025; ++i) t->ind2[i] = MNDOD_IND2[i];
    for (int i = 0; i < 492; ++i) t->isym[i] = MNDOD_ISYM[i];
    for (int i = 0; i < 9; ++i) t->indpp[i] = MNDOD_INDPP[i];
    for (int i = 0; i < 15; ++i) t->inddp[i] = MNDOD_INDDP[i];
    for (int i = 0; i < 25; ++i) t->inddd[i] = MNDOD_INDDD[i];
    for (int i = 0; i < 675; ++i) t->ch[i] = MNDOD_CH[i];
    gauss_legendre(48, t->gl48_t, t->gl48_w);
    gauss_legendre(40, t->gl40_t, t->gl40_w);
    return t;
  }();
  return *tab;
}

const ParamSet &param_set(int method) {
  static std::mutex mu;
  static ParamSet *sets[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  std::lock_guard<std::mutex> lock(mu);
  if (!sets[method]) sets[method] = new ParamSet(method);
  return *sets[method];
}

}  // namespace pm7
