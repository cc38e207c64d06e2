// Oracle (test infrastructure): post-SCF geometric corrections in kcal/mol.
// Restates pm7-rs src/dispersion.rs (D2-style dispersion), src/hbond.rs (EH+ H-bond,
// molecular path), src/mm_corrections.rs (C#C and Si-O-H) and src/hh_rep.rs (PM7-HH).
#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <tuple>
#include <vector>

#include "oracle_internal.hpp"

namespace oracle {
namespace {

// Tables of src/dispersion.rs:25-50 (index by Z, 0 = no parameter).
double c6_table(int z) {
  switch (z) {
    case 1: return 0.16; case 2: return 0.084; case 5: return 5.79; case 6: return 1.65; case 7: return 1.11;
    case 8: return 0.70; case 9: return 0.57; case 10: return 0.45; case 15: return 3.25; case 16: return 5.79;
    case 17: return 5.97; case 18: return 3.71; case 27: return 0.04; case 35: return 11.60; case 36: return 4.47;
    case 53: return 25.80; case 54: return 16.50; default: return 0.0;
  }
}
double r0_table(int z) {
  switch (z) {
    case 1: return 156.0; case 2: return 140.0; case 5: return 180.0; case 6: return 170.0; case 7: return 155.0;
    case 8: return 152.0; case 9: return 147.0; case 10: return 154.0; case 15: return 180.0; case 16: return 180.0;
    case 17: return 175.0; case 18: return 188.0; case 28: return 140.0; case 35: return 185.0; case 36: return 202.0;
    case 53: return 198.0; case 54: return 216.0; default: return 0.0;
  }
}
double neff_table(int z) {
  switch (z) {
    case 1: return 0.80; case 2: return 1.42; case 5: return 2.16; case 6: return 2.50; case 7: return 2.82;
    case 8: return 3.15; case 9: return 3.48; case 10: return 3.81; case 15: return 4.50; case 16: return 4.80;
    case 17: return 5.10; case 18: return 5.40; case 27: return 2.90; case 35: return 6.00; case 36: return 6.30;
    case 53: return 6.95; case 54: return 7.25; default: return 0.0;
  }
}
bool has_disp(int z) { return z >= 1 && z <= 86 && c6_table(z) != 0.0 && r0_table(z) != 0.0 && neff_table(z) != 0.0; }

// covalent_radius_angstrom (src/constants.rs:62-74).
double covalent_radius(int z) {
  static const double RAD[87] = {
      0.0,  0.31, 0.28, 1.28, 0.96, 0.84, 0.76, 0.71, 0.66, 0.57, 0.58, 1.66, 1.41, 1.21, 1.11, 1.07, 1.05, 1.02,
      1.06, 2.03, 1.76, 1.70, 1.60, 1.53, 1.39, 1.39, 1.32, 1.26, 1.24, 1.32, 1.22, 1.22, 1.20, 1.19, 1.20, 1.20,
      1.16, 2.20, 1.95, 1.90, 1.75, 1.64, 1.54, 1.47, 1.46, 1.42, 1.39, 1.45, 1.44, 1.42, 1.39, 1.39, 1.38, 1.39,
      1.40, 2.44, 2.15, 2.07, 2.04, 2.03, 2.01, 1.99, 1.98, 1.98, 1.96, 1.94, 1.92, 1.92, 1.89, 1.90, 1.87, 1.87,
      1.75, 1.70, 1.62, 1.51, 1.44, 1.41, 1.36, 1.36, 1.32, 1.45, 1.46, 1.48, 1.40, 1.50, 1.50};
  return (z >= 0 && z < 87) ? RAD[z] : 1.5;
}

// pair_dispersion_with_c6 (src/dispersion.rs:337-364).
double pair_disp(int zi, int zj, double c6i, double c6j, double r) {
  const double ALPHA = 15.450118, S = 1.226593, CSCALE = 2.286419;
  if (!has_disp(zi) || !has_disp(zj)) return 0.0;
  double ni = neff_table(zi), nj = neff_table(zj);
  double c6 = 2.0 * std::pow(c6i * c6i * c6j * c6j * ni * nj, 1.0 / 3.0) /
              (std::pow(c6i * nj * nj, 1.0 / 3.0) + std::pow(c6j * ni * ni, 1.0 / 3.0));
  double ri = r0_table(zi), rj = r0_table(zj);
  double r0 = (ri * ri * ri + rj * rj * rj) / (ri * ri + rj * rj) / 1000.0 * 2.0;
  double rij = r * (A0 * 0.1);
  double damp = std::exp((rij * (1.0 / (S * r0)) - 1.0) * (-ALPHA)) + 1.0;
  double e = (1.0 / std::pow(rij, 6)) * (c6 / (1000.0 * 4.184)) / damp;
  return e * (-CSCALE);
}

double c6_atom(int z, int nb) { return z == 6 ? (nb == 4 ? 0.95 : 1.65) : c6_table(z); }

double c6_atom_smooth(int z, double count) {  // src/dispersion.rs:133-140
  if (z != 6) return c6_table(z);
  double s = 1.0 / (1.0 + std::exp(-(count - 3.5) * 40.0));
  return 1.65 + (0.95 - 1.65) * s;
}

// ---- EH+ hydrogen-bond correction (src/hbond.rs) ----------------------

const double PI = 3.14159265358979323846;
const double MOPAC_TWO_PI = 6.28318530717959;
const double SHORTCUT = 2.4, LONGCUT = 7.0, COVCUT = 1.2;

double deg(double d) { return PI / (180.0 / d); }

struct HBond {
  int s[9];
  int nra, nrb;
  bool disabled;
};

double dist(const std::vector<Vec3> &c, int a, int b) { return (c[a] - c[b]).norm(); }

double bangle(const std::vector<Vec3> &c, int i, int j, int k) {  // src/hbond.rs:79-90
  double d2ij = (c[i] - c[j]).norm2(), d2jk = (c[j] - c[k]).norm2(), d2ik = (c[i] - c[k]).norm2();
  double xy = std::sqrt(d2ij * d2jk);
  if (xy < 1.0e-20) return 0.0;
  double t = std::min(std::max(0.5 * (d2ij + d2jk - d2ik) / xy, -1.0), 1.0);
  return std::acos(t);
}

double dang(double a1, double a2, double b1, double b2) {  // src/hbond.rs:93-113
  const double zero = 1.0e-6;
  if ((std::fabs(a1) >= zero || std::fabs(a2) >= zero) && (std::fabs(b1) >= zero || std::fabs(b2) >= zero)) {
    double an = 1.0 / std::sqrt(a1 * a1 + a2 * a2), bn = 1.0 / std::sqrt(b1 * b1 + b2 * b2);
    a1 *= an;
    a2 *= an;
    b1 *= bn;
    b2 *= bn;
    double sinth = a1 * b2 - a2 * b1;
    double costh = std::min(std::max(a1 * b1 + a2 * b2, -1.0), 1.0);
    double rcos = std::acos(costh);
    if (std::fabs(rcos) >= 4.0e-5) {
      if (sinth > 0.0) rcos = MOPAC_TWO_PI - rcos;
      return -rcos;
    }
  }
  return 0.0;
}

double dihed(const std::vector<Vec3> &c, int i, int j, int k, int l) {  // src/hbond.rs:116-168
  double xi1 = c[i].x - c[k].x, xj1 = c[j].x - c[k].x, xl1 = c[l].x - c[k].x;
  double yi1 = c[i].y - c[k].y, yj1 = c[j].y - c[k].y, yl1 = c[l].y - c[k].y;
  double zi1 = c[i].z - c[k].z, zj1 = c[j].z - c[k].z, zl1 = c[l].z - c[k].z;
  double d = std::sqrt(xj1 * xj1 + yj1 * yj1 + zj1 * zj1);
  double cosa = d > 0.0 ? std::min(std::max(zj1 / d, -1.0), 1.0) : 0.0;
  double ddd = 1.0 - cosa * cosa;
  double xi2, xl2, yi2, yl2, costh, sinth;
  double yxdist = ddd > 0.0 ? d * std::sqrt(ddd) : 0.0;
  if (ddd > 0.0 && yxdist > 1.0e-6) {
    double cosph = yj1 / yxdist, sinph = xj1 / yxdist;
    xi2 = xi1 * cosph - yi1 * sinph;
    xl2 = xl1 * cosph - yl1 * sinph;
    yi2 = xi1 * sinph + yi1 * cosph;
    double yj2 = xj1 * sinph + yj1 * cosph;
    yl2 = xl1 * sinph + yl1 * cosph;
    costh = cosa;
    sinth = yj2 / d;
  } else {
    xi2 = xi1;
    xl2 = xl1;
    yi2 = yi1;
    yl2 = yl1;
    costh = cosa;
    sinth = 0.0;
  }
  double yi3 = yi2 * costh - zi1 * sinth, yl3 = yl2 * costh - zl1 * sinth;
  double angle = dang(xl2, yl3, xi2, yi3);
  if (angle < 0.0) angle += 2.0 * PI;
  if (angle >= MOPAC_TWO_PI) angle = 0.0;
  return angle;
}

double covrad_scaled(int z) {  // src/hbond.rs:174-190
  static const double COVRAD[94] = {
      0.32, 0.46, 1.20, 0.94, 0.77, 0.75, 0.71, 0.63, 0.64, 0.67, 1.40, 1.25, 1.13, 1.04, 1.10, 1.02, 0.99, 0.96, 1.76,
      1.54, 1.33, 1.22, 1.21, 1.10, 1.07, 1.04, 1.00, 0.99, 1.01, 1.09, 1.12, 1.09, 1.15, 1.10, 1.14, 1.17, 1.89, 1.67,
      1.47, 1.39, 1.32, 1.24, 1.15, 1.13, 1.13, 1.08, 1.15, 1.23, 1.28, 1.26, 1.26, 1.23, 1.32, 1.31, 2.09, 1.76, 1.62,
      1.47, 1.58, 1.57, 1.56, 1.55, 1.51, 1.52, 1.51, 1.50, 1.49, 1.49, 1.48, 1.53, 1.46, 1.37, 1.31, 1.23, 1.18, 1.16,
      1.11, 1.12, 1.13, 1.32, 1.30, 1.30, 1.36, 1.31, 1.38, 1.42, 2.01, 1.81, 1.67, 1.58, 1.52, 1.53, 1.54, 1.55};
  if (z <= 0 || z > 94) return 1.5 * 4.0 / 3.0;
  return COVRAD[z - 1] * 4.0 / 3.0;
}

double bonding(const std::vector<int> &nat, int x, int y) { return covrad_scaled(nat[x]) + covrad_scaled(nat[y]); }

// Covalent neighbours capped at 4 (src/hbond.rs:411-435): ascending scan order.
std::vector<int> neighbours_capped(const std::vector<Vec3> &c, const std::vector<int> &nat, int atom) {
  std::vector<int> list;
  int n = (int)c.size();
  for (int j = 0; j < n; ++j) {
    if (j != atom && dist(c, j, atom) < bonding(nat, j, atom)) {
      list.push_back(j);
      if (list.size() == 5) {
        size_t worst = 0;
        double wd = -1.0;
        for (size_t idx = 0; idx < list.size(); ++idx) {
          double d = dist(c, atom, list[idx]);
          if (d > wd) {
            wd = d;
            worst = idx;
          }
        }
        list.erase(list.begin() + worst);
      }
    }
  }
  return list;
}

std::vector<int> neighbours_all(const std::vector<Vec3> &c, const std::vector<int> &nat, int atom) {
  std::vector<int> list;
  for (int k = 0; k < (int)c.size(); ++k)
    if (k != atom && dist(c, k, atom) < bonding(nat, k, atom)) list.push_back(k);
  return list;
}

// assign_refs (src/hbond.rs:439-505).
void assign_refs(const std::vector<Vec3> &c, const std::vector<int> &nat, const std::vector<int> &nb, int x, int h,
                 int s[9], int base) {
  int i2 = base, i3 = base + 1, i4 = base + 2;
  auto dh = [&](int a) { return dist(c, a, h); };
  size_t n = nb.size();
  int fill = dist(c, x, h) < bonding(nat, x, h) ? h : x;
  if (n == 3 || n == 4) {
    std::vector<int> order = nb;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dh(b) < dh(a); });
    s[i2] = order[0];
    s[i3] = order[1];
    s[i4] = order[2];
  } else if (n == 2) {
    int far = dh(nb[0]) >= dh(nb[1]) ? nb[0] : nb[1];
    int other = far == nb[0] ? nb[1] : nb[0];
    if (dh(nb[0]) >= dh(nb[1])) {
      far = nb[0];
      other = nb[1];
    } else {
      far = nb[1];
      other = nb[0];
    }
    s[i2] = far;
    s[i3] = other;
    s[i4] = fill;
  } else if (n == 1) {
    s[i2] = nb[0];
    std::vector<int> ncn = neighbours_all(c, nat, nb[0]);
    int best = nb[0];
    double bd = -1.0;
    for (int k : ncn) {
      double d = dh(k);
      if (d > bd) {
        bd = d;
        best = k;
      }
    }
    s[i3] = best;
    s[i4] = fill;
  } else {
    s[i2] = s[i3] = s[i4] = fill;
  }
}

// build_hbonds (src/hbond.rs:263-406), plain scans in ascending atom order.
std::vector<HBond> build_hbonds(const std::vector<Vec3> &c, const std::vector<int> &nat) {
  int numat = (int)c.size();
  bool any = false;
  for (int z : nat) any = any || z == 7 || z == 8;
  if (!any) return {};
  const double rah2 = 1.4 * 1.4;
  std::vector<int> acceptors, bonding_h;
  std::vector<char> used(numat, 0);
  for (int i = 0; i < numat; ++i) {
    if (nat[i] == 7 || nat[i] == 8) {
      acceptors.push_back(i);
      for (int j = 0; j < numat; ++j)
        if (nat[j] == 1 && !used[j] && (c[i] - c[j]).norm2() < rah2) {
          bonding_h.push_back(j);
          used[j] = 1;
        }
    }
  }
  const double cutoff2 = 7.0 * 7.0;
  std::vector<std::tuple<int, int, int>> pairs;
  std::set<std::tuple<int, int, int>> seen;
  for (int i : acceptors) {
    for (int j : bonding_h) {
      if ((c[i] - c[j]).norm2() >= rah2) continue;
      for (int k : acceptors) {
        if (k == i) continue;
        if ((c[k] - c[i]).norm2() >= cutoff2) continue;
        if (bangle(c, k, j, i) <= PI * 0.5) continue;
        auto key = std::make_tuple(j, std::min(i, k), std::max(i, k));
        if (!seen.insert(key).second) continue;
        pairs.push_back(std::make_tuple(i, j, k));
      }
    }
  }
  std::vector<HBond> out;
  for (auto &t : pairs) {
    int a1 = std::get<0>(t), h = std::get<1>(t), a5 = std::get<2>(t);
    HBond hb;
    for (int &v : hb.s) v = 0;
    hb.s[0] = a1;
    hb.s[4] = a5;
    hb.s[8] = h;
    std::vector<int> na = neighbours_capped(c, nat, a1), nb = neighbours_capped(c, nat, a5);
    hb.nra = (int)na.size();
    hb.nrb = (int)nb.size();
    bool disabled = false;
    for (int j : na) {
      if (j == a5) disabled = true;
      for (int kk : nb)
        if (j == kk && kk != h) disabled = true;
    }
    hb.disabled = disabled;
    if (!disabled) {
      assign_refs(c, nat, na, a1, h, hb.s, 1);
      assign_refs(c, nat, nb, a5, h, hb.s, 5);
    }
    out.push_back(hb);
  }
  return out;
}

double wrap_pi(double v) {
  if (v <= -PI) v += 2.0 * PI;
  if (v > PI) v -= 2.0 * PI;
  return v;
}

// side_terms (src/hbond.rs:627-743).
bool side_terms(const std::vector<Vec3> &c, const std::vector<int> &nat, int nrb, int heavy, int r1, int r2, int r3,
                int h, double &a2c_out, double &tc_out) {
  double a2s = 0.0, a2s2 = 0.0, ts = 0.0;
  bool tcs = false, tcs2 = false;
  if (nat[heavy] == 8) {
    if (nrb == 1) {
      a2s = PI;
      a2s2 = deg(120.0);
      ts = 0.0;
      tcs2 = true;
    } else {
      a2s = deg(109.48);
      a2s2 = a2s;
      ts = deg(54.74);
    }
  } else if (nat[heavy] == 7) {
    if (nrb == 2) {
      a2s = deg(120.0);
      a2s2 = a2s;
      ts = 0.0;
    } else {
      a2s = deg(109.48);
      a2s2 = a2s;
      ts = deg(54.74);
      tcs = true;
    }
  }
  double tcheck = 0.0;
  if (tcs) {
    double tc = dihed(c, r2, r1, heavy, r3);
    if (tc <= -PI) tc += 2.0 * PI;
    if (tc > PI) tc -= 2.0 * PI;
    tc = tc < 0.0 ? -PI - tc : PI - tc;
    double bac = tc;
    double tcp = tc < 0.0 ? -tc : tc;
    tcp *= 180.0 / PI;
    ts += deg((54.74 - tcp) / 54.74 * 35.26);
    a2s -= deg((54.74 - tcp) / 54.74 * 19.48);
    a2s2 = a2s;
    tcheck = bac;
  }
  double angle2 = bangle(c, r1, heavy, h);
  double a2c = std::cos(a2s - angle2);
  double a2c2 = std::cos(a2s2 - angle2);
  if (a2c2 > a2c) a2c = a2c2;
  if (a2c <= 0.0) return false;
  double tcorr = dihed(c, r2, r1, heavy, h);
  if (tcorr <= -PI) tcorr += 2.0 * PI;
  if (tcorr > PI) tcorr -= 2.0 * PI;
  if (!tcs2 || std::fabs(tcorr * 180.0 / PI) > 90.0) tcorr = tcorr < 0.0 ? -PI - tcorr : PI - tcorr;
  double tcos;
  if (tcheck < 0.0) tcos = std::cos(wrap_pi(ts - tcorr));
  else if (tcheck > 0.0) tcos = std::cos(wrap_pi(-ts - tcorr));
  else {
    double c1 = std::cos(wrap_pi(ts - tcorr)), c2 = std::cos(wrap_pi(-ts - tcorr));
    tcos = c2 > c1 ? c2 : c1;
  }
  if (dist(c, h, heavy) > dist(c, h, r1) && tcs2) tcos = 0.0;
  if (r2 == r3 || h == r3) tcos = 1.0;
  a2c_out = a2c;
  tc_out = tcos;
  return true;
}

// eh_plus, PM7 branch (src/hbond.rs:525-620).
double eh_plus(const std::vector<Vec3> &c, const HBond &hb, const std::vector<int> &nat) {
  if (hb.disabled) return 0.0;
  double a0 = A0;
  double scale_nsp3 = -0.171271 * a0 * a0, scale_osp3 = -0.098822 * a0 * a0, scale_nsp2 = -0.171271 * a0 * a0,
         scale_osp2 = scale_osp3;
  double hartree2kcal = EV * EV_TO_KCAL;
  int s1 = hb.s[0], s2 = hb.s[1], s3 = hb.s[2], s4 = hb.s[3], s5 = hb.s[4], s6 = hb.s[5], s7 = hb.s[6], s8 = hb.s[7],
      h = hb.s[8];
  double angle_cos = -std::cos(bangle(c, s1, h, s5));
  if (angle_cos <= 0.0) return 0.0;
  double a2c, tc, a2cn, tcn;
  if (!side_terms(c, nat, hb.nra, s1, s2, s3, s4, h, a2c, tc)) return 0.0;
  if (!side_terms(c, nat, hb.nrb, s5, s6, s7, s8, h, a2cn, tcn)) return 0.0;
  tcn = std::fabs(tcn);
  double sa = nat[s1] == 7 ? (hb.nra >= 3 ? scale_nsp3 : scale_nsp2) : (hb.nra >= 2 ? scale_osp3 : scale_osp2);
  double sb = nat[s5] == 7 ? (hb.nrb >= 3 ? scale_nsp3 : scale_nsp2) : (hb.nrb >= 2 ? scale_osp3 : scale_osp2);
  double sc = (sa + sb) / 2.0;
  double had = dist(c, h, s1), hbd = dist(c, h, s5);
  double xc_min = std::min(had, hbd);
  double xy_gap = std::max(had, hbd) - xc_min;
  double damping = xy_gap > 0.5 ? 1.0 - 1.0 / (1.0 + std::exp(-60.0 * (xc_min / COVCUT - 1.0))) : 1.0;
  double oo = dist(c, s1, s5);
  damping /= 1.0 + std::exp(-100.0 * (oo / SHORTCUT - 1.0));
  damping *= 1.0 - 1.0 / (1.0 + std::exp(-10.0 * (oo / LONGCUT - 1.0)));
  double xy = dist(c, s1, s5);
  double inner = 1.0 - a2c * tc * a2cn * tcn;
  double e = sc / std::pow(xy, 2.0) * (angle_cos * angle_cos) * (1.0 - inner * inner) * hartree2kcal * damping;
  if (nat[s1] == 8 && nat[s5] == 8) {
    double t = std::max(xy - 2.67, 0.0);
    e += -2.5 * std::exp(-80.0 * t * t) * std::pow(angle_cos, 4);
  }
  return e;
}

}  // namespace

// bond_counts + dispersion_energy_cut, molecular (src/dispersion.rs:186-284).
double dispersion_energy(const Molecule &mol) {
  int n = mol.size();
  std::vector<int> nb(n, 0);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      double d = (mol.pos[j] - mol.pos[i]).norm();
      if (d * A0 < 1.3 * (covalent_radius(mol.z[i]) + covalent_radius(mol.z[j]))) {
        nb[i]++;
        nb[j]++;
      }
    }
  double s = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      s += pair_disp(mol.z[i], mol.z[j], c6_atom(mol.z[i], nb[i]), c6_atom(mol.z[j], nb[j]),
                     (mol.pos[j] - mol.pos[i]).norm());
  return s;
}

// smooth_counts + dispersion_energy_smooth_cut (src/dispersion.rs:147-184, 383-426).
double dispersion_energy_smooth(const Molecule &mol) {
  int n = mol.size();
  std::vector<double> cnt(n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      double r = (mol.pos[j] - mol.pos[i]).norm();
      double rc = 1.3 * (covalent_radius(mol.z[i]) + covalent_radius(mol.z[j])) / A0;
      double e = std::exp(-26.0 * (rc / r - 1.0));
      double w = std::isfinite(e) ? 1.0 / (1.0 + e) : 0.0;
      cnt[i] += w;
      cnt[j] += w;
    }
  std::vector<double> c6(n);
  for (int i = 0; i < n; ++i) c6[i] = c6_atom_smooth(mol.z[i], cnt[i]);
  double s = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) s += pair_disp(mol.z[i], mol.z[j], c6[i], c6[j], (mol.pos[j] - mol.pos[i]).norm());
  return s;
}

// hydrogen_bond_energy, molecular (src/hbond.rs:1294-1321).
double hydrogen_bond_energy(const Molecule &mol) {
  std::vector<Vec3> c;
  for (const Vec3 &p : mol.pos) c.push_back(p * A0);
  std::vector<int> nat = mol.z;
  std::vector<HBond> bonds = build_hbonds(c, nat);
  double s = 0.0;
  for (const HBond &hb : bonds) s += eh_plus(c, hb, nat);
  return s;
}

// c_triple_bond_energy (src/mm_corrections.rs:81-101).
double c_triple_bond_energy(const Molecule &mol) {
  const double YMIN = 1.21, YMAX = 1.33, SCALE = 12.0, P1 = -5.0, P2 = 25.0;
  int n = mol.size();
  double sum = 0.0;
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      if (!(mol.z[a] == 6 && mol.z[b] == 6)) continue;
      double r = (mol.pos[b] - mol.pos[a]).norm() * A0;
      if (r >= YMAX) continue;
      double w;
      if (r < YMIN) w = 1.0;
      else {
        double x = (r - YMIN) / (YMAX - YMIN);
        double x3 = x * x * x, x4 = std::pow(x, 4), x5 = std::pow(x, 5), x6 = std::pow(x, 6);
        double smooth = 1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5;
        double tail = x3 - 3.0 * x4 + 3.0 * x5 - x6;
        w = smooth + (P1 + P2 * x) * tail;
      }
      sum += w;
    }
  return sum * SCALE;
}

// si_o_h_energy (src/mm_corrections.rs:154-224).
double si_o_h_energy(const Molecule &mol) {
  int n = mol.size();
  double s = 0.0;
  for (int o = 0; o < n; ++o) {
    if (mol.z[o] != 8) continue;
    auto nearest = [&](int z, double cut) {
      int best = -1;
      double bd = 0.0;
      for (int k = 0; k < n; ++k) {
        if (k == o || mol.z[k] != z) continue;
        double r = (mol.pos[k] - mol.pos[o]).norm() * A0;
        if (r < cut && (best < 0 || r < bd)) {
          bd = r;
          best = k;
        }
      }
      return best;
    };
    int si = nearest(14, 2.4), h = nearest(1, 1.4);
    if (si < 0 || h < 0) continue;
    Vec3 S = mol.pos[si], O = mol.pos[o], H = mol.pos[h];
    double rso = (O - S).norm() * A0, roh = (O - H).norm() * A0;
    double damp = std::exp(-33.0 * std::max(rso * rso - 1.7 * 1.7, 0.0)) * std::exp(-68.0 * std::max(roh * roh - 1.0, 0.0));
    double ref = 125.0 * PI / 180.0;
    Vec3 u = S - O, v = H - O;
    double cs = std::min(std::max(u.dot(v) / (u.norm() * v.norm()), -1.0), 1.0);
    double ang = std::acos(cs);
    s += 15.0 * damp * (ang - ref) * (ang - ref);
  }
  return s;
}

// hh_repulsion_energy (src/hh_rep.rs), PM7-HH only.
double hh_repulsion_energy(const Molecule &mol) {
  int n = mol.size();
  double s = 0.0;
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) {
      if (mol.z[a] != 1 || mol.z[b] != 1) continue;
      double r = (mol.pos[b] - mol.pos[a]).norm() * A0;
      double v;
      if (r <= 1.0) v = 25.46293603147693;
      else if (r < 1.5)
        v = std::pow(r, 5) * (-2714.9523516034697) + std::pow(r, 4) * 17103.650110591705 +
            std::pow(r, 3) * (-42511.85798221796) + std::pow(r, 2) * 52063.19679913834 + r * (-31430.65833597229) +
            7516.08469609514;
      else v = std::exp(std::pow(r, 1.72905) * (-1.53965)) * 118.7326;
      s += v;
    }
  return s;
}

}  // namespace oracle
