// Oracle (test infrastructure): core Hamiltonian, Fock build, SCF driver and the
// oracle's C entry points. Restates pm7-rs src/hamiltonian.rs, src/fock.rs,
// src/scf.rs, src/repulsion.rs, src/dipole.rs and src/memory.rs (molecular path,
// no field, no cell).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <string>
#include <tuple>
#include <unordered_map>

#include "oracle_internal.hpp"
#include "pm7_param_data.h"

namespace oracle {

bool set_lapack(const char *path, int threads);

static int pack9(int a, int b) { return pack(a, b); }

static double beta_of(const Element &e, int orb) {  // src/hamiltonian.rs:226-232
  return orb == 0 ? e.beta_s : (orb <= 3 ? e.beta_p : e.beta_d);
}

static bool molecule_has_d(const Molecule &mol, const Params &p) {
  for (int z : mol.z)
    if (p.element(z).n_orb == 9) return true;
  return false;
}

// build_core_generic, molecular branch (src/hamiltonian.rs:310-638).
CoreHamiltonian build_core(const Molecule &mol, const Basis &basis, const Params &p, bool force_dpath) {
  int nao = basis.nao, n = mol.size();
  CoreHamiltonian core;
  core.h = Mat(nao);
  for (int mu = 0; mu < nao; ++mu) {
    const Element &e = p.element(mol.z[basis.ao_atom[mu]]);
    int orb = basis.ao_orb[mu];
    core.h(mu, mu) = orb == 0 ? e.u_ss : (orb <= 3 ? e.u_pp : e.u_dd);
  }
  bool has_any_d = force_dpath || molecule_has_d(mol, p);
  std::vector<std::pair<int, int>> list;
  list.reserve((size_t)n * (n > 0 ? n - 1 : 0) / 2);
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b) list.push_back({a, b});
  size_t np = list.size();
  core.pairs.resize(np);
  std::vector<std::array<double, 81>> sblk(np);
  // Exceptions must not leave an OpenMP region: the first one is kept and rethrown.
  std::string err_msg;
  pm7_status err_code = PM7_OK;
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t k = 0; k < np; ++k) {
    try {
    int u = list[k].first, v = list[k].second;
    const Element &eu = p.element(mol.z[u]), &ev = p.element(mol.z[v]);
    Vec3 d = mol.pos[v] - mol.pos[u];
    int a = u, b = v;
    if (!(eu.n_orb >= ev.n_orb)) {
      a = v;
      b = u;
      d = d * -1.0;
    }
    const Element &ea = p.element(mol.z[a]), &eb = p.element(mol.z[b]);
    double s[9][9];
    double dv[3] = {d.x, d.y, d.z};
    PairIntegral &pi = core.pairs[k];
    pi.a = a;
    pi.b = b;
    if (has_any_d) {
      pi.te = pair_two_electron_d(ea, eb, dv);
      diat_overlap_d(ea, eb, dv, s);
    } else {
      diatom_overlap_sp(ea, eb, d, s);
      double r = d.norm();
      double x[3] = {d.x / r * r, d.y / r * r, d.z / r * r};
      pi.te = pair_two_electron(ea, eb, x);
    }
    for (int i = 0; i < 9; ++i)
      for (int j = 0; j < 9; ++j) sblk[k][i * 9 + j] = s[i][j];
    } catch (const Error &e) {
#pragma omp critical
      if (err_code == PM7_OK) {
        err_code = e.code;
        err_msg = e.what();
      }
    }
  }
  if (err_code != PM7_OK) throw Error(err_code, err_msg);
  // Serial assembly in pair order (src/hamiltonian.rs:507-582).
  for (size_t k = 0; k < np; ++k) {
    const PairIntegral &pi = core.pairs[k];
    const Element &ea = p.element(mol.z[pi.a]), &eb = p.element(mol.z[pi.b]);
    int oa = basis.atom_offset[pi.a], ob = basis.atom_offset[pi.b];
    int na = basis.atom_norb[pi.a], nb = basis.atom_norb[pi.b];
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < na; ++j) core.h(oa + i, oa + j) += pi.te.e1b[i][j];
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) core.h(ob + i, ob + j) += pi.te.e2a[i][j];
    for (int i = 0; i < na; ++i) {
      double bi = beta_of(ea, basis.ao_orb[oa + i]);
      for (int j = 0; j < nb; ++j) {
        double bj = beta_of(eb, basis.ao_orb[ob + j]);
        double value = 0.5 * (bi + bj) * sblk[k][i * 9 + j];
        core.h(oa + i, ob + j) += value;
        core.h(ob + j, oa + i) += value;
      }
    }
  }
  return core;
}

// oc_two_electron (src/fock.rs:69-107).
static double oc_two_electron(int a, int b, int c, int d, const Element &e) {
  if (a == b && c == d) {
    if (a == 0 && c == 0) return e.g_ss;
    if (a == 0 || c == 0) return e.g_sp;
    return a == c ? e.g_pp : e.g_p2;
  }
  int ba = std::min(a, b), bb = std::max(a, b), kc = std::min(c, d), kd = std::max(c, d);
  if (ba == 0 && bb != 0 && kc == 0 && kd != 0 && bb == kd) return e.h_sp;
  if (ba != 0 && bb != 0 && ba != bb && ba == kc && bb == kd) return 0.5 * (e.g_pp - e.g_p2);
  return 0.0;
}

// build_fock_spin_x with no exchange cutoff, molecular (src/fock.rs:149-418).
Mat build_fock_spin(const Molecule &mol, const Basis &basis, const Params &p, const CoreHamiltonian &core,
                    const Mat &pt, const Mat &ps) {
  Mat f = core.h;
  int n = mol.size();
  for (int ia = 0; ia < n; ++ia) {
    const Element &e = p.element(mol.z[ia]);
    int off = basis.atom_offset[ia], no = basis.atom_norb[ia];
    for (int mu = 0; mu < no; ++mu)
      for (int nu = 0; nu < no; ++nu) {
        double acc = 0.0;
        for (int la = 0; la < no; ++la)
          for (int si = 0; si < no; ++si) {
            if (no == 9) {
              const std::vector<double> &oc = e.dshell.onecenter;
              acc += pt(off + la, off + si) * oc[pack9(mu, nu) * 45 + pack9(la, si)];
              acc -= ps(off + la, off + si) * oc[pack9(mu, la) * 45 + pack9(nu, si)];
            } else {
              acc += pt(off + la, off + si) * oc_two_electron(mu, nu, la, si, e);
              acc -= ps(off + la, off + si) * oc_two_electron(mu, la, nu, si, e);
            }
          }
        f(off + mu, off + nu) += acc;
      }
  }
  size_t np = core.pairs.size();
  const size_t batch = 2048;
  for (size_t start = 0; start < np; start += batch) {
    size_t end = std::min(np, start + batch);
    std::vector<std::array<double, 81 * 3>> blk(end - start);
#pragma omp parallel for schedule(dynamic, 16)
    for (size_t k = start; k < end; ++k) {
      const PairIntegral &pi = core.pairs[k];
      const PairBlock &te = pi.te;
      int oa = basis.atom_offset[pi.a], ob = basis.atom_offset[pi.b];
      int na = basis.atom_norb[pi.a], nb = basis.atom_norb[pi.b];
      int stride = te.npair_j;
      double *jaa = &blk[k - start][0], *jbb = jaa + 81, *kab = jaa + 162;
      for (int mu = 0; mu < na; ++mu)
        for (int nu = 0; nu < na; ++nu) {
          int row = pack9(mu, nu) * stride;
          double acc = 0.0;
          for (int la = 0; la < nb; ++la)
            for (int si = 0; si < nb; ++si) acc += pt(ob + la, ob + si) * te.w[row + pack9(la, si)];
          jaa[mu * na + nu] = acc;
        }
      for (int la = 0; la < nb; ++la)
        for (int si = 0; si < nb; ++si) {
          int col = pack9(la, si);
          double acc = 0.0;
          for (int mu = 0; mu < na; ++mu)
            for (int nu = 0; nu < na; ++nu) acc += pt(oa + mu, oa + nu) * te.w[pack9(mu, nu) * stride + col];
          jbb[la * nb + si] = acc;
        }
      for (int mu = 0; mu < na; ++mu)
        for (int la = 0; la < nb; ++la) {
          double acc = 0.0;
          for (int nu = 0; nu < na; ++nu) {
            int row = pack9(mu, nu) * stride;
            for (int si = 0; si < nb; ++si) acc += ps(oa + nu, ob + si) * te.w[row + pack9(la, si)];
          }
          kab[mu * nb + la] = -acc;
        }
    }
    for (size_t k = start; k < end; ++k) {
      const PairIntegral &pi = core.pairs[k];
      int oa = basis.atom_offset[pi.a], ob = basis.atom_offset[pi.b];
      int na = basis.atom_norb[pi.a], nb = basis.atom_norb[pi.b];
      const double *jaa = &blk[k - start][0], *jbb = jaa + 81, *kab = jaa + 162;
      for (int mu = 0; mu < na; ++mu)
        for (int nu = 0; nu < na; ++nu) f(oa + mu, oa + nu) += jaa[mu * na + nu];
      for (int la = 0; la < nb; ++la)
        for (int si = 0; si < nb; ++si) f(ob + la, ob + si) += jbb[la * nb + si];
      for (int mu = 0; mu < na; ++mu)
        for (int la = 0; la < nb; ++la) {
          double v = kab[mu * nb + la];
          f(oa + mu, ob + la) += v;
          f(ob + la, oa + mu) += v;
        }
    }
  }
  return f;
}

// ---- core-core repulsion (src/repulsion.rs:16-36,164-263) --------------

static double core_gaussian_slot(const Element &src, double zz, double r_ang, size_t slot) {
  if (slot >= src.gauss.size()) return 0.0;
  double k = src.gauss[slot][0], l = src.gauss[slot][1], m = src.gauss[slot][2];
  double ax = std::pow(r_ang - m, 2) * l;
  if (ax >= 25.0) return 0.0;
  return std::exp(-ax) * (zz * k) / r_ang;
}

double pair_core_energy(const Element &ei, const Element &ej, int zi, int zj, double r, const Params &p) {
  double r_ang = r * A0;
  double zz = ei.core_charge * ej.core_charge;
  double gab_nddo = (1.0 / std::sqrt(r * r + std::pow(ei.po9() + ej.po9(), 2))) * EV;
  double cfrac, point;
  feather_to_point(r, cfrac, point);
  double gab = gab_nddo * cfrac + point * (1.0 - cfrac);
  double enuc = gab * zz;
  PairParam pair = p.pair(zi, zj);
  bool defined = std::fabs(pair.xfac) > 1.0e-5;
  if (defined) {
    double alpb = pair.alpb < 1.0e-6 ? 1.2 : pair.alpb;
    double scale = 1.0 + std::exp(-(r_ang + std::pow(r_ang, 6) * 0.0003) * alpb) * (2.0 * pair.xfac);
    int hi = std::max(zi, zj), lo = std::min(zi, zj);
    if (lo == 1 && (hi == 6 || hi == 7)) {
      scale = 1.0 + std::exp(-(r_ang * r_ang) * alpb) * (2.0 * pair.xfac);
    } else if (lo == 1 && hi == 8) {
      scale = 1.0 + std::exp(-(r_ang * r_ang) * alpb) * (2.0 * pair.xfac) -
              std::exp(r_ang * (-2.0 * p.vpar(4))) * p.vpar(3);
    } else if (lo == 6 && hi == 6) {
      scale = scale + std::exp(r_ang * (-p.vpar(2))) * p.vpar(1);
    } else if (lo == 8 && hi == 14) {
      scale = scale - std::exp(-std::pow(r_ang - 2.9, 2)) * 0.0007;
    }
    enuc = enuc * scale;
  } else {
    double exponent = ((zi >= 57 && zi <= 71) || (zj >= 57 && zj <= 71)) ? -3.0 : -2.18;
    enuc = enuc * (1.0 + std::exp(r_ang * exponent) * 10.0);
  }
  double corr = core_gaussian_slot(ei, zz, r_ang, 0);
  corr = corr + core_gaussian_slot(ej, zz, r_ang, 0);
  if (!defined)
    for (size_t s = 0; s < 4; ++s) {
      corr = corr + core_gaussian_slot(ei, zz, r_ang, s);
      corr = corr + core_gaussian_slot(ej, zz, r_ang, s);
    }
  double reduced = r_ang / (std::pow((double)zi, 0.3333) + std::pow((double)zj, 0.3333));
  if (reduced < 3.0) {
    double guard = (1.0 / std::pow(reduced, 12)) * 1.0e-8;
    corr = corr + (guard < 1.0e5 ? guard : 1.0e5);
  }
  return enuc + corr;
}

// Diagnostic only: PM7_ORACLE_EXACT_SUMS=1 replaces the reference's plain sequential sums of
// the energy (Frobenius products, core-core) by Neumaier's compensated summation, which shows
// how much of a large system's energy is the rounding of those sums.
static bool exact_sums() {
  static const bool on = std::getenv("PM7_ORACLE_EXACT_SUMS") != nullptr;
  return on;
}

static double neumaier(const double *t, size_t n) {
  double s = 0.0, c = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double x = t[i], u = s + x;
    c += std::fabs(s) >= std::fabs(x) ? (s - u) + x : (x - u) + s;
    s = u;
  }
  return s + c;
}

// `Matrix::frobenius_dot` (src/linalg.rs:138-141): a plain left-to-right fold.
static double frob(const Mat &a, const Mat &b) {
  if (exact_sums()) {
    std::vector<double> t(a.a.size());
    for (size_t i = 0; i < t.size(); ++i) t[i] = a.a[i] * b.a[i];
    return neumaier(t.data(), t.size());
  }
  double s = 0.0;
  for (size_t i = 0; i < a.a.size(); ++i) s += a.a[i] * b.a[i];
  return s;
}

double core_core_energy(const Molecule &mol, const Params &p) {
  int n = mol.size();
  std::vector<double> terms((size_t)n * (n > 0 ? n - 1 : 0) / 2);
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < n; ++i) {
    size_t base = (size_t)i * (2 * (size_t)n - i - 1) / 2;
    for (int j = i + 1; j < n; ++j)
      terms[base + (j - i - 1)] = pair_core_energy(p.element(mol.z[i]), p.element(mol.z[j]), mol.z[i], mol.z[j],
                                                    (mol.pos[j] - mol.pos[i]).norm(), p);
  }
  if (exact_sums()) return neumaier(terms.data(), terms.size());
  double s = 0.0;
  for (double t : terms) s += t;
  return s;
}

// ---- SCF helpers (src/scf.rs) ------------------------------------------



// sad_density (src/scf.rs:1050-1114).
Mat sad_density(const Molecule &mol, const Basis &basis, const Params &p, double n_electrons) {
  int nao = basis.nao;
  Mat P(nao);
  double total_tore = 0.0;
  for (int z : mol.z) total_tore += p.element(z).core_charge;
  double yy = nao > 0 ? (total_tore - n_electrons) / nao : 0.0;
  for (int ia = 0; ia < mol.size(); ++ia) {
    const Element &e = p.element(mol.z[ia]);
    int off = basis.atom_offset[ia], n = basis.atom_norb[ia], z = mol.z[ia];
    double tore = e.core_charge;
    if (n == 1) {
      P(off, off) = tore - yy;
    } else if (n == 4) {
      double w = tore * 0.25 - yy;
      for (int k = 0; k < 4; ++k) P(off + k, off + k) = w;
    } else if (n == 9) {
      bool mg = z < 21 || (z > 30 && z < 39) || (z > 48 && z < 57);
      if (mg) {
        double w = tore * 0.25 - yy;
        for (int k = 0; k < 4; ++k) P(off + k, off + k) = w;
        for (int k = 4; k < 9; ++k) P(off + k, off + k) = -yy;
      } else {
        double sum = tore - 9.0 * yy;
        P(off, off) = std::min(std::max(sum, 0.0), 2.0);
        sum -= 2.0;
        if (sum > 0.0) {
          for (int k = 4; k < 9; ++k) P(off + k, off + k) = std::min(std::max(sum * 0.2, 0.0), 2.0);
          sum -= 10.0;
          if (sum > 0.0)
            for (int k = 1; k < 4; ++k) P(off + k, off + k) = sum / 3.0;
        }
      }
    }
  }
  return P;
}

static void commutator_into(const Mat &f, const Mat &p, Mat &out) {
  Mat fp;
  matmul(f, p, fp);
  int n = fp.n;
  out = Mat(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) out(i, j) = fp(i, j) - fp(j, i);
}

static double rms_diff(const Mat &a, const Mat &b) {
  size_t n = std::max<size_t>(a.a.size(), 1);
  double s = 0.0;
  for (size_t i = 0; i < a.a.size(); ++i) s += (a.a[i] - b.a[i]) * (a.a[i] - b.a[i]);
  return std::sqrt(s / (double)n);
}

static void push_history(std::vector<Mat> &h, const Mat &m, size_t max) {
  if (h.size() >= max) h.erase(h.begin());
  h.push_back(m);
}

static void apply_level_shift(Mat &f, const Mat &d, double occ, double shift) {  // src/scf.rs:1558-1571
  if (shift <= 0.0) return;
  int n = f.n;
  double inv = 1.0 / occ;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double q = d(i, j) * inv;
      f(i, j) += shift * (i == j ? 1.0 - q : -q);
    }
}

// StallGuard (src/scf.rs:1581-1656).
struct StallGuard {
  double floor, shift;
  std::vector<double> steps, energies;
  explicit StallGuard(double f) : floor(f), shift(f) {}
  void update(double step, double energy) {
    const size_t W = 5;
    const double MAX_SHIFT = 64.0, EPROG = 1.0e-9;
    steps.push_back(step);
    energies.push_back(energy);
    size_t n = steps.size();
    if (n < 2 * W) return;
    auto smallest = [](const std::vector<double> &v, size_t a, size_t b) {
      double m = std::numeric_limits<double>::infinity();
      for (size_t i = a; i < b; ++i) m = std::min(m, v[i]);
      return m;
    };
    double step_now = smallest(steps, n - W, n), step_was = smallest(steps, n - 2 * W, n - W);
    double e_now = smallest(energies, n - W, n), e_was = smallest(energies, n - 2 * W, n - W);
    bool moved;
    if (step_now <= step_was * 0.1) {
      if (shift <= floor) moved = false;
      else {
        double relaxed = std::max(shift * 0.5, floor);
        shift = relaxed < 0.25 ? floor : relaxed;
        moved = true;
      }
    } else if (step_now > step_was * 0.9 && e_now > e_was - EPROG && shift < MAX_SHIFT) {
      shift = shift < 1.0 ? 1.0 : std::min(shift * 2.0, MAX_SHIFT);
      moved = true;
    } else {
      moved = false;
    }
    if (moved) {
      steps.clear();
      energies.clear();
    } else {
      steps.erase(steps.begin());
      energies.erase(energies.begin());
    }
  }
};

static Mat combine(const std::vector<Mat> &fs, size_t skip, const std::vector<double> &c) {
  Mat out(fs[0].n);
  for (size_t i = 0; i + skip < fs.size(); ++i) {
    const Mat &f = fs[i + skip];
    for (size_t k = 0; k < out.a.size(); ++k) out.a[k] += c[i] * f.a[k];
  }
  return out;
}

// solve_bordered_small (src/scf.rs:1755-1801).
static bool solve_bordered_small(std::vector<double> m, int n, std::vector<double> rhs, std::vector<double> &x) {
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double best = std::fabs(m[col * n + col]);
    for (int row = col + 1; row < n; ++row) {
      double v = std::fabs(m[row * n + col]);
      if (v > best) {
        best = v;
        piv = row;
      }
    }
    if (best < 1.0e-12) return false;
    if (piv != col) {
      for (int j = 0; j < n; ++j) std::swap(m[col * n + j], m[piv * n + j]);
      std::swap(rhs[col], rhs[piv]);
    }
    for (int row = col + 1; row < n; ++row) {
      double factor = m[row * n + col] / m[col * n + col];
      if (factor == 0.0) continue;
      for (int j = col; j < n; ++j) m[row * n + j] -= factor * m[col * n + j];
      rhs[row] -= factor * rhs[col];
    }
  }
  x.assign(n, 0.0);
  for (int col = n - 1; col >= 0; --col) {
    double s = rhs[col];
    for (int j = col + 1; j < n; ++j) s -= m[col * n + j] * x[j];
    x[col] = s / m[col * n + col];
  }
  return true;
}

// diis_coeffs + diis_window_coeffs (src/scf.rs:1684-1751).
static bool diis_coeffs(const std::vector<Mat> &es, size_t &skip_out, std::vector<double> &c_out) {
  size_t n = es.size();
  if (n < 2) return false;
  std::vector<double> gram(n * n);
  for (size_t i = 0; i < n; ++i)
    for (size_t j = i; j < n; ++j) gram[i * n + j] = gram[j * n + i] = frob(es[i], es[j]);
  for (size_t skip = 0; skip + 1 < n; ++skip) {
    size_t m = n - skip;
    if (m < 2) continue;
    double scale = 0.0;
    for (size_t i = 0; i < m; ++i) scale = std::max(scale, std::fabs(gram[(skip + i) * n + skip + i]));
    if (!std::isfinite(scale) || scale <= 0.0) continue;
    int dim = (int)m + 1;
    std::vector<double> b((size_t)dim * dim, 0.0), rhs(dim, 0.0), c;
    for (size_t i = 0; i < m; ++i) {
      for (size_t j = 0; j < m; ++j) b[i * dim + j] = gram[(skip + i) * n + skip + j] / scale;
      b[i * dim + m] = -1.0;
      b[m * dim + i] = -1.0;
    }
    rhs[m] = -1.0;
    if (!solve_bordered_small(b, dim, rhs, c)) continue;
    bool finite = true;
    for (double v : c) finite = finite && std::isfinite(v);
    if (!finite) continue;
    double wsum = 0.0;
    for (size_t i = 0; i < m; ++i) wsum += std::fabs(c[i]);
    if (wsum <= 25.0) {
      skip_out = skip;
      c_out = c;
      return true;
    }
  }
  return false;
}

// simplex_project + solve_adiis_simplex (src/scf.rs:1860-1916).
static std::vector<double> simplex_project(const std::vector<double> &v) {
  std::vector<double> u = v;
  std::sort(u.begin(), u.end(), [](double a, double b) { return a > b; });
  double css = 0.0, theta = 0.0;
  for (size_t j = 0; j < u.size(); ++j) {
    css += u[j];
    double t = (css - 1.0) / (j + 1.0);
    if (u[j] - t > 0.0) theta = t;
  }
  std::vector<double> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = std::max(v[i] - theta, 0.0);
  return out;
}

static std::vector<double> solve_adiis(const std::vector<double> &d, const std::vector<double> &s, size_t n) {
  double l = 1.0e-12;
  for (size_t i = 0; i < n; ++i) {
    double row = 0.0;
    for (size_t j = 0; j < n; ++j) row += std::fabs(s[i * n + j] + s[j * n + i]);
    l = std::max(l, row);
  }
  double lr = 1.0 / l;
  std::vector<double> c(n, 0.0), g(n);
  c[n - 1] = 1.0;
  for (int it = 0; it < 400; ++it) {
    for (size_t k = 0; k < n; ++k) {
      double acc = 2.0 * d[k];
      for (size_t j = 0; j < n; ++j) acc += (s[k * n + j] + s[j * n + k]) * c[j];
      g[k] = acc;
    }
    std::vector<double> trial(n);
    for (size_t i = 0; i < n; ++i) trial[i] = c[i] - lr * g[i];
    std::vector<double> proj = simplex_project(trial);
    double delta = 0.0;
    for (size_t i = 0; i < n; ++i) delta += std::fabs(proj[i] - c[i]);
    c = proj;
    if (delta < 1.0e-12) break;
  }
  return c;
}

// adiis_extrapolate (src/scf.rs:1812-1857).
static bool adiis_extrapolate(const std::vector<Mat> &ds, const std::vector<Mat> &fs, Mat &out) {
  size_t n = ds.size();
  if (n < 2) return false;
  const Mat &dn = ds[n - 1], &fn = fs[n - 1];
  std::vector<double> d(n), s(n * n);
  for (size_t i = 0; i < n; ++i) {
    double acc = 0.0;
    for (size_t k = 0; k < dn.a.size(); ++k) acc += (ds[i].a[k] - dn.a[k]) * fn.a[k];
    d[i] = acc;
    for (size_t j = 0; j < n; ++j) {
      double a2 = 0.0;
      for (size_t k = 0; k < dn.a.size(); ++k) a2 += (ds[i].a[k] - dn.a[k]) * (fs[j].a[k] - fn.a[k]);
      s[i * n + j] = a2;
    }
  }
  std::vector<double> c = solve_adiis(d, s, n);
  out = combine(fs, 0, c);
  return true;
}

struct ScfState {
  Mat density, spin;
  bool has_spin = false;
  std::vector<double> eps_a, vt_a, eps_b, vt_b;
  int n_occ = 0, n_occ_beta = -1;
  double electronic_ev = 0, density_error = 0;
  bool converged = false, unrestricted = false;
  int iterations = 0;
};

static const char *trace_env() { return std::getenv("PM7_SCF_TRACE"); }

// rhf_loop (src/scf.rs:1189-1322).
static ScfState rhf_loop(const Molecule &mol, const Basis &basis, const Params &p, const CoreHamiltonian &core,
                         int n_occ, const pm7_options &o) {
  int nao = basis.nao;
  Mat density;
  if (o.initial_density) {
    density = Mat(nao);
    std::memcpy(density.a.data(), o.initial_density, sizeof(double) * (size_t)nao * nao);
  } else {
    density = sad_density(mol, basis, p, 2.0 * n_occ);
  }
  double e_old = 0.0;
  ScfState st;
  st.eps_a.assign(nao, 0.0);
  st.density_error = std::numeric_limits<double>::infinity();
  std::vector<Mat> hf, he, hd;
  const size_t max_diis = 8;
  int accel = o.use_diis ? o.accelerator : PM7_ACCEL_NONE;
  StallGuard guard(o.level_shift);
  bool trace = trace_env() != nullptr;
  for (int iter = 0; iter < o.max_scf; ++iter) {
    st.iterations = iter + 1;
    Mat half = density;
    for (double &v : half.a) v *= 0.5;
    Mat f = build_fock_spin(mol, basis, p, core, density, half);
    double e_elec = 0.5 * (frob(density, core.h) + frob(density, f));
    push_history(hf, f, max_diis);
    Mat e;
    commutator_into(f, density, e);
    push_history(he, e, max_diis);
    push_history(hd, density, max_diis);
    double err_norm = std::sqrt(frob(he.back(), he.back()));
    Mat f_use;
    size_t skip;
    std::vector<double> c;
    auto cdiis = [&]() {
      if (diis_coeffs(he, skip, c)) f_use = combine(hf, skip, c);
      else f_use = f;
    };
    if (accel == PM7_ACCEL_NONE) f_use = f;
    else if (accel == PM7_ACCEL_CDIIS) cdiis();
    else if (err_norm > o.adiis_switch) {
      if (!adiis_extrapolate(hd, hf, f_use)) f_use = f;
    } else cdiis();
    apply_level_shift(f_use, density, 2.0, guard.shift);
    std::vector<double> eps, vt;
    symmetric_eigen(f_use, eps, vt);
    Mat p_new;
    density_from_vectors(vt, nao, n_occ, 2.0, p_new);
    double dp = rms_diff(p_new, density);
    st.density_error = dp;
    double de = std::fabs(e_elec - e_old);
    st.eps_a = eps;
    st.vt_a = vt;
    density = p_new;
    e_old = e_elec;
    bool residual_ok = guard.shift == 0.0 && err_norm < 1.0e-7;
    if (iter > 0 && de < o.e_tol && (dp < o.p_tol || residual_ok)) {
      st.converged = true;
      break;
    }
    guard.update(dp, e_elec);
    if (trace)
      std::fprintf(stderr, "oracle scf %4d E %.10f dp %.3e err %.3e shift %.2f\n", st.iterations, e_elec, dp,
                   err_norm, guard.shift);
  }
  Mat half = density;
  for (double &v : half.a) v *= 0.5;
  Mat f_final = build_fock_spin(mol, basis, p, core, density, half);
  st.electronic_ev = 0.5 * (frob(density, core.h) + frob(density, f_final));
  if (guard.shift > 0.0) symmetric_eigen(f_final, st.eps_a, st.vt_a);
  st.density = density;
  st.n_occ = n_occ;
  return st;
}

// uhf_loop (src/scf.rs:1325-1532); the reference disables DIIS on this path.
static ScfState uhf_loop(const Molecule &mol, const Basis &basis, const Params &p, const CoreHamiltonian &core,
                         int n_alpha, int n_beta, const pm7_options &o) {
  int nao = basis.nao;
  Mat total;
  if (o.initial_density) {
    total = Mat(nao);
    std::memcpy(total.a.data(), o.initial_density, sizeof(double) * (size_t)nao * nao);
  } else {
    total = sad_density(mol, basis, p, (double)(n_alpha + n_beta));
  }
  double n_tot = std::max(n_alpha + n_beta, 1);
  double fa_ = n_alpha / n_tot, fb_ = n_beta / n_tot;
  Mat pa = total, pb = total;
  for (double &v : pa.a) v *= fa_;
  for (double &v : pb.a) v *= fb_;
  if (o.initial_spin_density)
    for (size_t k = 0; k < pa.a.size(); ++k) {
      pa.a[k] += 0.5 * o.initial_spin_density[k];
      pb.a[k] -= 0.5 * o.initial_spin_density[k];
    }
  double e_old = 0.0;
  ScfState st;
  st.density_error = std::numeric_limits<double>::infinity();
  StallGuard guard(o.level_shift);
  bool trace = trace_env() != nullptr;
  for (int iter = 0; iter < o.max_scf; ++iter) {
    st.iterations = iter + 1;
    Mat pt = pa;
    for (size_t k = 0; k < pt.a.size(); ++k) pt.a[k] += pb.a[k];
    Mat fa = build_fock_spin(mol, basis, p, core, pt, pa);
    Mat fb = build_fock_spin(mol, basis, p, core, pt, pb);
    double e_elec = 0.5 * (frob(pt, core.h) + frob(pa, fa) + frob(pb, fb));
    Mat ea, eb;
    commutator_into(fa, pa, ea);
    commutator_into(fb, pb, eb);
    double err_norm = std::sqrt(frob(ea, ea) + frob(eb, eb));
    Mat fa_use = fa, fb_use = fb;
    apply_level_shift(fa_use, pa, 1.0, guard.shift);
    apply_level_shift(fb_use, pb, 1.0, guard.shift);
    std::vector<double> eps_a, vt_a, eps_b, vt_b;
    symmetric_eigen(fa_use, eps_a, vt_a);
    symmetric_eigen(fb_use, eps_b, vt_b);
    Mat pa_new, pb_new;
    density_from_vectors(vt_a, nao, n_alpha, 1.0, pa_new);
    density_from_vectors(vt_b, nao, n_beta, 1.0, pb_new);
    double dp = rms_diff(pa_new, pa) + rms_diff(pb_new, pb);
    st.density_error = dp;
    double de = std::fabs(e_elec - e_old);
    st.eps_a = eps_a;
    st.vt_a = vt_a;
    pa = pa_new;
    pb = pb_new;
    e_old = e_elec;
    bool residual_ok = guard.shift == 0.0 && err_norm < 1.0e-7;
    if (iter > 0 && de < o.e_tol && (dp < o.p_tol || residual_ok)) {
      st.converged = true;
      break;
    }
    guard.update(dp, e_elec);
    if (trace)
      std::fprintf(stderr, "oracle scf %4d E %.10f dp %.3e err %.3e shift %.2f (uhf)\n", st.iterations, e_elec, dp,
                   err_norm, guard.shift);
  }
  Mat density = pa, spin = pa;
  for (size_t k = 0; k < density.a.size(); ++k) {
    density.a[k] += pb.a[k];
    spin.a[k] -= pb.a[k];
  }
  Mat fa = build_fock_spin(mol, basis, p, core, density, pa);
  Mat fb = build_fock_spin(mol, basis, p, core, density, pb);
  st.electronic_ev = 0.5 * (frob(density, core.h) + frob(pa, fa) + frob(pb, fb));
  if (guard.shift > 0.0) symmetric_eigen(fa, st.eps_a, st.vt_a);
  symmetric_eigen(fb, st.eps_b, st.vt_b);
  st.density = density;
  st.spin = spin;
  st.has_spin = true;
  st.n_occ = n_alpha;
  st.n_occ_beta = n_beta;
  st.unrestricted = true;
  return st;
}

// ---- input validation and memory guard ----------------------------------

void validate_input(const Molecule &mol, const pm7_options &o) {  // src/scf.rs:937-1040
  auto bad = [](const std::string &m) { throw Error(PM7_ERR_INVALID_INPUT, m); };
  if (mol.size() == 0) bad("a PM7 calculation needs at least one atom");
  if (!std::isfinite(o.charge)) bad("charge must be finite");
  if (o.max_scf <= 0) bad("max_scf must be greater than zero");
  if (!std::isfinite(o.e_tol) || o.e_tol <= 0.0) bad("e_tol must be finite and positive");
  if (!std::isfinite(o.p_tol) || o.p_tol <= 0.0) bad("p_tol must be finite and positive");
  if (!std::isfinite(o.level_shift) || o.level_shift < 0.0) bad("level_shift must be finite and non-negative");
  if (!std::isfinite(o.adiis_switch) || o.adiis_switch < 0.0) bad("adiis_switch must be finite and non-negative");
  for (int i = 0; i < mol.size(); ++i) {
    const Vec3 &q = mol.pos[i];
    if (!std::isfinite(q.x) || !std::isfinite(q.y) || !std::isfinite(q.z))
      bad("atom " + std::to_string(i + 1) + " has non-finite coordinates");
  }
  struct Key {
    long long a, b, c;
    bool operator==(const Key &o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct KH {
    size_t operator()(const Key &k) const { return (size_t)(k.a * 73856093LL ^ k.b * 19349663LL ^ k.c * 83492791LL); }
  };
  const double spacing = 1.0e-6;
  std::unordered_map<Key, std::vector<int>, KH> buckets;
  for (int i = 0; i < mol.size(); ++i) {
    const Vec3 &q = mol.pos[i];
    Key k{(long long)std::floor(q.x / spacing), (long long)std::floor(q.y / spacing), (long long)std::floor(q.z / spacing)};
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          auto it = buckets.find(Key{k.a + dx, k.b + dy, k.c + dz});
          if (it == buckets.end()) continue;
          for (int j : it->second)
            if ((q - mol.pos[j]).norm2() < 1.0e-20)
              bad("atoms " + std::to_string(std::min(i, j) + 1) + " and " + std::to_string(std::max(i, j) + 1) +
                  " occupy the same position");
        }
    buckets[k].push_back(i);
  }
}

static uint64_t available_memory_bytes() {
  std::ifstream f("/proc/meminfo");
  std::string key;
  uint64_t val;
  std::string unit;
  while (f >> key >> val >> unit)
    if (key == "MemAvailable:") return val * 1024ULL;
  return 0;
}

void memory_guard(int nao, size_t n_pairs, bool has_d, int64_t explicit_mb) {  // src/memory.rs:95-118
  uint64_t budget = 0;
  bool have = false;
  if (explicit_mb >= 0) {
    budget = (uint64_t)explicit_mb << 20;
    have = true;
  } else if (const char *s = std::getenv("PM7_MEM_BUDGET_MB")) {
    char *end = nullptr;
    unsigned long long mb = std::strtoull(s, &end, 10);
    if (end != s) {
      budget = mb << 20;
      have = true;
    }
  }
  if (!have) {
    uint64_t av = available_memory_bytes();
    if (av > 0) {
      budget = av / 5 * 4;
      have = true;
    }
  }
  if (!have) return;
  uint64_t mat = (uint64_t)nao * nao * 8;
  uint64_t need = mat * 30 + (uint64_t)n_pairs * (has_d ? 18000 : 2400);
  if (need > budget)
    throw Error(PM7_ERR_INSUFFICIENT_MEMORY,
                "estimated SCF memory ~" + std::to_string((need + (1 << 20) - 1) >> 20) + " MB exceeds the " +
                    std::to_string(budget >> 20) + " MB budget");
}

// ---- post-SCF quantities -------------------------------------------------

double correction_energy(const Molecule &mol, const pm7_options &o, double parts[5]) {
  for (int k = 0; k < 5; ++k) parts[k] = 0.0;
  if (o.method == PM7_METHOD_PM7_MINUS) return 0.0;  // src/method.rs:35-37
  parts[0] = o.smooth_dispersion ? dispersion_energy_smooth(mol) : dispersion_energy(mol);
  parts[1] = hydrogen_bond_energy(mol);
  if (o.method == PM7_METHOD_PM7_HH) parts[4] = hh_repulsion_energy(mol);
  parts[2] = c_triple_bond_energy(mol);
  parts[3] = si_o_h_energy(mol);
  double c = parts[0];
  c += parts[1];
  c += parts[4];
  c += parts[2];
  c += parts[3];
  return c;
}

static const double INV_SQRT3 = 0.5773502691896258;

// dipole::breakdown, molecular (src/dipole.rs:282-350).
static void dipole_breakdown(const Molecule &mol, const Basis &basis, const Params &p, const Mat &P,
                             const std::vector<double> &q, int origin_choice, pm7_result *r) {
  Vec3 origin;
  double net = 0.0;
  for (double v : q) net += v;
  if (std::fabs(net) > 0.5) {
    if (origin_choice == PM7_DIPOLE_CENTRE_OF_MASS) {
      Vec3 c;
      double tot = 0.0;
      for (int i = 0; i < mol.size(); ++i) {
        double m = mol.z[i] < 87 ? PM7_MASS[mol.z[i]] : 0.0;
        c = c + mol.pos[i] * m;
        tot += m;
      }
      if (tot > 0.0) origin = c * (1.0 / tot);
    } else if (origin_choice == PM7_DIPOLE_CENTRE_OF_CHARGE) {
      Vec3 c;
      double tot = 0.0;
      for (int i = 0; i < mol.size(); ++i) {
        double z = p.element(mol.z[i]).core_charge;
        c = c + mol.pos[i] * z;
        tot += z;
      }
      if (tot > 0.0) origin = c * (1.0 / tot);
    }
  }
  Vec3 pc, sp, pd;
  for (int ia = 0; ia < mol.size(); ++ia) {
    pc = pc + (mol.pos[ia] - origin) * q[ia];
    const Element &e = p.element(mol.z[ia]);
    int off = basis.atom_offset[ia];
    if (e.has_p()) {
      double hyb = -2.0 * e.dd;
      sp = sp + Vec3(hyb * P(off, off + 1), hyb * P(off, off + 2), hyb * P(off, off + 3));
    }
    if (e.has_d()) {
      auto d = [&](int i, int j) { return P(off + i, off + j); };
      double hyb = -2.0 * e.ddp_pd();
      double dx = d(5, 3) + d(4, 1) + d(8, 2) - INV_SQRT3 * d(6, 1);
      double dy = d(7, 3) - d(4, 2) + d(8, 1) - INV_SQRT3 * d(6, 2);
      double dz = d(5, 1) + d(7, 2) + 2.0 * INV_SQRT3 * d(6, 3);
      pd = pd + Vec3(hyb * dx, hyb * dy, hyb * dz);
    }
  }
  pc = pc * AU_DIPOLE_TO_DEBYE;
  sp = sp * AU_DIPOLE_TO_DEBYE;
  pd = pd * AU_DIPOLE_TO_DEBYE;
  Vec3 tot = pc + sp + pd;
  for (int k = 0; k < 3; ++k) {
    r->dipole_point_charge[k] = pc.get(k);
    r->dipole_sp_hybrid[k] = sp.get(k);
    r->dipole_pd_hybrid[k] = pd.get(k);
    r->dipole_debye[k] = tot.get(k);
  }
  r->dipole_magnitude = tot.norm();
}

static double *copy_out(const std::vector<double> &v) {
  double *out = (double *)std::malloc(sizeof(double) * std::max<size_t>(v.size(), 1));
  std::memcpy(out, v.data(), sizeof(double) * v.size());
  return out;
}

static std::vector<double> coeff_rows(const std::vector<double> &vt, int n) {
  std::vector<double> c((size_t)n * n);
  for (int k = 0; k < n; ++k)
    for (int mu = 0; mu < n; ++mu) c[(size_t)mu * n + k] = vt[(size_t)k * n + mu];
  return c;
}

// run_pm7_once, molecular (src/scf.rs:524-867).
static void run(const Molecule &mol, const pm7_options &o, pm7_result *r) {
  validate_input(mol, o);
  if (o.multiplicity < 1) throw Error(PM7_ERR_INVALID_INPUT, "multiplicity must be >= 1");
  const Params &p = params_for(o.method);
  Basis basis = build_basis(mol, p);
  int n = mol.size();
  bool has_d = o.force_dpath || molecule_has_d(mol, p);
  memory_guard(basis.nao, (size_t)n * (n > 0 ? n - 1 : 0) / 2, has_d, o.max_memory_mb);
  CoreHamiltonian core = build_core(mol, basis, p, o.force_dpath != 0);
  double n_elec = 0.0;
  for (int z : mol.z) n_elec += p.element(z).core_charge;
  n_elec -= o.charge;
  long long n_int = (long long)std::llround(n_elec);
  if (std::fabs(n_elec - (double)n_int) > 1.0e-6 || n_int < 0)
    throw Error(PM7_ERR_INVALID_INPUT, "invalid electron count");
  long long unp = o.multiplicity - 1;
  if (n_int - unp < 0 || (n_int - unp) % 2 != 0)
    throw Error(PM7_ERR_INVALID_INPUT, "electron count " + std::to_string(n_int) +
                                           " is incompatible with multiplicity " + std::to_string(o.multiplicity) +
                                           " (need same parity)");
  int n_alpha = (int)((n_int + unp) / 2), n_beta = (int)((n_int - unp) / 2);
  bool uhf;
  if (o.reference == PM7_REF_AUTO) uhf = n_alpha != n_beta;
  else if (o.reference == PM7_REF_UNRESTRICTED) uhf = true;
  else {
    if (n_alpha != n_beta)
      throw Error(PM7_ERR_INVALID_INPUT, "restricted (RHF) needs a closed shell; use UHF");
    uhf = false;
  }
  ScfState st = uhf ? uhf_loop(mol, basis, p, core, n_alpha, n_beta, o) : rhf_loop(mol, basis, p, core, n_alpha, o);
  double core_ev = core_core_energy(mol, p);
  double parts[5];
  double corr = correction_energy(mol, o, parts);
  double total = st.electronic_ev + core_ev + corr * KCAL_TO_EV;
  double e_isol = 0.0, eheat = 0.0;
  for (int z : mol.z) {
    e_isol += p.element(z).e_isol;
    eheat += p.element(z).eheat_ev;
  }
  double dhf = (st.electronic_ev + core_ev - e_isol + eheat) * EV_TO_KCAL + corr;
  std::memset(r, 0, sizeof(*r));
  r->iterations = st.iterations;
  r->density_error = st.density_error;
  if (!st.converged) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "PM7 SCF did not converge after %d iterations (error=%.3e)", st.iterations,
                  st.density_error);
    throw Error(PM7_ERR_SCF_NOT_CONVERGED, buf);
  }
  int nao = basis.nao;
  std::vector<double> q(n);
  for (int ia = 0; ia < n; ++ia) {
    double pop = 0.0;
    for (int mu = 0; mu < basis.atom_norb[ia]; ++mu) pop += st.density(basis.atom_offset[ia] + mu, basis.atom_offset[ia] + mu);
    q[ia] = p.element(mol.z[ia]).core_charge - pop;
  }
  r->n_atoms = n;
  r->nao = nao;
  r->n_occ = st.n_occ;
  r->n_occ_beta = st.n_occ_beta;
  r->unrestricted = st.unrestricted;
  r->converged = 1;
  r->electronic_ev = st.electronic_ev;
  r->core_ev = core_ev;
  r->total_ev = total;
  r->heat_of_formation_kcal = dhf;
  r->correction_kcal = corr;
  dipole_breakdown(mol, basis, p, st.density, q, o.dipole_origin, r);
  const double nan = std::numeric_limits<double>::quiet_NaN();
  r->homo_ev = st.n_occ >= 1 ? st.eps_a[st.n_occ - 1] : nan;
  r->lumo_ev = st.n_occ < nao ? st.eps_a[st.n_occ] : nan;
  r->homo_ev_beta = r->lumo_ev_beta = nan;
  if (st.unrestricted) {
    r->homo_ev_beta = st.n_occ_beta >= 1 ? st.eps_b[st.n_occ_beta - 1] : nan;
    r->lumo_ev_beta = st.n_occ_beta < nao ? st.eps_b[st.n_occ_beta] : nan;
  }
  r->charges = copy_out(q);
  r->mo_energies = copy_out(st.eps_a);
  if (st.unrestricted) r->mo_energies_beta = copy_out(st.eps_b);
  if (o.want_matrices) {
    r->density = copy_out(st.density.a);
    if (st.has_spin) r->spin_density = copy_out(st.spin.a);
    r->mo_coeff = copy_out(coeff_rows(st.vt_a, nao));
    if (st.unrestricted) r->mo_coeff_beta = copy_out(coeff_rows(st.vt_b, nao));
  }
}

Molecule to_molecule(const pm7_molecule *m) {
  Molecule mol;
  if (!m || m->n_atoms < 0) throw Error(PM7_ERR_INVALID_INPUT, "null molecule");
  for (int i = 0; i < m->n_atoms; ++i) {
    mol.z.push_back(m->z[i]);
    mol.pos.push_back(Vec3(m->xyz_bohr[3 * i], m->xyz_bohr[3 * i + 1], m->xyz_bohr[3 * i + 2]));
  }
  return mol;
}

thread_local std::string g_error;

template <class F>
static pm7_status guarded(F f) {
  try {
    f();
    return PM7_OK;
  } catch (const Error &e) {
    g_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_error = e.what();
    return PM7_ERR_INVALID_INPUT;
  }
}

}  // namespace oracle

using namespace oracle;

// Fixed-density energy and the five-point difference of the gradient entry points below.
static double fixed_density_energy(const Molecule &mol, const Params &p, bool force_dpath, const Mat &pt,
                                   const Mat &pa, const Mat &pb) {
  Basis b = build_basis(mol, p);
  CoreHamiltonian core = build_core(mol, b, p, force_dpath);
  Mat fa = build_fock_spin(mol, b, p, core, pt, pa);
  Mat fb = build_fock_spin(mol, b, p, core, pt, pb);
  return 0.5 * (frob(pt, core.h) + frob(pa, fa) + frob(pb, fb)) + core_core_energy(mol, p);
}

template <class Energy>
static void five_point_gradient(const Molecule &mol, double h, Energy energy, double *grad) {
  const double t[4] = {1.0, -1.0, 2.0, -2.0};
  for (int a = 0; a < mol.size(); ++a)
    for (int k = 0; k < 3; ++k) {
      double e[4];
      for (int j = 0; j < 4; ++j) {
        Molecule m2 = mol;
        Vec3 &r = m2.pos[a];
        (k == 0 ? r.x : (k == 1 ? r.y : r.z)) += t[j] * h;
        e[j] = energy(m2);
      }
      grad[3 * a + k] = (8.0 * (e[0] - e[1]) - (e[2] - e[3])) / (12.0 * h);
    }
}
// The derivative rule for energies with hard switches (the post-SCF corrections): from the
// energies at -2h, -h, 0, +h, +2h, the five-point formula when both third differences stay
// below `tol` (one smooth curve), else the second-order one-sided formula of the side whose
// second difference is the smaller -- the side without the break, i.e. the derivative of the
// branch the geometry is on, which is what the reference's analytic gradient gives there. A
// break at the geometry itself (both outer second differences below 1% of the middle one, as
// at a symmetric tie) has no branch of its own: the right-hand one is taken; breaks on both
// sides leave the central difference on +-h. A side counts as the cleaner one only when its
// second difference is under half the other's, so rounding does not tip the choice.
static double break_aware_derivative(double em2, double em1, double e0, double ep1, double ep2, double h, double tol) {
  const double d0 = em1 - em2, d1 = e0 - em1, d2 = ep1 - e0, d3 = ep2 - ep1;
  const double t1 = (d2 - d1) - (d1 - d0), t2 = (d3 - d2) - (d2 - d1);
  if (std::fabs(t1) <= tol && std::fabs(t2) <= tol) return (8.0 * (ep1 - em1) - (ep2 - em2)) / (12.0 * h);
  const double sl = std::fabs(d1 - d0), sr = std::fabs(d3 - d2), sm = std::fabs(d2 - d1);
  const double left = (3.0 * e0 - 4.0 * em1 + em2) / (2.0 * h), right = (-3.0 * e0 + 4.0 * ep1 - ep2) / (2.0 * h);
  if (std::max(sl, sr) < 0.01 * sm) return right;  // the break is at the geometry
  if (sl < 0.5 * sr) return left;
  if (sr < 0.5 * sl) return right;
  return (ep1 - em1) / (2.0 * h);
}

extern "C" {

int pm7_oracle_set_lapack(const char *path, int threads) { return set_lapack(path, threads) ? 1 : 0; }

void pm7_oracle_set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
}

const char *pm7_oracle_last_error(void) { return g_error.c_str(); }

pm7_status pm7_oracle_run(const pm7_molecule *m, const pm7_options *o, pm7_result *r) {
  return guarded([&] { run(to_molecule(m), *o, r); });
}

void pm7_oracle_result_free(pm7_result *r) {
  if (!r) return;
  double **arrs[] = {&r->charges, &r->density, &r->spin_density, &r->mo_energies, &r->mo_coeff,
                     &r->mo_energies_beta, &r->mo_coeff_beta};
  for (double **a : arrs) {
    std::free(*a);
    *a = nullptr;
  }
}

pm7_status pm7_oracle_core_hamiltonian(const pm7_molecule *m, int method, int force_dpath, double *h, int *nao) {
  return guarded([&] {
    Molecule mol = to_molecule(m);
    const Params &p = params_for(method);
    Basis b = build_basis(mol, p);
    CoreHamiltonian core = build_core(mol, b, p, force_dpath != 0);
    if (nao) *nao = b.nao;
    if (h) std::memcpy(h, core.h.a.data(), sizeof(double) * core.h.a.size());
  });
}

pm7_status pm7_oracle_fock(const pm7_molecule *m, int method, int force_dpath, const double *pt, const double *ps,
                           double *f_out) {
  return guarded([&] {
    Molecule mol = to_molecule(m);
    const Params &p = params_for(method);
    Basis b = build_basis(mol, p);
    CoreHamiltonian core = build_core(mol, b, p, force_dpath != 0);
    Mat PT(b.nao), PS(b.nao);
    std::memcpy(PT.a.data(), pt, sizeof(double) * PT.a.size());
    std::memcpy(PS.a.data(), ps, sizeof(double) * PS.a.size());
    Mat f = build_fock_spin(mol, b, p, core, PT, PS);
    std::memcpy(f_out, f.a.data(), sizeof(double) * f.a.size());
  });
}

pm7_status pm7_oracle_pair(int method, int zi, int zj, const double d[3], int force_dpath, double *w, double *e1b,
                           double *e2a, double *s, int *npi, int *npj) {
  return guarded([&] {
    const Params &p = params_for(method);
    const Element &ei = p.element(zi), &ej = p.element(zj);
    PairBlock pb;
    double s9[9][9];
    if (force_dpath || ei.n_orb == 9 || ej.n_orb == 9) {
      pb = pair_two_electron_d(ei, ej, d);
      diat_overlap_d(ei, ej, d, s9);
    } else {
      pb = pair_two_electron_sp(ei, ej, d);
      diatom_overlap_sp(ei, ej, Vec3(d[0], d[1], d[2]), s9);
    }
    *npi = pb.npair_i;
    *npj = pb.npair_j;
    std::memcpy(w, pb.w.data(), sizeof(double) * pb.w.size());
    for (int i = 0; i < 9; ++i)
      for (int j = 0; j < 9; ++j) {
        e1b[i * 9 + j] = pb.e1b[i][j];
        e2a[i * 9 + j] = pb.e2a[i][j];
        s[i * 9 + j] = s9[i][j];
      }
  });
}

// Timed bounded sample of a solve, for the CPU baseline: the core-Hamiltonian build,
// `n_iter` RHF iterations (no convergence required) and the post-SCF terms.
// out = {build seconds, seconds of the n_iter iterations, post-SCF seconds, iterations run}.
pm7_status pm7_oracle_sample(const pm7_molecule *m, const pm7_options *o, int n_iter, double out[4]) {
  return guarded([&] {
    Molecule mol = to_molecule(m);
    const Params &p = params_for(o->method);
    auto now = [] { return omp_get_wtime(); };
    double t0 = now();
    Basis basis = build_basis(mol, p);
    CoreHamiltonian core = build_core(mol, basis, p, o->force_dpath != 0);
    double t1 = now();
    double n_elec = -o->charge;
    for (int z : mol.z) n_elec += p.element(z).core_charge;
    int n_occ = (int)std::llround(n_elec) / 2;
    pm7_options oo = *o;
    oo.max_scf = n_iter;
    ScfState st = rhf_loop(mol, basis, p, core, n_occ, oo);
    double t2 = now();
    double parts[5];
    volatile double sink = core_core_energy(mol, p) + correction_energy(mol, oo, parts) + st.electronic_ev;
    (void)sink;
    double t3 = now();
    out[0] = t1 - t0;
    out[1] = t2 - t1;
    out[2] = t3 - t2;
    out[3] = st.iterations;
  });
}

pm7_status pm7_oracle_core_core(const pm7_molecule *m, int method, double *e) {
  return guarded([&] { *e = core_core_energy(to_molecule(m), params_for(method)); });
}

pm7_status pm7_oracle_corrections(const pm7_molecule *m, int method, int smooth, double out[5]) {
  return guarded([&] {
    pm7_options o;
    std::memset(&o, 0, sizeof o);
    o.method = method;
    o.smooth_dispersion = smooth;
    correction_energy(to_molecule(m), o, out);
  });
}

// ---- nuclear gradient (src/gradient.rs) ----------------------------------------
// The oracle restates the reference's *independent* check of its closed-form gradient,
// `analytic_gradient` (src/gradient.rs:365-432): the electronic energy at a fixed density
// (`energy_at_fixed_density_with`, :312-363: 1/2 [tr(P H) + tr(P^a F^a) + tr(P^b F^b)] from a
// full core build, plus core-core) differentiated by central differences of the geometry,
// here the five-point form (8 [E(+h) - E(-h)] - [E(+2h) - E(-2h)]) / 12h per component; and
// the correction gradient (:208-261) as the same difference of the correction energy.

// Core-core + electronic gradient at the density p_total (spin density p_spin, or null for
// a closed shell: P^a = P^b = P / 2), eV/Bohr.
pm7_status pm7_oracle_fixed_density_gradient(const pm7_molecule *m, int method, int force_dpath, const double *pt,
                                             const double *ps, double step, double *grad) {
  return guarded([&] {
    Molecule mol = to_molecule(m);
    const Params &p = params_for(method);
    const int nao = build_basis(mol, p).nao;
    Mat PT(nao), PA(nao), PB(nao);
    std::memcpy(PT.a.data(), pt, sizeof(double) * PT.a.size());
    for (size_t i = 0; i < PT.a.size(); ++i) {
      const double s = ps ? ps[i] : 0.0;
      PA.a[i] = 0.5 * (PT.a[i] + s);
      PB.a[i] = 0.5 * (PT.a[i] - s);
    }
    five_point_gradient(mol, step, [&](const Molecule &x) { return fixed_density_energy(x, p, force_dpath != 0, PT, PA, PB); },
                        grad);
  });
}

// Post-SCF correction gradient, eV/Bohr: differences of the correction energy under the
// break-aware rule above (its EH+ H-bond term has jumps and kinks).
pm7_status pm7_oracle_correction_gradient(const pm7_molecule *m, int method, int smooth, double step, double *grad) {
  return guarded([&] {
    pm7_options o;
    std::memset(&o, 0, sizeof o);
    o.method = method;
    o.smooth_dispersion = smooth;
    double parts[5];
    const Molecule mol = to_molecule(m);
    const double e0 = correction_energy(mol, o, parts);
    const double t[4] = {-2.0, -1.0, 1.0, 2.0};
    for (int a = 0; a < mol.size(); ++a)
      for (int k = 0; k < 3; ++k) {
        double e[4];
        for (int j = 0; j < 4; ++j) {
          Molecule m2 = mol;
          Vec3 &r = m2.pos[a];
          (k == 0 ? r.x : (k == 1 ? r.y : r.z)) += t[j] * step;
          e[j] = correction_energy(m2, o, parts);
        }
        // kcal/mol; a smooth term's third differences stay far below 1e-9 kcal/mol
        grad[3 * a + k] = break_aware_derivative(e[0], e[1], e0, e[2], e[3], step, 1.0e-9) * KCAL_TO_EV;
      }
  });
}

// Derived element quantities, for checks against the reference's own unit tests:
// out = {n_orb, core_charge, e_isol, eheat_ev, dd, qq, rho0, rho1, rho2, po[1..9], ddp[2..6], eiscor}.
pm7_status pm7_oracle_element(int method, int z, double *out) {
  return guarded([&] {
    const Element &e = params_for(method).element(z);
    double v[] = {(double)e.n_orb, e.core_charge, e.e_isol, e.eheat_ev, e.dd, e.qq, e.rho0, e.rho1, e.rho2};
    int k = 0;
    for (double x : v) out[k++] = x;
    for (int i = 1; i <= 9; ++i) out[k++] = e.dshell.po[i];
    for (int i = 2; i <= 6; ++i) out[k++] = e.dshell.ddp[i];
    out[k++] = e.dshell.eiscor;
  });
}

}  // extern "C"
