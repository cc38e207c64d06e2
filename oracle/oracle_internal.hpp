// Oracle internals: a CPU restatement of pm7-rs `run_pm7` (molecular path).
//
// TEST INFRASTRUCTURE ONLY. This code is the correctness oracle and the timed
// CPU baseline; the product (pm7-rs_b200/) never links or calls it. Every
// function cites the pm7-rs file:line it restates. Parity is pinned by
// tests/test_oracle_golden.py against the 175 recorded pm7-rs results of
// tools/oracle/baselines/reference.json.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "pm7_b200.h"

namespace oracle {

// src/constants.rs:14-26
constexpr double EV = 27.211386245988;
constexpr double A0 = 0.529177210903;
constexpr double EV_TO_KCAL = 23.06054783061903;
constexpr double KCAL_TO_EV = 1.0 / EV_TO_KCAL;
constexpr double ANG_TO_BOHR = 1.0 / A0;
constexpr double AU_DIPOLE_TO_DEBYE = 2.541746473;

// Error carrying a pm7_status, mirroring `Pm7Error` (src/error.rs:8-30).
struct Error : std::runtime_error {
  pm7_status code;
  Error(pm7_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// `DShell` (src/mndod.rs:193-212). Fortran 1-based slots kept.
struct DShell {
  double repd[53] = {0};
  double po[10] = {0};
  double ddp[7] = {0};
  double aij[7] = {0};
  double eiscor = 0.0;
  bool has_d = false;
  std::vector<double> onecenter;  // 45*45, d elements only
};

// `Pm7Element` (src/params.rs:18-63).
struct Element {
  int z = 0, n = 0, ios = 0, iop = 0, iod = 0;
  double u_ss = 0, u_pp = 0, u_dd = 0;
  double zeta_s = 0, zeta_p = 0, zeta_d = 0;
  double beta_s = 0, beta_p = 0, beta_d = 0;
  double g_ss = 0, g_sp = 0, g_pp = 0, g_p2 = 0, h_sp = 0;
  double zsn = 0, zpn = 0, zdn = 0, f0sd = 0, g2sd = 0;
  double alpha = 0, poc = 0, polvol = 0;
  std::vector<std::array<double, 3>> gauss;
  int n_orb = 0;
  double core_charge = 0, eheat_ev = 0, e_isol = 0;
  double dd = 0, qq = 0, rho0 = 0, rho1 = 0, rho2 = 0;
  bool is_sparkle = false;
  bool has_dshell = false;
  DShell dshell;

  bool has_p() const { return n_orb >= 4; }
  bool has_d() const { return n_orb == 9; }
  // src/params.rs:78-85
  double po9() const { return poc > 1.0e-5 ? poc : rho0; }
  // src/params.rs:95-97
  double ddp_pd() const { return has_dshell ? dshell.ddp[5] : 0.0; }
};

struct PairParam {
  double alpb = 0, xfac = 0;
};

// `Pm7Parameters` (src/params.rs:104-111).
struct Params {
  int method = 0;
  std::map<int, Element> elements;
  std::map<std::pair<int, int>, PairParam> pairs;
  double vpar_table[60] = {0};

  const Element &element(int z) const;
  PairParam pair(int zi, int zj) const;
  double vpar(int index) const { return (index >= 1 && index <= 60) ? vpar_table[index - 1] : 0.0; }
};

const Params &params_for(int method);

struct Vec3 {
  double x = 0, y = 0, z = 0;
  Vec3() = default;
  Vec3(double a, double b, double c) : x(a), y(b), z(c) {}
  Vec3 operator+(const Vec3 &o) const { return {x + o.x, y + o.y, z + o.z}; }
  Vec3 operator-(const Vec3 &o) const { return {x - o.x, y - o.y, z - o.z}; }
  Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
  double dot(const Vec3 &o) const { return x * o.x + y * o.y + z * o.z; }
  double norm2() const { return x * x + y * y + z * z; }
  double norm() const { return std::sqrt(norm2()); }
  double get(int k) const { return k == 0 ? x : (k == 1 ? y : z); }
};

struct Molecule {
  std::vector<int> z;
  std::vector<Vec3> pos;  // Bohr
  int size() const { return (int)z.size(); }
};

// Dense row-major square matrix.
struct Mat {
  int n = 0;
  std::vector<double> a;
  Mat() = default;
  explicit Mat(int n_) : n(n_), a((size_t)n_ * n_, 0.0) {}
  double &operator()(int i, int j) { return a[(size_t)i * n + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * n + j]; }
};

// `Basis` (src/basis.rs:25-62).
struct Basis {
  std::vector<int> atom_offset, atom_norb, ao_atom, ao_orb;
  int nao = 0;
};
Basis build_basis(const Molecule &mol, const Params &p);

// One atom pair's two-centre block (`PairTwoElecG`, src/integrals.rs:120-132).
struct PairBlock {
  int norb_i = 0, norb_j = 0, npair_i = 0, npair_j = 0;
  std::vector<double> w;  // npair_i * npair_j
  double e1b[9][9] = {{0}};
  double e2a[9][9] = {{0}};
  double at(int pi, int pj) const { return w[(size_t)pi * npair_j + pj]; }
};

inline int pack(int a, int b) {
  int h = a >= b ? a : b, l = a >= b ? b : a;
  return h * (h + 1) / 2 + l;
}

// sp integrals (src/integrals.rs) and the MNDO/d kernel (src/mndod_twocenter.rs).
PairBlock pair_two_electron(const Element &ei, const Element &ej, const double d[3]);
PairBlock pair_two_electron_sp(const Element &ei, const Element &ej, const double d[3]);
PairBlock pair_two_electron_d(const Element &ei, const Element &ej, const double d[3]);
void rotation_to_x(double vx, double vy, double vz, double r[3][3]);
void feather_to_point(double r, double &cfrac, double &point);

// Overlaps (src/overlap.rs, src/overlap_d.rs): S in the i-first orientation, 9x9.
void diatom_overlap_sp(const Element &ei, const Element &ej, const Vec3 &d, double s[9][9]);
void diat_overlap_d(const Element &ei, const Element &ej, const double d[3], double s[9][9]);
void slater_locals_numeric(int na, double zsa, double zpa, int nb, double zsb, double zpb, double r,
                           double out[5]);

struct PairIntegral {
  int a = 0, b = 0;  // ordered heavier-first as in src/hamiltonian.rs:388-392
  PairBlock te;
};

struct CoreHamiltonian {
  Mat h;
  std::vector<PairIntegral> pairs;
};
CoreHamiltonian build_core(const Molecule &mol, const Basis &basis, const Params &p, bool force_dpath);

Mat build_fock_spin(const Molecule &mol, const Basis &basis, const Params &p, const CoreHamiltonian &core,
                    const Mat &p_tot, const Mat &p_spin);

double core_core_energy(const Molecule &mol, const Params &p);
double pair_core_energy(const Element &ei, const Element &ej, int zi, int zj, double r, const Params &p);

// Post-SCF corrections (kcal/mol).
double dispersion_energy(const Molecule &mol);
double dispersion_energy_smooth(const Molecule &mol);
double hydrogen_bond_energy(const Molecule &mol);
double c_triple_bond_energy(const Molecule &mol);
double si_o_h_energy(const Molecule &mol);
double hh_repulsion_energy(const Molecule &mol);

// Symmetric eigendecomposition: eigenvalues ascending; vectors returned as
// rows of `vt` (vt[k*n + i] = component i of eigenvector k).
void symmetric_eigen(const Mat &a, std::vector<double> &eval, std::vector<double> &vt);
// C = A * B for square row-major matrices.
void matmul(const Mat &a, const Mat &b, Mat &c);
// P = w * V_occ^T V_occ from the first n_occ rows of vt.
void density_from_vectors(const std::vector<double> &vt, int n, int n_occ, double w, Mat &p);

// Shared by the divide-and-conquer restatement (dandc.cpp).
Molecule to_molecule(const pm7_molecule *m);
void validate_input(const Molecule &mol, const pm7_options &o);                    // src/scf.rs:937-1040
void memory_guard(int nao, size_t n_pairs, bool has_d, int64_t explicit_mb);       // src/memory.rs:95-118
Mat sad_density(const Molecule &mol, const Basis &basis, const Params &p, double n_electrons);  // scf.rs:1050-1114
double correction_energy(const Molecule &mol, const pm7_options &o, double parts[5]);  // src/scf.rs:907-932
extern thread_local std::string g_error;

}  // namespace oracle
