// Per-element constants as the kernels read them: one flat record per atomic number,
// built once per PM7 method on the host (params.cpp) and copied to device memory.
#pragma once

#include <cstdint>

namespace pm7 {

constexpr double kEv = 27.211386245988;         // eV per Hartree (CODATA 2018)
constexpr double kA0 = 0.529177210903;          // Bohr radius in Angstrom
constexpr double kEvToKcal = 23.06054783061903;
constexpr double kKcalToEv = 1.0 / kEvToKcal;
constexpr double kAuDipoleToDebye = 2.541746473;
constexpr int kMaxZ = 110;

struct ElementRec {
  int32_t present;     // 1 when the method parameterises this element
  int32_t z, n, n_orb;  // n: principal quantum number of the valence shell
  int32_t is_sparkle, n_gauss, ios, iop;
  double core;          // core charge (tore)
  double u_ss, u_pp, u_dd;
  double beta_s, beta_p, beta_d;
  double zeta_s, zeta_p, zeta_d;
  double g_ss, g_sp, g_pp, g_p2, h_sp;
  double dd, qq, rho0, rho1, rho2;  // sp multipole separations and additive terms (Bohr)
  double po[10];        // MNDO/d additive terms, slots 1..9
  double ddp[7];        // MNDO/d charge separations, slots 2..6
  double gauss[4][3];   // core Gaussians (K, L, M)
  double e_isol, eheat_ev, poc;
  double repd[53];      // MNDO/d one-centre integrals, slots 1..52
  int32_t onecenter_slot;  // index into the 45x45 one-centre table array, -1 if none
  int32_t iod;             // ground-state d occupation (PM7 d-balance switch)
};

struct PairParamRec {
  double alpb, xfac;
};

// Index tables of the MNDO/d two-centre integrals (MOPAC fordd: 1-based values) and the
// Gauss-Legendre rules of the numerical Slater overlaps, one copy per device.
struct DTables {
  uint16_t ind2[2025];   // (ij, kl) -> local integral number, 0 = none
  int16_t isym[492];     // 0: evaluate; +-n (n >= 35): copy (negated) integral n
  uint8_t indpp[9], inddp[15], inddd[25], pad_[7];
  double ch[675];        // multipole coefficients ch(ij, l, m)
  double gl48_t[48], gl48_w[48];  // 48-point rule on [-1, 1]
  double gl40_t[40], gl40_w[40];  // 40-point rule on [-1, 1]
};

// Everything a kernel needs about the parameter set, in device memory.
struct DeviceParams {
  const ElementRec *elements;   // kMaxZ entries
  const PairParamRec *pairs;    // kMaxZ*kMaxZ, already completed with the diagonal-average rule
  const double *onecenter;      // n_onecenter * 2025
  const DTables *tab;           // MNDO/d index tables and quadrature rules
  double vpar[61];              // 1-based
};

}  // namespace pm7
