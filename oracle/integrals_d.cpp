// Oracle (test infrastructure): MNDO/d two-centre integrals and general Slater overlaps.
// Placeholder until the restatement of pm7-rs src/mndod_twocenter.rs and src/overlap_d.rs lands.
#include "oracle_internal.hpp"

namespace oracle {

PairBlock pair_two_electron_d(const Element &, const Element &, const double *) {
  throw Error(PM7_ERR_UNSUPPORTED, "MNDO/d pair integrals are not restated yet");
}

void diat_overlap_d(const Element &, const Element &, const double *, double (*)[9]) {
  throw Error(PM7_ERR_UNSUPPORTED, "MNDO/d overlaps are not restated yet");
}

void slater_locals_numeric(int, double, double, int, double, double, double, double *) {
  throw Error(PM7_ERR_UNSUPPORTED, "numerical Slater overlaps (n >= 4) are not restated yet");
}

}  // namespace oracle
