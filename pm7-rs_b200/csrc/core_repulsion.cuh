// PM7 core-core repulsion of one atom pair (pm7-rs src/repulsion.rs:164-263), shared by
// the sp-frame and MNDO/d-frame pair kernels.
#pragma once

#include "device_params.hpp"
#include "nddo_sp.cuh"

namespace pm7 {

// Core Gaussian of element `src` for slot `s` (repulsion.rs:250-263).
__device__ __forceinline__ double core_gaussian(const ElementRec &src, double zz, double ra, int s) {
  if (s >= src.n_gauss) return 0.0;
  const double k = src.gauss[s][0], l = src.gauss[s][1], m = src.gauss[s][2];
  const double ax = (ra - m) * (ra - m) * l;
  if (ax >= 25.0) return 0.0;
  return exp(-ax) * (zz * k) / ra;
}

// PM7 ccrep for one pair at distance r (Bohr), eV (repulsion.rs:164-248).
__device__ inline double pair_core_energy(const DeviceParams &P, const ElementRec &ei, const ElementRec &ej, double r) {
  const int zi = ei.z, zj = ej.z;
  const double ra = r * kA0;
  const double zz = ei.core * ej.core;
  const double po9i = ei.poc > 1.0e-5 ? ei.poc : ei.rho0;
  const double po9j = ej.poc > 1.0e-5 ? ej.poc : ej.rho0;
  const double gnddo = (1.0 / sqrt(r * r + (po9i + po9j) * (po9i + po9j))) * kEv;
  double cf, pt;
  d_feather(r, cf, pt);
  double enuc = (gnddo * cf + pt * (1.0 - cf)) * zz;
  const PairParamRec pp = P.pairs[zi * kMaxZ + zj];
  const bool defined = fabs(pp.xfac) > 1.0e-5;
  if (defined) {
    const double alpb = pp.alpb < 1.0e-6 ? 1.2 : pp.alpb;
    const double ra6 = ra * ra * ra * ra * ra * ra;
    double scale = 1.0 + exp(-(ra + ra6 * 0.0003) * alpb) * (2.0 * pp.xfac);
    const int hi = zi > zj ? zi : zj, lo = zi > zj ? zj : zi;
    if (lo == 1 && (hi == 6 || hi == 7)) {
      scale = 1.0 + exp(-(ra * ra) * alpb) * (2.0 * pp.xfac);
    } else if (lo == 1 && hi == 8) {
      scale = 1.0 + exp(-(ra * ra) * alpb) * (2.0 * pp.xfac) - exp(ra * (-2.0 * P.vpar[4])) * P.vpar[3];
    } else if (lo == 6 && hi == 6) {
      scale = scale + exp(ra * (-P.vpar[2])) * P.vpar[1];
    } else if (lo == 8 && hi == 14) {
      scale = scale - exp(-(ra - 2.9) * (ra - 2.9)) * 0.0007;
    }
    enuc *= scale;
  } else {
    const bool ln = (zi >= 57 && zi <= 71) || (zj >= 57 && zj <= 71);
    enuc *= 1.0 + exp(ra * (ln ? -3.0 : -2.18)) * 10.0;
  }
  double corr = core_gaussian(ei, zz, ra, 0) + core_gaussian(ej, zz, ra, 0);
  if (!defined)
    for (int s = 0; s < 4; ++s) corr += core_gaussian(ei, zz, ra, s) + core_gaussian(ej, zz, ra, s);
  const double red = ra / (pow((double)zi, 0.3333) + pow((double)zj, 0.3333));
  if (red < 3.0) {
    const double r2 = red * red, r4 = r2 * r2, r12 = r4 * r4 * r4;
    const double guard = (1.0 / r12) * 1.0e-8;
    corr += guard < 1.0e5 ? guard : 1.0e5;
  }
  return enuc + corr;
}

}  // namespace pm7
