// Parameter set of one PM7 method: element records, pair core-core scalings and the
// global correction table, derived once per process (like the reference's
// `Pm7Parameters::shared`, pm7-rs src/params.rs:139-155).
#pragma once

#include <vector>

#include "device_params.hpp"

namespace pm7 {

class ParamSet {
 public:
  explicit ParamSet(int method);
  int method() const { return method_; }
  const ElementRec *element(int z) const;
  const std::vector<ElementRec> &elements() const { return elements_; }
  const std::vector<PairParamRec> &pairs() const { return pairs_; }
  const std::vector<double> &onecenter() const { return onecenter_; }
  const double *vpar() const { return vpar_; }  // 1-based, 61 entries
  PairParamRec pair(int zi, int zj) const { return pairs_[(size_t)zi * kMaxZ + zj]; }

 private:
  int method_;
  std::vector<ElementRec> elements_;
  std::vector<PairParamRec> pairs_;
  std::vector<double> onecenter_;
  double vpar_[61];
};

// Process-global, thread-safe cache (method 0..4).
const ParamSet &param_set(int method);

// MNDO/d index tables and the Gauss-Legendre rules (built once, method independent).
const DTables &mndod_tables();

}  // namespace pm7
