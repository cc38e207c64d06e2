// Autotuner of result-identical launch variants (autotune.cpp).
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>

namespace pm7 {

// Launches variant launch(v) of `key` on stream st. On the first use of `key` on this device
// (and with no entry in the PM7_AUTOTUNE_CACHE file) every variant is run once untimed and
// once timed with CUDA events, synchronously, and the fastest is kept; afterwards only the
// kept variant is launched; PM7_AUTOTUNE_FORCE="prefix=variant,..." overrides both for keys
// with that prefix. Returns the variant used. Every variant must write the same results. Not
// for use inside a stream capture.
int autotune(cudaStream_t st, const std::string &key, int n_variants, const std::function<void(int)> &launch);

// The decisions so far as JSON ({"<device>|<key>": variant, ...}).
std::string autotune_report();

}  // namespace pm7
