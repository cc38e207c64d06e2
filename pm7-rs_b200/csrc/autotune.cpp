// Autotuner: for a launch with several result-identical variants (tile shapes, threads per
// block, items per warp), the fastest one for this device and this key (kernel + size bucket)
// is found on first use by timing every variant with CUDA events on the caller's stream, and
// kept for the process. When PM7_AUTOTUNE_CACHE names a file, decisions are read from it at
// first use and the file is rewritten (JSON) after each new decision, so later processes skip
// the timing. PM7_AUTOTUNE_FORCE="prefix=variant,..." pins every key that starts with a prefix
// (e.g. "b_fock_near=4") to a variant, for all size buckets. Variants never change results
// (same summation order per output element), so the timing runs also produce the caller's
// result.
#include "autotune.hpp"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

namespace pm7 {
namespace {

struct Entry {
  int choice = 0;
  std::vector<float> ms;
};

struct Store {
  std::mutex mu;
  bool loaded = false;
  std::map<std::string, Entry> entries;  // "device name|key"
  std::vector<std::pair<std::string, int>> forced;  // (key prefix, variant)
  std::string path;
};

Store &store() {
  static Store s;
  return s;
}

// The current device's name, queried once per device (the property query costs
// milliseconds; every autotuned launch needs the name for its key).
const std::string &device_name() {
  static std::mutex mu;
  static std::string names[64];
  static const std::string unknown = "unknown";
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return unknown;
  std::lock_guard<std::mutex> lock(mu);
  if (names[dev].empty()) {
    cudaDeviceProp p{};
    names[dev] = cudaGetDeviceProperties(&p, dev) == cudaSuccess ? std::string(p.name) : unknown;
  }
  return names[dev];
}

// The cache is a flat JSON object {"<device>|<key>": {"choice": c, "ms": [..]}, ...} written by
// save(); load() reads back exactly that shape.
void load(Store &s) {
  s.loaded = true;
  if (const char *f = std::getenv("PM7_AUTOTUNE_FORCE")) {
    std::stringstream fs(f);
    std::string item;
    while (std::getline(fs, item, ',')) {
      const size_t eq = item.find('=');
      if (eq == std::string::npos || eq == 0) continue;
      s.forced.emplace_back(item.substr(0, eq), std::atoi(item.c_str() + eq + 1));
    }
  }
  const char *p = std::getenv("PM7_AUTOTUNE_CACHE");
  if (!p || !*p) return;
  s.path = p;
  std::ifstream in(s.path);
  if (!in) return;
  std::stringstream ss;
  ss << in.rdbuf();
  const std::string t = ss.str();
  size_t i = 0;
  while (true) {
    const size_t k0 = t.find('"', i);
    if (k0 == std::string::npos) break;
    const size_t k1 = t.find('"', k0 + 1);
    if (k1 == std::string::npos) break;
    const std::string key = t.substr(k0 + 1, k1 - k0 - 1);
    const size_t c = t.find("\"choice\"", k1);
    const size_t close = t.find('}', k1);
    if (c == std::string::npos || close == std::string::npos || c > close) {
      i = k1 + 1;
      continue;
    }
    Entry e;
    e.choice = std::atoi(t.c_str() + t.find(':', c) + 1);
    s.entries[key] = e;
    i = close + 1;
  }
}

void save(const Store &s) {
  if (s.path.empty()) return;
  std::ofstream out(s.path, std::ios::trunc);
  if (!out) return;
  out << "{\n";
  size_t k = 0;
  for (const auto &kv : s.entries) {
    out << "  \"" << kv.first << "\": {\"choice\": " << kv.second.choice << ", \"ms\": [";
    for (size_t j = 0; j < kv.second.ms.size(); ++j) out << (j ? ", " : "") << kv.second.ms[j];
    out << "]}" << (++k < s.entries.size() ? "," : "") << "\n";
  }
  out << "}\n";
}

}  // namespace

int autotune(cudaStream_t st, const std::string &key, int n_variants, const std::function<void(int)> &launch) {
  if (n_variants <= 1) {
    launch(0);
    return 0;
  }
  Store &s = store();
  const std::string full = device_name() + "|" + key;
  {
    std::lock_guard<std::mutex> lock(s.mu);
    if (!s.loaded) load(s);
    for (const auto &f : s.forced)
      if (key.compare(0, f.first.size(), f.first) == 0 && f.second >= 0 && f.second < n_variants) {
        s.entries[full].choice = f.second;
        launch(f.second);
        return f.second;
      }
    auto it = s.entries.find(full);
    if (it != s.entries.end() && it->second.choice >= 0 && it->second.choice < n_variants) {
      launch(it->second.choice);
      return it->second.choice;
    }
  }
  // one untimed run of every variant (first-launch costs), then one timed run each
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    launch(0);
    return 0;
  }
  std::vector<float> ms(n_variants, 0.0f);
  for (int v = 0; v < n_variants; ++v) launch(v);
  for (int v = 0; v < n_variants; ++v) {
    cudaEventRecord(a, st);
    launch(v);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms[v], a, b);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  int best = 0;
  for (int v = 1; v < n_variants; ++v)
    if (ms[v] < ms[best]) best = v;
  std::lock_guard<std::mutex> lock(s.mu);
  Entry e;
  e.choice = best;
  e.ms = ms;
  s.entries[full] = e;
  save(s);
  return best;
}

std::string autotune_report() {
  Store &s = store();
  std::lock_guard<std::mutex> lock(s.mu);
  std::ostringstream o;
  o << "{";
  size_t k = 0;
  for (const auto &kv : s.entries) o << (k++ ? "," : "") << "\"" << kv.first << "\":" << kv.second.choice;
  o << "}";
  return o.str();
}

}  // namespace pm7
