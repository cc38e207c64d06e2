// An allocation-free variant of the post-SCF corrections (dispersion, EH+ hydrogen
// bonds, C#C, Si-O-H, PM7-HH), for callers that cannot call cudaMalloc: a host that
// owns all device memory through its own pool (a framework's caching allocator, a
// serving process holding a fixed HBM budget), or a loop that must not take the
// implicit device-wide synchronisation a cudaMalloc can cause.
//
// The caller passes device inputs and outputs and a stream. The scratch the kernels
// need lives in one file-scope __device__ array sized for kMaxAtoms atoms, which every
// GPU that loads this library holds until the process exits. Host code cannot use the
// array's name as a device address, so the first call on each device looks the address
// up with cudaGetSymbolAddress (with that device current) and caches it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kernels.hpp"
#include "pm7_b200.h"

namespace pm7 {
namespace {

constexpr int kMaxAtoms = 2048;
// corrections_scratch(kMaxAtoms): three per-block partial arrays of the pair sweep,
// per-atom C6 / H-bond / Si-O-H values and the capped neighbour lists.
constexpr size_t kScratchDoubles =
    3 * (size_t)((kMaxAtoms + 127) / 128) * (size_t)kMaxAtoms + 3 * (size_t)kMaxAtoms + 8 * (size_t)kMaxAtoms;

static __device__ __align__(256) double g_corrections_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_addr[kMaxDevices] = {nullptr};

thread_local std::string g_noalloc_error;

}  // namespace

// Device address of the static scratch on the current device (set up once per device).
static cudaError_t scratch_for_current_device(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_corrections_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace pm7

extern "C" {

pm7_status pm7_corrections_noalloc(int32_t n_atoms, const int32_t *z_dev, const double *xyz_bohr_dev,
                                   int32_t method, int32_t smooth_dispersion, double *out_dev, void *stream) {
  using namespace pm7;
  if (n_atoms < 1 || n_atoms > kMaxAtoms) {
    g_noalloc_error = "pm7_corrections_noalloc handles 1 to " + std::to_string(kMaxAtoms) + " atoms, got " +
                      std::to_string(n_atoms);
    return PM7_ERR_INVALID_INPUT;
  }
  if (!z_dev || !xyz_bohr_dev || !out_dev) {
    g_noalloc_error = "pm7_corrections_noalloc needs device pointers for z, xyz and out";
    return PM7_ERR_INVALID_INPUT;
  }
  if (method < 0 || method > 4) {
    g_noalloc_error = "unknown PM7 method";
    return PM7_ERR_INVALID_INPUT;
  }
  double *scratch = nullptr;
  cudaError_t e = scratch_for_current_device(&scratch);
  if (e != cudaSuccess) {
    g_noalloc_error = std::string("scratch set-up failed: ") + cudaGetErrorString(e);
    return PM7_ERR_CUDA;
  }
  // Every scratch entry is written by the kernels before it is read, so nothing needs
  // clearing between calls.
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_corrections(st, n_atoms, z_dev, xyz_bohr_dev, method, smooth_dispersion, scratch,
                     corrections_scratch(n_atoms), out_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_noalloc_error = std::string("launch failed: ") + cudaGetErrorString(e);
    return PM7_ERR_CUDA;
  }
  return PM7_OK;
}

const char *pm7_corrections_noalloc_error(void) { return pm7::g_noalloc_error.c_str(); }

int32_t pm7_corrections_noalloc_max_atoms(void) { return pm7::kMaxAtoms; }

}  // extern "C"
