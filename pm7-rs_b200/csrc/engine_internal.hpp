// Internal interface of the host runtime shared by the single-molecule engine
// (engine.cu) and the batched engine (batch.cu): errors, the per-device context, device
// buffers, the AO / near-pair layout of a molecule and its validation.
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "params.hpp"
#include "pm7_b200.h"

namespace pm7 {

struct Failure {
  pm7_status code;
  std::string msg;
};
extern thread_local std::string g_last_error;

#define CUDA_OK(expr)                                                                            \
  do {                                                                                           \
    cudaError_t e_ = (expr);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      throw Failure{PM7_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " + \
                                      __FILE__ + ":" + std::to_string(__LINE__)};                \
  } while (0)
#define SOLVER_OK(expr)                                                                           \
  do {                                                                                            \
    cusolverStatus_t s_ = (expr);                                                                 \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                                            \
      throw Failure{PM7_ERR_LINEAR_ALGEBRA, "cuSOLVER status " + std::to_string((int)s_) + " at " + \
                                                std::to_string(__LINE__)};                        \
  } while (0)

struct StageProfiler {
  std::mutex mu;
  bool on = false;
  struct Open {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Open> pending;
  std::vector<std::string> names;
  std::vector<double> total_ms;
  std::vector<long long> calls;
  int index(const char *name) {
    for (size_t i = 0; i < names.size(); ++i)
      if (names[i] == name) return (int)i;
    names.push_back(name);
    total_ms.push_back(0.0);
    calls.push_back(0);
    return (int)names.size() - 1;
  }
  // Returns a token for end(); -1 when profiling is off.
  int begin(cudaStream_t st, const char *name) {
    std::lock_guard<std::mutex> g(mu);
    if (!on) return -1;
    Open o;
    o.stage = index(name);
    cudaEventCreate(&o.a);
    cudaEventCreate(&o.b);
    cudaEventRecord(o.a, st);
    pending.push_back(o);
    return (int)pending.size() - 1;
  }
  void end(cudaStream_t st, int token) {
    if (token < 0) return;
    std::lock_guard<std::mutex> g(mu);
    if (token < (int)pending.size()) cudaEventRecord(pending[token].b, st);
  }
  // Forget the last `count` pending measurements of stage `name` (launches whose work the
  // device skipped, e.g. SP2 steps queued past the step that stopped the purification).
  void drop_last(const char *name, int count) {
    std::lock_guard<std::mutex> g(mu);
    if (!on || count <= 0) return;
    int idx = -1;
    for (size_t i = 0; i < names.size(); ++i)
      if (names[i] == name) idx = (int)i;
    for (int i = (int)pending.size() - 1; i >= 0 && count > 0 && idx >= 0; --i)
      if (pending[i].stage == idx) {
        pending[i].stage = -1;
        --count;
      }
  }
  void flush() {
    std::lock_guard<std::mutex> g(mu);
    for (Open &o : pending) {
      cudaEventSynchronize(o.b);
      float ms = 0.0f;
      if (o.stage >= 0 && cudaEventElapsedTime(&ms, o.a, o.b) == cudaSuccess) {
        total_ms[o.stage] += ms;
        calls[o.stage] += 1;
      }
      cudaEventDestroy(o.a);
      cudaEventDestroy(o.b);
    }
    pending.clear();
  }
  void reset(bool enable) {
    flush();
    std::lock_guard<std::mutex> g(mu);
    on = enable;
    names.clear();
    total_ms.clear();
    calls.clear();
  }
};
extern StageProfiler g_prof;

// RAII stage timer on a stream.
struct Stage {
  cudaStream_t st;
  int token;
  Stage(cudaStream_t s, const char *name) : st(s), token(g_prof.begin(s, name)) {}
  ~Stage() { g_prof.end(st, token); }
};

// Grow-only device scratch of the eigenvalue solver (stream-ordered growth): repeated
// solves reuse it instead of re-allocating their workspace every call.
struct EigvalsScratch {
  double *work = nullptr;
  size_t cap = 0;  // doubles
  unsigned char *meta = nullptr;
  size_t meta_cap = 0;  // bytes
  unsigned char *pinned = nullptr;  // host staging of the task table (same capacity)
  cudaEvent_t uploaded = nullptr;   // the last upload from `pinned` has been read
  // stream-ordered release (the owner's stream); the owner calls it before it goes away
  void release(cudaStream_t st) {
    if (uploaded) cudaEventSynchronize(uploaded);
    if (work) cudaFreeAsync(work, st);
    if (meta) cudaFreeAsync(meta, st);
    if (pinned) cudaFreeHost(pinned);
    if (uploaded) cudaEventDestroy(uploaded);
    work = nullptr;
    meta = pinned = nullptr;
    uploaded = nullptr;
    cap = meta_cap = 0;
  }
};

struct DeviceContext {
  int device = 0;
  cudaStream_t stream = nullptr;
  cusolverDnHandle_t solver = nullptr;
  std::mutex run_mutex;
  DeviceParams params[5];
  bool params_ready[5] = {false, false, false, false, false};
  // Pinned staging area for the small per-iteration transfers (pointer lists,
  // extrapolation weights, scalars), so they never go through pageable memory.
  unsigned char *pinned = nullptr;
  EigvalsScratch eig_scratch;  // eigenvalue solves of this context's stream
};
static constexpr size_t kPinnedBytes = 1 << 16;

DeviceContext &context_for(int device);
const DeviceParams &device_params(DeviceContext &ctx, int method);

template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  void alloc(size_t count, cudaStream_t s) {
    release();
    st = s;
    n = count;
    CUDA_OK(cudaMallocAsync((void **)&p, sizeof(T) * std::max<size_t>(count, 1), s));
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
  }
  ~DevBuf() { release(); }
};

struct Molecule {
  int n = 0;
  std::vector<int> z;
  std::vector<double> xyz;  // Bohr
};

struct Layout {
  int nao = 0;
  std::vector<int> aoff, norb, ao_atom, ao_orb;
  std::vector<NearPair> near;
  std::vector<int> csr_start;
  std::vector<int2> csr;
  std::vector<int> csr_eoff;  // per csr entry: the packed Coulomb partials of the row's atom in that pair
  int64_t w_len = 0;
  int32_t e_len = 0;
  bool has_d = false;
};

void validate(const Molecule &m, const pm7_options &o);  // src/scf.rs:937-1040
Layout build_layout(const Molecule &m, const ParamSet &ps);
std::vector<double> sad_diag(const Molecule &m, const Layout &L, const ParamSet &ps, double n_electrons);
double *host_copy(const double *src_dev, size_t count, cudaStream_t st);
double *host_vec(const std::vector<double> &v);
uint64_t device_budget(int64_t explicit_mb);
Molecule to_molecule(const pm7_molecule *mol);
const double *pm7_mass_table();

// What a finished SCF hands to fill_result.
struct ResultParts {
  int iterations = 0, fp32_iterations = 0;
  double density_error = 0.0;
  bool converged = false, unrestricted = false;
  double electronic_ev = 0.0, core_ev = 0.0, corr[5] = {0, 0, 0, 0, 0};
  int n_occ = 0, n_occ_beta = -1;
  std::vector<double> eps_a, eps_b;
  double device_ms = 0.0;
};

// The reported quantities of run_pm7 (scf.rs:757-823, dipole.rs:282-350): energies, heat
// of formation, Mulliken charges, dipole breakdown, frontier orbitals. `pops` are the atom
// populations and Pm(atom, i, j) the atom-block density elements. Throws
// PM7_ERR_SCF_NOT_CONVERGED (with iterations and error set in res) when not converged.
void fill_result(pm7_result *res, const Molecule &m, const Layout &L, const ParamSet &ps, const pm7_options &o,
                 const ResultParts &S, const std::vector<double> &pops,
                 const std::function<double(int, int, int)> &Pm);

// One symmetric device matrix (order n, leading dimension ld) whose eigenvalues go,
// ascending, to the device array eps.
struct EigvalsRequest {
  const double *src;
  int n, ld;
  double *eps;
};
// Eigenvalues only, many matrices at once (kernels_eig.cu): grouped by cluster size, one
// tridiagonalisation and one Sturm launch per group; workspace from `scr` (grown in
// stream order as needed). Every order must satisfy eigvals_supported().
void eigvals_device(cudaStream_t st, const std::vector<EigvalsRequest> &req, EigvalsScratch &scr);

template <class T>
inline void upload(DevBuf<T> &b, const std::vector<T> &v, cudaStream_t st) {
  b.alloc(v.size(), st);
  if (!v.empty()) CUDA_OK(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
}

// Core Hamiltonian and stored pair integrals on the device (hamiltonian.rs:310-638).

// One molecule's geometry, integrals and core Hamiltonian on the device (engine.cu).
struct DeviceMolecule {
  cudaStream_t st;
  int n = 0, nao = 0, n_near = 0;
  DevBuf<int> z, aoff, ao_atom, csr_start, csr_eoff;
  DevBuf<double> xyz, H, w, ecore, jbuf, pop, cc_terms, scal, gfar;  // cc_terms: pair energies in pair order
  DevBuf<NearPair> near;
  DevBuf<int2> csr;
  DevBuf<unsigned char> mask;
  DevBuf<int> status;
  double core_core_ev = 0.0;

  FockGeometry geometry() const {
    FockGeometry g;
    g.n_atoms = n;
    g.nao = nao;
    g.n_near = n_near;
    g.z = z.p;
    g.aoff = aoff.p;
    g.ao_atom = ao_atom.p;
    g.xyz = xyz.p;
    g.near_mask = mask.p;
    g.np = near.p;
    g.csr_start = csr_start.p;
    g.csr = csr.p;
    g.csr_eoff = csr_eoff.p;
    g.w = w.p;
    g.gfar = gfar.p;
    return g;
  }
};
// Uploads m / L and evaluates every pair's integrals, H_core and the core-core energy;
// `dpath` selects the MNDO/d frame for every pair (hamiltonian.rs:346-355). With `wait` false
// the call only queues the work: D.status (nonzero: a pair outside the sp-frame kernels) and
// D.scal[0] (the core-core energy) are then the caller's to read.
void build_device_molecule(DeviceMolecule &D, const Molecule &m, const Layout &L, const DeviceParams &P, bool dpath,
                           cudaStream_t st, bool wait = true);

// Nuclear gradient (eV/Bohr, 3 per atom) of a molecule on the device at the density g.Pt / g.Ps
// (engine.cu); g.E and g.status are provided by the call.
struct GradGeometry;
std::vector<double> geometry_gradient(cudaStream_t st, const DeviceParams &P, GradGeometry g, bool dpath, int method,
                                      int smooth, bool corrections, bool any_si);
}  // namespace pm7
