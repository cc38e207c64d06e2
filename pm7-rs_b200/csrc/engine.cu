// Host runtime of the engine and the C ABI of include/pm7_b200.h.
//
// `pm7_run` restates pm7-rs `run_pm7_once` (src/scf.rs:524-867) for molecules: input
// validation, electron counting, the memory guard, the core Hamiltonian, the RHF/UHF
// SCF loops (src/scf.rs:1189-1532) with A-DIIS/CDIIS and the stall guard
// (src/scf.rs:1534-1916), and the reported quantities. All O(n^2) and O(n^3) work runs
// on the device; the host keeps only the <= 9x9 extrapolation solves and the control flow.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <thread>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "gradient.cuh"
#include "kernels.hpp"
#include "params.hpp"
#include "pm7_b200.h"
#include "scf_host.hpp"
#include "autotune.hpp"
#include "engine_internal.hpp"

namespace pm7 {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
thread_local std::string g_last_error = "";

// ---------------------------------------------------------------------------
// diagnostics: launch counter and per-stage CUDA-event timing
// ---------------------------------------------------------------------------
static std::atomic<long long> g_launches{0};
void note_launch(int kernels) { g_launches.fetch_add(kernels, std::memory_order_relaxed); }

StageProfiler g_prof;

// ---------------------------------------------------------------------------
// per-device context: stream, solver handle, parameter tables
// ---------------------------------------------------------------------------
static std::mutex g_ctx_mutex;
static std::unordered_map<int, DeviceContext *> g_contexts;

DeviceContext &context_for(int device) {
  std::lock_guard<std::mutex> lock(g_ctx_mutex);
  auto it = g_contexts.find(device);
  if (it != g_contexts.end()) return *it->second;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    throw Failure{PM7_ERR_CUDA, "no CUDA device is available; this engine has no CPU fallback"};
  if (device < 0 || device >= count) throw Failure{PM7_ERR_CUDA, "invalid CUDA device ordinal"};
  CUDA_OK(cudaSetDevice(device));
  auto *ctx = new DeviceContext();
  ctx->device = device;
  CUDA_OK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  {
    // Keep freed stream-ordered allocations in the pool across synchronisations, so the
    // per-solve buffers are recycled instead of being remapped on every call.
    cudaMemPool_t pool;
    CUDA_OK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    CUDA_OK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  CUDA_OK(cudaMallocHost((void **)&ctx->pinned, kPinnedBytes));
  SOLVER_OK(cusolverDnCreate(&ctx->solver));
  SOLVER_OK(cusolverDnSetStream(ctx->solver, ctx->stream));
  g_contexts[device] = ctx;
  return *ctx;
}

const DeviceParams &device_params(DeviceContext &ctx, int method) {
  if (ctx.params_ready[method]) return ctx.params[method];
  const ParamSet &ps = param_set(method);
  DeviceParams &d = ctx.params[method];
  ElementRec *el = nullptr;
  PairParamRec *pr = nullptr;
  double *oc = nullptr;
  CUDA_OK(cudaMalloc(&el, sizeof(ElementRec) * kMaxZ));
  CUDA_OK(cudaMemcpy(el, ps.elements().data(), sizeof(ElementRec) * kMaxZ, cudaMemcpyHostToDevice));
  CUDA_OK(cudaMalloc(&pr, sizeof(PairParamRec) * kMaxZ * kMaxZ));
  CUDA_OK(cudaMemcpy(pr, ps.pairs().data(), sizeof(PairParamRec) * kMaxZ * kMaxZ, cudaMemcpyHostToDevice));
  const size_t noc = std::max<size_t>(ps.onecenter().size(), 1);
  CUDA_OK(cudaMalloc(&oc, sizeof(double) * noc));
  if (!ps.onecenter().empty())
    CUDA_OK(cudaMemcpy(oc, ps.onecenter().data(), sizeof(double) * ps.onecenter().size(), cudaMemcpyHostToDevice));
  DTables *tab = nullptr;
  CUDA_OK(cudaMalloc(&tab, sizeof(DTables)));
  CUDA_OK(cudaMemcpy(tab, &mndod_tables(), sizeof(DTables), cudaMemcpyHostToDevice));
  d.elements = el;
  d.pairs = pr;
  d.onecenter = oc;
  d.tab = tab;
  for (int i = 0; i <= 60; ++i) d.vpar[i] = ps.vpar()[i];
  ctx.params_ready[method] = true;
  return d;
}

// ---------------------------------------------------------------------------
// device buffers with stream-ordered allocation
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// the molecule on the device
// ---------------------------------------------------------------------------
void validate(const Molecule &m, const pm7_options &o) {  // src/scf.rs:937-1040
  auto bad = [](const std::string &s) { throw Failure{PM7_ERR_INVALID_INPUT, s}; };
  if (m.n == 0) bad("a PM7 calculation needs at least one atom");
  if (!std::isfinite(o.charge)) bad("charge must be finite");
  if (o.max_scf <= 0) bad("max_scf must be greater than zero");
  if (!std::isfinite(o.e_tol) || o.e_tol <= 0.0) bad("e_tol must be finite and positive");
  if (!std::isfinite(o.p_tol) || o.p_tol <= 0.0) bad("p_tol must be finite and positive");
  if (!std::isfinite(o.level_shift) || o.level_shift < 0.0) bad("level_shift must be finite and non-negative");
  if (!std::isfinite(o.adiis_switch) || o.adiis_switch < 0.0) bad("adiis_switch must be finite and non-negative");
  for (int i = 0; i < m.n; ++i)
    if (!std::isfinite(m.xyz[3 * i]) || !std::isfinite(m.xyz[3 * i + 1]) || !std::isfinite(m.xyz[3 * i + 2]))
      bad("atom " + std::to_string(i + 1) + " has non-finite coordinates");
  // Coincident atoms in O(N): buckets much wider than the 1e-10 Bohr threshold.
  struct K {
    long long a, b, c;
    bool operator==(const K &o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct KH {
    size_t operator()(const K &k) const { return std::hash<long long>()(k.a * 1000003LL ^ k.b * 10007LL ^ k.c); }
  };
  std::unordered_map<K, std::vector<int>, KH> cells;
  const double sp = 1.0e-6;
  for (int i = 0; i < m.n; ++i) {
    K k{(long long)std::floor(m.xyz[3 * i] / sp), (long long)std::floor(m.xyz[3 * i + 1] / sp),
        (long long)std::floor(m.xyz[3 * i + 2] / sp)};
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          auto it = cells.find(K{k.a + dx, k.b + dy, k.c + dz});
          if (it == cells.end()) continue;
          for (int j : it->second) {
            const double ex = m.xyz[3 * i] - m.xyz[3 * j], ey = m.xyz[3 * i + 1] - m.xyz[3 * j + 1],
                         ez = m.xyz[3 * i + 2] - m.xyz[3 * j + 2];
            if (ex * ex + ey * ey + ez * ez < 1.0e-20)
              bad("atoms " + std::to_string(std::min(i, j) + 1) + " and " + std::to_string(std::max(i, j) + 1) +
                  " occupy the same position");
          }
        }
    cells[k].push_back(i);
  }
}

// AO layout and the list of atom pairs inside the 7 Angstrom feather range, from a
// cell list (pairs come out sorted by (u, v), u < v).
Layout build_layout(const Molecule &m, const ParamSet &ps) {
  Layout L;
  for (int i = 0; i < m.n; ++i) {
    const ElementRec *e = ps.element(m.z[i]);
    if (!e) throw Failure{PM7_ERR_MISSING_ELEMENT, "missing PM7 parameter block for Z=" + std::to_string(m.z[i])};
    L.aoff.push_back(L.nao);
    L.norb.push_back(e->n_orb);
    for (int o = 0; o < e->n_orb; ++o) {
      L.ao_atom.push_back(i);
      L.ao_orb.push_back(o);
    }
    L.nao += e->n_orb;
    if (e->n_orb == 9) L.has_d = true;
  }
  const double cut = 7.0 / kA0;  // Bohr
  struct K {
    long long a, b, c;
    bool operator==(const K &o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct KH {
    size_t operator()(const K &k) const { return std::hash<long long>()(k.a * 1000003LL ^ k.b * 10007LL ^ k.c); }
  };
  std::unordered_map<K, std::vector<int>, KH> cells;
  std::vector<K> key(m.n);
  for (int i = 0; i < m.n; ++i) {
    key[i] = K{(long long)std::floor(m.xyz[3 * i] / cut), (long long)std::floor(m.xyz[3 * i + 1] / cut),
               (long long)std::floor(m.xyz[3 * i + 2] / cut)};
    cells[key[i]].push_back(i);
  }
  // partners of each atom, on several host threads for large molecules (atom ranges,
  // concatenated in atom order: the pair list is the same as a serial scan's)
  const int workers = m.n >= 512 ? (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency())) : 1;
  std::vector<std::vector<NearPair>> part(workers);
  auto scan = [&](int w) {
    const int a0 = (int)((long long)m.n * w / workers), a1 = (int)((long long)m.n * (w + 1) / workers);
    std::vector<int> partners;
    for (int u = a0; u < a1; ++u) {
      partners.clear();
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            auto it = cells.find(K{key[u].a + dx, key[u].b + dy, key[u].c + dz});
            if (it == cells.end()) continue;
            for (int v : it->second) {
              if (v <= u) continue;
              const double ex = m.xyz[3 * v] - m.xyz[3 * u], ey = m.xyz[3 * v + 1] - m.xyz[3 * u + 1],
                           ez = m.xyz[3 * v + 2] - m.xyz[3 * u + 2];
              if (std::sqrt(ex * ex + ey * ey + ez * ez) * kA0 < 7.0) partners.push_back(v);
            }
          }
      std::sort(partners.begin(), partners.end());
      for (int v : partners) {
        NearPair q;
        q.u = u;
        q.v = v;
        part[w].push_back(q);
      }
    }
  };
  if (workers == 1) {
    scan(0);
  } else {
    std::vector<std::thread> th;
    for (int w = 0; w < workers; ++w) th.emplace_back(scan, w);
    for (auto &t : th) t.join();
  }
  for (auto &pp : part) L.near.insert(L.near.end(), pp.begin(), pp.end());
  std::vector<std::vector<int2>> lists(m.n);
  int64_t woff = 0;
  int32_t eoff = 0;
  for (size_t p = 0; p < L.near.size(); ++p) {
    NearPair &q = L.near[p];
    const int nu = L.norb[q.u], nv = L.norb[q.v];
    const int pu = nu * (nu + 1) / 2, pv = nv * (nv + 1) / 2;
    q.woff = woff;
    woff += (int64_t)pu * pv;
    q.eoff_u = eoff;
    eoff += pu;
    q.eoff_v = eoff;
    eoff += pv;
    lists[q.u].push_back(make_int2(q.v, (int)p));
    lists[q.v].push_back(make_int2(q.u, (int)p));
  }
  L.w_len = woff;
  L.e_len = eoff;
  L.csr_start.assign(m.n + 1, 0);
  for (int a = 0; a < m.n; ++a) {
    std::sort(lists[a].begin(), lists[a].end(), [](const int2 &x, const int2 &y) { return x.x < y.x; });
    L.csr_start[a + 1] = L.csr_start[a] + (int)lists[a].size();
  }
  L.csr.reserve(L.csr_start[m.n]);
  for (int a = 0; a < m.n; ++a) L.csr.insert(L.csr.end(), lists[a].begin(), lists[a].end());
  L.csr_eoff.resize(L.csr.size());
  for (int a = 0; a < m.n; ++a)
    for (int c = L.csr_start[a]; c < L.csr_start[a + 1]; ++c) {
      const NearPair &q = L.near[L.csr[c].y];
      L.csr_eoff[c] = q.u == a ? q.eoff_u : q.eoff_v;
    }
  return L;
}


__global__ void k_fill_mask(int n_near, int n_atoms, const NearPair *np, unsigned char *mask) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_near) return;
  mask[(size_t)np[p].u * n_atoms + np[p].v] = 1;
  mask[(size_t)np[p].v * n_atoms + np[p].u] = 1;
}

// `dpath`: the molecule has a d-shell atom (or the caller forced it), so every pair is
// evaluated in the MNDO/d frame (hamiltonian.rs:346-355).
void build_device_molecule(DeviceMolecule &D, const Molecule &m, const Layout &L, const DeviceParams &P,
                                  bool dpath, cudaStream_t st, bool wait) {
  D.st = st;
  D.n = m.n;
  D.nao = L.nao;
  D.n_near = (int)L.near.size();
  upload(D.z, m.z, st);
  upload(D.xyz, m.xyz, st);
  upload(D.aoff, L.aoff, st);
  upload(D.ao_atom, L.ao_atom, st);
  upload(D.csr_start, L.csr_start, st);
  upload(D.near, L.near, st);
  upload(D.csr, L.csr, st);
  upload(D.csr_eoff, L.csr_eoff, st);
  D.mask.alloc((size_t)m.n * m.n, st);
  CUDA_OK(cudaMemsetAsync(D.mask.p, 0, (size_t)m.n * m.n, st));
  if (D.n_near) k_fill_mask<<<(D.n_near + 255) / 256, 256, 0, st>>>(D.n_near, m.n, D.near.p, D.mask.p);
  D.gfar.alloc((size_t)m.n * m.n, st);
  launch_far_coulomb(st, m.n, D.xyz.p, D.mask.p, D.gfar.p);
  const size_t nao2 = (size_t)L.nao * L.nao;
  D.H.alloc(nao2, st);
  CUDA_OK(cudaMemsetAsync(D.H.p, 0, sizeof(double) * nao2, st));
  D.w.alloc((size_t)L.w_len, st);
  D.ecore.alloc((size_t)L.e_len, st);
  D.jbuf.alloc((size_t)L.e_len, st);
  D.pop.alloc(m.n, st);
  D.scal.alloc(8, st);
  D.status.alloc(1, st);
  CUDA_OK(cudaMemsetAsync(D.status.p, 0, sizeof(int), st));
  // the pair energies in pair order, summed as the reference's fold (repulsion.rs:16-36)
  const size_t npairs = (size_t)m.n * (m.n > 0 ? m.n - 1 : 0) / 2;
  D.cc_terms.alloc(npairs, st);
  DevBuf<unsigned char> ss_scratch;
  ss_scratch.alloc(seqsum_scratch_bytes(npairs, 1), st);
  if (dpath) {
    launch_pairs_all_d(st, m.n, D.z.p, D.xyz.p, D.aoff.p, L.nao, P, D.H.p, D.cc_terms.p);
    launch_near_integrals_d(st, D.n_near, D.z.p, D.xyz.p, D.near.p, P, D.w.p, D.ecore.p);
  } else {
    launch_pairs_all(st, m.n, D.z.p, D.xyz.p, D.aoff.p, L.nao, P, D.H.p, D.cc_terms.p, D.status.p);
    launch_near_integrals(st, D.n_near, D.z.p, D.xyz.p, D.near.p, P, D.w.p, D.ecore.p, D.status.p);
  }
  launch_hcore_diag(st, m.n, D.z.p, D.xyz.p, D.aoff.p, D.csr_start.p, D.csr.p, D.near.p, D.ecore.p, D.mask.p, P,
                    L.nao, D.H.p);
  SeqSumBatch fold{};
  fold.job[0] = {D.cc_terms.p, nullptr, npairs, D.scal.p};
  fold.count = 1;
  launch_seqsum(st, fold, ss_scratch.p);
  if (!wait) return;  // the caller reads D.status and D.scal[0] itself
  int status = 0;
  double cc = 0.0;
  CUDA_OK(cudaMemcpyAsync(&status, D.status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(&cc, D.scal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  CUDA_OK(cudaGetLastError());
  if (status != 0) throw Failure{PM7_ERR_UNSUPPORTED, "a pair's shells are outside the sp-frame integral kernels"};
  D.core_core_ev = cc;
}

// ---------------------------------------------------------------------------
// SCF on the device
// ---------------------------------------------------------------------------
struct Eigen {
  DeviceContext &ctx;
  int n;
  DevBuf<double> work, eps;
  DevBuf<int> info;
  int lwork = 0;
  Eigen(DeviceContext &c, int n_, double *probe) : ctx(c), n(n_) {
    SOLVER_OK(cusolverDnDsyevd_bufferSize(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, probe,
                                          n, nullptr, &lwork));
    work.alloc((size_t)std::max(lwork, 1), ctx.stream);
    eps.alloc(n, ctx.stream);
    info.alloc(1, ctx.stream);
  }
  // In place: A (n x n symmetric) becomes the eigenvectors, one per row when read
  // row-major (vectors = true; else A is overwritten); eigenvalues ascending in eps.
  void solve(double *A, bool vectors = true) {
    SOLVER_OK(cusolverDnDsyevd(ctx.solver, vectors ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR,
                               CUBLAS_FILL_MODE_LOWER, n, A, n, eps.p, work.p, lwork, info.p));
  }
};

// Eigendecomposition on the SCF path (`symmetric_eigen`, src/linalg.rs:231-278): cuSOLVER
// dsyevd, or with PM7_DENSITY_SOLVER=jacobi the repo's Jacobi kernel for orders up to
// kJacobiMax, warm-started from this object's previous eigenvectors (one object per spin
// channel). Jacobi is not the default: measured per solve it is no faster than dsyevd at
// ~60 orbitals and slower from ~100 (40 against 28 ms at 108), and on exactly degenerate
// frontier levels (the reference's O2++ triplet and Cl- cases) its choice of vectors inside
// the degenerate space leads the SCF to another state than the reference's. In place: A
// becomes the eigenvectors, one per row (row-major), eigenvalues ascending in eps(). A Jacobi
// solve that ends unconverged or non-finite raises PM7_ERR_LINEAR_ALGEBRA at the next
// check(), which the caller makes after a stream synchronisation.
static bool use_jacobi(int n) {
  const char *env = std::getenv("PM7_DENSITY_SOLVER");
  return env && std::strcmp(env, "jacobi") == 0 && n <= kJacobiMax;
}

constexpr int kOwnEigvalsMax = 511;  // eigenvalues alone: the cluster tridiagonalisation up to here

struct Diag {
  DeviceContext &ctx;
  cudaStream_t st;
  int n;
  bool jac;
  std::unique_ptr<Eigen> lib;
  DevBuf<double> basis, ev;
  DevBuf<int> info;
  DevBuf<JacobiJob> job;
  double *slot = nullptr;
  bool warm = false, pending = false;
  int *pin;  // pinned copy of the Jacobi status
  Diag(DeviceContext &ctx, int n_, double *probe, int *pinned_info)
      : ctx(ctx), st(ctx.stream), n(n_), jac(use_jacobi(n_)), pin(pinned_info) {
    if (jac) {
      basis.alloc((size_t)n * n, st);
      ev.alloc(n, st);
      info.alloc(1, st);
      prepare_jacobi_eigen(n);
    } else {
      lib = std::make_unique<Eigen>(ctx, n, probe);
    }
  }
  void solve(double *A, bool vectors = true) {
    if (!jac) {
      lib->solve(A, vectors);
      return;
    }
    if (A != slot) {
      upload(job, std::vector<JacobiJob>{JacobiJob{A, ev.p, basis.p, info.p, n, n}}, st);
      slot = A;
    }
    launch_jacobi_eigen(st, job.p, 1, n, warm ? 1 : 0, 0.0);
    warm = true;
    CUDA_OK(cudaMemcpyAsync(pin, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    pending = true;
  }
  // Eigenvalues of A into eps(); A keeps its contents unless the solver is Jacobi or
  // cuSOLVER (which leave eigenvectors). Up to kOwnEigvalsMax the values come from the
  // repo's cluster tridiagonalisation and Sturm multisection.
  void values(double *A) {
    const char *env = std::getenv("PM7_DENSITY_SOLVER");
    const bool library_only = env && std::strcmp(env, "syevd") == 0;
    if (jac || library_only || n > kOwnEigvalsMax) {
      solve(A, false);
      return;
    }
    eigvals_device(st, {EigvalsRequest{A, n, n, lib->eps.p}}, ctx.eig_scratch);
  }
  void check() {
    if (!pending) return;
    pending = false;
    if (*pin != 0)
      throw Failure{PM7_ERR_LINEAR_ALGEBRA, *pin == 1 ? "Jacobi eigensolver did not converge"
                                                      : "Jacobi eigensolver: non-finite matrix"};
  }
  const double *eps() const { return jac ? ev.p : lib->eps.p; }
};

// Density from F by SP2 purification: P = w X with X the aufbau projector onto the
// n_occ lowest eigenvectors of F. Returns false when the iteration does not settle on
// an idempotent X (degenerate frontier levels), so the caller diagonalises instead.
struct Purifier {
  cudaStream_t st;
  int n;
  DevBuf<double> X, X2, scratch, bounds, state, parts;
  int last_iterations = 0;
  double *pin = nullptr;  // kSp2Len pinned doubles for the purification state
  Purifier(cudaStream_t s, int n_, double *pinned_state) : st(s), n(n_), pin(pinned_state) {
    X.alloc((size_t)n * n, st);
    X2.alloc((size_t)n * n, st);
    scratch.alloc(1024, st);
    bounds.alloc(2, st);
    state.alloc(kSp2Len, st);
  }
  // fp32 iterate of the mixed-precision purification: X, its tf32 split, X^2 (ld x ld)
  int ld = 0;
  DevBuf<float> X32, hi32, lo32, C32;
  DevBuf<int> err32;
  alignas(64) unsigned char map_hi[128], map_lo[128];
  void ensure32() {
    if (ld) return;
    ld = ((n + 31) / 32) * 32;
    const size_t ll = (size_t)ld * ld;
    for (DevBuf<float> *b : {&X32, &hi32, &lo32, &C32}) {
      b->alloc(ll, st);
      CUDA_OK(cudaMemsetAsync(b->p, 0, sizeof(float) * ll, st));  // the padding stays zero
    }
    err32.alloc(1, st);
    CUDA_OK(cudaMemsetAsync(err32.p, 0, sizeof(int), st));
    if (!make_square_map(hi32.p, ld, map_hi) || !make_square_map(lo32.p, ld, map_lo))
      throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
  }
  // X = F P at fp32 accuracy on the tcgen05 tensor cores (3xTF32), for the DIIS error of
  // the fp32 cycles: F into its own split pair, P into the SP2 split buffers (free between
  // purifications; the next purification re-initialises them).
  DevBuf<float> Fhi32, Flo32;
  alignas(64) unsigned char mapF_hi[128], mapF_lo[128];
  void product32(const double *F, const double *Pm, double *X) {
    ensure32();
    if (!Fhi32.p) {
      const size_t ll = (size_t)ld * ld;
      for (DevBuf<float> *b : {&Fhi32, &Flo32}) {
        b->alloc(ll, st);
        CUDA_OK(cudaMemsetAsync(b->p, 0, sizeof(float) * ll, st));
      }
      if (!make_square_map(Fhi32.p, ld, mapF_hi) || !make_square_map(Flo32.p, ld, mapF_lo))
        throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    }
    launch_split_tf32(st, n, ld, F, Fhi32.p, Flo32.p);
    launch_split_tf32(st, n, ld, Pm, hi32.p, lo32.p);
    launch_product_tf32x3(st, n, ld, mapF_hi, mapF_lo, map_hi, map_lo, C32.p, err32.p);
    launch_widen(st, n, ld, C32.p, X);
  }

  // Queue SP2 steps in chunks and read the device state once per chunk: the device stops
  // the purification itself (Sp2Rule) and skips the steps queued after that. The first
  // chunk is sized from the previous purification's step count. Returns the steps run.
  static constexpr int kMaxSteps = 100;
  int hint64 = 0, hint32 = 0;
  template <class Launch>
  int run_chunks(Launch launch_step, const char *gemm_stage, int &hint) {
    launch_sp2_reset(st, state.p);
    int launched = 0, chunk = std::max(4, hint + 1);
    while (launched < kMaxSteps) {
      for (int c = 0; c < chunk && launched < kMaxSteps; ++c) launch_step(launched++);
      CUDA_OK(cudaMemcpyAsync(pin, state.p, kSp2Len * sizeof(double), cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaStreamSynchronize(st));
      if (pin[kSp2Stop] < 1.0e8) break;
      chunk = 4;
    }
    const int steps = pin[kSp2Stop] < 1.0e8 ? (int)pin[kSp2Stop] + 1 : launched;
    g_prof.drop_last(gemm_stage, launched - steps);
    hint = steps;
    return steps;
  }

  // SP2 with the squarings on the tcgen05 tensor cores (3xTF32, fp32 accumulation). The
  // fp32 iterate reaches idempotency only to its rounding floor, so the density carries
  // about 1e-5 relative error: the SCF uses it for its early cycles only.
  bool project32(const double *F, int n_occ, double w, double *P) {
    ensure32();
    launch_gershgorin(st, n, F, scratch.p, bounds.p);
    launch_sp2_init32(st, n, ld, F, bounds.p, X32.p, hi32.p, lo32.p);
    const double scale = std::max(1, n_occ);
    const Sp2Rule rule{1.0e-6 * scale, 1.0e-2 * scale, kMaxSteps};
    last_iterations = run_chunks(
        [&](int s) {
          {
            Stage g_(st, "sp2_square_tf32");
            launch_square_tf32x3(st, n, ld, map_hi, map_lo, C32.p, err32.p, state.p, s);
          }
          launch_sp2_trace32(st, n, ld, X32.p, C32.p, (double)n_occ, state.p, s, rule);
          launch_sp2_update32(st, n, ld, X32.p, C32.p, state.p, hi32.p, lo32.p, s);
        },
        "sp2_square_tf32", hint32);
    bool ok = pin[kSp2Ok] != 0.0;
    // an idempotent X whose trace is not n_occ is a wrong projector (degenerate frontier)
    if (ok && std::fabs(pin[kSp2TrX] - (double)n_occ) > 1.0e-2 * scale) ok = false;
    int bad = 0;
    CUDA_OK(cudaMemcpyAsync(&bad, err32.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (bad) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 squaring: a pipeline wait expired"};
    if (!ok) return false;
    launch_sp2_density32(st, n, ld, X32.p, w, P);
    return true;
  }

  // Lanczos workspace for the tighter interval; once a refined interval has failed, this
  // purifier keeps to Gershgorin.
  DevBuf<double> lz;
  bool tight = true;

  // FP64-accuracy squarings on the integer tensor cores (int8 digit planes, kernels_i8.cu):
  // two plane sets, read and written alternately with X and X2, and their tensor maps.
  bool i8 = false;
  DevBuf<int8_t> dig0, dig1;
  DevBuf<int> i8err;
  alignas(64) unsigned char dmap[4][128];
  void ensure_i8() {
    if (dig0.p) return;
    dig0.alloc(sp2_i8_digit_bytes(n), st);
    dig1.alloc(sp2_i8_digit_bytes(n), st);
    i8err.alloc(1, st);
    CUDA_OK(cudaMemsetAsync(i8err.p, 0, sizeof(int), st));
    if (!make_digit_maps(dig0.p, n, dmap[0], dmap[1]) || !make_digit_maps(dig1.p, n, dmap[2], dmap[3]))
      throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
  }
  // 1: a pipeline wait expired (raised), 2: an iterate element left the digits' range (the
  // purification is treated as failed); the flag is cleared.
  int i8_status() {
    int e = 0;
    CUDA_OK(cudaMemcpyAsync(&e, i8err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (e == 1) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 i8 squaring: a pipeline wait expired"};
    if (e) CUDA_OK(cudaMemsetAsync(i8err.p, 0, sizeof(int), st));
    return e;
  }
  bool project(const double *F, int n_occ, double w, double *P) {
    if (tight && !lz.p) lz.alloc(lanczos_doubles(n), st);
    for (int attempt = 0; attempt < 2; ++attempt) {
      const bool refine = tight && attempt == 0;
      launch_gershgorin(st, n, F, scratch.p, bounds.p);
      if (refine) {
        Stage l_(st, "sp2_bounds");
        launch_lanczos_bounds(st, n, F, lz.p, bounds.p);
      }
      launch_sp2_init(st, n, F, bounds.p, X.p);
      const Sp2Rule rule{1.0e-13 * std::max(1, n_occ), 1.0e-6, kMaxSteps};
      // Fused steps on the ping-pong pair (X, X2): step s reads the iterate from one and
      // writes the next, already updated, to the other; its traces come from the previous
      // step's epilogue (the first from k_sp2_norms).
      if (!parts.p) parts.alloc(std::max(sp2_parts_doubles(n), 2 * (size_t)sp2_i8_tiles(n) + 8), st);
      if (i8) {
        ensure_i8();
        launch_sp2_digits(st, n, X.p, dig0.p, nullptr, -1, i8err.p);
      }
      const char *stage = i8 ? "sp2_square_i8" : "sp2_square_gemm";
      last_iterations = run_chunks(
          [&](int s) {
            if (s == 0) launch_sp2_norms(st, n, X.p, state.p, parts.p);
            launch_sp2_decide(st, (double)n_occ, state.p, parts.p, s, rule);
            Stage g_(st, stage);
            const double *in = s % 2 == 0 ? X.p : X2.p;
            double *out = s % 2 == 0 ? X2.p : X.p;
            if (i8)
              launch_sp2_step_i8(st, n, dmap[2 * (s % 2)], dmap[2 * (s % 2) + 1], in, out,
                                 s % 2 == 0 ? dig1.p : dig0.p, state.p, parts.p, s, i8err.p);
            else
              launch_sp2_step(st, n, in, out, state.p, parts.p, s);
          },
          stage, hint64);
      bool ok = pin[kSp2Ok] != 0.0;
      if (i8 && i8_status() != 0) ok = false;
      // an idempotent X whose trace is not n_occ is a wrong projector (degenerate frontier)
      if (ok && std::fabs(pin[kSp2TrX] - (double)n_occ) > 1.0e-3) ok = false;
      if (ok) {
        const int stop = (int)pin[kSp2Stop];  // the iterate after the last step is in its output
        launch_scale(st, (size_t)n * n, w, stop % 2 == 0 ? X2.p : X.p, P);
        return true;
      }
      if (!refine) return false;
      tight = false;  // the refined interval missed part of the spectrum: Gershgorin from now on
    }
    return false;
  }
};

// The fp64 SP2 squarings run on the integer tensor cores (kernels_i8.cu) from kI8MinN orbitals
// up, on the DMMA GEMM below (the two are level at ~600 orbitals: 0.051 ms per squaring at
// 600, 0.224 against 0.314 ms at 2,004, 4.2 against 6.9 ms at 6,000); PM7_SP2_GEMM=dmma|i8
// forces one.
constexpr int kI8MinN = 768;
static bool use_i8_sp2(int n) {
  const char *env = std::getenv("PM7_SP2_GEMM");
  if (env && std::strcmp(env, "dmma") == 0) return false;
  if (env && std::strcmp(env, "i8") == 0) return true;
  return n >= kI8MinN;
}

// Density solver for the SCF loop: SP2 above kJacobiMax orbitals (tensor-core squarings;
// 16 against 37 ms per solve at 240 orbitals), the eigendecomposition (Diag) up to it and
// when SP2 cannot settle. PM7_DENSITY_SOLVER=sp2|jacobi|syevd forces one (jacobi and syevd
// turn SP2 off; syevd also keeps the final eigenvalues on cuSOLVER).
// DIIS error below which the mixed-precision SCF switches to fp64 densities.
static constexpr double kMixedSwitch = 1.0e-3;
static constexpr double kMixedSwitchStep = 1.0e-6;  // rms density step that also ends the fp32 phase
// DIIS error (eV) above which an fp32 cycle also builds its Fock matrix in FP32: the guess and
// the first A-DIIS cycles. The FP32 build's ~1e-6 relative error stays in the DIIS history's
// Fock matrices, so the SCF may not end while the history holds one: the reported orbitals come
// from the last extrapolated Fock (on a 1,002-atom water cluster a switch at 0.1 took 20
// iterations instead of 17, one at 1 shifted the HOMO by 1e-3 eV; at 10 the last FP32 build is
// cycle 6 and the SCF still ends at 17 from a clean history).
static constexpr double kFock32Switch = 10.0;

static bool use_sp2(int n) {
  const char *env = std::getenv("PM7_DENSITY_SOLVER");
  if (env && (std::strcmp(env, "syevd") == 0 || std::strcmp(env, "jacobi") == 0)) return false;
  if (env && std::strcmp(env, "sp2") == 0) return true;
  return n > kJacobiMax;
}

static thread_local double *t_pinned_scalar = nullptr;  // set per solve from the context

static double host_sum(const DevBuf<double> &partials, size_t count, double *dscal, cudaStream_t st) {
  launch_sum(st, partials.p, count, dscal);
  double local = 0.0;
  double *v = t_pinned_scalar ? t_pinned_scalar : &local;
  CUDA_OK(cudaMemcpyAsync(v, dscal, sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  return *v;
}

// The reference's energy folds on the device (scf.rs:1237,1297-1298,1405,1503-1504): one
// reference-order sum per (density, matrix) pair, d[i] = fold of a[i] * b[i] over nn
// elements, queued on st. The host adds them left to right, as the reference's
// expression does.
static void queue_energy_folds(cudaStream_t st, size_t nn, int count, const double *const *a,
                               const double *const *b, double *d, void *scratch) {
  SeqSumBatch B{};
  for (int i = 0; i < count; ++i) B.job[i] = {a[i], b[i], nn, d + i};
  B.count = count;
  launch_seqsum(st, B, scratch);
}

struct ScfOut {
  bool converged = false;
  int iterations = 0;
  double density_error = std::numeric_limits<double>::infinity();
  double electronic_ev = 0.0;
  std::vector<double> eps_a, eps_b;
  DevBuf<double> P, Pspin, Va, Vb;  // total density, spin density, eigenvectors (rows)
  bool unrestricted = false;
  int n_occ = 0, n_occ_beta = -1;
  int fp32_iterations = 0;
};

// SAD guess diagonal (scf.rs:1050-1114).
std::vector<double> sad_diag(const Molecule &m, const Layout &L, const ParamSet &ps, double n_electrons) {
  std::vector<double> d(L.nao, 0.0);
  double tore = 0.0;
  for (int zz : m.z) tore += ps.element(zz)->core;
  const double yy = L.nao > 0 ? (tore - n_electrons) / L.nao : 0.0;
  for (int a = 0; a < m.n; ++a) {
    const ElementRec *e = ps.element(m.z[a]);
    const int off = L.aoff[a], no = L.norb[a], z = m.z[a];
    const double t = e->core;
    if (no == 1) {
      d[off] = t - yy;
    } else if (no == 4) {
      for (int k = 0; k < 4; ++k) d[off + k] = t * 0.25 - yy;
    } else if (no == 9) {
      const bool mg = z < 21 || (z > 30 && z < 39) || (z > 48 && z < 57);
      if (mg) {
        for (int k = 0; k < 4; ++k) d[off + k] = t * 0.25 - yy;
        for (int k = 4; k < 9; ++k) d[off + k] = -yy;
      } else {
        double sum = t - 9.0 * yy;
        d[off] = std::min(std::max(sum, 0.0), 2.0);
        sum -= 2.0;
        if (sum > 0.0) {
          for (int k = 4; k < 9; ++k) d[off + k] = std::min(std::max(sum * 0.2, 0.0), 2.0);
          sum -= 10.0;
          if (sum > 0.0)
            for (int k = 1; k < 4; ++k) d[off + k] = sum / 3.0;
        }
      }
    }
  }
  return d;
}

static void run_rhf(DeviceContext &ctx, const DeviceParams &P, DeviceMolecule &D, const Molecule &m,
                    const Layout &L, const ParamSet &ps, int n_occ, const pm7_options &o, ScfOut &out) {
  cudaStream_t st = ctx.stream;
  const int n = L.nao;
  const size_t nn = (size_t)n * n;
  const FockGeometry g = D.geometry();
  out.P.alloc(nn, st);
  DevBuf<double> Pnew, F, Fuse, X, partials, dscal, coef, dots;
  Pnew.alloc(nn, st);
  F.alloc(nn, st);
  Fuse.alloc(nn, st);
  X.alloc(nn, st);
  const int kmax = 8;
  std::vector<DevBuf<double>> hF(kmax), hE(kmax), hD(kmax);
  const bool accel_on = o.use_diis && o.accelerator != PM7_ACCEL_NONE;
  partials.alloc(std::max<size_t>(((size_t)(n + 31) / 32) * ((n + 31) / 32), 4096), st);
  dscal.alloc(8, st);
  DevBuf<unsigned char> folds;
  folds.alloc(seqsum_scratch_bytes(nn, 2), st);
  coef.alloc(kmax + 1, st);
  const int dot_blocks = 296;
  dots.alloc((size_t)dot_blocks * 32, st);
  DevBuf<double> dotout;
  dotout.alloc(64, st);
  DevBuf<const double *> ptrs;
  ptrs.alloc(64, st);

  if (o.initial_density) {
    CUDA_OK(cudaMemcpyAsync(out.P.p, o.initial_density, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
  } else {
    std::vector<double> diag = sad_diag(m, L, ps, 2.0 * n_occ);
    DevBuf<double> dd;
    upload(dd, diag, st);
    launch_set_diag(st, n, dd.p, out.P.p);
    CUDA_OK(cudaStreamSynchronize(st));
  }
  Diag eig(ctx, n, Fuse.p, reinterpret_cast<int *>(ctx.pinned + 8192));
  const bool sp2 = use_sp2(n);
  Purifier pur(st, sp2 ? n : 1, reinterpret_cast<double *>(ctx.pinned + 4096));
  pur.i8 = sp2 && use_i8_sp2(n);
  bool diagonalised = false;  // whether Fuse holds the eigenvectors of the last iteration
  // Mixed precision: fp32 (tcgen05) densities while the DIIS error is large, then fp64
  // refinement cycles; only an fp64 cycle may end the SCF.
  bool phase32 = sp2 && o.precision == PM7_PRECISION_MIXED;
  DevBuf<float> P32, w32;  // float copies of the density and the w store for the FP32 Fock build
  bool w32_ready = false;
  double last_err = std::numeric_limits<double>::infinity();
  std::vector<char> fock32_slot(kmax, 0);  // ring slots whose Fock matrix came from the FP32 build
  HistoryHost hist(kmax);
  StallGuardHost guard(o.level_shift);
  const bool trace = std::getenv("PM7_SCF_TRACE") != nullptr;
  double e_old = 0.0;
  for (int iter = 0; iter < o.max_scf; ++iter) {
    out.iterations = iter + 1;
    const int slot = hist.push();  // chronological bookkeeping of the ring
    if (!hF[slot].p) {
      hF[slot].alloc(nn, st);
      hE[slot].alloc(nn, st);
      hD[slot].alloc(nn, st);
    }
    double *Fk = hF[slot].p;
    fock32_slot[slot] = phase32 && last_err > kFock32Switch;
    if (fock32_slot[slot]) {
      Stage s_(st, "fock_fp32");
      if (!w32_ready) {
        P32.alloc(nn, st);
        w32.alloc((size_t)L.w_len, st);
        launch_to_float(st, (size_t)L.w_len, D.w.p, w32.p);
        w32_ready = true;
      }
      launch_to_float(st, nn, out.P.p, P32.p);
      launch_fock32(st, g, P, D.H.p, out.P.p, P32.p, P32.p, 0.5, Fk, D.pop.p, D.jbuf.p, w32.p);
    } else {
      Stage s_(st, "fock");
      launch_fock(st, g, P, D.H.p, out.P.p, out.P.p, 0.5, Fk, D.pop.p, D.jbuf.p);
    }
    // the iteration's energy for the convergence test, summed accurately: the reference's
    // folds carry ~1e-8 eV of rounding noise at a thousand atoms, the size of e_tol itself,
    // so they are kept for the reported energy only
    size_t ne = launch_energy(st, nn, out.P.p, D.H.p, Fk, partials.p);
    launch_sum(st, partials.p, ne, dscal.p + 0);
    CUDA_OK(cudaMemcpyAsync(hD[slot].p, out.P.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    // DIIS error e = F P - P F = F P - (F P)^T
    if (phase32) {
      // fp32 cycles: the product at fp32 accuracy (tcgen05), like their densities
      Stage s_(st, "commutator_tf32");
      pur.product32(Fk, out.P.p, X.p);
    } else {
      Stage s_(st, "commutator_gemm");
      launch_gemm_tn(st, n, n, n, 1.0, Fk, n, out.P.p, n, X.p, n);
    }
    size_t na = launch_antisym(st, n, X.p, hE[slot].p, partials.p);
    launch_sum(st, partials.p, na, dscal.p + 1);
    // inner products of the new entry with the history (chronological, newest last)
    const std::vector<int> older = hist.order();
    const int k = (int)older.size();
    std::vector<const double *> hp;
    for (int i = 0; i < k; ++i) hp.push_back(hE[older[i]].p);
    hp.push_back(hE[slot].p);
    for (int i = 0; i < k; ++i) hp.push_back(hF[older[i]].p);
    hp.push_back(Fk);
    for (int i = 0; i < k; ++i) hp.push_back(hD[older[i]].p);
    hp.push_back(hD[slot].p);
    const double **pin_ptrs = reinterpret_cast<const double **>(ctx.pinned + 1024);
    std::copy(hp.begin(), hp.end(), pin_ptrs);
    CUDA_OK(cudaMemcpyAsync(ptrs.p, pin_ptrs, sizeof(double *) * hp.size(), cudaMemcpyHostToDevice, st));
    const double *const *dE = ptrs.p, *const *dF = ptrs.p + (k + 1), *const *dD = ptrs.p + 2 * (k + 1);
    { Stage s_(st, "diis_dots"); launch_dot_many(st, nn, 1, dE + k, k + 1, dE, dots.p, dot_blocks); }  // <e_new, e_i>
    launch_reduce_rows(st, dots.p, dot_blocks, k + 1, dotout.p);
    { Stage s_(st, "diis_dots"); launch_dot_many(st, nn, 1, dD + k, k + 1, dF, dots.p, dot_blocks); }  // <D_new, F_j>
    launch_reduce_rows(st, dots.p, dot_blocks, k + 1, dotout.p + 16);
    if (k > 0) {
      { Stage s_(st, "diis_dots"); launch_dot_many(st, nn, 1, dF + k, k, dD, dots.p, dot_blocks); }  // <D_i, F_new>
      launch_reduce_rows(st, dots.p, dot_blocks, k, dotout.p + 32);
    }
    double *sc = reinterpret_cast<double *>(ctx.pinned), *dh = sc + 8;
    CUDA_OK(cudaMemcpyAsync(sc, dscal.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(dh, dotout.p, sizeof(double) * 48, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const double e_elec = 0.5 * sc[0];
    const double err_norm = std::sqrt(sc[1]);
    last_err = err_norm;
    hist.record(std::vector<double>(dh, dh + k + 1), std::vector<double>(dh + 16, dh + 16 + k + 1),
                std::vector<double>(dh + 32, dh + 32 + k));
    // extrapolation weights over the chronological history
    std::vector<double> w;
    if (accel_on) {
      if (o.accelerator == PM7_ACCEL_CDIIS || err_norm <= o.adiis_switch) w = hist.cdiis();
      else w = hist.adiis();
    }
    std::vector<const double *> fp;
    std::vector<double> cw;
    if (w.empty()) {
      fp.push_back(Fk);
      cw.push_back(1.0);
    } else {
      const std::vector<int> &ent = hist.entries();
      for (size_t i = 0; i < ent.size(); ++i)
        if (w[i] != 0.0) {  // an exact zero weight adds exactly nothing
          fp.push_back(hF[ent[i]].p);
          cw.push_back(w[i]);
        }
    }
    const double **pin_fp = reinterpret_cast<const double **>(ctx.pinned + 2048);
    double *pin_cw = reinterpret_cast<double *>(ctx.pinned + 3072);
    std::copy(fp.begin(), fp.end(), pin_fp);
    std::copy(cw.begin(), cw.end(), pin_cw);
    CUDA_OK(cudaMemcpyAsync(ptrs.p + 48, pin_fp, sizeof(double *) * fp.size(), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(coef.p, pin_cw, sizeof(double) * cw.size(), cudaMemcpyHostToDevice, st));
    { Stage s_(st, "combine"); launch_combine(st, n, (int)fp.size(), ptrs.p + 48, coef.p, out.P.p, 2.0, guard.shift, Fuse.p); }
    bool purified = false;
    // (the first cycles' error says nothing: a SAD guess proportional to I commutes with F;
    // for a large molecule the commutator norm can stall at the fp32 noise floor while the
    // density step is already small, so either criterion, or 40 fp32 cycles, ends the phase)
    if (phase32 && iter >= 2 &&
        (err_norm < kMixedSwitch || out.density_error < kMixedSwitchStep || out.fp32_iterations >= 40))
      phase32 = false;
    const bool used32 = phase32;
    if (sp2) {
      Stage s_(st, "sp2_purify");
      purified = used32 ? pur.project32(Fuse.p, n_occ, 2.0, Pnew.p) : pur.project(Fuse.p, n_occ, 2.0, Pnew.p);
    }
    if (used32) ++out.fp32_iterations;
    diagonalised = !purified;
    if (!purified) {
      { Stage s_(st, "eigensolve"); eig.solve(Fuse.p); }
      { Stage s_(st, "density_gemm"); launch_density(st, n, n_occ, 2.0, Fuse.p, n, Pnew.p); }
    }
    size_t nd = launch_sqdiff(st, nn, Pnew.p, out.P.p, partials.p);
    const double dp = std::sqrt(host_sum(partials, nd, dscal.p + 2, st) / (double)std::max<size_t>(nn, 1));
    eig.check();
    out.density_error = dp;
    const double de = std::fabs(e_elec - e_old);
    std::swap(out.P.p, Pnew.p);
    e_old = e_elec;
    const bool residual_ok = guard.shift == 0.0 && err_norm < 1.0e-7;
    bool hist64 = true;  // no Fock matrix of the DIIS history came from the FP32 build
    for (int e : hist.entries()) hist64 = hist64 && !fock32_slot[e];
    if (!used32 && hist64 && iter > 0 && de < o.e_tol && (dp < o.p_tol || residual_ok)) {
      out.converged = true;
      break;
    }
    guard.update(dp, e_elec);
    if (trace)
      std::fprintf(stderr, "scf %4d E %.10f dp %.3e err %.3e shift %.2f%s%s\n", out.iterations, e_elec, dp, err_norm,
                   guard.shift, used32 ? " fp32" : "", fock32_slot[slot] ? " fock32" : "");
  }
  // final Fock and energy at the converged density
  { Stage s_(st, "fock"); launch_fock(st, g, P, D.H.p, out.P.p, out.P.p, 0.5, F.p, D.pop.p, D.jbuf.p); }
  {
    const double *fa[2] = {out.P.p, out.P.p}, *fb[2] = {D.H.p, F.p};
    queue_energy_folds(st, nn, 2, fa, fb, dscal.p, folds.p);
    double *sc = reinterpret_cast<double *>(ctx.pinned);
    CUDA_OK(cudaMemcpyAsync(sc, dscal.p, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    out.electronic_ev = 0.5 * (sc[0] + sc[1]);
  }
  // Reported orbitals: the eigenvectors of the last extrapolated Fock, or of the real
  // Fock when a level shift was active (scf.rs:1299-1305); their energies alone when no
  // matrices are returned.
  const bool vectors = o.want_matrices != 0;
  if (guard.shift > 0.0) {
    CUDA_OK(cudaMemcpyAsync(Fuse.p, F.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    Stage s_(st, "eigensolve");
    if (vectors) eig.solve(Fuse.p, true);
    else eig.values(Fuse.p);
  } else if (!diagonalised) {
    Stage s_(st, "eigensolve");
    if (vectors) eig.solve(Fuse.p, true);
    else eig.values(Fuse.p);
  }
  if (vectors) {
    out.Va.alloc(nn, st);
    CUDA_OK(cudaMemcpyAsync(out.Va.p, Fuse.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
  }
  out.eps_a.resize(n);
  CUDA_OK(cudaMemcpyAsync(out.eps_a.data(), eig.eps(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  eig.check();
  out.n_occ = n_occ;
}

void eigvals_device(cudaStream_t st, const std::vector<EigvalsRequest> &req, EigvalsScratch &scr) {
  if (req.empty()) return;
  std::map<int, std::vector<int>> groups;  // cluster size -> requests
  size_t work = 0;
  for (size_t i = 0; i < req.size(); ++i) {
    const int n = req[i].n;
    if (!eigvals_supported(n) || req[i].ld < n)
      throw Failure{PM7_ERR_INVALID_INPUT, "eigenvalue solve: order " + std::to_string(n) + " not supported"};
    groups[tridiag_cluster_size(n)].push_back((int)i);
    work += (eigvals_work_doubles(n) + 31) / 32 * 32;
  }
  // per group: its tasks, then its prefix sums (int), in one uploaded block
  std::vector<unsigned char> meta;
  struct G {
    int c, count, max_n, total;
    size_t tasks_off, prefix_off;
  };
  std::vector<G> gs;
  std::vector<std::vector<EigvalsTask>> tasks_of;
  for (auto &kv : groups) {
    G g{kv.first, (int)kv.second.size(), 0, 0, 0, 0};
    std::vector<int> prefix;
    for (int i : kv.second) {
      prefix.push_back(g.total);
      g.total += req[i].n;
      g.max_n = std::max(g.max_n, req[i].n);
    }
    g.tasks_off = (meta.size() + 63) / 64 * 64;
    meta.resize(g.tasks_off + sizeof(EigvalsTask) * kv.second.size());
    g.prefix_off = (meta.size() + 63) / 64 * 64;
    meta.resize(g.prefix_off + sizeof(int) * prefix.size());
    std::memcpy(meta.data() + g.prefix_off, prefix.data(), sizeof(int) * prefix.size());
    gs.push_back(g);
  }
  if (work > scr.cap) {
    if (scr.work) CUDA_OK(cudaFreeAsync(scr.work, st));
    scr.cap = work + work / 4;
    CUDA_OK(cudaMallocAsync((void **)&scr.work, sizeof(double) * scr.cap, st));
  }
  if (!scr.uploaded) CUDA_OK(cudaEventCreateWithFlags(&scr.uploaded, cudaEventDisableTiming));
  CUDA_OK(cudaEventSynchronize(scr.uploaded));  // the previous table was read: pinned is free
  if (meta.size() > scr.meta_cap) {
    if (scr.meta) CUDA_OK(cudaFreeAsync(scr.meta, st));
    if (scr.pinned) CUDA_OK(cudaFreeHost(scr.pinned));
    scr.meta_cap = meta.size() + meta.size() / 4 + 256;
    CUDA_OK(cudaMallocAsync((void **)&scr.meta, scr.meta_cap, st));
    CUDA_OK(cudaMallocHost((void **)&scr.pinned, scr.meta_cap));
  }
  size_t woff = 0;
  size_t k = 0;
  for (auto &kv : groups) {
    EigvalsTask *out = reinterpret_cast<EigvalsTask *>(meta.data() + gs[k].tasks_off);
    for (size_t q = 0; q < kv.second.size(); ++q) {
      const EigvalsRequest &r = req[kv.second[q]];
      EigvalsTask t{};
      t.src = r.src;
      t.n = r.n;
      t.ld = r.ld;
      t.eps = r.eps;
      eigvals_task_layout(t, scr.work + woff);
      woff += (eigvals_work_doubles(t.n) + 31) / 32 * 32;
      std::memcpy(out + q, &t, sizeof(t));
    }
    ++k;
  }
  std::memcpy(scr.pinned, meta.data(), meta.size());
  CUDA_OK(cudaMemcpyAsync(scr.meta, scr.pinned, meta.size(), cudaMemcpyHostToDevice, st));
  CUDA_OK(cudaEventRecord(scr.uploaded, st));
  for (const G &g : gs) {
    const cudaError_t err =
        launch_eigvals(st, reinterpret_cast<const EigvalsTask *>(scr.meta + g.tasks_off), g.count, g.c, g.max_n,
                       reinterpret_cast<const int *>(scr.meta + g.prefix_off), g.total);
    if (err != cudaSuccess) throw Failure{PM7_ERR_CUDA, std::string("eigenvalue solve: ") + cudaGetErrorString(err)};
  }
}

static void run_uhf(DeviceContext &ctx, const DeviceParams &P, DeviceMolecule &D, const Molecule &m,
                    const Layout &L, const ParamSet &ps, int n_alpha, int n_beta, const pm7_options &o,
                    ScfOut &out) {
  cudaStream_t st = ctx.stream;
  const int n = L.nao;
  const size_t nn = (size_t)n * n;
  const FockGeometry g = D.geometry();
  DevBuf<double> Pa, Pb, Pt, Fa, Fb, X, E, Ua, Ub, partials, dscal, Pan, Pbn;
  for (DevBuf<double> *b : {&Pa, &Pb, &Pt, &Fa, &Fb, &X, &E, &Ua, &Ub, &Pan, &Pbn}) b->alloc(nn, st);
  partials.alloc(std::max<size_t>(((size_t)(n + 31) / 32) * ((n + 31) / 32), 4096), st);
  dscal.alloc(8, st);
  DevBuf<unsigned char> folds;
  folds.alloc(seqsum_scratch_bytes(nn, 3), st);
  const double ntot = std::max(n_alpha + n_beta, 1);
  {
    DevBuf<double> total;
    total.alloc(nn, st);
    if (o.initial_density) {
      CUDA_OK(cudaMemcpyAsync(total.p, o.initial_density, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
    } else {
      std::vector<double> diag = sad_diag(m, L, ps, (double)(n_alpha + n_beta));
      DevBuf<double> dd;
      upload(dd, diag, st);
      launch_set_diag(st, n, dd.p, total.p);
      CUDA_OK(cudaStreamSynchronize(st));
    }
    launch_scale(st, nn, n_alpha / ntot, total.p, Pa.p);
    launch_scale(st, nn, n_beta / ntot, total.p, Pb.p);
    if (o.initial_spin_density) {
      DevBuf<double> s;
      s.alloc(nn, st);
      CUDA_OK(cudaMemcpyAsync(s.p, o.initial_spin_density, sizeof(double) * nn, cudaMemcpyHostToDevice, st));
      launch_axpby(st, nn, 1.0, Pa.p, 0.5, s.p, Pa.p);
      launch_axpby(st, nn, 1.0, Pb.p, -0.5, s.p, Pb.p);
      CUDA_OK(cudaStreamSynchronize(st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
  }
  Diag eig(ctx, n, Ua.p, reinterpret_cast<int *>(ctx.pinned + 8192));
  Diag eig_b(ctx, n, Ub.p, reinterpret_cast<int *>(ctx.pinned + 8192 + 64));
  const bool sp2 = use_sp2(n);
  Purifier pur(st, sp2 ? n : 1, reinterpret_cast<double *>(ctx.pinned + 4096));
  pur.i8 = sp2 && use_i8_sp2(n);
  bool diag_a = false;  // whether Ua holds the alpha eigenvectors of the last iteration
  DevBuf<double> eps_b;
  eps_b.alloc(n, st);
  StallGuardHost guard(o.level_shift);
  const bool trace = std::getenv("PM7_SCF_TRACE") != nullptr;
  double e_old = 0.0;
  // <Pt, H>, <Pa, Fa>, <Pb, Fb> into dscal[0..3): summed accurately for the iterations'
  // convergence test, as the reference's folds for the reported energy (`folds`)
  auto energy = [&](const double *pt, const double *pa, const double *fa, const double *pb, const double *fb,
                    bool folds_order) {
    if (folds_order) {
      const double *xa[3] = {pt, pa, pb}, *xb[3] = {D.H.p, fa, fb};
      queue_energy_folds(st, nn, 3, xa, xb, dscal.p, folds.p);
      return;
    }
    size_t c1 = launch_dot(st, nn, pt, D.H.p, partials.p);
    launch_sum(st, partials.p, c1, dscal.p + 0);
    c1 = launch_dot(st, nn, pa, fa, partials.p);
    launch_sum(st, partials.p, c1, dscal.p + 1);
    c1 = launch_dot(st, nn, pb, fb, partials.p);
    launch_sum(st, partials.p, c1, dscal.p + 2);
  };
  for (int iter = 0; iter < o.max_scf; ++iter) {
    out.iterations = iter + 1;
    launch_axpby(st, nn, 1.0, Pa.p, 1.0, Pb.p, Pt.p);
    { Stage s_(st, "fock"); launch_fock(st, g, P, D.H.p, Pt.p, Pa.p, 1.0, Fa.p, D.pop.p, D.jbuf.p); }
    { Stage s_(st, "fock"); launch_fock(st, g, P, D.H.p, Pt.p, Pb.p, 1.0, Fb.p, D.pop.p, D.jbuf.p); }
    energy(Pt.p, Pa.p, Fa.p, Pb.p, Fb.p, false);
    { Stage s_(st, "commutator_gemm"); launch_gemm_tn(st, n, n, n, 1.0, Fa.p, n, Pa.p, n, X.p, n); }
    size_t c = launch_antisym(st, n, X.p, E.p, partials.p);
    launch_sum(st, partials.p, c, dscal.p + 3);
    { Stage s_(st, "commutator_gemm"); launch_gemm_tn(st, n, n, n, 1.0, Fb.p, n, Pb.p, n, X.p, n); }
    c = launch_antisym(st, n, X.p, E.p, partials.p);
    launch_sum(st, partials.p, c, dscal.p + 4);
    double sc[5];
    CUDA_OK(cudaMemcpyAsync(sc, dscal.p, sizeof(double) * 5, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const double e_elec = 0.5 * (sc[0] + sc[1] + sc[2]);
    const double err_norm = std::sqrt(sc[3] + sc[4]);
    const double one = 1.0;
    double *dcoef = dscal.p + 6;
    CUDA_OK(cudaMemcpyAsync(dcoef, &one, sizeof(double), cudaMemcpyHostToDevice, st));
    DevBuf<const double *> ptr;
    ptr.alloc(2, st);
    const double *pp[2] = {Fa.p, Fb.p};
    CUDA_OK(cudaMemcpyAsync(ptr.p, pp, sizeof(pp), cudaMemcpyHostToDevice, st));
    { Stage s_(st, "combine"); launch_combine(st, n, 1, ptr.p, dcoef, Pa.p, 1.0, guard.shift, Ua.p); }
    { Stage s_(st, "combine"); launch_combine(st, n, 1, ptr.p + 1, dcoef, Pb.p, 1.0, guard.shift, Ub.p); }
    std::vector<double> ea(n, 0.0);
    bool pa_ok = false, pb_ok = false;
    if (sp2) {
      Stage s_(st, "sp2_purify");
      pa_ok = pur.project(Ua.p, n_alpha, 1.0, Pan.p);
      pb_ok = pur.project(Ub.p, n_beta, 1.0, Pbn.p);
    }
    diag_a = !pa_ok;
    if (!pa_ok) {
      { Stage s_(st, "eigensolve"); eig.solve(Ua.p); }
      { Stage s_(st, "density_gemm"); launch_density(st, n, n_alpha, 1.0, Ua.p, n, Pan.p); }
      CUDA_OK(cudaMemcpyAsync(ea.data(), eig.eps(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    }
    if (!pb_ok) {
      { Stage s_(st, "eigensolve"); eig_b.solve(Ub.p); }
      { Stage s_(st, "density_gemm"); launch_density(st, n, n_beta, 1.0, Ub.p, n, Pbn.p); }
    }
    size_t c2 = launch_sqdiff(st, nn, Pan.p, Pa.p, partials.p);
    const double dpa = std::sqrt(host_sum(partials, c2, dscal.p + 5, st) / (double)nn);
    c2 = launch_sqdiff(st, nn, Pbn.p, Pb.p, partials.p);
    const double dpb = std::sqrt(host_sum(partials, c2, dscal.p + 5, st) / (double)nn);
    eig.check();
    eig_b.check();
    const double dp = dpa + dpb;
    out.density_error = dp;
    out.eps_a = ea;
    const double de = std::fabs(e_elec - e_old);
    std::swap(Pa.p, Pan.p);
    std::swap(Pb.p, Pbn.p);
    e_old = e_elec;
    const bool residual_ok = guard.shift == 0.0 && err_norm < 1.0e-7;
    if (iter > 0 && de < o.e_tol && (dp < o.p_tol || residual_ok)) {
      out.converged = true;
      break;
    }
    guard.update(dp, e_elec);
    if (trace)
      std::fprintf(stderr, "scf %4d E %.10f dp %.3e err %.3e shift %.2f (uhf)\n", out.iterations, e_elec, dp,
                   err_norm, guard.shift);
  }
  out.P.alloc(nn, st);
  out.Pspin.alloc(nn, st);
  launch_axpby(st, nn, 1.0, Pa.p, 1.0, Pb.p, out.P.p);
  launch_axpby(st, nn, 1.0, Pa.p, -1.0, Pb.p, out.Pspin.p);
  { Stage s_(st, "fock"); launch_fock(st, g, P, D.H.p, out.P.p, Pa.p, 1.0, Fa.p, D.pop.p, D.jbuf.p); }
  { Stage s_(st, "fock"); launch_fock(st, g, P, D.H.p, out.P.p, Pb.p, 1.0, Fb.p, D.pop.p, D.jbuf.p); }
  energy(out.P.p, Pa.p, Fa.p, Pb.p, Fb.p, true);
  double sc[3];
  CUDA_OK(cudaMemcpyAsync(sc, dscal.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  out.electronic_ev = 0.5 * (sc[0] + sc[1] + sc[2]);
  out.Va.alloc(nn, st);
  out.Vb.alloc(nn, st);
  if (guard.shift > 0.0) {
    CUDA_OK(cudaMemcpyAsync(Ua.p, Fa.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
    { Stage s_(st, "eigensolve"); eig.solve(Ua.p); }
    out.eps_a.resize(n);
    CUDA_OK(cudaMemcpyAsync(out.eps_a.data(), eig.eps(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  } else if (!diag_a) {
    { Stage s_(st, "eigensolve"); eig.solve(Ua.p); }
    out.eps_a.resize(n);
    CUDA_OK(cudaMemcpyAsync(out.eps_a.data(), eig.eps(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  }
  CUDA_OK(cudaMemcpyAsync(out.Va.p, Ua.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
  CUDA_OK(cudaMemcpyAsync(Ub.p, Fb.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
  { Stage s_(st, "eigensolve"); eig_b.solve(Ub.p); }
  CUDA_OK(cudaMemcpyAsync(out.Vb.p, Ub.p, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st));
  out.eps_b.resize(n);
  CUDA_OK(cudaMemcpyAsync(out.eps_b.data(), eig_b.eps(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  eig.check();
  eig_b.check();
  out.unrestricted = true;
  out.n_occ = n_alpha;
  out.n_occ_beta = n_beta;
}

// ---------------------------------------------------------------------------
// run_pm7
// ---------------------------------------------------------------------------
double *host_copy(const double *src_dev, size_t count, cudaStream_t st) {
  double *h = (double *)std::malloc(sizeof(double) * std::max<size_t>(count, 1));
  if (count) CUDA_OK(cudaMemcpyAsync(h, src_dev, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
  return h;
}

double *host_vec(const std::vector<double> &v) {
  double *h = (double *)std::malloc(sizeof(double) * std::max<size_t>(v.size(), 1));
  std::memcpy(h, v.data(), sizeof(double) * v.size());
  return h;
}

uint64_t device_budget(int64_t explicit_mb) {
  if (explicit_mb >= 0) return (uint64_t)explicit_mb << 20;
  if (const char *s = std::getenv("PM7_MEM_BUDGET_MB")) {
    char *end = nullptr;
    unsigned long long mb = std::strtoull(s, &end, 10);
    if (end != s) return (uint64_t)mb << 20;
  }
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
  return free_b / 5 * 4;
}

Molecule to_molecule(const pm7_molecule *mol) {
  if (!mol || mol->n_atoms < 0 || (mol->n_atoms > 0 && (!mol->z || !mol->xyz_bohr)))
    throw Failure{PM7_ERR_INVALID_INPUT, "null molecule"};
  Molecule m;
  m.n = mol->n_atoms;
  m.z.assign(mol->z, mol->z + m.n);
  m.xyz.assign(mol->xyz_bohr, mol->xyz_bohr + 3 * (size_t)m.n);
  return m;
}

void fill_result(pm7_result *res, const Molecule &m, const Layout &L, const ParamSet &ps, const pm7_options &o,
                 const ResultParts &S, const std::vector<double> &pops,
                 const std::function<double(int, int, int)> &Pm) {
  // correction sum in the reference's order (scf.rs:907-932)
  double corr = S.corr[0];
  corr += S.corr[1];
  corr += S.corr[4];
  corr += S.corr[2];
  corr += S.corr[3];
  const double total = S.electronic_ev + S.core_ev + corr * kKcalToEv;
  double e_isol = 0.0, eheat = 0.0;
  for (int zz : m.z) {
    e_isol += ps.element(zz)->e_isol;
    eheat += ps.element(zz)->eheat_ev;
  }
  const double dhf = (S.electronic_ev + S.core_ev - e_isol + eheat) * kEvToKcal + corr;
  std::memset(res, 0, sizeof(*res));
  res->iterations = S.iterations;
  res->density_error = S.density_error;
  res->fp32_iterations = S.fp32_iterations;
  if (!S.converged) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "PM7 SCF did not converge after %d iterations (error=%.3e)", S.iterations,
                  S.density_error);
    throw Failure{PM7_ERR_SCF_NOT_CONVERGED, buf};
  }
  const int nao = L.nao;
  std::vector<double> q(m.n);
  for (int a = 0; a < m.n; ++a) q[a] = ps.element(m.z[a])->core - pops[a];
  res->n_atoms = m.n;
  res->nao = nao;
  res->n_occ = S.n_occ;
  res->n_occ_beta = S.n_occ_beta;
  res->unrestricted = S.unrestricted;
  res->converged = 1;
  res->electronic_ev = S.electronic_ev;
  res->core_ev = S.core_ev;
  res->total_ev = total;
  res->heat_of_formation_kcal = dhf;
  res->correction_kcal = corr;
  res->device_ms = S.device_ms;
  // dipole breakdown (dipole.rs:282-350)
  {
    double ox = 0, oy = 0, oz = 0, net = 0;
    for (double v : q) net += v;
    if (std::fabs(net) > 0.5 && o.dipole_origin != PM7_DIPOLE_COORDINATES) {
      double tx = 0, ty = 0, tz = 0, tot = 0;
      for (int a = 0; a < m.n; ++a) {
        const double wgt = o.dipole_origin == PM7_DIPOLE_CENTRE_OF_MASS ? (m.z[a] < 87 ? pm7_mass_table()[m.z[a]] : 0.0)
                                                                        : ps.element(m.z[a])->core;
        tx += m.xyz[3 * a] * wgt;
        ty += m.xyz[3 * a + 1] * wgt;
        tz += m.xyz[3 * a + 2] * wgt;
        tot += wgt;
      }
      if (tot > 0.0) {
        ox = tx / tot;
        oy = ty / tot;
        oz = tz / tot;
      }
    }
    double pc[3] = {0, 0, 0}, sp[3] = {0, 0, 0}, pd[3] = {0, 0, 0};
    const double inv3 = 0.5773502691896258;
    for (int a = 0; a < m.n; ++a) {
      pc[0] += (m.xyz[3 * a] - ox) * q[a];
      pc[1] += (m.xyz[3 * a + 1] - oy) * q[a];
      pc[2] += (m.xyz[3 * a + 2] - oz) * q[a];
      const ElementRec *e = ps.element(m.z[a]);
      if (e->n_orb >= 4) {
        const double hyb = -2.0 * e->dd;
        for (int k = 0; k < 3; ++k) sp[k] += hyb * Pm(a, 0, 1 + k);
      }
      if (e->n_orb == 9) {
        const double hyb = -2.0 * e->ddp[5];
        pd[0] += hyb * (Pm(a, 5, 3) + Pm(a, 4, 1) + Pm(a, 8, 2) - inv3 * Pm(a, 6, 1));
        pd[1] += hyb * (Pm(a, 7, 3) - Pm(a, 4, 2) + Pm(a, 8, 1) - inv3 * Pm(a, 6, 2));
        pd[2] += hyb * (Pm(a, 5, 1) + Pm(a, 7, 2) + 2.0 * inv3 * Pm(a, 6, 3));
      }
    }
    double mag = 0.0;
    for (int k = 0; k < 3; ++k) {
      res->dipole_point_charge[k] = pc[k] * kAuDipoleToDebye;
      res->dipole_sp_hybrid[k] = sp[k] * kAuDipoleToDebye;
      res->dipole_pd_hybrid[k] = pd[k] * kAuDipoleToDebye;
      res->dipole_debye[k] = res->dipole_point_charge[k] + res->dipole_sp_hybrid[k] + res->dipole_pd_hybrid[k];
      mag += res->dipole_debye[k] * res->dipole_debye[k];
    }
    res->dipole_magnitude = std::sqrt(mag);
  }
  const double nan = std::numeric_limits<double>::quiet_NaN();
  res->homo_ev = S.n_occ >= 1 ? S.eps_a[S.n_occ - 1] : nan;
  res->lumo_ev = S.n_occ < nao ? S.eps_a[S.n_occ] : nan;
  res->homo_ev_beta = res->lumo_ev_beta = nan;
  if (S.unrestricted) {
    res->homo_ev_beta = S.n_occ_beta >= 1 ? S.eps_b[S.n_occ_beta - 1] : nan;
    res->lumo_ev_beta = S.n_occ_beta < nao ? S.eps_b[S.n_occ_beta] : nan;
  }
  res->charges = host_vec(q);
  res->mo_energies = host_vec(S.eps_a);
  if (S.unrestricted) res->mo_energies_beta = host_vec(S.eps_b);
}

// Displaced geometry copies per pass of the correction gradient: all 12 n at once when they fit
// in ~1 GB of device memory (and the grid's z extent), else as many as do.
static int correction_copies(int n, int smooth) {
  const size_t per = corrections_gradient_work(n, 1, smooth) - corrections_gradient_work(n, 0, smooth);
  return (int)std::max<size_t>(1, std::min<size_t>({(size_t)kStencil * n + 1, (size_t)65535, ((size_t)1 << 27) / per}));
}

// Nuclear gradient (eV/Bohr) of a molecule on the device at the density g.Pt (total) / g.Ps
// (spin, null for a closed shell): core-core + electronic pair terms (src/gradient.rs:654-700,
// 1082-1247) and, with `corrections`, the post-SCF correction gradient (:208-261). g's atoms,
// AO offsets, coordinates, near mask and near pairs are the molecule's; g.E and g.status are set
// here.
std::vector<double> geometry_gradient(cudaStream_t st, const DeviceParams &P, GradGeometry g, bool dpath, int method,
                                      int smooth, bool corrections, bool any_si) {
  const int n = g.n_atoms;
  std::vector<double> grad(3 * (size_t)n, 0.0);
  if (n == 0) return grad;
  const size_t npairs = (size_t)n * (size_t)(n - 1) / 2;
  {
    // the stencil energies (12 per atom pair) are the gradient's one large buffer
    size_t free_b = 0, total_b = 0;
    CUDA_OK(cudaMemGetInfo(&free_b, &total_b));
    const size_t need = npairs * kStencil * sizeof(double);
    if (need > free_b)
      throw Failure{PM7_ERR_INSUFFICIENT_MEMORY, "gradient needs " + std::to_string(need >> 20) +
                                                     " MB of stencil energies, " + std::to_string(free_b >> 20) +
                                                     " MB free on the device"};
  }
  DevBuf<double> E, G;
  DevBuf<int> status;
  E.alloc(npairs * kStencil, st);
  G.alloc(3 * (size_t)n, st);
  status.alloc(1, st);
  CUDA_OK(cudaMemsetAsync(status.p, 0, sizeof(int), st));
  g.E = E.p;
  g.status = status.p;
  {
    Stage s_(st, "gradient_pairs");
    if (dpath) {
      launch_grad_pairs_d(st, g, P);
      launch_grad_near_d(st, g, P);
    } else {
      launch_grad_pairs_sp(st, g, P);
      launch_grad_near_sp(st, g, P);
    }
    launch_grad_atoms(st, g, G.p);
  }
  if (corrections && method != 3) {
    Stage s_(st, "gradient_corrections");
    const int copies = correction_copies(n, smooth);
    DevBuf<double> work, energies, cg;
    work.alloc(corrections_gradient_work(n, copies, smooth), st);
    energies.alloc((size_t)kStencil * n + 1, st);
    cg.alloc(3 * (size_t)n, st);
    launch_corrections_gradient(st, n, g.z, g.xyz, method, smooth, any_si, copies, work.p, energies.p, cg.p);
    launch_grad_add(st, n, kKcalToEv, cg.p, G.p);
  }
  int bad = 0;
  CUDA_OK(cudaMemcpyAsync(grad.data(), G.p, sizeof(double) * grad.size(), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(&bad, status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  CUDA_OK(cudaGetLastError());
  if (bad & 1) throw Failure{PM7_ERR_UNSUPPORTED, "gradient: a shell pair without an overlap formula"};
  if (bad & 2) throw Failure{PM7_ERR_INVALID_INPUT, "gradient: d-shell pair in the sp frame"};
  return grad;
}

// The same for the built single-molecule device state D.
static std::vector<double> device_gradient(cudaStream_t st, const DeviceParams &P, const DeviceMolecule &D, bool dpath,
                                           const double *Pt, const double *Ps, int method, int smooth,
                                           bool corrections, bool any_si) {
  GradGeometry g{};
  g.n_atoms = D.n;
  g.nao = D.nao;
  g.n_near = D.n_near;
  g.z = D.z.p;
  g.aoff = D.aoff.p;
  g.xyz = D.xyz.p;
  g.near_mask = D.mask.p;
  g.np = D.near.p;
  g.Pt = Pt;
  g.Ps = Ps;
  return geometry_gradient(st, P, g, dpath, method, smooth, corrections, any_si);
}

// Host-side phase times of one pm7_run on stderr (PM7_HOST_TRACE set): where the wall time
// beyond the device's goes.
struct HostTrace {
  bool on = std::getenv("PM7_HOST_TRACE") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  std::string line;
  void mark(const char *what) {
    if (!on) return;
    const auto now = std::chrono::steady_clock::now();
    char buf[64];
    std::snprintf(buf, sizeof buf, " %s %.3f", what, std::chrono::duration<double, std::milli>(now - t).count());
    line += buf;
    t = now;
  }
  ~HostTrace() {
    if (on) std::fprintf(stderr, "pm7_run host ms:%s\n", line.c_str());
  }
};

static void run_impl(const pm7_molecule *mol, const pm7_params *params, const pm7_options *opt, pm7_result *res,
                     std::vector<double> *gradient = nullptr) {
  if (!opt || !res || !params) throw Failure{PM7_ERR_INVALID_INPUT, "null argument"};
  HostTrace ht;
  const pm7_options &o = *opt;
  Molecule m = to_molecule(mol);
  validate(m, o);
  ht.mark("validate");
  const int pmethod = *reinterpret_cast<const int *>(params);
  if (o.method != pmethod)
    throw Failure{PM7_ERR_INVALID_INPUT, "options method does not match parameter method"};
  if (o.multiplicity < 1) throw Failure{PM7_ERR_INVALID_INPUT, "multiplicity must be >= 1"};
  if (o.precision != PM7_PRECISION_FP64 && o.precision != PM7_PRECISION_MIXED)
    throw Failure{PM7_ERR_INVALID_INPUT, "unknown precision mode"};
  const ParamSet &ps = param_set(o.method);
  Layout L = build_layout(m, ps);
  ht.mark("layout");
  DeviceContext &ctx = context_for(o.device);
  std::lock_guard<std::mutex> lock(ctx.run_mutex);
  CUDA_OK(cudaSetDevice(ctx.device));
  {
    // Pre-flight memory guard (memory.rs:95-118) against the device's HBM.
    const bool has_d = o.force_dpath || L.has_d;
    const uint64_t mat = (uint64_t)L.nao * L.nao * 8;
    const uint64_t pairs = (uint64_t)m.n * (m.n > 0 ? m.n - 1 : 0) / 2;
    const uint64_t need = mat * 30 + pairs * (has_d ? 18000 : 2400);
    const uint64_t budget = device_budget(o.max_memory_mb);
    if (budget > 0 && need > budget)
      throw Failure{PM7_ERR_INSUFFICIENT_MEMORY, "estimated SCF memory ~" + std::to_string((need + (1 << 20) - 1) >> 20) +
                                                     " MB exceeds the " + std::to_string(budget >> 20) + " MB budget"};
  }
  const DeviceParams &P = device_params(ctx, o.method);
  cudaStream_t st = ctx.stream;
  t_pinned_scalar = reinterpret_cast<double *>(ctx.pinned + 4608);
  cudaEvent_t t0, t1;
  CUDA_OK(cudaEventCreate(&t0));
  CUDA_OK(cudaEventCreate(&t1));
  CUDA_OK(cudaEventRecord(t0, st));
  DeviceMolecule D;
  { Stage s_(st, "build"); build_device_molecule(D, m, L, P, o.force_dpath || L.has_d, st); }
  ht.mark("build_queued");
  // electron count and spin (scf.rs:588-627)
  double n_elec = 0.0;
  for (int zz : m.z) n_elec += ps.element(zz)->core;
  n_elec -= o.charge;
  const long long ni = std::llround(n_elec);
  if (std::fabs(n_elec - (double)ni) > 1.0e-6 || ni < 0)
    throw Failure{PM7_ERR_INVALID_INPUT, "invalid electron count " + std::to_string(n_elec)};
  const long long unp = o.multiplicity - 1;
  if (ni - unp < 0 || (ni - unp) % 2 != 0)
    throw Failure{PM7_ERR_INVALID_INPUT, "electron count " + std::to_string(ni) + " is incompatible with multiplicity " +
                                             std::to_string(o.multiplicity) + " (need same parity)"};
  const int n_alpha = (int)((ni + unp) / 2), n_beta = (int)((ni - unp) / 2);
  bool uhf;
  if (o.reference == PM7_REF_AUTO) uhf = n_alpha != n_beta;
  else if (o.reference == PM7_REF_UNRESTRICTED) uhf = true;
  else {
    if (n_alpha != n_beta)
      throw Failure{PM7_ERR_INVALID_INPUT, "restricted (RHF) needs a closed shell, but multiplicity " +
                                               std::to_string(o.multiplicity) + " gives " + std::to_string(n_alpha) +
                                               "a/" + std::to_string(n_beta) + "b; use UHF"};
    uhf = false;
  }
  ScfOut S;
  if (uhf) run_uhf(ctx, P, D, m, L, ps, n_alpha, n_beta, o, S);
  else run_rhf(ctx, P, D, m, L, ps, n_alpha, o, S);
  ht.mark("scf");
  // post-SCF corrections on the device (scf.rs:907-932)
  DevBuf<double> cscratch, cout;
  cscratch.alloc(corrections_scratch(m.n), st);
  cout.alloc(5, st);
  { Stage s_(st, "corrections"); launch_corrections(st, m.n, D.z.p, D.xyz.p, o.method, o.smooth_dispersion, cscratch.p, cscratch.n, cout.p); }
  double parts[5];
  CUDA_OK(cudaMemcpyAsync(parts, cout.p, sizeof(parts), cudaMemcpyDeviceToHost, st));
  // per-atom populations and the hybrid-dipole density elements
  std::vector<double> diag_blocks;
  {
    DevBuf<double> pop;
    pop.alloc(m.n, st);
    launch_atom_pop(st, m.n, D.aoff.p, D.z.p, P, L.nao, S.P.p, pop.p);
    diag_blocks.resize(m.n);
    CUDA_OK(cudaMemcpyAsync(diag_blocks.data(), pop.p, sizeof(double) * m.n, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
  }
  CUDA_OK(cudaEventRecord(t1, st));
  CUDA_OK(cudaEventSynchronize(t1));
  ht.mark("corrections");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, t0, t1);
  g_prof.flush();
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);

  ResultParts R;
  R.iterations = S.iterations;
  R.density_error = S.density_error;
  R.converged = S.converged;
  R.electronic_ev = S.electronic_ev;
  R.core_ev = D.core_core_ev;
  for (int k = 0; k < 5; ++k) R.corr[k] = parts[k];
  R.n_occ = S.n_occ;
  R.n_occ_beta = S.n_occ_beta;
  R.unrestricted = S.unrestricted;
  R.eps_a = S.eps_a;
  R.eps_b = S.eps_b;
  R.device_ms = ms;
  R.fp32_iterations = S.fp32_iterations;
  const int nao = L.nao;
  const size_t nn = (size_t)nao * nao;
  // The density back on the host: all of it when it is returned, else only the atom
  // blocks the dipole needs (a full nao^2 copy is ~30 MB at 2,000 basis functions).
  std::vector<double> Ph, blocks;
  if (S.converged) {
    if (o.want_matrices) {
      Ph.resize(nn);
      CUDA_OK(cudaMemcpyAsync(Ph.data(), S.P.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    } else {
      DevBuf<double> B;
      B.alloc((size_t)81 * m.n, st);
      launch_atom_blocks(st, m.n, D.aoff.p, D.z.p, P, nao, S.P.p, B.p);
      blocks.resize((size_t)81 * m.n);
      CUDA_OK(cudaMemcpyAsync(blocks.data(), B.p, sizeof(double) * blocks.size(), cudaMemcpyDeviceToHost, st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
  }
  ht.mark("readback");
  if (gradient && S.converged)
    *gradient = device_gradient(st, P, D, o.force_dpath || L.has_d, S.P.p, S.unrestricted ? S.Pspin.p : nullptr,
                                o.method, o.smooth_dispersion, true,
                                std::find(m.z.begin(), m.z.end(), 14) != m.z.end());
  fill_result(res, m, L, ps, o, R, diag_blocks, [&](int a, int i, int j) {
    return o.want_matrices ? Ph[(size_t)(L.aoff[a] + i) * nao + L.aoff[a] + j] : blocks[(size_t)81 * a + 9 * i + j];
  });
  ht.mark("result");
  if (o.want_matrices) {
    res->density = host_vec(Ph);
    if (S.unrestricted) res->spin_density = host_copy(S.Pspin.p, nn, st);
    DevBuf<double> T;
    T.alloc(nn, st);
    launch_transpose(st, nao, S.Va.p, T.p);
    res->mo_coeff = host_copy(T.p, nn, st);
    if (S.unrestricted) {
      launch_transpose(st, nao, S.Vb.p, T.p);
      res->mo_coeff_beta = host_copy(T.p, nn, st);
    }
    CUDA_OK(cudaStreamSynchronize(st));
  }
}

template <class Fn>
static pm7_status guarded(Fn fn) {
  try {
    fn();
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    return f.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return PM7_ERR_INVALID_INPUT;
  }
}

// ---- stage entry points ----------------------------------------------------

static void stage_core(const pm7_molecule *mol, const pm7_params *params, int force_dpath, double *h_out,
                       int32_t *nao_out, const double *p_tot, const double *p_spin, double *f_out,
                       bool fp32 = false) {
  Molecule m = to_molecule(mol);
  const int method = *reinterpret_cast<const int *>(params);
  const ParamSet &ps = param_set(method);
  Layout L = build_layout(m, ps);
  if (nao_out) *nao_out = L.nao;
  if (!h_out && !f_out) return;
  DeviceContext &ctx = context_for(0);
  std::lock_guard<std::mutex> lock(ctx.run_mutex);
  CUDA_OK(cudaSetDevice(ctx.device));
  const DeviceParams &P = device_params(ctx, method);
  cudaStream_t st = ctx.stream;
  DeviceMolecule D;
  build_device_molecule(D, m, L, P, force_dpath || L.has_d, st);
  const size_t nn = (size_t)L.nao * L.nao;
  if (h_out) CUDA_OK(cudaMemcpyAsync(h_out, D.H.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
  if (f_out) {
    DevBuf<double> Pt, Ps, F;
    upload(Pt, std::vector<double>(p_tot, p_tot + nn), st);
    upload(Ps, std::vector<double>(p_spin, p_spin + nn), st);
    F.alloc(nn, st);
    if (fp32) {
      DevBuf<float> Pt32, Ps32, w32;
      Pt32.alloc(nn, st);
      Ps32.alloc(nn, st);
      w32.alloc(D.w.n, st);
      launch_to_float(st, nn, Pt.p, Pt32.p);
      launch_to_float(st, nn, Ps.p, Ps32.p);
      launch_to_float(st, D.w.n, D.w.p, w32.p);
      launch_fock32(st, D.geometry(), P, D.H.p, Pt.p, Pt32.p, Ps32.p, 1.0, F.p, D.pop.p, D.jbuf.p, w32.p);
      CUDA_OK(cudaMemcpyAsync(f_out, F.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaStreamSynchronize(st));
      return;
    }
    launch_fock(st, D.geometry(), P, D.H.p, Pt.p, Ps.p, 1.0, F.p, D.pop.p, D.jbuf.p);
    CUDA_OK(cudaMemcpyAsync(f_out, F.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
  }
  CUDA_OK(cudaStreamSynchronize(st));
}

// Fixed-density gradient of host densities (src/gradient.rs:626-700 and the UHF form :1249-1350).
static void stage_gradient(const pm7_molecule *mol, const pm7_params *params, int force_dpath, const double *p_total,
                           const double *p_spin, double *grad_out) {
  Molecule m = to_molecule(mol);
  const int method = *reinterpret_cast<const int *>(params);
  const ParamSet &ps = param_set(method);
  Layout L = build_layout(m, ps);
  DeviceContext &ctx = context_for(0);
  std::lock_guard<std::mutex> lock(ctx.run_mutex);
  CUDA_OK(cudaSetDevice(ctx.device));
  const DeviceParams &P = device_params(ctx, method);
  cudaStream_t st = ctx.stream;
  DeviceMolecule D;
  const bool dpath = force_dpath || L.has_d;
  build_device_molecule(D, m, L, P, dpath, st);
  const size_t nn = (size_t)L.nao * L.nao;
  DevBuf<double> Pt, Ps;
  upload(Pt, std::vector<double>(p_total, p_total + nn), st);
  if (p_spin) upload(Ps, std::vector<double>(p_spin, p_spin + nn), st);
  const std::vector<double> g = device_gradient(st, P, D, dpath, Pt.p, p_spin ? Ps.p : nullptr, method, 0, false, false);
  std::memcpy(grad_out, g.data(), sizeof(double) * g.size());
}

// Correction-energy gradient alone, eV/Bohr (src/gradient.rs:208-261).
static void stage_correction_gradient(const pm7_molecule *mol, int method, int smooth, double *grad_out) {
  Molecule m = to_molecule(mol);
  DeviceContext &ctx = context_for(0);
  std::lock_guard<std::mutex> lock(ctx.run_mutex);
  CUDA_OK(cudaSetDevice(ctx.device));
  cudaStream_t st = ctx.stream;
  const int n = m.n;
  if (n == 0) return;
  DevBuf<int> z;
  DevBuf<double> xyz, work, energies, cg, G;
  upload(z, m.z, st);
  upload(xyz, m.xyz, st);
  const int copies = correction_copies(n, smooth);
  work.alloc(corrections_gradient_work(n, copies, smooth), st);
  energies.alloc((size_t)kStencil * n + 1, st);
  cg.alloc(3 * (size_t)n, st);
  G.alloc(3 * (size_t)n, st);
  CUDA_OK(cudaMemsetAsync(G.p, 0, sizeof(double) * 3 * n, st));
  launch_corrections_gradient(st, n, z.p, xyz.p, method, smooth, std::find(m.z.begin(), m.z.end(), 14) != m.z.end(),
                              copies, work.p, energies.p, cg.p);
  launch_grad_add(st, n, kKcalToEv, cg.p, G.p);
  CUDA_OK(cudaMemcpyAsync(grad_out, G.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  CUDA_OK(cudaGetLastError());
}

}  // namespace pm7

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace pm7;

#include "pm7_param_data.h"
namespace pm7 {
const double *pm7_mass_table() { return PM7_MASS; }
}

struct pm7_params {
  int method;
};

extern "C" {

pm7_status pm7_params_load(int32_t method, const pm7_params **out) {
  static pm7_params sets[5] = {{0}, {1}, {2}, {3}, {4}};
  if (!out) return PM7_ERR_INVALID_INPUT;
  if (method < 0 || method > 4) {
    g_last_error = "unknown PM7 method";
    return PM7_ERR_INVALID_INPUT;
  }
  return guarded([&] {
    param_set(method);
    *out = &sets[method];
  });
}

void pm7_options_default(pm7_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->method = PM7_METHOD_PM7;
  o->charge = 0.0;
  o->multiplicity = 1;
  o->max_scf = 200;
  o->e_tol = 1.0e-8;
  o->p_tol = 1.0e-7;
  o->use_diis = 1;
  o->accelerator = PM7_ACCEL_ADIIS_CDIIS;
  o->adiis_switch = 0.1;
  o->level_shift = 0.0;
  o->reference = PM7_REF_AUTO;
  o->force_dpath = 0;
  o->smooth_dispersion = 0;
  o->max_memory_mb = -1;
  o->dipole_origin = PM7_DIPOLE_CENTRE_OF_MASS;
  o->initial_density = nullptr;
  o->initial_spin_density = nullptr;
  o->precision = PM7_PRECISION_FP64;
  o->device = 0;
  o->want_matrices = 1;
}

pm7_status pm7_run(const pm7_molecule *molecule, const pm7_params *params, const pm7_options *options,
                   pm7_result *result) {
  return guarded([&] { run_impl(molecule, params, options, result); });
}

pm7_status pm7_gradient(const pm7_molecule *molecule, const pm7_params *params, const pm7_options *options,
                        pm7_result *result, double *gradient, double *max_gradient) {
  return guarded([&] {
    if (!gradient) throw Failure{PM7_ERR_INVALID_INPUT, "null gradient buffer"};
    std::vector<double> g;
    run_impl(molecule, params, options, result, &g);
    std::memcpy(gradient, g.data(), sizeof(double) * g.size());
    if (max_gradient) {
      double mx = 0.0;
      for (double v : g) mx = std::max(mx, std::fabs(v));
      *max_gradient = mx;
    }
  });
}

pm7_status pm7_fixed_density_gradient(const pm7_molecule *molecule, const pm7_params *params, int32_t force_dpath,
                                      const double *p_total, const double *p_spin, double *gradient) {
  return guarded([&] {
    if (!params || !p_total || !gradient) throw Failure{PM7_ERR_INVALID_INPUT, "null argument"};
    stage_gradient(molecule, params, force_dpath, p_total, p_spin, gradient);
  });
}

pm7_status pm7_correction_gradient(const pm7_molecule *molecule, int32_t method, int32_t smooth_dispersion,
                                   double *gradient) {
  return guarded([&] {
    if (!gradient) throw Failure{PM7_ERR_INVALID_INPUT, "null gradient buffer"};
    if (method < 0 || method > 4) throw Failure{PM7_ERR_INVALID_INPUT, "unknown PM7 method"};
    stage_correction_gradient(molecule, method, smooth_dispersion, gradient);
  });
}

void pm7_result_free(pm7_result *r) {
  if (!r) return;
  double **arrs[] = {&r->charges, &r->density, &r->spin_density, &r->mo_energies, &r->mo_coeff,
                     &r->mo_energies_beta, &r->mo_coeff_beta};
  for (double **a : arrs) {
    std::free(*a);
    *a = nullptr;
  }
}

const char *pm7_last_error_message(void) { return g_last_error.c_str(); }

int32_t pm7_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) return 0;
  return c;
}

pm7_status pm7_stage_core_hamiltonian(const pm7_molecule *molecule, const pm7_params *params, int32_t force_dpath,
                                      double *h_out, int32_t *nao_out) {
  return guarded([&] { stage_core(molecule, params, force_dpath, h_out, nao_out, nullptr, nullptr, nullptr); });
}

pm7_status pm7_stage_fock(const pm7_molecule *molecule, const pm7_params *params, int32_t force_dpath,
                          const double *p_tot, const double *p_spin, double *f_out) {
  return guarded([&] { stage_core(molecule, params, force_dpath, nullptr, nullptr, p_tot, p_spin, f_out); });
}

pm7_status pm7_stage_fock_fp32(const pm7_molecule *molecule, const pm7_params *params, int32_t force_dpath,
                               const double *p_tot, const double *p_spin, double *f_out) {
  return guarded([&] { stage_core(molecule, params, force_dpath, nullptr, nullptr, p_tot, p_spin, f_out, true); });
}

pm7_status pm7_stage_pair(const pm7_params *params, int32_t z_i, int32_t z_j, const double d[3], int32_t force_dpath,
                          double *w_out, double *e1b_out, double *e2a_out, double *s_out, int32_t *npair_i,
                          int32_t *npair_j) {
  return guarded([&] {
    const int method = *reinterpret_cast<const int *>(params);
    const ParamSet &ps = param_set(method);
    const ElementRec *ei = ps.element(z_i), *ej = ps.element(z_j);
    if (!ei) throw Failure{PM7_ERR_MISSING_ELEMENT, "missing PM7 parameter block for Z=" + std::to_string(z_i)};
    if (!ej) throw Failure{PM7_ERR_MISSING_ELEMENT, "missing PM7 parameter block for Z=" + std::to_string(z_j)};
    if (ei->n_orb < ej->n_orb) throw Failure{PM7_ERR_INVALID_INPUT, "the first atom must carry at least as many orbitals"};
    const bool dpath = force_dpath || ei->n_orb == 9 || ej->n_orb == 9;
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    const DeviceParams &P = device_params(ctx, method);
    cudaStream_t st = ctx.stream;
    DevBuf<double> buf;
    buf.alloc(2025 + 3 * 81, st);
    DevBuf<int> ib;
    ib.alloc(3, st);
    CUDA_OK(cudaMemsetAsync(ib.p, 0, 3 * sizeof(int), st));
    if (dpath)
      launch_stage_pair_d(st, P, z_i, z_j, d, buf.p, buf.p + 2025, buf.p + 2025 + 81, buf.p + 2025 + 162, ib.p);
    else
      launch_stage_pair(st, P, z_i, z_j, d, buf.p, buf.p + 2025, buf.p + 2025 + 81, buf.p + 2025 + 162, ib.p,
                        ib.p + 2);
    int h[3];
    std::vector<double> hb(2025 + 3 * 81);
    CUDA_OK(cudaMemcpyAsync(hb.data(), buf.p, sizeof(double) * hb.size(), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(h, ib.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (h[2]) throw Failure{PM7_ERR_UNSUPPORTED, "a pair's shells are outside the sp-frame integral kernels"};
    *npair_i = h[0];
    *npair_j = h[1];
    std::memcpy(w_out, hb.data(), sizeof(double) * h[0] * h[1]);
    std::memcpy(e1b_out, hb.data() + 2025, sizeof(double) * 81);
    std::memcpy(e2a_out, hb.data() + 2025 + 81, sizeof(double) * 81);
    std::memcpy(s_out, hb.data() + 2025 + 162, sizeof(double) * 81);
  });
}

pm7_status pm7_stage_square_tf32(int32_t n, const double *x, double *c_out) {
  return guarded([&] {
    if (n < 1 || !x || !c_out) throw Failure{PM7_ERR_INVALID_INPUT, "square_tf32 needs n >= 1 and buffers"};
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    const int ld = ((n + 31) / 32) * 32;
    const size_t nn = (size_t)n * n, ll = (size_t)ld * ld;
    DevBuf<double> X, C;
    DevBuf<float> hi, lo, C32;
    DevBuf<int> err;
    upload(X, std::vector<double>(x, x + nn), st);
    hi.alloc(ll, st);
    lo.alloc(ll, st);
    C32.alloc(ll, st);
    C.alloc(nn, st);
    err.alloc(1, st);
    CUDA_OK(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    CUDA_OK(cudaMemsetAsync(C32.p, 0, sizeof(float) * ll, st));
    launch_split_tf32(st, n, ld, X.p, hi.p, lo.p);
    alignas(64) unsigned char map_hi[128], map_lo[128];
    if (!make_square_map(hi.p, ld, map_hi) || !make_square_map(lo.p, ld, map_lo))
      throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    launch_square_tf32x3(st, n, ld, map_hi, map_lo, C32.p, err.p);
    launch_widen(st, n, ld, C32.p, C.p);
    int e = 0;
    CUDA_OK(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(c_out, C.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    if (e) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 squaring: a pipeline wait expired"};
  });
}

pm7_status pm7_stage_tf32_wait_drill(int32_t n) {
  return guarded([&] {
    if (n < 1 || n > 4096) throw Failure{PM7_ERR_INVALID_INPUT, "wait drill needs 1 <= n <= 4096"};
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    const int ld = ((n + 31) / 32) * 32;
    const size_t ll = (size_t)ld * ld;
    DevBuf<float> hi, lo, C32;
    DevBuf<int> err;
    for (DevBuf<float> *b : {&hi, &lo, &C32}) {
      b->alloc(ll, st);
      CUDA_OK(cudaMemsetAsync(b->p, 0, sizeof(float) * ll, st));
    }
    err.alloc(1, st);
    CUDA_OK(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    alignas(64) unsigned char map_hi[128], map_lo[128];
    if (!make_square_map(hi.p, ld, map_hi) || !make_square_map(lo.p, ld, map_lo))
      throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    launch_square_tf32x3(st, n, ld, map_hi, map_lo, C32.p, err.p, nullptr, 0, 1);
    int e = 0;
    CUDA_OK(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    if (e) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 squaring: a pipeline wait expired (drill)"};
  });
}

pm7_status pm7_stage_sp2_step_i8(int32_t n, const double *x, int32_t square, double *x_out, double *norms) {
  return guarded([&] {
    if (n < 1 || !x || !x_out) throw Failure{PM7_ERR_INVALID_INPUT, "sp2_step_i8 needs n >= 1 and buffers"};
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    const size_t nn = (size_t)n * n;
    const int tiles = sp2_i8_tiles(n);
    DevBuf<double> X, Y, state, parts;
    DevBuf<int8_t> dig0, dig1;
    DevBuf<int> err;
    upload(X, std::vector<double>(x, x + nn), st);
    Y.alloc(nn, st);
    state.alloc(kSp2Len, st);
    parts.alloc(2 * (size_t)tiles, st);
    dig0.alloc(sp2_i8_digit_bytes(n), st);
    dig1.alloc(sp2_i8_digit_bytes(n), st);
    err.alloc(1, st);
    CUDA_OK(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    launch_sp2_reset(st, state.p);
    const double sq = square ? 1.0 : 0.0;
    CUDA_OK(cudaMemcpyAsync(state.p + kSp2Square, &sq, sizeof(double), cudaMemcpyHostToDevice, st));
    launch_sp2_digits(st, n, X.p, dig0.p, nullptr, -1, err.p);
    alignas(64) unsigned char map_a[128], map_b[128];
    if (!make_digit_maps(dig0.p, n, map_a, map_b)) throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    launch_sp2_step_i8(st, n, map_a, map_b, X.p, Y.p, dig1.p, state.p, parts.p, 0, err.p);
    std::vector<double> ph(2 * (size_t)tiles);
    int e = 0;
    CUDA_OK(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(x_out, Y.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(ph.data(), parts.p, sizeof(double) * ph.size(), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    if (e == 1) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 i8 squaring: a pipeline wait expired"};
    if (e == 2) throw Failure{PM7_ERR_INVALID_INPUT, "sp2_step_i8: an element outside [-1.98, 1.98]"};
    if (norms) {
      norms[0] = norms[1] = 0.0;
      for (int t = 0; t < tiles; ++t) {
        norms[0] += ph[2 * t];
        norms[1] += ph[2 * t + 1];
      }
    }
  });
}

pm7_status pm7_stage_product_tf32(int32_t n, const double *a, const double *b, double *c_out) {
  return guarded([&] {
    if (n < 1 || !a || !b || !c_out) throw Failure{PM7_ERR_INVALID_INPUT, "product_tf32 needs n >= 1 and buffers"};
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    const int ld = ((n + 31) / 32) * 32;
    const size_t nn = (size_t)n * n, ll = (size_t)ld * ld;
    DevBuf<double> A, B, Cm;
    DevBuf<float> ahi, alo, bhi, blo, C32;
    DevBuf<int> err;
    upload(A, std::vector<double>(a, a + nn), st);
    upload(B, std::vector<double>(b, b + nn), st);
    for (DevBuf<float> *q : {&ahi, &alo, &bhi, &blo, &C32}) q->alloc(ll, st);
    Cm.alloc(nn, st);
    err.alloc(1, st);
    CUDA_OK(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    launch_split_tf32(st, n, ld, A.p, ahi.p, alo.p);
    launch_split_tf32(st, n, ld, B.p, bhi.p, blo.p);
    alignas(64) unsigned char m_ahi[128], m_alo[128], m_bhi[128], m_blo[128];
    if (!make_square_map(ahi.p, ld, m_ahi) || !make_square_map(alo.p, ld, m_alo) ||
        !make_square_map(bhi.p, ld, m_bhi) || !make_square_map(blo.p, ld, m_blo))
      throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    launch_product_tf32x3(st, n, ld, m_ahi, m_alo, m_bhi, m_blo, C32.p, err.p);
    launch_widen(st, n, ld, C32.p, Cm.p);
    int e = 0;
    CUDA_OK(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(c_out, Cm.p, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    if (e) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 product: a pipeline wait expired"};
  });
}

pm7_status pm7_stage_eigenvalues(int32_t count, const int32_t *orders, const double *a, double *w,
                                 int32_t device) {
  return guarded([&] {
    if (count < 0 || (count > 0 && (!orders || !a || !w)))
      throw Failure{PM7_ERR_INVALID_INPUT, "eigenvalues: bad count or null arrays"};
    if (count == 0) return;
    DeviceContext &ctx = context_for(device);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    size_t na = 0, nw = 0;
    for (int i = 0; i < count; ++i) {
      if (!eigvals_supported(orders[i]))
        throw Failure{PM7_ERR_INVALID_INPUT, "eigenvalues: order " + std::to_string(orders[i]) + " outside 1..4096"};
      na += (size_t)orders[i] * orders[i];
      nw += orders[i];
    }
    DevBuf<double> A, E;
    upload(A, std::vector<double>(a, a + na), st);
    E.alloc(nw, st);
    std::vector<EigvalsRequest> req;
    size_t oa = 0, ow = 0;
    for (int i = 0; i < count; ++i) {
      req.push_back({A.p + oa, orders[i], orders[i], E.p + ow});
      oa += (size_t)orders[i] * orders[i];
      ow += orders[i];
    }
    eigvals_device(st, req, ctx.eig_scratch);
    CUDA_OK(cudaMemcpyAsync(w, E.p, sizeof(double) * nw, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
  });
}

pm7_status pm7_stage_core_core(const pm7_molecule *molecule, const pm7_params *params, double *energy_ev) {
  return guarded([&] {
    Molecule m = to_molecule(molecule);
    const int method = *reinterpret_cast<const int *>(params);
    const ParamSet &ps = param_set(method);
    Layout L = build_layout(m, ps);
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    const DeviceParams &P = device_params(ctx, method);
    DeviceMolecule D;
    build_device_molecule(D, m, L, P, L.has_d, ctx.stream);
    *energy_ev = D.core_core_ev;
  });
}

pm7_status pm7_stage_seqsum(int64_t n, const double *a, const double *b, double *out, int32_t device) {
  return guarded([&] {
    if (n < 0 || !out || (n > 0 && !a)) throw Failure{PM7_ERR_INVALID_INPUT, "seqsum: bad length or null arrays"};
    DeviceContext &ctx = context_for(device);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    DevBuf<double> A, B, R;
    DevBuf<unsigned char> scratch;
    A.alloc((size_t)n, st);
    if (n > 0) CUDA_OK(cudaMemcpyAsync(A.p, a, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    if (b) {
      B.alloc((size_t)n, st);
      if (n > 0) CUDA_OK(cudaMemcpyAsync(B.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    }
    R.alloc(1, st);
    scratch.alloc(seqsum_scratch_bytes((size_t)n, 1), st);
    SeqSumBatch job{};
    job.job[0] = {A.p, b ? B.p : nullptr, (size_t)n, R.p};
    job.count = 1;
    launch_seqsum(st, job, scratch.p);
    CUDA_OK(cudaMemcpyAsync(out, R.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
  });
}

pm7_status pm7_stage_corrections(const pm7_molecule *molecule, int32_t method, int32_t smooth_dispersion,
                                 double out[5]) {
  return guarded([&] {
    Molecule m = to_molecule(molecule);
    DeviceContext &ctx = context_for(0);
    std::lock_guard<std::mutex> lock(ctx.run_mutex);
    CUDA_OK(cudaSetDevice(ctx.device));
    cudaStream_t st = ctx.stream;
    DevBuf<int> z;
    DevBuf<double> xyz, scratch, res;
    upload(z, m.z, st);
    upload(xyz, m.xyz, st);
    scratch.alloc(corrections_scratch(m.n), st);
    res.alloc(5, st);
    launch_corrections(st, m.n, z.p, xyz.p, method, smooth_dispersion, scratch.p, scratch.n, res.p);
    CUDA_OK(cudaMemcpyAsync(out, res.p, sizeof(double) * 5, cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
  });
}

int64_t pm7_launch_count(void) { return g_launches.load(); }

const char *pm7_autotune_report(void) {
  static thread_local std::string r;
  r = autotune_report();
  return r.c_str();
}

void pm7_profile_enable(int32_t on) { g_prof.reset(on != 0); }

int32_t pm7_profile_count(void) {
  g_prof.flush();
  return (int32_t)g_prof.names.size();
}

pm7_status pm7_profile_entry(int32_t i, const char **name, double *total_ms, int64_t *calls) {
  if (i < 0 || i >= (int32_t)g_prof.names.size()) return PM7_ERR_INVALID_INPUT;
  if (name) *name = g_prof.names[i].c_str();
  if (total_ms) *total_ms = g_prof.total_ms[i];
  if (calls) *calls = g_prof.calls[i];
  return PM7_OK;
}

// sizeof of the ABI structs, for the ctypes mirror's self-check.
void pm7_abi_sizes(int64_t out[3]) {
  out[0] = (int64_t)sizeof(pm7_molecule);
  out[1] = (int64_t)sizeof(pm7_options);
  out[2] = (int64_t)sizeof(pm7_result);
}

}  // extern "C"
