// Divide-and-conquer SCF of a molecule on the device (pm7-rs src/dandc/mod.rs:143-428,
// src/dandc/partition.rs, src/dandc/sparse.rs) and its energy and gradient
// (`dandc_derivatives`, src/dandc/mod.rs:446-506).
//
// Every subsystem (a core of atoms from recursive median bisection plus a buffer shell) is a
// small device molecule of its own: its pair integrals and core Hamiltonian are built once by
// the engine's build kernels, and every iteration runs one Fock build on it (the engine's Fock
// kernel on the global density restricted to the subsystem). The subsystem Fock matrices are
// padded into size buckets and diagonalised together: up to order 112 by a shared-memory Jacobi
// kernel (one block per matrix, warm-started from the previous iteration's eigenvectors), above
// that by cuSOLVER (XsyevBatched below order 512, dsyevd above). One Fermi level for the whole
// molecule is found by bisection in a single
// thread block; each subsystem's Fermi-weighted density (V^T diag(f) V on the FP64 tensor
// cores) is scattered with the Dixon-Merz weights into a global density kept dense in HBM
// (zeros outside the stored atom-pair pattern: a 180 GB device holds it at any size this
// method is used for), normalised per pair, compared and mixed.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <deque>
#include <functional>
#include <exception>
#include <memory>
#include <thread>
#include <unordered_map>

#include "common.cuh"
#include "engine_internal.hpp"
#include "gradient.cuh"

namespace pm7 {
namespace {

constexpr double kDcPad = 1.0e5;  // diagonal of the padding rows of a bucket matrix (eV)
constexpr int kDcPartials = 128;   // blocks of the reductions (fixed: the sums are deterministic)
constexpr size_t kDcLanes = 16;    // side streams for the subsystems' independent launch sequences
constexpr int kDcAssembleBlocks = 148 * 8;  // grid of the global assembly (8 blocks per SM)

// ---------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum in a fixed order (warps, then warp 0 over the warp sums); result in thread 0.
__device__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    t = warp_sum(t);
  }
  __syncthreads();
  return t;
}

// Fermi-Dirac occupation in electrons per spin-degenerate orbital (src/dandc/mod.rs:563-573).
__device__ __forceinline__ double dc_occupation(double e, double fermi, double width) {
  const double x = (e - fermi) / width;
  if (x > 40.0) return 0.0;
  if (x < -40.0) return 2.0;
  return 2.0 / (1.0 + exp(x));
}

// out[a] = sum_{b != a} EV q[b] / r_ab over every atom (src/dandc/mod.rs:889-902, 932-944):
// one warp per atom.
__global__ void k_dc_coulomb(int n, const double *__restrict__ xyz, const double *__restrict__ q,
                             double *__restrict__ out) {
  const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= n) return;
  const double xa = xyz[3 * a], ya = xyz[3 * a + 1], za = xyz[3 * a + 2];
  double s = 0.0;
  for (int b = lane; b < n; b += 32) {
    if (b == a) continue;
    const double dx = xyz[3 * b] - xa, dy = xyz[3 * b + 1] - ya, dz = xyz[3 * b + 2] - za;
    s += kEv * q[b] / sqrt(dx * dx + dy * dy + dz * dz);
  }
  s = warp_sum(s);
  if (lane == 0) out[a] = s;
}

// The environment of subsystem atom i: the global sum at its parent minus what the subsystem
// holds itself (src/dandc/mod.rs:972-996). One warp per subsystem atom.
__global__ void k_dc_env(int n_sub, const int *__restrict__ parent, const double *__restrict__ xyz,
                         const double *__restrict__ q, const double *__restrict__ global, double *__restrict__ out) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n_sub) return;
  const int a = parent[i];
  const double xa = xyz[3 * a], ya = xyz[3 * a + 1], za = xyz[3 * a + 2];
  double s = 0.0;
  for (int j = lane; j < n_sub; j += 32) {
    if (j == i) continue;
    const int b = parent[j];
    const double dx = xyz[3 * b] - xa, dy = xyz[3 * b + 1] - ya, dz = xyz[3 * b + 2] - za;
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (r < 1.0e-8) continue;
    s += kEv * q[b] / r;
  }
  s = warp_sum(s);
  if (lane == 0) out[i] = global[a] - s;
}

// H_kk -= v of the atom of AO k: the nuclear half of the environment (src/dandc/mod.rs:560-566).
__global__ void k_dc_hdiag(int nao, const int *__restrict__ ao_atom, const double *__restrict__ v,
                           double *__restrict__ H) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nao) H[(size_t)k * nao + k] -= v[ao_atom[k]];
}

// Atom populations of the global density (SparseDensity::population).
__global__ void k_dc_pops(int n, const int *__restrict__ aoff, const int *__restrict__ norb, int nao,
                          const double *__restrict__ P, double *__restrict__ pop) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double s = 0.0;
  for (int m = 0; m < norb[a]; ++m) s += P[(size_t)(aoff[a] + m) * nao + aoff[a] + m];
  pop[a] = s;
}

// The global density restricted to a subsystem (src/dandc/mod.rs:672-690): elements of atom
// pairs outside the stored pattern read as zero. Unrestricted: the spin densities too,
// Pa = (P + S) / 2, Pb = (P - S) / 2 (:602-608, :617-622).
__global__ void k_dc_gather(int nao, const int *__restrict__ map, const int *__restrict__ ao_par, int n_glob,
                            int nao_glob, const unsigned char *__restrict__ wcnt, const double *__restrict__ Pg,
                            const double *__restrict__ Sg, double *__restrict__ P, double *__restrict__ Pa,
                            double *__restrict__ Pb) {
  const size_t nn = (size_t)nao * nao;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / nao), l = (int)(e % nao);
    const bool stored = wcnt[(size_t)ao_par[k] * n_glob + ao_par[l]] != 0;
    const size_t g = (size_t)map[k] * nao_glob + map[l];
    const double p = stored ? Pg[g] : 0.0;
    P[e] = p;
    if (Sg) {
      const double s = stored ? Sg[g] : 0.0;
      Pa[e] = 0.5 * (p + s);
      Pb[e] = 0.5 * (p - s);
    }
  }
}

// A subsystem Fock matrix plus the electronic half of its environment on the diagonal
// (src/dandc/mod.rs:568-576) into its np x np bucket slot, padded with kDcPad.
__global__ void k_dc_pack(int nao, int np, const double *__restrict__ F, const int *__restrict__ ao_atom,
                          const double *__restrict__ env, double *__restrict__ slot) {
  const size_t nn = (size_t)np * np;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / np), l = (int)(e % np);
    double v;
    if (k < nao && l < nao) v = F[(size_t)k * nao + l] + (k == l ? env[ao_atom[k]] : 0.0);
    else v = k == l ? kDcPad : 0.0;
    slot[e] = v;
  }
}

// Partials of sum_{kl} 1/2 w_kl P_kl (H + F)_kl with the Dixon-Merz weights (core AOs first:
// 1 core-core, 1/2 core-buffer, 0 buffer-buffer), src/dandc/mod.rs:634-653.
__global__ void k_dc_energy(int nao, int np, int core_ao, const double *__restrict__ P, const double *__restrict__ H,
                            const double *__restrict__ slot, double *__restrict__ partials) {
  __shared__ double sh[32];
  const size_t nn = (size_t)nao * nao;
  double s = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / nao), l = (int)(e % nao);
    const bool ck = k < core_ao, cl = l < core_ao;
    const double w = (ck && cl) ? 1.0 : ((ck || cl) ? 0.5 : 0.0);
    if (w == 0.0) continue;
    s += 0.5 * w * P[e] * (H[e] + slot[(size_t)k * np + l]);
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Eigenvalue and weighted norm sum_{core AOs} C^2 of every state (src/dandc/mod.rs:584-637):
// one warp per state; V holds the eigenvectors as rows (ld np).
__global__ void k_dc_norms(int nao, int np, int core_ao, double scale, const double *__restrict__ V,
                           const double *__restrict__ eps, double *__restrict__ se, double *__restrict__ sw) {
  const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= nao) return;
  double t = 0.0;
  for (int k = lane; k < core_ao; k += 32) {
    const double v = V[(size_t)s * np + k];
    t += v * v;
  }
  t = warp_sum(t);
  if (lane == 0) {
    se[s] = eps[s];
    sw[s] = scale * t;
  }
}

// The common chemical potential (src/dandc/mod.rs:641-700): bisection on [-500, 500] eV for
// the electron count sum_states f(e) w (occupations below 1e-14 count zero), at most 200 halvings
// or until the bracket is narrower than 1e-12. out[0] = E_F, out[1] = 1 when no potential in the
// range holds n_elec. One block of 1024 threads; the count's summation order is fixed.
__global__ void __launch_bounds__(1024) k_dc_fermi(size_t n_states, const double *__restrict__ se,
                                                   const double *__restrict__ sw, double n_elec, double width,
                                                   double *__restrict__ out) {
  __shared__ double sh[32];
  __shared__ double bracket[2];
  __shared__ int outside;
  auto count = [&](double fermi) {
    double s = 0.0;
    for (size_t i = threadIdx.x; i < n_states; i += blockDim.x) {
      const double f = dc_occupation(se[i], fermi, width);
      s += f < 1.0e-14 ? 0.0 : f * sw[i];
    }
    return block_sum(s, sh);
  };
  const double c_lo = count(-500.0);
  const double c_hi = count(500.0);
  if (threadIdx.x == 0) {  // the block sums are valid in thread 0; it decides for the block
    bracket[0] = -500.0;
    bracket[1] = 500.0;
    outside = (c_lo > n_elec || c_hi < n_elec) ? 1 : 0;
    out[1] = outside ? 1.0 : 0.0;
  }
  __syncthreads();
  if (outside) return;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (bracket[0] + bracket[1]);
    const double c = count(mid);
    if (threadIdx.x == 0) {
      if (c < n_elec) bracket[0] = mid;
      else bracket[1] = mid;
    }
    __syncthreads();
    if (bracket[1] - bracket[0] < 1.0e-12) break;
  }
  if (threadIdx.x == 0) out[0] = 0.5 * (bracket[0] + bracket[1]);
}

// Rows of the occupation-scaled eigenvectors: Vf[s] = f_s V[s] with f_s = f(e_s) * scale,
// zero when |f_s| < 1e-14 and for the padding states (src/dandc/mod.rs:770-800).
__global__ void k_dc_occupy(int nao, int np, double scale, const double *__restrict__ V,
                            const double *__restrict__ eps, const double *__restrict__ fermi, double width,
                            double *__restrict__ Vf) {
  const size_t nn = (size_t)np * np;
  const double ef = fermi[0];
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(e / np);
    double f = s < nao ? dc_occupation(eps[s], ef, width) * scale : 0.0;
    if (fabs(f) < 1.0e-14) f = 0.0;
    Vf[e] = f * V[e];
  }
}

// One stored atom pair's contributions to the next global density: at most two subsystems
// weight it, the one whose core holds A and the one whose core holds B (a pair with both atoms
// in one core has a single contribution of weight 1). Per contribution: the offset of that
// subsystem's density in the product buffer, its order, A's and B's local AO offsets, the weight.
struct DcPairSrc {
  long long off[2];
  int nao[2], la[2], lb[2];
  double w[2];
  int n;
};

// The next global density assembled from the subsystem densities (scatter_density +
// SparseDensity::accumulate, src/dandc/mod.rs:770-814, in the fixed order above), normalised by
// the realised weight total (:236-258), its RMS difference to P (rms_diff) and the mixing
// P <- (1 - m) P + m next (sparse.rs mix); the spin density likewise, without the error.
// Thread per global element; partial sums of (P - next)^2 per block.
__global__ void k_dc_assemble(int nao, int n_glob, const int *__restrict__ ao_atom, const int *__restrict__ aoff,
                              const int *__restrict__ pair_rec, const DcPairSrc *__restrict__ recs,
                              const double *__restrict__ D, const double *__restrict__ Ds, double mixing,
                              double *__restrict__ P, double *__restrict__ S, double *__restrict__ partials) {
  __shared__ double sh[32];
  const size_t nn = (size_t)nao * nao;
  double acc = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / nao), l = (int)(e % nao);
    const int A = ao_atom[k], B = ao_atom[l];
    const int r = pair_rec[(size_t)A * n_glob + B];
    if (r < 0) continue;
    const DcPairSrc &q = recs[r];
    const int mu = k - aoff[A], nu = l - aoff[B];
    double t = 0.0, wt = 0.0, ts = 0.0;
    for (int c = 0; c < q.n; ++c) {
      const size_t i = (size_t)q.off[c] + (size_t)(q.la[c] + mu) * q.nao[c] + q.lb[c] + nu;
      t += q.w[c] * D[i];
      if (Ds) ts += q.w[c] * Ds[i];
      wt += q.w[c];
    }
    const double norm = 1.0 / wt;
    const double nx = t * norm;
    const double d = P[e] - nx;
    acc += d * d;
    P[e] = (1.0 - mixing) * P[e] + mixing * nx;
    if (S) S[e] = (1.0 - mixing) * S[e] + mixing * (ts * norm);
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}


unsigned grid_for(size_t items) { return (unsigned)std::max<size_t>(1, std::min<size_t>((items + 255) / 256, 4096)); }

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------

// `partition::bisect` (src/dandc/partition.rs): split along the longest extent at the median of
// a stable sort, recursively, until a part holds at most `target` atoms. Among equal extents the
// last axis wins, as Iterator::max_by does.
void dc_bisect(std::vector<int> idx, const std::vector<double> &xyz, size_t target, std::vector<std::vector<int>> &out) {
  if (idx.size() <= target || idx.size() < 2) {
    out.push_back(std::move(idx));
    return;
  }
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i : idx)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], xyz[3 * i + k]);
      hi[k] = std::max(hi[k], xyz[3 * i + k]);
    }
  int axis = 0;
  for (int k = 1; k < 3; ++k)
    if (hi[k] - lo[k] >= hi[axis] - lo[axis]) axis = k;
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return xyz[3 * a + axis] < xyz[3 * b + axis]; });
  const size_t half = idx.size() / 2;
  std::vector<int> right(idx.begin() + (std::ptrdiff_t)half, idx.end());
  idx.resize(half);
  dc_bisect(std::move(idx), xyz, target, out);
  dc_bisect(std::move(right), xyz, target, out);
}

struct DcPart {
  std::vector<int> parent;  // core atoms (bisection order), then the buffer (ascending index)
  int n_core = 0;
};

// `partition` + `grow_buffer` (src/dandc/partition.rs) for a molecule: every atom within
// `buffer` Bohr of a core atom joins the core's subsystem (a cell grid of that width).
std::vector<DcPart> dc_partition(const Molecule &m, int core_size, double buffer) {
  std::vector<std::vector<int>> cores;
  std::vector<int> all(m.n);
  for (int i = 0; i < m.n; ++i) all[i] = i;
  dc_bisect(std::move(all), m.xyz, (size_t)std::max(core_size, 1), cores);
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  for (int i = 0; i < m.n; ++i)
    for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], m.xyz[3 * i + k]);
  auto key = [&](long long a, long long b, long long c) { return (a * 1000003LL + b) * 1000033LL + c; };
  auto cell = [&](int i, int k) { return (long long)std::floor((m.xyz[3 * i + k] - lo[k]) / buffer); };
  std::unordered_map<long long, std::vector<int>> grid;
  for (int i = 0; i < m.n; ++i) grid[key(cell(i, 0), cell(i, 1), cell(i, 2))].push_back(i);
  const double cut2 = buffer * buffer;
  std::vector<int> stamp(m.n, -1);
  std::vector<DcPart> parts;
  parts.reserve(cores.size());
  for (size_t s = 0; s < cores.size(); ++s) {
    DcPart p;
    p.parent = cores[s];
    p.n_core = (int)cores[s].size();
    for (int i : cores[s]) stamp[i] = (int)s;
    std::vector<int> buf;
    for (int i : cores[s]) {
      const long long cx = cell(i, 0), cy = cell(i, 1), cz = cell(i, 2);
      for (long long dx = -1; dx <= 1; ++dx)
        for (long long dy = -1; dy <= 1; ++dy)
          for (long long dz = -1; dz <= 1; ++dz) {
            auto it = grid.find(key(cx + dx, cy + dy, cz + dz));
            if (it == grid.end()) continue;
            for (int j : it->second) {
              if (stamp[j] == (int)s) continue;
              const double ex = m.xyz[3 * j] - m.xyz[3 * i], ey = m.xyz[3 * j + 1] - m.xyz[3 * i + 1],
                           ez = m.xyz[3 * j + 2] - m.xyz[3 * i + 2];
              if (ex * ex + ey * ey + ez * ez > cut2) continue;
              stamp[j] = (int)s;
              buf.push_back(j);
            }
          }
    }
    std::sort(buf.begin(), buf.end());
    p.parent.insert(p.parent.end(), buf.begin(), buf.end());
    parts.push_back(std::move(p));
  }
  return parts;
}

int dc_bucket(int nao) { return nao <= 256 ? ((nao + 15) / 16) * 16 : ((nao + 63) / 64) * 64; }

struct DcSub {
  DcPart part;
  Molecule m;
  Layout L;
  DeviceMolecule D;
  int nao = 0, core_ao = 0, np = 0;
  int bucket = -1, slot = 0;  // index into buckets, position inside it
  size_t spec = 0;            // first spectrum entry
  DevBuf<int> map, ao_par, parent, ao_atom;
};

struct DcBucket {
  int np = 0, count = 0;  // matrices (2 per subsystem when unrestricted)
  bool jacobi = false;    // solved by k_dc_jacobi (np <= kJacobiMax), else by cuSOLVER
  DevBuf<double> A, eps;
  DevBuf<int> info;
};

void check_dandc_options(const pm7_dandc_options &d) {  // src/dandc/mod.rs:83-110
  auto bad = [](const char *s) { throw Failure{PM7_ERR_INVALID_INPUT, s}; };
  if (!std::isfinite(d.buffer) || d.buffer <= 0.0) bad("the divide-and-conquer buffer must be finite and positive");
  if (d.core_size <= 0) bad("the divide-and-conquer core size must be at least 1");
  if (!std::isfinite(d.fermi_width_ev) || d.fermi_width_ev <= 0.0)
    bad("the divide-and-conquer Fermi width must be finite and positive");
  if (!(d.mixing > 0.0 && d.mixing <= 1.0)) bad("the divide-and-conquer mixing factor must lie in (0, 1]");
  if (d.max_scf < 0) bad("the divide-and-conquer max_scf must be non-negative");
}

void run_dandc_impl(const pm7_molecule *mol, const pm7_params *params, const pm7_options *opt,
                    const pm7_dandc_options *dco, int want_gradient, pm7_dandc_result *res) {
  if (!mol || !params || !opt || !dco || !res) throw Failure{PM7_ERR_INVALID_INPUT, "null argument"};
  const auto t_start = std::chrono::steady_clock::now();
  // PM7_DANDC_TRACE: setup sub-phases and per-phase iteration times on stderr (phases then end
  // in a synchronise)
  const bool trace = std::getenv("PM7_DANDC_TRACE") != nullptr;
  std::string setup_marks;
  auto t_mark = t_start;
  auto mark = [&](const char *what, cudaStream_t sync_st) {
    if (!trace) return;
    if (sync_st) cudaStreamSynchronize(sync_st);
    const auto now = std::chrono::steady_clock::now();
    char buf[64];
    std::snprintf(buf, sizeof buf, " %s %.1f", what, std::chrono::duration<double, std::milli>(now - t_mark).count());
    setup_marks += buf;
    t_mark = now;
  };
  const pm7_options &o = *opt;
  const pm7_dandc_options &dc = *dco;
  Molecule m = to_molecule(mol);
  validate(m, o);
  if (o.method != *reinterpret_cast<const int *>(params))
    throw Failure{PM7_ERR_INVALID_INPUT, "options method does not match parameter method"};
  check_dandc_options(dc);
  const ParamSet &ps = param_set(o.method);
  Layout Lg = build_layout(m, ps);
  const int N = m.n, nao_g = Lg.nao;
  std::vector<DcPart> parts = dc_partition(m, dc.core_size, dc.buffer);

  // per-subsystem layouts and the pre-flight memory check on the whole device footprint
  std::vector<std::unique_ptr<DcSub>> subs;
  subs.reserve(parts.size());
  int largest_atoms = 0, largest_nao = 0;
  for (DcPart &p : parts) {
    auto s = std::make_unique<DcSub>();
    s->part = std::move(p);
    s->m.n = (int)s->part.parent.size();
    for (int a : s->part.parent) {
      s->m.z.push_back(m.z[a]);
      for (int k = 0; k < 3; ++k) s->m.xyz.push_back(m.xyz[3 * a + k]);
    }
    subs.push_back(std::move(s));
  }
  {
    // the subsystems' layouts (pair lists, AO offsets) are independent host work: a few threads
    const int workers = (int)std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 16);
    std::vector<std::exception_ptr> errs(workers);
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w)
      pool.emplace_back([&, w] {
        try {
          for (size_t a = (size_t)w; a < subs.size(); a += (size_t)workers) subs[a]->L = build_layout(subs[a]->m, ps);
        } catch (...) {
          errs[w] = std::current_exception();
        }
      });
    for (std::thread &t : pool) t.join();
    for (auto &e : errs)
      if (e) std::rethrow_exception(e);
  }
  for (auto &sp : subs) {
    DcSub *s = sp.get();
    s->nao = s->L.nao;
    s->core_ao = s->part.n_core < s->m.n ? s->L.aoff[s->part.n_core] : s->nao;
    s->np = dc_bucket(s->nao);
    largest_atoms = std::max(largest_atoms, s->m.n);
    largest_nao = std::max(largest_nao, s->nao);
  }
  const bool unrestricted =
      o.reference == PM7_REF_UNRESTRICTED || (o.reference == PM7_REF_AUTO && o.multiplicity > 1);
  const int chan = unrestricted ? 2 : 1;
  {
    // global density (and spin channels), the stored-pair mask (N^2 bytes) and the int32
    // atom-pair table of the reassembly (4 N^2 bytes)
    uint64_t need = (uint64_t)nao_g * nao_g * 8 * (unrestricted ? 4 : 2) + (uint64_t)N * N * 5;
    for (const auto &s : subs) {
      const uint64_t pairs = (uint64_t)s->m.n * (s->m.n > 0 ? s->m.n - 1 : 0) / 2;
      need += (uint64_t)s->np * s->np * 8 * chan + (uint64_t)s->m.n * s->m.n * 9 + (uint64_t)s->nao * s->nao * 8 +
              pairs * (s->L.has_d ? 1200 : 200);
    }
    need += (uint64_t)largest_nao * largest_nao * 8 * (unrestricted ? 8 : 4);
    const uint64_t budget = device_budget(o.max_memory_mb);
    if (budget > 0 && need > budget)
      throw Failure{PM7_ERR_INVALID_INPUT,
                    "estimated divide-and-conquer memory ~" + std::to_string((need + (1 << 20) - 1) >> 20) +
                        " MB exceeds the " + std::to_string(budget >> 20) +
                        " MB budget\nThis is a divide-and-conquer subsystem, not the whole system: a " +
                        std::to_string(dc.buffer * 0.529177210903) + " Angstrom buffer around a " +
                        std::to_string(dc.core_size) + "-atom core gives a largest subsystem of " +
                        std::to_string(largest_atoms) + " atoms and " + std::to_string(largest_nao) +
                        " orbitals. Reduce the buffer, or drop divide and conquer and use the exact SCF."};
  }

  mark("layouts", nullptr);
  // the stored pattern and the realised weight totals, in half units (0, 1 or 2: a pair is
  // weighted only by the subsystems whose core holds one of its atoms)
  std::vector<unsigned char> wcnt((size_t)N * N, 0);
  for (const auto &s : subs) {
    const auto &par = s->part.parent;
    const int nc = s->part.n_core;
    for (int i = 0; i < (int)par.size(); ++i)
      for (int j = 0; j < (int)par.size(); ++j) {
        if (i >= nc && j >= nc) continue;
        wcnt[(size_t)par[i] * N + par[j]] += (i < nc && j < nc) ? 2 : 1;
      }
  }
  int64_t stored = 0;
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b)
      if (wcnt[(size_t)a * N + b]) stored += (int64_t)Lg.norb[a] * Lg.norb[b];

  double core_e = 0.0;
  std::vector<double> cores(N);
  for (int a = 0; a < N; ++a) core_e += (cores[a] = ps.element(m.z[a])->core);
  const double n_elec = core_e - o.charge;
  if (n_elec < -1.0e-9)
    throw Failure{PM7_ERR_INVALID_INPUT, "the divide-and-conquer driver was given a system with negative electron count"};
  const double n_beta_extra = (o.multiplicity - 1) * 0.5;

  mark("pattern", nullptr);
  DeviceContext &ctx = context_for(o.device);
  std::lock_guard<std::mutex> lock(ctx.run_mutex);
  CUDA_OK(cudaSetDevice(ctx.device));
  const DeviceParams &P = device_params(ctx, o.method);
  cudaStream_t st = ctx.stream;

  // global arrays
  const size_t nng = (size_t)nao_g * nao_g;
  DevBuf<double> xyz, q, gnuc, gelec, pops, Pg, Sg, partials, scal;
  DevBuf<int> aoff, norb, ao_atom;
  DevBuf<unsigned char> wdev;
  upload(xyz, m.xyz, st);
  upload(q, cores, st);
  upload(aoff, Lg.aoff, st);
  upload(norb, Lg.norb, st);
  upload(ao_atom, Lg.ao_atom, st);
  upload(wdev, wcnt, st);
  gnuc.alloc(N, st);
  gelec.alloc(N, st);
  pops.alloc(N, st);
  partials.alloc(kDcAssembleBlocks, st);
  scal.alloc(4, st);  // [0] error^2 sum, [1] Fermi level, [2] Fermi status
  {
    // atomic-density start on the diagonal blocks (src/dandc/mod.rs:289-301); the spin density
    // starts as a scaled copy of the total's diagonal (:302-323)
    std::vector<double> diag = sad_diag(m, Lg, ps, n_elec);
    DevBuf<double> dd;
    upload(dd, diag, st);
    Pg.alloc(nng, st);
    launch_set_diag(st, nao_g, dd.p, Pg.p);  // zero, then the diagonal
    if (unrestricted) {
      const double scale = core_e > 0.0 ? 2.0 * n_beta_extra / core_e : 0.0;
      for (double &v : diag) v *= scale;
      DevBuf<double> ds;
      upload(ds, diag, st);
      Sg.alloc(nng, st);
      launch_set_diag(st, nao_g, ds.p, Sg.p);
    }
  }
  if (N > 0) k_dc_coulomb<<<(N + 3) / 4, 128, 0, st>>>(N, xyz.p, q.p, gnuc.p);
  note_launch();

  mark("globals", st);
  // subsystems: device molecules, AO maps, the nuclear environment folded into H once
  int max_nao = 0, max_np = 0;
  size_t n_states = 0;
  std::deque<DcBucket> buckets;  // DevBuf is not movable: a deque never relocates its elements
  DevBuf<double> env;
  env.alloc(std::max(largest_atoms, 1), st);
  for (auto &sp : subs) {
    DcSub &s = *sp;
    build_device_molecule(s.D, s.m, s.L, P, s.L.has_d, st, false);
    std::vector<int> map(s.nao), par(s.nao);
    for (int i = 0; i < s.m.n; ++i)
      for (int mu = 0; mu < s.L.norb[i]; ++mu) {
        map[s.L.aoff[i] + mu] = Lg.aoff[s.part.parent[i]] + mu;
        par[s.L.aoff[i] + mu] = s.part.parent[i];
      }
    upload(s.map, map, st);
    upload(s.ao_par, par, st);
    upload(s.parent, s.part.parent, st);
    upload(s.ao_atom, s.L.ao_atom, st);
    k_dc_env<<<(s.m.n + 3) / 4, 128, 0, st>>>(s.m.n, s.parent.p, xyz.p, q.p, gnuc.p, env.p);
    note_launch();
    if (s.nao > 0) {
      k_dc_hdiag<<<(s.nao + 127) / 128, 128, 0, st>>>(s.nao, s.ao_atom.p, env.p, s.D.H.p);
      note_launch();
    }
    max_nao = std::max(max_nao, s.nao);
    max_np = std::max(max_np, s.np);
    s.spec = n_states;
    n_states += (size_t)chan * s.nao;
    if (s.nao == 0) continue;
    auto it = std::find_if(buckets.begin(), buckets.end(), [&](const DcBucket &b) { return b.np == s.np; });
    if (it == buckets.end()) {
      buckets.emplace_back();
      buckets.back().np = s.np;
      it = buckets.end() - 1;
    }
    s.bucket = (int)(it - buckets.begin());
    s.slot = it->count;
    it->count += chan;
  }
  {
    mark("builds_queued", nullptr);
    // the builds were queued without waiting: one synchronisation for all their statuses
    std::vector<int> status(subs.size(), 0);
    for (size_t a = 0; a < subs.size(); ++a)
      CUDA_OK(cudaMemcpyAsync(&status[a], subs[a]->D.status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    for (int x : status)
      if (x != 0) throw Failure{PM7_ERR_UNSUPPORTED, "a pair's shells are outside the sp-frame integral kernels"};
  }
  for (DcBucket &b : buckets) {
    b.A.alloc((size_t)b.count * b.np * b.np, st);
    b.eps.alloc((size_t)b.count * b.np, st);
    b.info.alloc(b.count, st);
    CUDA_OK(cudaMemsetAsync(b.info.p, 0, sizeof(int) * b.count, st));
    b.jacobi = b.np <= kJacobiMax;
  }
  // the Jacobi jobs (one block per matrix) and their kept eigenvector bases
  std::vector<JacobiJob> jac;
  DevBuf<double> jac_basis;
  DevBuf<JacobiJob> jac_d;
  int jac_n = 0;
  {
    size_t basis_len = 0;
    for (const auto &sp : subs)
      if (sp->nao > 0 && buckets[sp->bucket].jacobi) basis_len += (size_t)chan * sp->np * sp->np;
    jac_basis.alloc(std::max<size_t>(basis_len, 1), st);
    size_t off = 0;
    for (const auto &sp : subs) {
      if (sp->nao == 0 || !buckets[sp->bucket].jacobi) continue;
      DcBucket &b = buckets[sp->bucket];
      const size_t npp = (size_t)b.np * b.np;
      for (int c = 0; c < chan; ++c) {
        const size_t k = (size_t)sp->slot + c;
        jac.push_back(JacobiJob{b.A.p + k * npp, b.eps.p + k * b.np, jac_basis.p + off, b.info.p + k, sp->nao, b.np});
        off += npp;
      }
      jac_n = std::max(jac_n, sp->nao);
    }
    upload(jac_d, jac, st);
    if (!jac.empty())
      prepare_jacobi_eigen(jac_n);
  }
  // Lanes: the subsystems' launch sequences are independent, so they run on kDcLanes side
  // streams forked from and joined back into the main stream (parallel branches of the captured
  // graphs), each lane with its own scratch. The lanes synchronise before their buffers go.
  const size_t mm = (size_t)std::max(max_nao, 1) * std::max(max_nao, 1);
  const size_t vv = (size_t)chan * std::max(max_np, 1) * std::max(max_np, 1);
  struct Lane {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    DevBuf<double> Pl, Pa, Pb, Fa, Fb, Vf, env, part;
    ~Lane() {
      if (st) cudaStreamSynchronize(st);
      if (done) cudaEventDestroy(done);
      // the buffers are released (stream-ordered on the main stream) after this body
    }
  };
  const int n_lanes = (int)std::min<size_t>(kDcLanes, std::max<size_t>(subs.size(), 1));
  std::deque<Lane> lanes(n_lanes);
  struct LaneStreams {
    std::deque<Lane> &l;
    cudaEvent_t fork = nullptr;
    ~LaneStreams() {
      for (Lane &x : l)
        if (x.st) {
          cudaStreamSynchronize(x.st);
          cudaStreamDestroy(x.st);
          x.st = nullptr;
        }
      if (fork) cudaEventDestroy(fork);
    }
  } lane_streams{lanes};
  CUDA_OK(cudaEventCreateWithFlags(&lane_streams.fork, cudaEventDisableTiming));
  for (Lane &L : lanes) {
    CUDA_OK(cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
    L.Pl.alloc(mm, st);
    L.Fa.alloc(mm, st);
    if (unrestricted) {
      L.Pa.alloc(mm, st);
      L.Pb.alloc(mm, st);
      L.Fb.alloc(mm, st);
    }
    L.Vf.alloc(vv, st);
    L.env.alloc(std::max(largest_atoms, 1), st);
    L.part.alloc(kDcPartials, st);
  }
  auto fork = [&]() {
    CUDA_OK(cudaEventRecord(lane_streams.fork, st));
    for (Lane &L : lanes) CUDA_OK(cudaStreamWaitEvent(L.st, lane_streams.fork, 0));
  };
  auto join = [&]() {
    for (Lane &L : lanes) {
      CUDA_OK(cudaEventRecord(L.done, L.st));
      CUDA_OK(cudaStreamWaitEvent(st, L.done, 0));
    }
  };
  // each subsystem's Fermi-weighted density (and spin density), kept until the ordered scatter
  std::vector<size_t> dm_off(subs.size() + 1, 0);
  for (size_t a = 0; a < subs.size(); ++a) dm_off[a + 1] = dm_off[a] + (size_t)subs[a]->nao * subs[a]->nao;
  DevBuf<double> Dm, econ, se, sw;
  Dm.alloc(std::max<size_t>(dm_off.back(), 1) * (unrestricted ? 2 : 1), st);
  econ.alloc(std::max<size_t>(subs.size(), 1), st);
  se.alloc(std::max<size_t>(n_states, 1), st);
  sw.alloc(std::max<size_t>(n_states, 1), st);
  mark("builds_done+lanes", st);
  // the contributions of every stored atom pair (see DcPairSrc), indexed by an N x N table
  DevBuf<int> pair_rec_d;
  DevBuf<DcPairSrc> recs_d;
  {
    std::vector<int> core_of(N, -1), local(N, -1);
    for (size_t a = 0; a < subs.size(); ++a)
      for (int i = 0; i < subs[a]->part.n_core; ++i) core_of[subs[a]->part.parent[i]] = (int)a;
    // local atom index of a parent atom in a subsystem: (atom, local) sorted per subsystem, built
    // on demand (memory in proportion to the subsystems' sizes, not to N per subsystem)
    std::vector<std::vector<std::pair<int, int>>> where(subs.size());
    auto local_of = [&](int a, int atom) {
      std::vector<std::pair<int, int>> &w = where[a];
      if (w.empty()) {
        for (int i = 0; i < subs[a]->m.n; ++i) w.emplace_back(subs[a]->part.parent[i], i);
        std::sort(w.begin(), w.end());
      }
      const auto it = std::lower_bound(w.begin(), w.end(), std::make_pair(atom, -1));
      return (it != w.end() && it->first == atom) ? it->second : -1;
    };
    std::vector<int> rec((size_t)N * N, -1);
    std::vector<DcPairSrc> recs;
    // the stored pairs are exactly the (core, member) pairs of the subsystems, both ways round
    std::vector<std::pair<int, int>> stored_pairs;
    for (const auto &sp : subs) {
      const auto &par = sp->part.parent;
      for (int i = 0; i < sp->part.n_core; ++i)
        for (int j = 0; j < (int)par.size(); ++j) {
          stored_pairs.emplace_back(par[i], par[j]);
          stored_pairs.emplace_back(par[j], par[i]);
        }
    }
    for (const auto &ab : stored_pairs) {
      const int A = ab.first, B = ab.second;
      if (rec[(size_t)A * N + B] >= 0) continue;
      {
        DcPairSrc q{};
        const int sa = core_of[A], sb = core_of[B];
        for (int sub : {sa, sb}) {
          if (q.n == 1 && sub == sa) break;  // both atoms in one core: one contribution
          const int ia = local_of(sub, A), ib = local_of(sub, B);
          if (ia < 0 || ib < 0) continue;
          const DcSub &x = *subs[sub];
          const bool ca = ia < x.part.n_core, cb = ib < x.part.n_core;
          if (!ca && !cb) continue;
          q.off[q.n] = (long long)dm_off[sub];
          q.nao[q.n] = x.nao;
          q.la[q.n] = x.L.aoff[ia];
          q.lb[q.n] = x.L.aoff[ib];
          q.w[q.n] = (ca && cb) ? 1.0 : 0.5;
          ++q.n;
        }
        rec[(size_t)A * N + B] = (int)recs.size();
        recs.push_back(q);
      }
    }
    upload(pair_rec_d, rec, st);
    upload(recs_d, recs, st);
  }
  mark("pair_table", st);
  struct LaneSync {  // destroyed first: no lane work is pending when the buffers above are released
    std::deque<Lane> &l;
    ~LaneSync() {
      for (Lane &x : l)
        if (x.st) cudaStreamSynchronize(x.st);
    }
  } lane_sync{lanes};

  // eigensolver workspaces (the bucket shapes are fixed for the whole run)
  cusolverDnParams_t sparams = nullptr;
  SOLVER_OK(cusolverDnCreateParams(&sparams));
  struct ParamsGuard {
    cusolverDnParams_t p;
    ~ParamsGuard() { cusolverDnDestroyParams(p); }
  } pguard{sparams};
  size_t wd_max = 0, wh_max = 0;
  int lwork_max = 0;
  for (DcBucket &b : buckets) {
    if (b.jacobi) continue;
    if (b.np >= 512) {
      int lw = 0;
      SOLVER_OK(cusolverDnDsyevd_bufferSize(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, b.np, b.A.p,
                                            b.np, b.eps.p, &lw));
      lwork_max = std::max(lwork_max, lw);
    } else {
      size_t wd = 0, wh = 0;
      SOLVER_OK(cusolverDnXsyevBatched_bufferSize(ctx.solver, sparams, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                                  b.np, CUDA_R_64F, b.A.p, b.np, CUDA_R_64F, b.eps.p, CUDA_R_64F, &wd,
                                                  &wh, b.count));
      wd_max = std::max(wd_max, wd);
      wh_max = std::max(wh_max, wh);
    }
  }
  DevBuf<double> dwork;
  DevBuf<unsigned char> bwork;
  dwork.alloc(std::max(lwork_max, 1), st);
  bwork.alloc(std::max<size_t>(wd_max, 1), st);
  std::vector<unsigned char> hwork(wh_max);

  std::vector<double> econ_h(subs.size());
  double fermi = 0.0, err = INFINITY, electronic = 0.0;
  int iterations = 0;
  bool converged = false;
  // One iteration is three parts: the subsystem Fock builds (queue_pre), the eigensolves
  // (cuSOLVER, issued directly) and the Fermi level with the reassembly (queue_post). The first
  // iteration runs them as plain launches, which also settles the autotuned Fock shapes; from the
  // second on the two launch sequences (thousands of small kernels, identical every iteration)
  // are replayed as CUDA graphs.
  auto queue_pre = [&]() {
    // environment potential of the current populations (src/dandc/mod.rs:946-998)
    k_dc_pops<<<(N + 127) / 128, 128, 0, st>>>(N, aoff.p, norb.p, nao_g, Pg.p, pops.p);
    k_dc_coulomb<<<(N + 3) / 4, 128, 0, st>>>(N, xyz.p, pops.p, gelec.p);
    note_launch();
    note_launch();
    // every subsystem: Fock build, environment, packing, energy (src/dandc/mod.rs:526-663)
    fork();
    for (size_t a = 0; a < subs.size(); ++a) {
      DcSub &s = *subs[a];
      Lane &L = lanes[a % lanes.size()];
      const cudaStream_t ls = L.st;
      if (s.nao == 0) {
        CUDA_OK(cudaMemsetAsync(econ.p + a, 0, sizeof(double), ls));
        continue;
      }
      DcBucket &b = buckets[s.bucket];
      const size_t nn = (size_t)s.nao * s.nao;
      k_dc_env<<<(s.m.n + 3) / 4, 128, 0, ls>>>(s.m.n, s.parent.p, xyz.p, pops.p, gelec.p, L.env.p);
      k_dc_gather<<<grid_for(nn), 256, 0, ls>>>(s.nao, s.map.p, s.ao_par.p, N, nao_g, wdev.p, Pg.p,
                                                unrestricted ? Sg.p : nullptr, L.Pl.p, L.Pa.p, L.Pb.p);
      note_launch();
      note_launch();
      const FockGeometry g = s.D.geometry();
      double *slot_a = b.A.p + (size_t)s.slot * b.np * b.np;
      if (!unrestricted) {
        launch_fock(ls, g, P, s.D.H.p, L.Pl.p, L.Pl.p, 0.5, L.Fa.p, s.D.pop.p, s.D.jbuf.p);
      } else {
        launch_fock(ls, g, P, s.D.H.p, L.Pl.p, L.Pa.p, 1.0, L.Fa.p, s.D.pop.p, s.D.jbuf.p);
        launch_fock(ls, g, P, s.D.H.p, L.Pl.p, L.Pb.p, 1.0, L.Fb.p, s.D.pop.p, s.D.jbuf.p);
      }
      const size_t npp = (size_t)b.np * b.np;
      k_dc_pack<<<grid_for(npp), 256, 0, ls>>>(s.nao, b.np, L.Fa.p, s.ao_atom.p, L.env.p, slot_a);
      note_launch();
      if (unrestricted) {
        k_dc_pack<<<grid_for(npp), 256, 0, ls>>>(s.nao, b.np, L.Fb.p, s.ao_atom.p, L.env.p, slot_a + npp);
        note_launch();
      }
      k_dc_energy<<<kDcPartials, 256, 0, ls>>>(s.nao, b.np, s.core_ao, L.Pl.p, s.D.H.p, slot_a, L.part.p);
      note_launch();
      launch_sum(ls, L.part.p, kDcPartials, econ.p + a);
    }
    join();
  };
  int jac_warm = 0;  // the Jacobi bases hold the previous iteration's eigenvectors
  auto queue_eig = [&]() {
    // the subsystem eigenproblems: one Jacobi launch for every matrix of order <= kJacobiMax, the
    // larger buckets through cuSOLVER
    if (!jac.empty()) {
      launch_jacobi_eigen(st, jac_d.p, (int)jac.size(), jac_n, jac_warm, kDcPad);
      note_launch();
    }
    for (DcBucket &b : buckets) {
      if (b.jacobi) continue;
      if (b.np >= 512) {
        for (int k = 0; k < b.count; ++k)
          SOLVER_OK(cusolverDnDsyevd(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, b.np,
                                     b.A.p + (size_t)k * b.np * b.np, b.np, b.eps.p + (size_t)k * b.np, dwork.p,
                                     lwork_max, b.info.p + k));
      } else {
        SOLVER_OK(cusolverDnXsyevBatched(ctx.solver, sparams, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, b.np,
                                         CUDA_R_64F, b.A.p, b.np, CUDA_R_64F, b.eps.p, CUDA_R_64F, bwork.p, wd_max,
                                         hwork.empty() ? nullptr : hwork.data(), wh_max, b.info.p, b.count));
      }
    }
  };
  auto queue_post = [&]() {
    // weighted spectra and the common Fermi level
    fork();
    for (size_t a = 0; a < subs.size(); ++a) {
      DcSub &s = *subs[a];
      if (s.nao == 0) continue;
      const cudaStream_t ls = lanes[a % lanes.size()].st;
      DcBucket &b = buckets[s.bucket];
      for (int c = 0; c < chan; ++c) {
        const size_t k = (size_t)s.slot + c;
        k_dc_norms<<<(s.nao + 3) / 4, 128, 0, ls>>>(s.nao, b.np, s.core_ao, unrestricted ? 0.5 : 1.0,
                                                    b.A.p + k * b.np * b.np, b.eps.p + k * b.np,
                                                    se.p + s.spec + (size_t)c * s.nao, sw.p + s.spec + (size_t)c * s.nao);
        note_launch();
      }
    }
    join();
    k_dc_fermi<<<1, 1024, 0, st>>>(n_states, se.p, sw.p, n_elec, dc.fermi_width_ev, scal.p + 1);
    note_launch();
    // reassembly (src/dandc/mod.rs:354-393): V^T diag(f) V per subsystem on the lanes, then every
    // stored element of the global density gathers its (at most two) weighted contributions
    fork();
    for (size_t a = 0; a < subs.size(); ++a) {
      DcSub &s = *subs[a];
      if (s.nao == 0) continue;
      Lane &L = lanes[a % lanes.size()];
      DcBucket &b = buckets[s.bucket];
      const size_t npp = (size_t)b.np * b.np;
      for (int spin = 0; spin < (unrestricted ? 2 : 1); ++spin) {
        for (int c = 0; c < chan; ++c) {
          const double scale = !unrestricted ? 1.0 : (c == 0 ? 0.5 : (spin ? -0.5 : 0.5));
          const size_t k = (size_t)s.slot + c;
          k_dc_occupy<<<grid_for(npp), 256, 0, L.st>>>(s.nao, b.np, scale, b.A.p + k * npp, b.eps.p + k * b.np,
                                                       scal.p + 1, dc.fermi_width_ev, L.Vf.p + (size_t)c * npp);
          note_launch();
        }
        // the channels' slots are adjacent, so both enter one product of inner dimension chan*np
        launch_gemm_tn(L.st, s.nao, s.nao, chan * b.np, 1.0, L.Vf.p, b.np, b.A.p + (size_t)s.slot * npp, b.np,
                       Dm.p + (spin ? dm_off.back() : 0) + dm_off[a], s.nao);
      }
    }
    join();
    k_dc_assemble<<<kDcAssembleBlocks, 256, 0, st>>>(nao_g, N, ao_atom.p, aoff.p, pair_rec_d.p, recs_d.p, Dm.p,
                                               unrestricted ? Dm.p + dm_off.back() : nullptr, dc.mixing, Pg.p,
                                               unrestricted ? Sg.p : nullptr, partials.p);
    note_launch();
    launch_sum(st, partials.p, kDcAssembleBlocks, scal.p);
  };
  struct Graphs {
    cudaGraphExec_t pre = nullptr, post = nullptr;
    int n_pre = 0, n_post = 0;
    ~Graphs() {
      if (pre) cudaGraphExecDestroy(pre);
      if (post) cudaGraphExecDestroy(post);
    }
  } graphs;
  auto capture = [&](const std::function<void()> &fn, cudaGraphExec_t &exec, int &nodes) {
    const long long before = pm7_launch_count();
    cudaGraph_t graph = nullptr;
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    fn();
    CUDA_OK(cudaStreamEndCapture(st, &graph));
    nodes = (int)(pm7_launch_count() - before);
    note_launch(-nodes);  // counted when replayed
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    CUDA_OK(ie);
  };
  auto replay = [&](cudaGraphExec_t exec, int nodes) {
    CUDA_OK(cudaGraphLaunch(exec, st));
    note_launch(nodes);
  };
  // PM7_DANDC_TRACE: per-phase wall times on stderr (each phase then ends in a synchronise)
  double t_phase[4] = {0, 0, 0, 0};
  auto tick = [&](int k, std::chrono::steady_clock::time_point &t) {
    if (!trace) return;
    CUDA_OK(cudaStreamSynchronize(st));
    const auto now = std::chrono::steady_clock::now();
    t_phase[k] += std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
  };
  if (trace) CUDA_OK(cudaStreamSynchronize(st));
  auto t = std::chrono::steady_clock::now();
  const double t_setup = std::chrono::duration<double, std::milli>(t - t_start).count();
  for (int iter = 0; iter < dc.max_scf; ++iter) {
    iterations = iter + 1;
    jac_warm = iter > 0 ? 1 : 0;
    if (iter == 0) {
      queue_pre();
      tick(1, t);
      queue_eig();
      tick(2, t);
      queue_post();
      tick(3, t);
    } else {
      if (!graphs.pre) capture(queue_pre, graphs.pre, graphs.n_pre);
      replay(graphs.pre, graphs.n_pre);
      tick(1, t);
      queue_eig();
      tick(2, t);
      if (!graphs.post) capture(queue_post, graphs.post, graphs.n_post);
      replay(graphs.post, graphs.n_post);
      tick(3, t);
    }
    double sc[3];
    CUDA_OK(cudaMemcpyAsync(sc, scal.p, sizeof(sc), cudaMemcpyDeviceToHost, st));
    if (!subs.empty())
      CUDA_OK(cudaMemcpyAsync(econ_h.data(), econ.p, sizeof(double) * subs.size(), cudaMemcpyDeviceToHost, st));
    std::vector<std::vector<int>> infos(buckets.size());
    for (size_t k = 0; k < buckets.size(); ++k) {
      infos[k].resize(buckets[k].count);
      CUDA_OK(cudaMemcpyAsync(infos[k].data(), buckets[k].info.p, sizeof(int) * buckets[k].count,
                              cudaMemcpyDeviceToHost, st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
    CUDA_OK(cudaGetLastError());
    for (const auto &v : infos)
      for (int x : v)
        if (x != 0)
          throw Failure{PM7_ERR_LINEAR_ALGEBRA, "subsystem eigendecomposition failed (info " + std::to_string(x) + ")"};
    if (sc[2] != 0.0) {
      // the message of src/dandc/mod.rs:743-757: the span of the subsystems' (alpha) spectra
      std::vector<double> eh(n_states);
      CUDA_OK(cudaMemcpy(eh.data(), se.p, sizeof(double) * n_states, cudaMemcpyDeviceToHost));
      double lo = INFINITY, hi = -INFINITY;
      for (const auto &sp : subs)
        if (sp->nao > 0) {
          lo = std::min(lo, eh[sp->spec]);
          hi = std::max(hi, eh[sp->spec + sp->nao - 1]);
        }
      char buf[256];
      std::snprintf(buf, sizeof buf,
                    "no chemical potential in [-500, 500] eV holds %g electrons; the subsystem spectra span %.3f to "
                    "%.3f eV",
                    n_elec, lo, hi);
      throw Failure{PM7_ERR_INVALID_INPUT, buf};
    }
    const size_t n_st = (size_t)std::max<int64_t>(stored, 1);
    err = std::sqrt(sc[0] / (double)n_st);
    fermi = sc[1];
    electronic = 0.0;
    for (double e : econ_h) electronic += e;
    if (err < dc.p_tol) {
      converged = true;
      break;
    }
  }

  if (trace)
    std::fprintf(stderr,
                 "pm7_run_dandc ms: setup %.1f (%s) fock %.1f eigen %.1f reassembly %.1f (%d iterations, %zu buckets)\n",
                 t_setup, setup_marks.c_str(), t_phase[1], t_phase[2], t_phase[3], iterations, buckets.size());
  // energy, charges and (on request) the gradient at the divide-and-conquer density
  DeviceMolecule Dg;
  build_device_molecule(Dg, m, Lg, P, Lg.has_d, st);
  DevBuf<double> cscratch, cout;
  cscratch.alloc(corrections_scratch(N), st);
  cout.alloc(5, st);
  launch_corrections(st, N, Dg.z.p, Dg.xyz.p, o.method, o.smooth_dispersion, cscratch.p, cscratch.n, cout.p);
  k_dc_pops<<<(N + 127) / 128, 128, 0, st>>>(N, aoff.p, norb.p, nao_g, Pg.p, pops.p);
  note_launch();
  double parts5[5];
  std::vector<double> pop_h(N);
  CUDA_OK(cudaMemcpyAsync(parts5, cout.p, sizeof(parts5), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(pop_h.data(), pops.p, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  double corr = parts5[0];
  corr += parts5[1];
  corr += parts5[4];
  corr += parts5[2];
  corr += parts5[3];
  res->n_atoms = N;
  res->nao = nao_g;
  res->converged = converged ? 1 : 0;
  res->iterations = iterations;
  res->subsystems = (int)subs.size();
  res->largest_subsystem = largest_atoms;
  res->unrestricted = unrestricted ? 1 : 0;
  res->fermi_ev = fermi;
  res->electronic_ev = electronic;
  res->density_error = err;
  res->core_core_ev = Dg.core_core_ev;
  res->correction_ev = corr * kKcalToEv;
  res->energy_ev = electronic + Dg.core_core_ev + corr * kKcalToEv;
  res->stored_density_elements = stored;
  res->charges = static_cast<double *>(std::malloc(sizeof(double) * std::max(N, 1)));
  for (int a = 0; a < N; ++a) res->charges[a] = cores[a] - pop_h[a];
  if (want_gradient) {
    // electronic_gradient_sparse + core_core_gradient + the correction gradient
    // (src/dandc/mod.rs:462-481): the RHF fixed-density form on the total density
    GradGeometry g{};
    g.n_atoms = Dg.n;
    g.nao = Dg.nao;
    g.n_near = Dg.n_near;
    g.z = Dg.z.p;
    g.aoff = Dg.aoff.p;
    g.xyz = Dg.xyz.p;
    g.near_mask = Dg.mask.p;
    g.np = Dg.near.p;
    g.Pt = Pg.p;
    g.Ps = nullptr;
    const std::vector<double> gr = geometry_gradient(st, P, g, Lg.has_d, o.method, o.smooth_dispersion, true,
                                                     std::find(m.z.begin(), m.z.end(), 14) != m.z.end());
    res->gradient = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(gr.size(), 1)));
    std::memcpy(res->gradient, gr.data(), sizeof(double) * gr.size());
  }
  if (o.want_matrices) {
    res->density = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(nng, 1)));
    CUDA_OK(cudaMemcpyAsync(res->density, Pg.p, sizeof(double) * nng, cudaMemcpyDeviceToHost, st));
    if (unrestricted) {
      res->spin_density = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(nng, 1)));
      CUDA_OK(cudaMemcpyAsync(res->spin_density, Sg.p, sizeof(double) * nng, cudaMemcpyDeviceToHost, st));
    }
    CUDA_OK(cudaStreamSynchronize(st));
  }
}

}  // namespace
}  // namespace pm7

using namespace pm7;

extern "C" {

void pm7_dandc_abi_sizes(int64_t out[2]) {
  out[0] = (int64_t)sizeof(pm7_dandc_options);
  out[1] = (int64_t)sizeof(pm7_dandc_result);
}

void pm7_dandc_options_default(pm7_dandc_options *d) {  // src/dandc/mod.rs:70-81
  if (!d) return;
  d->buffer = 15.0;
  d->core_size = 12;
  d->fermi_width_ev = 0.1;
  d->max_scf = 200;
  d->p_tol = 1.0e-6;
  d->mixing = 0.4;
}

pm7_status pm7_run_dandc(const pm7_molecule *molecule, const pm7_params *params, const pm7_options *options,
                         const pm7_dandc_options *dandc, int32_t want_gradient, pm7_dandc_result *result) {
  if (result) std::memset(result, 0, sizeof(*result));
  try {
    run_dandc_impl(molecule, params, options, dandc, want_gradient, result);
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    if (result) pm7_dandc_result_free(result);
    return f.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    if (result) pm7_dandc_result_free(result);
    return PM7_ERR_INVALID_INPUT;
  }
}

pm7_status pm7_stage_dandc_partition(const pm7_molecule *molecule, int32_t core_size, double buffer, int32_t *core_of,
                                     int32_t *sizes, int32_t *n_subsystems, int64_t *stored_pairs) {
  try {
    if (!molecule || !core_of || !sizes || !n_subsystems || !stored_pairs)
      throw Failure{PM7_ERR_INVALID_INPUT, "null argument"};
    // the same option checks as the solve (src/dandc/mod.rs:83-110)
    pm7_dandc_options d;
    pm7_dandc_options_default(&d);
    d.core_size = core_size;
    d.buffer = buffer;
    check_dandc_options(d);
    const Molecule m = to_molecule(molecule);
    const std::vector<DcPart> parts = dc_partition(m, core_size, buffer);
    // stored (ordered) atom pairs: those with at least one atom in some subsystem's core,
    // counted as sorted unique keys over the subsystems (memory linear in their sizes)
    std::vector<int64_t> keys;
    for (size_t a = 0; a < parts.size(); ++a) {
      const DcPart &p = parts[a];
      sizes[a] = (int32_t)p.parent.size();
      for (int i = 0; i < p.n_core; ++i) core_of[p.parent[i]] = (int32_t)a;
      for (int i = 0; i < (int)p.parent.size(); ++i)
        for (int j = 0; j < (int)p.parent.size(); ++j)
          if (i < p.n_core || j < p.n_core) keys.push_back((int64_t)p.parent[i] * m.n + p.parent[j]);
    }
    std::sort(keys.begin(), keys.end());
    const int64_t pairs = (int64_t)(std::unique(keys.begin(), keys.end()) - keys.begin());
    *n_subsystems = (int32_t)parts.size();
    *stored_pairs = pairs;
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

void pm7_dandc_result_free(pm7_dandc_result *r) {
  if (!r) return;
  std::free(r->charges);
  std::free(r->gradient);
  std::free(r->density);
  std::free(r->spin_density);
  r->charges = r->gradient = r->density = r->spin_density = nullptr;
}

}  // extern "C"
