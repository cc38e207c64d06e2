// Batched RHF SCF of many molecules on one device (pm7-rs src/scf.rs:1189-1322 per
// molecule), one launch per SCF phase over every active molecule:
//
//   push -> Fock (far rows | near pairs | atoms) -> energy + density copy -> F P (DMMA,
//   tiles of all molecules) -> E = FP - PF and |E| -> DIIS inner products -> control
//   (history, A-DIIS / CDIIS weights) -> extrapolation into padded size buckets ->
//   batched eigensolve per bucket -> P' = 2 C_occ C_occ^T (DMMA) -> convergence test,
//   stall guard, density swap.
//
// Molecules join (admit) and leave (retire) between iterations, so the same runner
// serves a fixed batch and a continuous request stream. Every per-molecule decision is
// taken on the device from the molecule's MolCtl; the host only rebuilds the work lists
// and reads one done-flag per molecule per iteration.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>
#include <functional>

#include "batch.hpp"
#include "common.cuh"
#include "gradient.cuh"
#include "engine_internal.hpp"

namespace pm7 {

// ===========================================================================
// device side
// ===========================================================================
namespace {

constexpr int RB = 256;        // threads of the block-per-molecule kernels
constexpr double kPad = 1.0e5;  // diagonal of the padding rows of a bucket matrix (eV)

// Sums NV values over the block; the totals are valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum_n(double (&v)[NV]) {
  __shared__ double red[NV][RB / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[k][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = 0.0;
      for (int w = 0; w < RB / 32; ++w) x += red[k][w];
      v[k] = x;
    }
  }
  __syncthreads();
}

// Zero H; P = the SAD diagonal (or the caller's full density staged in Pn).
__global__ void __launch_bounds__(RB) k_b_init(BatchList L, const MolDesc *__restrict__ D,
                                               const MolCtl *__restrict__ C, const double *const *__restrict__ sad) {
  const int slot = L.slot[blockIdx.x];
  const MolDesc &d = D[slot];
  const int n = d.g.nao;
  const size_t nn = (size_t)n * n;
  const double *diag = sad[blockIdx.x];
  for (size_t i = threadIdx.x; i < nn; i += RB) {
    d.H[i] = 0.0;
    const size_t r = i / n, c = i - r * n;
    d.P[i] = diag ? (r == c ? diag[r] : 0.0) : d.Pn[i];
  }
  if (d.X32) {  // the fp32 arrays' padding must stay zero
    const size_t l32 = (size_t)d.ld32 * d.ld32;
    for (size_t i = threadIdx.x; i < l32; i += RB) d.X32[i] = d.hi32[i] = d.lo32[i] = d.C32[i] = 0.0f;
  }
}

// The two energy fold jobs of each listed molecule, <P, H> and <P, F> (F: this iteration's
// Fock in the history ring, or with final_pass the final Fock in X), from the device
// descriptors: P and Pn swap on the device, so only D knows the density.
__global__ void k_b_fold_jobs(int n, const int *__restrict__ slots, const MolDesc *__restrict__ D,
                              MolCtl *__restrict__ C, SeqSumJob *__restrict__ jobs, int final_pass) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const MolDesc &d = D[slots[m]];
  MolCtl &c = C[slots[m]];
  const size_t nn = (size_t)d.g.nao * d.g.nao;
  jobs[2 * m] = {d.P, d.H, nn, &c.e_fold[0]};
  jobs[2 * m + 1] = {d.P, final_pass ? d.X : hist_F(d, c.slot), nn, &c.e_fold[1]};
}

// e_final = 1/2 (<P, H> + <P, F>) from the two folds of the final density (scf.rs:1297-1298).
__global__ void k_b_fold_energy(int n, const int *__restrict__ slots, MolCtl *__restrict__ C) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  MolCtl &c = C[slots[m]];
  c.e_final = 0.5 * (c.e_fold[0] + c.e_fold[1]);
}

// Make room in the DIIS ring (HistoryHost::push).
__global__ void k_b_push(int n, const int *__restrict__ slots, MolCtl *__restrict__ C) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  MolCtl &c = C[slots[m]];
  if (c.n_ord < kHist) {
    c.slot = c.n_ord;
  } else {
    c.slot = c.ord[0];
    for (int i = 0; i + 1 < c.n_ord; ++i) c.ord[i] = c.ord[i + 1];
    c.n_ord -= 1;
  }
}

// Partial of E_el = 1/2 sum P (H + F) (scf.rs:1237) into part[0]; in the SCF loop also
// D_slot = P. Item = a chunk.
__global__ void __launch_bounds__(RB) k_b_energy_c(BatchList L, const MolDesc *__restrict__ D,
                                                   const MolCtl *__restrict__ C, int final_pass) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const MolCtl &c = C[r.slot];
  const double *F = final_pass ? d.X : hist_F(d, c.slot);
  double *Dc = final_pass ? nullptr : hist_D(d, c.slot);
  double v[1] = {0.0};
  for (size_t i = r.e0 + threadIdx.x; i < r.e1; i += RB) {
    const double p = d.P[i];
    v[0] += p * (d.H[i] + F[i]);
    if (Dc) Dc[i] = p;
  }
  block_sum_n<1>(v);
  if (threadIdx.x == 0) d.part[(size_t)r.q * kPart + 0] = v[0];
}

// E_slot = X - X^T with X = F P (scf.rs:1148-1156), partial |E|^2 into part[1].
__global__ void __launch_bounds__(RB) k_b_antisym_c(BatchList L, const MolDesc *__restrict__ D,
                                                    const MolCtl *__restrict__ C) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const int n = d.g.nao;
  double *E = hist_E(d, C[r.slot].slot);
  double v[1] = {0.0};
  for (size_t i = r.e0 + threadIdx.x; i < r.e1; i += RB) {
    const size_t row = i / n, col = i - row * n;
    const double e = d.X[i] - d.X[col * n + row];
    E[i] = e;
    v[0] += e * e;
  }
  block_sum_n<1>(v);
  if (threadIdx.x == 0) d.part[(size_t)r.q * kPart + 1] = v[0];
}

// Partials of the inner products of the new history entry with the older ones
// (chronological) into part[2..27]: <E_i, E_new> (i < k) and <E_new, E_new>; <D_new, F_j>
// and <D_new, F_new>; <D_i, F_new>.
__global__ void __launch_bounds__(RB) k_b_dots_c(BatchList L, const MolDesc *__restrict__ D,
                                                 const MolCtl *__restrict__ C) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const MolCtl &c = C[r.slot];
  const int k = c.n_ord;
  const double *En = hist_E(d, c.slot), *Fn = hist_F(d, c.slot), *Dn = hist_D(d, c.slot);
  const double *Eo[kHist], *Fo[kHist], *Do[kHist];
#pragma unroll
  for (int i = 0; i < kHist; ++i) {
    const int o = i < k ? c.ord[i] : c.slot;
    Eo[i] = hist_E(d, o);
    Fo[i] = hist_F(d, o);
    Do[i] = hist_D(d, o);
  }
  double v[3 * kHist + 2];
#pragma unroll
  for (int i = 0; i < 3 * kHist + 2; ++i) v[i] = 0.0;
  for (size_t e = r.e0 + threadIdx.x; e < r.e1; e += RB) {
    const double en = En[e], dn = Dn[e], fn = Fn[e];
#pragma unroll
    for (int i = 0; i < kHist; ++i) {
      if (i < k) {
        v[i] += Eo[i][e] * en;
        v[kHist + 1 + i] += dn * Fo[i][e];
        v[2 * kHist + 2 + i] += Do[i][e] * fn;
      }
    }
    v[kHist] += en * en;
    v[2 * kHist + 1] += dn * fn;
  }
  block_sum_n<3 * kHist + 2>(v);
  if (threadIdx.x == 0)
    for (int i = 0; i < 3 * kHist + 2; ++i) d.part[(size_t)r.q * kPart + 2 + i] = v[i];
}

// Per molecule: the chunk partials summed in chunk order: E_el of the iteration (for the
// convergence test; the reported energy is the reference's fold, k_b_fold_energy), |E|^2
// and the DIIS inner products.
__global__ void k_b_reduce(int n, const int *__restrict__ slots, const MolDesc *__restrict__ D,
                           MolCtl *__restrict__ C) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const MolDesc &d = D[slots[m]];
  MolCtl &c = C[slots[m]];
  const int nc = items_chunks(d.g.nao);
  double e = 0.0;
  for (int q = 0; q < nc; ++q) e += d.part[(size_t)q * kPart + 0];
  c.e_elec = 0.5 * e;
  double err2 = 0.0;
  for (int q = 0; q < nc; ++q) err2 += d.part[(size_t)q * kPart + 1];
  c.err2 = err2;
  const int k = c.n_ord;
  for (int t = 0; t < 3 * kHist + 2; ++t) {
    const bool used = t < k || t == kHist || (t > kHist && t < kHist + 1 + k) || t == 2 * kHist + 1 ||
                      (t >= 2 * kHist + 2 && t < 2 * kHist + 2 + k);
    if (!used) continue;
    double s = 0.0;
    for (int q = 0; q < nc; ++q) s += d.part[(size_t)q * kPart + 2 + t];
    if (t < kHist) c.ee[t] = s;
    else if (t == kHist) c.ee[k] = s;
    else if (t < 2 * kHist + 1) c.df_row[t - kHist - 1] = s;
    else if (t == 2 * kHist + 1) c.df_row[k] = s;
    else c.df_col[t - 2 * kHist - 2] = s;
  }
}

// ---- the <= 9x9 extrapolation algebra (HistoryHost in scf_host.hpp) on the device ----

__device__ __forceinline__ double g_at(const MolCtl &c, int i, int j) { return c.gram[c.ord[i] * kHist + c.ord[j]]; }
__device__ __forceinline__ double x_at(const MolCtl &c, int i, int j) { return c.xdf[c.ord[i] * kHist + c.ord[j]]; }

// Gaussian elimination with partial pivoting on an n x n system (n <= kHist + 1).
__device__ bool small_solve(double *m, int n, double *rhs, double *x) {
  for (int col = 0; col < n; ++col) {
    int piv = col;
    double best = fabs(m[col * n + col]);
    for (int r = col + 1; r < n; ++r)
      if (fabs(m[r * n + col]) > best) {
        best = fabs(m[r * n + col]);
        piv = r;
      }
    if (best < 1.0e-12) return false;
    if (piv != col) {
      for (int j = 0; j < n; ++j) {
        const double t = m[col * n + j];
        m[col * n + j] = m[piv * n + j];
        m[piv * n + j] = t;
      }
      const double t = rhs[col];
      rhs[col] = rhs[piv];
      rhs[piv] = t;
    }
    for (int r = col + 1; r < n; ++r) {
      const double f = m[r * n + col] / m[col * n + col];
      if (f == 0.0) continue;
      for (int j = col; j < n; ++j) m[r * n + j] -= f * m[col * n + j];
      rhs[r] -= f * rhs[col];
    }
  }
  for (int col = n - 1; col >= 0; --col) {
    double s = rhs[col];
    for (int j = col + 1; j < n; ++j) s -= m[col * n + j] * x[j];
    x[col] = s / m[col * n + col];
  }
  return true;
}

// CDIIS weights over the chronological entries (scf.rs:1684-1806); false = fall back.
__device__ bool dev_cdiis(const MolCtl &c, double *w) {
  const int n = c.n_ord;
  if (n < 2) return false;
  double b[(kHist + 1) * (kHist + 1)], rhs[kHist + 1], x[kHist + 1];
  for (int skip = 0; skip + 1 < n; ++skip) {
    const int m = n - skip;
    if (m < 2) continue;
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(g_at(c, skip + i, skip + i)));
    if (!isfinite(scale) || scale <= 0.0) continue;
    const int dim = m + 1;
    for (int i = 0; i < dim * dim; ++i) b[i] = 0.0;
    for (int i = 0; i < dim; ++i) rhs[i] = 0.0;
    for (int i = 0; i < m; ++i) {
      for (int j = 0; j < m; ++j) b[i * dim + j] = g_at(c, skip + i, skip + j) / scale;
      b[i * dim + m] = -1.0;
      b[m * dim + i] = -1.0;
    }
    rhs[m] = -1.0;
    if (!small_solve(b, dim, rhs, x)) continue;
    bool finite = true;
    for (int i = 0; i < dim; ++i) finite = finite && isfinite(x[i]);
    if (!finite) continue;
    double wsum = 0.0;
    for (int i = 0; i < m; ++i) wsum += fabs(x[i]);
    if (wsum <= 25.0) {
      for (int i = 0; i < n; ++i) w[i] = 0.0;
      for (int i = 0; i < m; ++i) w[skip + i] = x[i];
      return true;
    }
  }
  return false;
}

// Euclidean projection onto the probability simplex (sort-based).
__device__ void simplex_project(const double *v, int n, double *out) {
  double u[kHist];
  for (int i = 0; i < n; ++i) u[i] = v[i];
  for (int i = 1; i < n; ++i) {  // descending insertion sort
    const double x = u[i];
    int j = i - 1;
    while (j >= 0 && u[j] < x) {
      u[j + 1] = u[j];
      --j;
    }
    u[j + 1] = x;
  }
  double css = 0.0, theta = 0.0;
  for (int j = 0; j < n; ++j) {
    css += u[j];
    const double t = (css - 1.0) / (j + 1.0);
    if (u[j] - t > 0.0) theta = t;
  }
  for (int i = 0; i < n; ++i) out[i] = fmax(v[i] - theta, 0.0);
}

// A-DIIS weights (scf.rs:1812-1916): projected gradient on the simplex.
__device__ bool dev_adiis(const MolCtl &c, double *cw) {
  const int n = c.n_ord;
  if (n < 2) return false;
  const int last = n - 1;
  double d[kHist], s[kHist * kHist], gr[kHist], trial[kHist], proj[kHist];
  for (int i = 0; i < n; ++i) {
    d[i] = x_at(c, i, last) - x_at(c, last, last);
    for (int j = 0; j < n; ++j) s[i * n + j] = x_at(c, i, j) - x_at(c, i, last) - x_at(c, last, j) + x_at(c, last, last);
  }
  double l = 1.0e-12;
  for (int i = 0; i < n; ++i) {
    double row = 0.0;
    for (int j = 0; j < n; ++j) row += fabs(s[i * n + j] + s[j * n + i]);
    l = fmax(l, row);
  }
  const double lr = 1.0 / l;
  for (int i = 0; i < n; ++i) cw[i] = 0.0;
  cw[last] = 1.0;
  for (int it = 0; it < 400; ++it) {
    for (int k = 0; k < n; ++k) {
      double acc = 2.0 * d[k];
      for (int j = 0; j < n; ++j) acc += (s[k * n + j] + s[j * n + k]) * cw[j];
      gr[k] = acc;
    }
    for (int i = 0; i < n; ++i) trial[i] = cw[i] - lr * gr[i];
    simplex_project(trial, n, proj);
    double delta = 0.0;
    for (int i = 0; i < n; ++i) delta += fabs(proj[i] - cw[i]);
    for (int i = 0; i < n; ++i) cw[i] = proj[i];
    if (delta < 1.0e-12) break;
  }
  return true;
}

// Record the new entry's inner products and choose this iteration's extrapolation.
// DIIS error below which a mixed-precision molecule switches to fp64 densities.
constexpr double kMixedSwitch = 1.0e-3;
constexpr double kMixedSwitchStep = 1.0e-6;  // rms density step that also ends the fp32 phase

__global__ void k_b_control(int n, const int *__restrict__ slots, MolCtl *__restrict__ C,
                            unsigned char *__restrict__ use32) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  MolCtl &c = C[slots[m]];
  // mixed precision: fp32 densities until the DIIS error is small, fp64 from then on
  // (the first cycles' error says nothing: a SAD guess proportional to I commutes with F;
  // for a large molecule the commutator norm can stall at the fp32 noise floor while the
  // density step is already small, so either criterion, or 40 fp32 cycles, ends the phase)
  if (c.mixed && c.iter >= 2 && (sqrt(c.err2) < kMixedSwitch || c.dp < kMixedSwitchStep || c.fp32_iters >= 40))
    c.mixed = 0;
  c.use32 = c.mixed;
  use32[m] = (unsigned char)c.use32;
  const int s = c.slot, k = c.n_ord;
  for (int i = 0; i < k; ++i) {
    const int o = c.ord[i];
    c.gram[o * kHist + s] = c.gram[s * kHist + o] = c.ee[i];
    c.xdf[s * kHist + o] = c.df_row[i];
    c.xdf[o * kHist + s] = c.df_col[i];
  }
  c.gram[s * kHist + s] = c.ee[k];
  c.xdf[s * kHist + s] = c.df_row[k];
  c.ord[k] = s;
  c.n_ord = k + 1;
  double w[kHist];
  bool have = false;
  if (c.accel != 0) {
    if (c.accel == 2 || sqrt(c.err2) <= c.adiis_switch) have = dev_cdiis(c, w);
    else have = dev_adiis(c, w);
  }
  if (!have) {
    c.ncoef = 1;
    c.csrc[0] = s;
    c.coef[0] = 1.0;
  } else {
    int q = 0;
    for (int i = 0; i < c.n_ord; ++i)
      if (w[i] != 0.0) {  // an exact zero weight adds exactly nothing
        c.csrc[q] = c.ord[i];
        c.coef[q] = w[i];
        ++q;
      }
    c.ncoef = q;
  }
}

// Element (r, col) of this iteration's extrapolated Fock sum_i c_i F_i + shift (I - P/2)
// (the combine of scf.rs:1169-1176 with the level shift of :1537-1580).
__device__ __forceinline__ double fuse_elem(const MolDesc &d, const MolCtl &c, const double *const *Fs, int r,
                                            int col) {
  const size_t ij = (size_t)r * d.g.nao + col;
  double v = 0.0;
  for (int i = 0; i < c.ncoef; ++i) v += c.coef[i] * Fs[i][ij];
  if (c.shift > 0.0) {
    const double q = d.P[ij] * 0.5;
    v += c.shift * ((r == col) ? 1.0 - q : -q);
  }
  return v;
}

// The molecule's padded bucket matrix from: the extrapolated Fock (src 0), the final
// Fock in X (src 1), or, for reporting orbitals, the final Fock when a level shift was
// active and the last extrapolated Fock otherwise (src 2, scf.rs:1299-1305).
// Grid: x = molecule, y = blocks sharing its matrix (kBucketBlocks).
constexpr int kBucketBlocks = 32;
__global__ void __launch_bounds__(RB) k_b_to_bucket(BatchList L, const MolDesc *__restrict__ D,
                                                    const MolCtl *__restrict__ C, const EigSlot *__restrict__ E,
                                                    int src) {
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const MolCtl &c = C[slot];
  const int n = d.g.nao, np = E[m].ldv;
  if (src == 2) src = c.shift > 0.0 ? 1 : 0;
  double *out = E[m].in;
  const double *Fs[kHist];
  for (int i = 0; i < kHist; ++i) Fs[i] = hist_F(d, i < c.ncoef ? c.csrc[i] : 0);
  const size_t len = (size_t)np * np;
  for (size_t e = (size_t)blockIdx.y * RB + threadIdx.x; e < len; e += (size_t)gridDim.y * RB) {
    const int r = (int)(e / np), col = (int)(e - (size_t)r * np);
    double v;
    if (r < n && col < n) v = src == 1 ? d.X[(size_t)r * n + col] : fuse_elem(d, c, Fs, r, col);
    else v = r == col ? kPad : 0.0;
    out[e] = v;
  }
}

// SP2 start, item = 8 rows: X = the extrapolated Fock, and the rows' Gershgorin bounds
// (min of F_ii - sum_j |F_ij|, max of F_ii + sum_j |F_ij|) into part[0..1].
__global__ void __launch_bounds__(RB) k_b_sp2_fuse(BatchList L, const MolDesc *__restrict__ D,
                                                   const MolCtl *__restrict__ C) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const MolCtl &c = C[slot];
  const int n = d.g.nao, q = item - L.prefix[m];
  const double *Fs[kHist];
  for (int i = 0; i < kHist; ++i) Fs[i] = hist_F(d, i < c.ncoef ? c.csrc[i] : 0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = q * 8 + warp;
  double lo = 1.0e300, hi = -1.0e300;
  if (r < n) {
    double off = 0.0, diag = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double v = fuse_elem(d, c, Fs, r, j);
      d.X[(size_t)r * n + j] = v;
      if (j == r) diag = v;
      else off += fabs(v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_down_sync(0xffffffffu, off, o);
      diag += __shfl_down_sync(0xffffffffu, diag, o);
    }
    lo = diag - off;
    hi = diag + off;
  }
  __shared__ double slo[RB / 32], shi[RB / 32];
  if (lane == 0) {
    slo[warp] = lo;
    shi[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 1.0e300, b = -1.0e300;
    for (int w = 0; w < RB / 32; ++w) {
      a = fmin(a, slo[w]);
      b = fmax(b, shi[w]);
    }
    d.part[(size_t)q * kPart + 0] = a;
    d.part[(size_t)q * kPart + 1] = b;
  }
}

// Per molecule: the spectrum interval from the row partials, widened so that no level
// starts on 0 or 1 (fixed points of both SP2 maps); the purification state is reset.
__global__ void k_b_sp2_bounds(int n, const int *__restrict__ slots, const MolDesc *__restrict__ D,
                               MolCtl *__restrict__ C) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const MolDesc &d = D[slots[m]];
  MolCtl &c = C[slots[m]];
  double a = 1.0e300, b = -1.0e300;
  const int rows = (d.g.nao + 7) / 8;
  for (int q = 0; q < rows; ++q) {
    a = fmin(a, d.part[(size_t)q * kPart + 0]);
    b = fmax(b, d.part[(size_t)q * kPart + 1]);
  }
  const double pad = 1.0e-3 * (b - a) + 1.0e-6;
  c.sp2_emin = a - pad;
  c.sp2_emax = b + pad;
  c.sp2_state = 0;
  c.sp2_steps = 0;
  c.sp2_apply = 0;
}

// Per molecule (one 1,024-thread CTA): kLzSteps Lanczos steps on its extrapolated Fock
// (d.X, before the SP2 map), the vectors in shared memory (3 nao doubles), and the SP2
// interval narrowed to [theta_min - 3% R, theta_max + 5% R] inside the Gershgorin one that
// k_b_sp2_bounds left in sp2_emin / sp2_emax (widened like it). Orders below 2 kLzSteps or
// above kLzMaxOrder keep the Gershgorin interval. Deterministic: fixed-order reductions.
constexpr int kLzMaxOrder = 4096;
__device__ __forceinline__ double lz_block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double s = red[lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[32] = s;
  }
  __syncthreads();
  return red[32];
}
__device__ int lz_sturm(const double *a, const double *b, int m, double x) {
  int c = 0;
  double q = a[0] - x;
  if (q == 0.0) q = -1.0e-300;
  c += q < 0.0;
  for (int i = 1; i < m; ++i) {
    q = a[i] - x - b[i] * b[i] / q;
    if (q == 0.0) q = -1.0e-300;
    c += q < 0.0;
  }
  return c;
}
__global__ void __launch_bounds__(1024) k_b_lanczos(BatchList L, const MolDesc *__restrict__ D,
                                                    MolCtl *__restrict__ C) {
  extern __shared__ double lzs[];
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  const int n = d.g.nao;
  if (n < 2 * kLzSteps || n > kLzMaxOrder) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *vp = lzs, *v = lzs + n, *w = lzs + 2 * n, *red = lzs + 3 * n;
  __shared__ double alpha[kLzSteps], beta[kLzSteps + 1];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 1024) {
    const double x = 1.0 + 0.5 * sin(0.7 * i);
    v[i] = x;
    vp[i] = 0.0;
    s += x * x;
  }
  s = lz_block_sum(s, red);
  const double inv0 = 1.0 / sqrt(s);
  for (int i = threadIdx.x; i < n; i += 1024) v[i] *= inv0;
  double bj = 0.0;
  for (int j = 0; j < kLzSteps; ++j) {
    __syncthreads();
    for (int i = warp; i < n; i += 32) {  // w = X v, a warp per row
      const double *xi = d.X + (size_t)i * n;
      double acc = 0.0;
      for (int base = lane; base < n; base += 256) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int k = base + 32 * u;
          t[u] = k < n ? xi[k] * v[k] : 0.0;
        }
        acc += ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7]));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) w[i] = acc;
    }
    __syncthreads();
    double a = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) a += w[i] * v[i];
    a = lz_block_sum(a, red);
    double q = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) {
      const double x = w[i] - a * v[i] - bj * vp[i];
      w[i] = x;
      q += x * x;
    }
    q = lz_block_sum(q, red);
    const double b = sqrt(q);
    if (threadIdx.x == 0) {
      alpha[j] = a;
      beta[j + 1] = b;
    }
    const double inv = b > 1.0e-280 ? 1.0 / b : 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) {
      vp[i] = v[i];
      v[i] = w[i] * inv;
    }
    bj = b;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double g_lo = 1.0e300, g_hi = -1.0e300;
  for (int i = 0; i < kLzSteps; ++i) {
    const double r = (i > 0 ? fabs(beta[i]) : 0.0) + (i + 1 < kLzSteps ? fabs(beta[i + 1]) : 0.0);
    g_lo = fmin(g_lo, alpha[i] - r);
    g_hi = fmax(g_hi, alpha[i] + r);
  }
  double lo = g_lo, hi = g_hi;
  for (int it = 0; it < 100; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (lz_sturm(alpha, beta, kLzSteps, mid) >= 1) hi = mid;
    else lo = mid;
  }
  const double tmin = hi;
  lo = g_lo;
  hi = g_hi;
  for (int it = 0; it < 100; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (lz_sturm(alpha, beta, kLzSteps, mid) >= kLzSteps) hi = mid;
    else lo = mid;
  }
  const double tmax = hi, R = tmax - tmin;
  if (!(R > 0.0) || !isfinite(R)) return;
  const double elo = fmax(tmin - 0.03 * R, c.sp2_emin), ehi = fmin(tmax + 0.05 * R, c.sp2_emax);
  const double pad = 1.0e-3 * (ehi - elo) + 1.0e-6;
  c.sp2_emin = fmax(elo - pad, c.sp2_emin);
  c.sp2_emax = fmin(ehi + pad, c.sp2_emax);
}

// X <- (emax I - X) / (emax - emin): spectrum in [0, 1], occupied levels near 1. Item = a
// chunk; the chunk's tr X and |X|_F^2 go to part[q kPart + 0 / 1] (the first fused step's
// decision).
__global__ void __launch_bounds__(RB) k_b_sp2_x0(BatchList L, const MolDesc *__restrict__ D,
                                                 const MolCtl *__restrict__ C) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const MolCtl &c = C[r.slot];
  const int n = d.g.nao;
  const double emax = c.sp2_emax, inv = 1.0 / (c.sp2_emax - c.sp2_emin);
  double v[2] = {0.0, 0.0};
  for (size_t e = r.e0 + threadIdx.x; e < r.e1; e += RB) {
    const size_t i = e / n, j = e - i * n;
    const double x = ((i == j ? emax : 0.0) - d.X[e]) * inv;
    d.X[e] = x;
    if (i == j) v[0] += x;
    v[1] += x * x;
  }
  block_sum_n<2>(v);
  if (threadIdx.x == 0) {
    d.part[(size_t)r.q * kPart + 0] = v[0];
    d.part[(size_t)r.q * kPart + 1] = v[1];
  }
}

// The fused fp64 SP2 step's decision (block per molecule), before the squaring: tr X and
// tr X^2 = |X|_F^2 of the current iterate from its partials (the first step: x0's chunk
// partials; later: the previous squaring's 64 x 64 tile partials, both summed in a fixed
// order), then the trace rule (X^2 or 2X - X^2, whichever moves tr X toward n_occ) and the
// stopping rule: idempotency (tr X - tr X^2 at the rounding floor) with tr X = n_occ, or
// failure (non-finite, 100 steps, or an idempotent X of the wrong trace), which leaves the
// molecule to the eigensolver; flags[m]: 0 running, 1 done, 2 failed. sp2_apply marks the
// molecules whose step runs now.
__global__ void __launch_bounds__(RB) k_b_sp2_decide64(BatchList L, const MolDesc *__restrict__ D,
                                                       MolCtl *__restrict__ C, unsigned char *__restrict__ flags) {
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  if (c.sp2_state != 0) {
    if (threadIdx.x == 0) c.sp2_apply = 0;
    return;
  }
  const int n = d.g.nao, k = c.sp2_steps;
  const int t = (n + 63) / 64;
  const int count = k == 0 ? items_chunks(n) : t * (t + 1) / 2;
  const size_t stride = k == 0 ? kPart : 2;
  double v[2] = {0.0, 0.0};
  for (int i = threadIdx.x; i < count; i += RB) {
    v[0] += d.part[(size_t)i * stride + 0];
    v[1] += d.part[(size_t)i * stride + 1];
  }
  block_sum_n<2>(v);
  if (threadIdx.x == 0) {
    const double a = v[0], b = v[1], nocc = (double)d.n_occ;
    c.sp2_square = fabs(b - nocc) < fabs(2.0 * a - b - nocc) ? 1 : 0;
    const double e = a - b;
    int state = 0;
    if (!isfinite(e)) {
      state = 2;
    } else if (fabs(e) <= 1.0e-13 * fmax(1.0, nocc)) {
      state = 1;
    } else if (k >= 2 && fabs(e) < 1.0e-6 && fabs(e) >= fabs(c.sp2_err[(k + 1) % 3])) {
      state = 1;  // at the rounding floor: no further progress
    } else if (k + 1 >= 100) {
      state = 2;
    }
    if (state == 1 && fabs(a - nocc) > 1.0e-3) state = 2;
    c.sp2_err[k % 3] = e;
    c.sp2_steps = k + 1;
    c.sp2_state = state;
    c.sp2_apply = 1;
    flags[m] = (unsigned char)state;
  }
}

// After the fused steps: a converged molecule whose last iterate landed in X gets the
// density Pn = 2 X (one landing in Pn was written doubled by the squaring). Item = a chunk.
__global__ void __launch_bounds__(RB) k_b_sp2_final64(BatchList L, const MolDesc *__restrict__ D,
                                                      const MolCtl *__restrict__ C) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const MolCtl &c = C[r.slot];
  if (c.sp2_state != 1 || (c.sp2_steps - 1) % 2 == 0) return;
  for (size_t e = r.e0 + threadIdx.x; e < r.e1; e += RB) d.Pn[e] = 2.0 * d.X[e];
}

// Stall guard (StallGuardHost::update, scf.rs:1581-1656).
__device__ void guard_update(MolCtl &c, double step, double energy) {
  const int W = 5;
  c.win_step[c.n_win] = step;
  c.win_e[c.n_win] = energy;
  c.n_win += 1;
  const int n = c.n_win;
  if (n < 2 * W) return;
  double s_now = INFINITY, s_was = INFINITY, e_now = INFINITY, e_was = INFINITY;
  for (int i = n - W; i < n; ++i) {
    s_now = fmin(s_now, c.win_step[i]);
    e_now = fmin(e_now, c.win_e[i]);
  }
  for (int i = n - 2 * W; i < n - W; ++i) {
    s_was = fmin(s_was, c.win_step[i]);
    e_was = fmin(e_was, c.win_e[i]);
  }
  bool moved = false;
  if (s_now <= s_was * 0.1) {
    if (c.shift > c.shift_floor) {
      const double relaxed = fmax(c.shift * 0.5, c.shift_floor);
      c.shift = relaxed < 0.25 ? c.shift_floor : relaxed;
      moved = true;
    }
  } else if (s_now > s_was * 0.9 && e_now > e_was - 1.0e-9 && c.shift < 64.0) {
    c.shift = c.shift < 1.0 ? 1.0 : fmin(c.shift * 2.0, 64.0);
    moved = true;
  }
  if (moved) {
    c.n_win = 0;
  } else {
    for (int i = 0; i + 1 < n; ++i) {
      c.win_step[i] = c.win_step[i + 1];
      c.win_e[i] = c.win_e[i + 1];
    }
    c.n_win = n - 1;
  }
}

// Partial of sum (P' - P)^2 into part[28]. Item = a chunk.
__global__ void __launch_bounds__(RB) k_b_sqdiff_c(BatchList L, const MolDesc *__restrict__ D) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  double v[1] = {0.0};
  for (size_t i = r.e0 + threadIdx.x; i < r.e1; i += RB) {
    const double t = d.Pn[i] - d.P[i];
    v[0] += t * t;
  }
  block_sum_n<1>(v);
  if (threadIdx.x == 0) d.part[(size_t)r.q * kPart + 28] = v[0];
}

// Density step, convergence test (scf.rs:1274-1287), stall guard, P <- P' (per molecule).
__global__ void k_b_converge(int n, const int *__restrict__ slots, MolDesc *__restrict__ D, MolCtl *__restrict__ C,
                             unsigned char *__restrict__ flags) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  MolDesc &d = D[slots[m]];
  MolCtl &c = C[slots[m]];
  const size_t nn = mol_nn(d);
  const int nc = items_chunks(d.g.nao);
  double sq = 0.0;
  for (int q = 0; q < nc; ++q) sq += d.part[(size_t)q * kPart + 28];
  const double dp = sqrt(sq / (double)(nn > 0 ? nn : 1));
  c.dp = dp;
  const double de = fabs(c.e_elec - c.e_old);
  double *t = d.P;
  d.P = d.Pn;
  d.Pn = t;
  c.e_old = c.e_elec;
  const bool residual_ok = c.shift == 0.0 && sqrt(c.err2) < 1.0e-7;
  bool hist64 = true;  // no Fock matrix of the DIIS history came from the FP32 build
  for (int i = 0; i < c.n_ord; ++i) hist64 = hist64 && !((c.f32_slots >> c.ord[i]) & 1);
  // only fp64 cycles end the SCF, and only from a history of FP64 Fock builds
  if (!c.use32 && hist64 && c.iter > 0 && de < c.e_tol && (dp < c.p_tol || residual_ok)) {
    c.converged = 1;
    c.done = 1;
  } else {
    guard_update(c, dp, c.e_elec);
  }
  if (c.use32) c.fp32_iters += 1;
  c.iter += 1;
  if (!c.done && c.iter >= c.max_scf) c.done = 1;
  flags[m] = (unsigned char)c.done;
}

// Reported orbitals (energies, and vectors when asked) from the bucket output.
__global__ void __launch_bounds__(RB) k_b_save_orbitals(BatchList L, const MolDesc *__restrict__ D,
                                                        const EigSlot *__restrict__ E) {
  const int m = blockIdx.x;
  const MolDesc &d = D[L.slot[m]];
  const int n = d.g.nao, ld = E[m].ldv;
  for (int i = threadIdx.x; i < n; i += RB) d.eps_out[i] = E[m].eps[i];
  if (d.want_matrices)
    for (size_t e = threadIdx.x; e < (size_t)n * n; e += RB) {
      const size_t r = e / n, col = e - r * n;
      d.V_out[e] = E[m].in[r * ld + col];
    }
}

// Per atom: population and the density elements of the hybrid dipole terms.
__global__ void k_b_atom_out(BatchList L, const MolDesc *__restrict__ D, DeviceParams P) {
  const MolDesc &d = D[L.slot[blockIdx.x]];
  const int n = d.g.nao;
  for (int a = threadIdx.x; a < d.g.n_atoms; a += blockDim.x) {
    const int off = d.g.aoff[a], no = P.elements[d.g.z[a]].n_orb;
    auto pm = [&](int i, int j) { return d.P[(size_t)(off + i) * n + off + j]; };
    double *o = d.atom_out + (size_t)kAtomOut * a;
    double s = 0.0;
    for (int k = 0; k < no; ++k) s += pm(k, k);
    o[0] = s;
    for (int k = 1; k < kAtomOut; ++k) o[k] = 0.0;
    if (no >= 4)
      for (int k = 0; k < 3; ++k) o[1 + k] = pm(0, 1 + k);
    if (no == 9) {
      const int ij[11][2] = {{5, 3}, {4, 1}, {8, 2}, {6, 1}, {7, 3}, {4, 2}, {8, 1}, {6, 2}, {5, 1}, {7, 2}, {6, 3}};
      for (int k = 0; k < 11; ++k) o[4 + k] = pm(ij[k][0], ij[k][1]);
    }
  }
}

// Packs what the host reports of each listed molecule into out + off[m]: 11 control
// scalars, the orbital energies (nao) and the per-atom outputs (kAtomOut n).
constexpr int kOutScalars = 12;
__global__ void k_b_gather_out(BatchList L, const MolDesc *__restrict__ D, const MolCtl *__restrict__ C,
                               const long long *__restrict__ off, double *__restrict__ out) {
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const MolCtl &c = C[slot];
  double *o = out + off[m];
  if (threadIdx.x == 0) {
    o[0] = c.iter;
    o[1] = c.dp;
    o[2] = c.converged;
    o[3] = c.e_final;
    o[4] = c.core_core;
    for (int k = 0; k < 5; ++k) o[5 + k] = c.corr[k];
    o[10] = c.shift;
    o[11] = c.fp32_iters;
  }
  const int nao = d.g.nao, na = kAtomOut * d.g.n_atoms;
  for (int i = threadIdx.x; i < nao; i += blockDim.x) o[kOutScalars + i] = d.eps_out[i];
  for (int i = threadIdx.x; i < na; i += blockDim.x) o[kOutScalars + nao + i] = d.atom_out[i];
}

}  // namespace

// Index of the density element (i, j) of an atom in MolDesc::atom_out.
static int atom_out_index(int i, int j) {
  if (i == 0 && j >= 1 && j <= 3) return j;
  static const int ij[11][2] = {{5, 3}, {4, 1}, {8, 2}, {6, 1}, {7, 3}, {4, 2}, {8, 1}, {6, 2}, {5, 1}, {7, 2}, {6, 3}};
  for (int k = 0; k < 11; ++k)
    if (ij[k][0] == i && ij[k][1] == j) return 4 + k;
  return -1;
}

// ===========================================================================
// host side
// ===========================================================================

// Packs int arrays into one pinned buffer and uploads them with one copy.
class ListUpload {
 public:
  ~ListUpload() {
    if (host_) cudaFreeHost(host_);
    if (dev_) cudaFree(dev_);
  }
  void begin() { used_ = 0; }
  // reserves `bytes` (16-byte aligned) and returns the host pointer and its device offset
  void *add(size_t bytes, size_t &offset) {
    bytes = (bytes + 15) & ~size_t(15);
    offset = used_;
    used_ += bytes;
    stage_.resize(used_);
    return stage_.data() + offset;
  }
  // copies the staged bytes to the device; returns the device base
  char *commit(cudaStream_t st) {
    if (used_ > cap_) {
      if (host_) CUDA_OK(cudaFreeHost(host_));
      if (dev_) CUDA_OK(cudaFree(dev_));
      cap_ = std::max<size_t>(used_ * 2, 1 << 16);
      CUDA_OK(cudaMallocHost((void **)&host_, cap_));
      CUDA_OK(cudaMalloc((void **)&dev_, cap_));
    }
    std::memcpy(host_, stage_.data(), used_);
    if (used_) CUDA_OK(cudaMemcpyAsync(dev_, host_, used_, cudaMemcpyHostToDevice, st));
    return dev_;
  }

 private:
  std::vector<char> stage_;
  char *host_ = nullptr, *dev_ = nullptr;
  size_t cap_ = 0, used_ = 0;
};

struct BatchMol {
  // request
  uint64_t ticket = 0;
  Molecule m;
  pm7_options o;
  Layout L;
  const ParamSet *ps = nullptr;
  int n_occ = 0;
  bool dframe = false;
  std::vector<double> init_density;  // optional caller density
  std::vector<double> init_spin;     // optional caller spin density (single-path requests)
  // device state
  int slot = -1;
  char *base = nullptr;
  size_t bytes = 0;
  MolDesc d{};
  int np = 0;  // bucket matrix size
  bool mixed = false;  // fp32 (tcgen05) SP2 cycles before the fp64 ones
  // outcome
  pm7_status status = PM7_OK;
  std::string error;
  pm7_result result{};
  double t_admit = 0.0;
  double *grad_out = nullptr;  // caller's 3 n_atoms doubles: the nuclear gradient at retirement
  pm7_status grad_status = PM7_OK;
  std::string grad_error;
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// fn(i) for i in [0, n) on the host's cores (contiguous chunks; fn must not throw).
template <class Fn>
static void parallel_for(int n, Fn fn) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int workers = std::min(hw, std::max(1, n / 16));
  if (workers <= 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> th;
  for (int w = 0; w < workers; ++w)
    th.emplace_back([&, w] {
      const int a = (int)((long long)n * w / workers), b = (int)((long long)n * (w + 1) / workers);
      for (int i = a; i < b; ++i) fn(i);
    });
  for (auto &t : th) t.join();
}

static int bucket_size(int nao) { return nao <= 256 ? ((nao + 15) / 16) * 16 : ((nao + 63) / 64) * 64; }

// Device bytes of one molecule (the footprint admission counts), with the layout filled
// into `d` when base != nullptr.
static size_t mol_layout(BatchMol &b, char *base) {
  const Layout &L = b.L;
  const int n = b.m.n, nao = L.nao;
  const size_t nn = (size_t)nao * nao;
  const int gx = (n + 127) / 128;
  size_t off = 0;
  auto take = [&](size_t bytes) -> char * {
    char *p = base ? base + off : nullptr;
    off += align256(std::max<size_t>(bytes, 8));
    return p;
  };
  MolDesc &d = b.d;
  d.H = (double *)take(8 * nn);
  d.P = (double *)take(8 * nn);
  d.Pn = (double *)take(8 * nn);
  d.X = (double *)take(8 * nn);
  d.hist = (double *)take(8 * nn * 3 * kHist);
  d.w = (double *)take(8 * (size_t)L.w_len);
  d.ecore = (double *)take(8 * (size_t)L.e_len);
  d.jbuf = (double *)take(8 * (size_t)L.e_len);
  d.pop = (double *)take(8 * (size_t)n);
  d.eps_out = (double *)take(8 * (size_t)nao);
  d.V_out = b.o.want_matrices ? (double *)take(8 * nn) : nullptr;
  d.atom_out = (double *)take(8 * (size_t)kAtomOut * n);
  d.part = (double *)take(8 * (size_t)kPart * std::max(items_chunks(nao), items_rows8(nao)));
  d.ld32 = b.mixed ? ((nao + 31) / 32) * 32 : 0;
  const size_t l32 = (size_t)d.ld32 * d.ld32;
  d.X32 = b.mixed ? (float *)take(4 * l32) : nullptr;
  d.hi32 = b.mixed ? (float *)take(4 * l32) : nullptr;
  d.lo32 = b.mixed ? (float *)take(4 * l32) : nullptr;
  d.C32 = b.mixed ? (float *)take(4 * l32) : nullptr;
  d.P32 = b.mixed ? (float *)take(4 * nn) : nullptr;
  d.w32 = b.mixed ? (float *)take(4 * (size_t)L.w_len) : nullptr;
  d.w_len = (size_t)L.w_len;
  d.corr_scratch = (double *)take(8 * corrections_scratch(n));
  // the uploaded tables, contiguous: xyz | sad | z | aoff | ao_atom | csr_start | csr | near | mask
  const size_t up0 = off;
  double *xyz = (double *)take(8 * 3 * (size_t)n);
  double *sad = (double *)take(8 * (size_t)nao);
  int *z = (int *)take(4 * (size_t)n);
  int *aoff = (int *)take(4 * (size_t)n);
  int *ao_atom = (int *)take(4 * (size_t)nao);
  int *csr_start = (int *)take(4 * ((size_t)n + 1));
  int2 *csr = (int2 *)take(8 * L.csr.size());
  NearPair *np = (NearPair *)take(sizeof(NearPair) * L.near.size());
  unsigned char *mask = (unsigned char *)take((size_t)n * n);
  (void)up0;
  d.g.n_atoms = n;
  d.g.nao = nao;
  d.g.n_near = (int)L.near.size();
  d.g.z = z;
  d.g.aoff = aoff;
  d.g.ao_atom = ao_atom;
  d.g.xyz = xyz;
  d.g.near_mask = mask;
  d.g.np = np;
  d.g.csr_start = csr_start;
  d.g.csr = csr;
  d.g.w = d.w;
  d.g.gfar = nullptr;  // the batched Fock kernels evaluate EV / r themselves
  d.g.csr_eoff = nullptr;
  d.n_occ = b.n_occ;
  d.dframe = b.dframe;
  d.cc_nx = gx;
  d.cc_terms = d.X;  // n (n - 1) / 2 <= nao^2 doubles, free until the first SCF step
  d.want_matrices = b.o.want_matrices;
  d.smooth_dispersion = b.o.smooth_dispersion;
  (void)sad;
  return off;
}

// Offset of the uploaded-table segment and its bytes.
static void upload_span(BatchMol &b, size_t &start, size_t &bytes) {
  const char *base = b.base;
  start = (size_t)((const char *)b.d.g.xyz - base);
  bytes = b.bytes - start;
}

static std::vector<char> upload_image(const BatchMol &b) {
  const Layout &L = b.L;
  const int n = b.m.n, nao = L.nao;
  const char *base = (const char *)b.d.g.xyz;
  std::vector<char> img((size_t)(b.base + b.bytes - base), 0);
  auto at = [&](const void *dev) { return img.data() + ((const char *)dev - base); };
  std::memcpy(at(b.d.g.xyz), b.m.xyz.data(), 8 * 3 * (size_t)n);
  const std::vector<double> sad = sad_diag(b.m, L, *b.ps, 2.0 * b.n_occ);
  const char *sad_dev = (const char *)b.d.g.xyz + align256(8 * 3 * (size_t)n);
  std::memcpy(at(sad_dev), sad.data(), 8 * (size_t)nao);
  std::memcpy(at(b.d.g.z), b.m.z.data(), 4 * (size_t)n);
  std::memcpy(at(b.d.g.aoff), L.aoff.data(), 4 * (size_t)n);
  std::memcpy(at(b.d.g.ao_atom), L.ao_atom.data(), 4 * (size_t)nao);
  std::memcpy(at(b.d.g.csr_start), L.csr_start.data(), 4 * ((size_t)n + 1));
  if (!L.csr.empty()) std::memcpy(at(b.d.g.csr), L.csr.data(), 8 * L.csr.size());
  if (!L.near.empty()) std::memcpy(at(b.d.g.np), L.near.data(), sizeof(NearPair) * L.near.size());
  unsigned char *mask = (unsigned char *)at(b.d.g.near_mask);
  for (const NearPair &q : L.near) {
    mask[(size_t)q.u * n + q.v] = 1;
    mask[(size_t)q.v * n + q.u] = 1;
  }
  return img;
}

static const double *sad_device(const BatchMol &b) {
  return (const double *)((const char *)b.d.g.xyz + align256(8 * 3 * (size_t)b.m.n));
}

// The batched SCF engine of one device and one PM7 method.
class BatchRunner {
 public:
  BatchRunner(int device, int method)
      : ctx_(context_for(device)), method_(method), ps_(param_set(method)) {
    CUDA_OK(cudaSetDevice(ctx_.device));
    P_ = &device_params(ctx_, method);
    CUDA_OK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    SOLVER_OK(cusolverDnCreate(&solver_));
    SOLVER_OK(cusolverDnSetStream(solver_, st_));
    SOLVER_OK(cusolverDnCreateParams(&sparams_));
    CUDA_OK(cudaMalloc((void **)&err32_, sizeof(int)));
    CUDA_OK(cudaMemset(err32_, 0, sizeof(int)));
    CUDA_OK(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    // kernel attributes of the SP2 steps, before any of them is captured into a graph
    prepare_gemm_kernels();
    prepare_tf32_kernels();
    CUDA_OK(cudaStreamCreateWithFlags(&eig_st_, cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreateWithFlags(&eig_done_, cudaEventDisableTiming));
    for (Side &sd : side_) {
      CUDA_OK(cudaStreamCreateWithFlags(&sd.st, cudaStreamNonBlocking));
      SOLVER_OK(cusolverDnCreate(&sd.solver));
      SOLVER_OK(cusolverDnSetStream(sd.solver, sd.st));
      CUDA_OK(cudaEventCreateWithFlags(&sd.done, cudaEventDisableTiming));
      CUDA_OK(cudaMalloc((void **)&sd.info, sizeof(int)));
    }
    // density of each SCF iteration: SP2 purification from sp2_min_nao_ basis functions up,
    // the eigensolver below; PM7_BATCH_DENSITY=eig|sp2 forces one of them for every molecule
    if (const char *e = std::getenv("PM7_BATCH_DENSITY")) {
      if (std::strcmp(e, "eig") == 0) sp2_min_nao_ = 1 << 30;
      if (std::strcmp(e, "sp2") == 0) sp2_min_nao_ = 0;
    }
  }
  ~BatchRunner() {
    cudaSetDevice(ctx_.device);
    cudaStreamSynchronize(st_);
    cudaStreamSynchronize(eig_st_);
    for (Side &sd : side_)
      if (sd.st) cudaStreamSynchronize(sd.st);
    for (auto &kv : active_) release(*kv);
    for (BatchMol *b : retiring_) release(*b);
    eig_scr_.release(eig_st_);
    cudaStreamSynchronize(eig_st_);
    cudaStreamSynchronize(st_);
    if (rarena_) cudaFree(rarena_);
    if (fold_scr_) cudaFree(fold_scr_);
    if (desc_) cudaFree(desc_);
    if (ctl_) cudaFree(ctl_);
    if (arena_) cudaFree(arena_);
    if (work_) cudaFree(work_);
    if (flags_h_) cudaFreeHost(flags_h_);
    if (flags_d_) cudaFree(flags_d_);
    if (pin_) cudaFreeHost(pin_);
    if (out_d_) cudaFree(out_d_);
    if (maps_) cudaFree(maps_);
    if (err32_) cudaFree(err32_);
    for (Side &sd : side_) {
      if (sd.st) cudaStreamSynchronize(sd.st);
      if (sd.work) cudaFree(sd.work);
      if (sd.info) cudaFree(sd.info);
      if (sd.solver) cusolverDnDestroy(sd.solver);
      if (sd.done) cudaEventDestroy(sd.done);
      if (sd.st) cudaStreamDestroy(sd.st);
    }
    if (fork_) cudaEventDestroy(fork_);
    if (eig_done_) cudaEventDestroy(eig_done_);
    if (eig_st_) cudaStreamDestroy(eig_st_);
    cusolverDnDestroyParams(sparams_);
    cusolverDnDestroy(solver_);
    cudaStreamDestroy(st_);
  }

  // Host-side preparation: validation, layout, electron count (throws Failure).
  std::unique_ptr<BatchMol> prepare(const Molecule &m, const pm7_options &o) {
    auto b = std::make_unique<BatchMol>();
    b->m = m;
    b->o = o;
    validate(m, o);
    if (o.method != method_) throw Failure{PM7_ERR_INVALID_INPUT, "options method does not match parameter method"};
    if (o.precision != PM7_PRECISION_FP64 && o.precision != PM7_PRECISION_MIXED)
      throw Failure{PM7_ERR_INVALID_INPUT, "unknown precision mode"};
    b->ps = &ps_;
    b->L = build_layout(m, ps_);
    double n_elec = 0.0;
    for (int zz : m.z) n_elec += ps_.element(zz)->core;
    n_elec -= o.charge;
    const long long ni = std::llround(n_elec);
    if (std::fabs(n_elec - (double)ni) > 1.0e-6 || ni < 0)
      throw Failure{PM7_ERR_INVALID_INPUT, "invalid electron count " + std::to_string(n_elec)};
    const long long unp = o.multiplicity - 1;
    if (o.multiplicity < 1 || ni - unp < 0 || (ni - unp) % 2 != 0)
      throw Failure{PM7_ERR_INVALID_INPUT, "electron count " + std::to_string(ni) +
                                               " is incompatible with multiplicity " + std::to_string(o.multiplicity)};
    b->n_occ = (int)(ni / 2);
    b->dframe = o.force_dpath || b->L.has_d;
    b->mixed = o.precision == PM7_PRECISION_MIXED && b->L.nao >= sp2_min_nao_;
    b->bytes = mol_layout(*b, nullptr);
    b->np = bucket_size(b->L.nao);
    const size_t nn = (size_t)b->L.nao * b->L.nao;
    if (o.initial_density) b->init_density.assign(o.initial_density, o.initial_density + nn);
    if (o.initial_spin_density) b->init_spin.assign(o.initial_spin_density, o.initial_spin_density + nn);
    b->o.initial_density = nullptr;
    b->o.initial_spin_density = nullptr;
    return b;
  }

  // Whether a prepared request runs in the batch (closed-shell RHF), else on the
  // single-molecule path.
  static bool batchable(const BatchMol &b) {
    const long long unp = b.o.multiplicity - 1;
    if (b.o.reference == PM7_REF_UNRESTRICTED || unp != 0) return false;
    return b.m.n >= 1;
  }

  size_t bytes_in_use() const { return bytes_in_use_; }
  long long sp2_fallbacks() const { return sp2_fallbacks_; }
  // Host wall time of each phase of iterate() so far (seconds), for PM7_BATCH_TRACE.
  static constexpr int kPhases = 8;
  static const char *phase_name(int k) {
    static const char *names[kPhases] = {"queue", "mixed_sync", "sp2", "eigensolve", "converge", "retire_end",
                                         "retire", "admit"};
    return names[k];
  }
  double phase_seconds(int k) const { return phase_s_[k]; }
  int active_count() const { return (int)active_.size(); }

  // Allocate, upload and build the integrals of the given molecules (one launch per
  // build phase for all of them); they join the next iteration.
  void admit(std::vector<BatchMol *> &in) {
    if (in.empty()) return;
    const auto t_admit0 = std::chrono::steady_clock::now();
    struct AdmitClock {  // host wall of admissions, for PM7_BATCH_TRACE
      double &acc;
      std::chrono::steady_clock::time_point t0;
      ~AdmitClock() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
    } admit_clock{phase_s_[kPhases - 1], t_admit0};
    CUDA_OK(cudaSetDevice(ctx_.device));
    const int n = (int)in.size();
    for (BatchMol *b : in) {
      b->slot = take_slot();
      CUDA_OK(cudaMallocAsync((void **)&b->base, b->bytes, st_));
      mol_layout(*b, b->base);
      bytes_in_use_ += b->bytes;
    }
    // one pinned staging area for the wave: table images, descriptors, control records
    std::vector<size_t> img_off(n + 1, 0);
    for (int i = 0; i < n; ++i) {
      size_t start, bytes;
      upload_span(*in[i], start, bytes);
      img_off[i + 1] = img_off[i] + align256(bytes);
    }
    const size_t desc_off = img_off[n], ctl_off = desc_off + align256(sizeof(MolDesc) * n);
    const size_t total = ctl_off + align256(sizeof(MolCtl) * n);
    char *host = pinned_stage(total);
    parallel_for(n, [&](int i) {
      BatchMol *b = in[i];
      std::vector<char> img = upload_image(*b);
      std::memcpy(host + img_off[i], img.data(), img.size());
      std::memcpy(host + desc_off + sizeof(MolDesc) * i, &b->d, sizeof(MolDesc));
      MolCtl c;
      std::memset(&c, 0, sizeof c);
      c.max_scf = b->o.max_scf;
      c.accel = (b->o.use_diis && b->o.accelerator != PM7_ACCEL_NONE) ? (b->o.accelerator == PM7_ACCEL_CDIIS ? 2 : 1) : 0;
      c.e_tol = b->o.e_tol;
      c.p_tol = b->o.p_tol;
      c.adiis_switch = b->o.adiis_switch;
      c.shift_floor = b->o.level_shift;
      c.shift = b->o.level_shift;
      c.mixed = b->mixed ? 1 : 0;
      std::memcpy(host + ctl_off + sizeof(MolCtl) * i, &c, sizeof(MolCtl));
    });
    for (int i = 0; i < n; ++i) {
      BatchMol *b = in[i];
      if (!b->mixed) continue;
      // tensor maps of the split fp32 iterate, read by the grouped tcgen05 squaring
      alignas(64) unsigned char maps[256];
      if (!make_square_map(b->d.hi32, b->d.ld32, maps) || !make_square_map(b->d.lo32, b->d.ld32, maps + 128))
        throw Failure{PM7_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
      std::memcpy(map_stage_.data() + 256 * (size_t)b->slot, maps, 256);
      CUDA_OK(cudaMemcpyAsync(maps_ + 256 * (size_t)b->slot, map_stage_.data() + 256 * (size_t)b->slot, 256,
                              cudaMemcpyHostToDevice, st_));
    }
    for (int i = 0; i < n; ++i) {
      BatchMol *b = in[i];
      size_t start, bytes;
      upload_span(*b, start, bytes);
      CUDA_OK(cudaMemcpyAsync(b->base + start, host + img_off[i], bytes, cudaMemcpyHostToDevice, st_));
      CUDA_OK(cudaMemcpyAsync(desc_ + b->slot, host + desc_off + sizeof(MolDesc) * i, sizeof(MolDesc),
                              cudaMemcpyHostToDevice, st_));
      CUDA_OK(cudaMemcpyAsync(ctl_ + b->slot, host + ctl_off + sizeof(MolCtl) * i, sizeof(MolCtl),
                              cudaMemcpyHostToDevice, st_));
      if (!b->init_density.empty())
        CUDA_OK(cudaMemcpyAsync(b->d.Pn, b->init_density.data(), 8 * b->init_density.size(), cudaMemcpyHostToDevice,
                                st_));
    }
    // build phase, batched over the newcomers
    Lists A = lists(in, false);
    std::vector<const double *> sad(in.size());
    for (size_t i = 0; i < in.size(); ++i) sad[i] = in[i]->init_density.empty() ? sad_device(*in[i]) : nullptr;
    const double **dsad = upload_ptrs(sad);
    {
      Stage s_(st_, "batch_build");
      k_b_init<<<A.mol.n, RB, 0, st_>>>(A.mol, desc_, ctl_, dsad);
      note_launch();
      if (A.sp_pairs.total) launch_b_pairs_all(st_, A.sp_pairs, desc_, *P_);
      if (A.d_pairs.total) launch_b_pairs_all_d(st_, A.d_pairs, desc_, *P_);
      if (A.sp_near.total) launch_b_near_integrals(st_, A.sp_near, desc_, *P_);
      if (A.d_near.total) launch_b_near_integrals_d(st_, A.d_near, desc_, *P_);
      launch_b_hcore_diag(st_, A.atoms, desc_, *P_);
      // core-core energies: the pair-order fold of each molecule (repulsion.rs:16-36)
      std::vector<SeqSumJob> jobs;
      for (BatchMol *b : in) {
        const size_t np = (size_t)b->m.n * (b->m.n > 0 ? b->m.n - 1 : 0) / 2;
        jobs.push_back({b->d.cc_terms, nullptr, np, &ctl_[b->slot].core_core});
      }
      queue_folds(jobs, fold_build_up_);
    }
    CUDA_OK(cudaStreamSynchronize(st_));
    CUDA_OK(cudaGetLastError());
    for (BatchMol *b : in) active_.push_back(b);
  }

  // One SCF iteration of every active molecule. Returns the molecules that finished
  // (their results filled, device memory released).
  std::vector<BatchMol *> iterate() {
    std::vector<BatchMol *> finished;
    CUDA_OK(cudaSetDevice(ctx_.device));
    auto t_last = std::chrono::steady_clock::now();
    auto mark = [&](int k) {
      const auto now = std::chrono::steady_clock::now();
      phase_s_[k] += std::chrono::duration<double>(now - t_last).count();
      t_last = now;
    };
    if (active_.empty()) return retiring_.empty() ? finished : retire_end();
    Lists A = lists(active_, false);
    const int n = A.mol.n;
    const int nb = (n + 127) / 128;
    {
      Stage s_(st_, "batch_fock");
      k_b_push<<<nb, 128, 0, st_>>>(n, A.mol.slot, ctl_);
      note_launch();
      launch_b_fock(st_, A.mol, A.rows, A.near, A.atoms, desc_, ctl_, *P_, 0);
      k_b_energy_c<<<A.chunks.total, RB, 0, st_>>>(A.chunks, desc_, ctl_, 0);
      note_launch();
    }
    {
      Stage s_(st_, "batch_commutator");
      launch_b_gemm(st_, A.gfull, desc_, ctl_, nullptr, 0);
      k_b_antisym_c<<<A.chunks.total, RB, 0, st_>>>(A.chunks, desc_, ctl_);
      note_launch();
    }
    {
      Stage s_(st_, "batch_diis");
      k_b_dots_c<<<A.chunks.total, RB, 0, st_>>>(A.chunks, desc_, ctl_);
      k_b_reduce<<<nb, 128, 0, st_>>>(n, A.mol.slot, desc_, ctl_);
      k_b_control<<<(n + 63) / 64, 64, 0, st_>>>(n, A.mol.slot, ctl_, flags_d_ + 2 * (size_t)cap_);
      note_launch(3);
    }
    // which molecules take an fp32 cycle (decided on the device from their DIIS error)
    bool any_mixed = false;
    for (const BatchMol *b : active_) any_mixed = any_mixed || b->mixed;
    mark(0);
    if (any_mixed) {
      CUDA_OK(cudaMemcpyAsync(flags_h_ + 2 * (size_t)cap_, flags_d_ + 2 * (size_t)cap_, n, cudaMemcpyDeviceToHost,
                              st_));
      CUDA_OK(cudaStreamSynchronize(st_));
    }
    mark(1);
    // density: SP2 purification on the tensor cores for the larger molecules (fp32 cycles
    // on tcgen05, fp64 cycles on DMMA), the batched eigensolver for the small ones (where
    // it is as fast) and for what SP2 leaves
    std::vector<BatchMol *> fallback, purify64, purify32;
    for (int m = 0; m < n; ++m) {
      BatchMol *b = active_[m];
      if (b->L.nao < sp2_min_nao_) fallback.push_back(b);
      else if (any_mixed && flags_h_[2 * (size_t)cap_ + m]) purify32.push_back(b);
      else purify64.push_back(b);
    }
    if (!purify64.empty() || !purify32.empty()) {
      Stage s_(st_, "batch_sp2");
      Lists S = lists(purify64, false, &up_sp2_);
      Lists T = lists(purify32, false, &up_sp32_);
      unsigned char *f64 = flags_d_, *f32 = flags_d_ + cap_;
      for (const Lists *L : {&S, &T}) {
        if (L->mol.n == 0) continue;
        k_b_sp2_fuse<<<L->rows.total, RB, 0, st_>>>(L->rows, desc_, ctl_);
        k_b_sp2_bounds<<<(L->mol.n + 127) / 128, 128, 0, st_>>>(L->mol.n, L->mol.slot, desc_, ctl_);
        launch_b_lanczos(*L, L == &S ? purify64 : purify32);
        k_b_sp2_x0<<<L->chunks.total, RB, 0, st_>>>(L->chunks, desc_, ctl_);
        note_launch(3);
      }
      if (T.mol.n) launch_b_to32(st_, T.chunks, desc_);
      const int chunk = 8;
      bool run64 = S.mol.n > 0, run32 = T.mol.n > 0;
      // A chunk is `chunk` purification steps of every molecule still purifying (steps of a
      // molecule that has stopped do nothing on the device), the same launches each time
      // within this iteration: captured once as a CUDA graph and replayed (the kernels'
      // attributes were set in the constructor, outside any capture).
      auto queue_chunk = [&](bool r64, bool r32) {
        for (int k = 0; k < chunk; ++k) {
          if (r64) {  // the fused step: decision, then the squaring that applies it
            k_b_sp2_decide64<<<S.mol.n, RB, 0, st_>>>(S.mol, desc_, ctl_, f64);
            note_launch();
            launch_b_gemm(st_, S.glow, desc_, ctl_, nullptr, 3);
          }
          if (r32) {
            launch_b_square_tf32x3(st_, T.tiles, desc_, ctl_, maps_, err32_);
            launch_b_sp2_decide32(st_, T.mol, desc_, ctl_, f32);
            launch_b_sp2_apply32(st_, T.chunks, desc_, ctl_);
          }
        }
      };
      cudaGraphExec_t exec = nullptr;
      bool g64 = false, g32 = false;
      int nodes = 0;
      for (int step = 0; step < 100 && (run64 || run32); step += chunk) {
        {
          if (!exec || g64 != run64 || g32 != run32) {
            if (exec) CUDA_OK(cudaGraphExecDestroy(exec));
            exec = nullptr;
            const long long before = pm7_launch_count();
            cudaGraph_t graph = nullptr;
            CUDA_OK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
            queue_chunk(run64, run32);
            CUDA_OK(cudaStreamEndCapture(st_, &graph));
            nodes = (int)(pm7_launch_count() - before);
            note_launch(-nodes);  // counted when replayed
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            CUDA_OK(ie);
            g64 = run64;
            g32 = run32;
          }
          CUDA_OK(cudaGraphLaunch(exec, st_));
          note_launch(nodes);
        }
        CUDA_OK(cudaMemcpyAsync(flags_h_, flags_d_, 2 * (size_t)cap_, cudaMemcpyDeviceToHost, st_));
        CUDA_OK(cudaStreamSynchronize(st_));
        run64 = false;
        for (int m = 0; m < S.mol.n; ++m) run64 = run64 || flags_h_[m] == 0;
        run32 = false;
        for (int m = 0; m < T.mol.n; ++m) run32 = run32 || flags_h_[cap_ + m] == 0;
      }
      if (exec) CUDA_OK(cudaGraphExecDestroy(exec));
      if (S.mol.n) {
        k_b_sp2_final64<<<S.chunks.total, RB, 0, st_>>>(S.chunks, desc_, ctl_);
        note_launch();
      }
      for (int m = 0; m < S.mol.n; ++m)
        if (flags_h_[m] != 1) {
          fallback.push_back(purify64[m]);
          ++sp2_fallbacks_;
        }
      for (int m = 0; m < T.mol.n; ++m)
        if (flags_h_[cap_ + m] != 1) {
          fallback.push_back(purify32[m]);
          ++sp2_fallbacks_;
        }
      if (T.mol.n) {
        int bad = 0;
        CUDA_OK(cudaMemcpyAsync(&bad, err32_, sizeof(int), cudaMemcpyDeviceToHost, st_));
        CUDA_OK(cudaStreamSynchronize(st_));
        if (bad) throw Failure{PM7_ERR_TIMEOUT, "tcgen05 squaring: a pipeline wait expired"};
      }
    }
    mark(2);
    if (!fallback.empty()) {
      Stage s_(st_, "batch_eigensolve");
      Lists B = lists(fallback, true, &up_fallback_);
      k_b_to_bucket<<<dim3(B.mol.n, kBucketBlocks), RB, 0, st_>>>(B.mol, desc_, ctl_, B.eig, 0);
      note_launch();
      eigensolve(B);
      launch_b_gemm(st_, B.glow, desc_, ctl_, B.eig, 1);
    }
    mark(3);
    {
      Stage s_(st_, "batch_converge");
      k_b_sqdiff_c<<<A.chunks.total, RB, 0, st_>>>(A.chunks, desc_);
      k_b_converge<<<nb, 128, 0, st_>>>(n, A.mol.slot, desc_, ctl_, flags_d_);
      note_launch(2);
    }
    CUDA_OK(cudaMemcpyAsync(flags_h_, flags_d_, n, cudaMemcpyDeviceToHost, st_));
    CUDA_OK(cudaStreamSynchronize(st_));
    CUDA_OK(cudaGetLastError());
    std::vector<BatchMol *> keep;
    for (int m = 0; m < n; ++m) (flags_h_[m] ? finished : keep).push_back(active_[m]);
    active_.swap(keep);
    // the previous iteration's retirement (its eigensolves ran alongside this step)
    mark(4);
    std::vector<BatchMol *> done;
    if (!retiring_.empty()) done = retire_end();
    mark(5);
    if (!finished.empty()) {
      bool vectors = false;
      for (const BatchMol *b : finished) vectors = vectors || b->o.want_matrices;
      if (vectors) {
        retire(finished);
        done.insert(done.end(), finished.begin(), finished.end());
      } else {
        retire_begin(finished);
      }
    }
    mark(6);
    return done;
  }

  // Molecules whose retirement eigensolves are still running.
  int retiring_count() const { return (int)retiring_.size(); }
  bool busy() const { return !active_.empty() || !retiring_.empty(); }

 private:
  struct Lists {
    BatchList mol, rows, chunks, near, atoms, gfull, glow, tiles, sp_pairs, d_pairs, sp_near, d_near, pairs;
    const EigSlot *eig = nullptr;
    std::vector<EigSlot> eig_h;
    std::map<int, std::vector<int>> buckets;  // np -> list positions
    int max_atoms = 0;
  };

  // A pinned host buffer of at least `bytes` (reused; the caller syncs before reuse).
  char *pinned_stage(size_t bytes) {
    if (bytes > pin_cap_) {
      if (pin_) CUDA_OK(cudaFreeHost(pin_));
      pin_cap_ = bytes + bytes / 4 + 4096;
      CUDA_OK(cudaMallocHost((void **)&pin_, pin_cap_));
    }
    return pin_;
  }

  int take_slot() {
    if (free_slots_.empty()) grow(std::max(cap_ * 2, 256));
    const int s = free_slots_.back();
    free_slots_.pop_back();
    return s;
  }

  void grow(int cap) {
    const int old_cap = cap_;
    MolDesc *nd = nullptr;
    MolCtl *nc = nullptr;
    CUDA_OK(cudaMalloc(&nd, sizeof(MolDesc) * cap));
    CUDA_OK(cudaMalloc(&nc, sizeof(MolCtl) * cap));
    if (desc_) {
      CUDA_OK(cudaMemcpyAsync(nd, desc_, sizeof(MolDesc) * cap_, cudaMemcpyDeviceToDevice, st_));
      CUDA_OK(cudaMemcpyAsync(nc, ctl_, sizeof(MolCtl) * cap_, cudaMemcpyDeviceToDevice, st_));
      CUDA_OK(cudaStreamSynchronize(st_));
      CUDA_OK(cudaFree(desc_));
      CUDA_OK(cudaFree(ctl_));
    }
    for (int s = cap - 1; s >= cap_; --s) free_slots_.push_back(s);
    desc_ = nd;
    ctl_ = nc;
    cap_ = cap;
    if (flags_h_) CUDA_OK(cudaFreeHost(flags_h_));
    if (flags_d_) CUDA_OK(cudaFree(flags_d_));
    CUDA_OK(cudaMallocHost((void **)&flags_h_, 3 * (size_t)cap));
    CUDA_OK(cudaMalloc((void **)&flags_d_, 3 * (size_t)cap));
    unsigned char *nm = nullptr;
    CUDA_OK(cudaMalloc((void **)&nm, 256 * (size_t)cap));
    if (maps_) {
      CUDA_OK(cudaMemcpy(nm, maps_, 256 * (size_t)old_cap, cudaMemcpyDeviceToDevice));
      CUDA_OK(cudaFree(maps_));
    }
    maps_ = nm;
    map_stage_.resize(256 * (size_t)cap);
  }

  // Reference-order sums (launch_seqsum_table) of `jobs` on the main stream; the job table
  // and its chunk offsets go up through `up` (one set in flight per upload buffer).
  // <P, H> and <P, F> of every molecule of the list into its MolCtl::e_fold; the job table is
  // filled on the device (the density pointer lives there).
  void queue_energy_folds(const Lists &A, const std::vector<BatchMol *> &mols, ListUpload &up, int final_pass) {
    const int n = A.mol.n;
    std::vector<SeqSumJob> jobs;
    for (const BatchMol *b : mols) {
      const size_t nn = (size_t)b->L.nao * b->L.nao;
      jobs.push_back({nullptr, nullptr, nn, nullptr});
      jobs.push_back({nullptr, nullptr, nn, nullptr});
    }
    queue_folds(jobs, up, [&](SeqSumJob *dev_jobs) {
      k_b_fold_jobs<<<(n + 127) / 128, 128, 0, st_>>>(n, A.mol.slot, desc_, ctl_, dev_jobs, final_pass);
      note_launch();
    });
  }

  // `fill`, when given, writes the device job table itself (after the upload, before the sums).
  void queue_folds(const std::vector<SeqSumJob> &jobs, ListUpload &up,
                   const std::function<void(SeqSumJob *)> &fill = nullptr) {
    if (jobs.empty()) return;
    const int count = (int)jobs.size();
    up.begin();
    size_t off_jobs, off_first;
    SeqSumJob *hj = (SeqSumJob *)up.add(sizeof(SeqSumJob) * count, off_jobs);
    std::memcpy(hj, jobs.data(), sizeof(SeqSumJob) * count);
    long long *hf = (long long *)up.add(sizeof(long long) * (count + 1), off_first);
    long long total = 0;
    for (int j = 0; j < count; ++j) {
      hf[j] = total;
      total += (long long)seqsum_chunks(jobs[j].n);
    }
    hf[count] = total;
    char *dev = up.commit(st_);
    if (fill) fill((SeqSumJob *)(dev + off_jobs));
    const size_t need = seqsum_table_scratch_bytes(total);
    if (need > fold_cap_) {
      if (fold_scr_) CUDA_OK(cudaFreeAsync(fold_scr_, st_));
      fold_cap_ = need + need / 4;
      CUDA_OK(cudaMallocAsync(&fold_scr_, fold_cap_, st_));
    }
    launch_seqsum_table(st_, (const SeqSumJob *)(dev + off_jobs), (const long long *)(dev + off_first), count,
                        total, fold_scr_);
  }

  void release(BatchMol &b) {
    if (b.base) cudaFreeAsync(b.base, st_);
    b.base = nullptr;
    bytes_in_use_ -= b.bytes;
    if (b.slot >= 0) free_slots_.push_back(b.slot);
    b.slot = -1;
  }

  const double **upload_ptrs(const std::vector<const double *> &v) {
    ptr_up_.begin();
    size_t off;
    void *h = ptr_up_.add(sizeof(double *) * std::max<size_t>(v.size(), 1), off);
    std::memcpy(h, v.data(), sizeof(double *) * v.size());
    return (const double **)(ptr_up_.commit(st_) + off);
  }

  // Work lists of one launch sequence over `mols` (list position = index in mols).
  // Each ListUpload backs at most one list set in flight: the host writes its pinned
  // buffer immediately, so a second set on the same buffer before a stream sync would
  // overwrite what queued copies have not yet read.
  Lists lists(const std::vector<BatchMol *> &mols, bool with_eig, ListUpload *upl = nullptr,
              bool retire_arena = false) {
    ListUpload &up_ = upl ? *upl : this->up_;
    double *&arena = retire_arena ? rarena_ : arena_;  // bucket matrices
    size_t &arena_cap = retire_arena ? rarena_cap_ : arena_cap_;
    Lists A;
    const int n = (int)mols.size();
    up_.begin();
    struct Spec {
      BatchList *L;
      std::function<int(const BatchMol &)> count;
      std::function<bool(const BatchMol &)> member;
    };
    auto all = [](const BatchMol &) { return true; };
    std::vector<Spec> specs = {
        {&A.mol, [](const BatchMol &) { return 1; }, all},
        {&A.rows, [](const BatchMol &b) { return items_rows8(b.L.nao); }, all},
        {&A.chunks, [](const BatchMol &b) { return items_chunks(b.L.nao); }, all},
        {&A.near, [](const BatchMol &b) { return items_near_chunks((int)b.L.near.size()); }, all},
        {&A.atoms, [](const BatchMol &b) { return b.m.n; }, all},
        {&A.gfull, [](const BatchMol &b) { return items_gemm_full(b.L.nao); }, all},
        {&A.glow, [](const BatchMol &b) { return items_gemm_lower(b.L.nao); }, all},
        {&A.tiles, [](const BatchMol &b) { return items_tiles128(b.L.nao); }, all},
        {&A.pairs, [](const BatchMol &b) { return items_pairs_all(b.m.n); }, all},
        {&A.sp_pairs, [](const BatchMol &b) { return items_pairs_all(b.m.n); },
         [](const BatchMol &b) { return !b.dframe; }},
        {&A.d_pairs, [](const BatchMol &b) { return items_pairs_all(b.m.n); }, [](const BatchMol &b) { return b.dframe; }},
        {&A.sp_near, [](const BatchMol &b) { return items_near_chunks((int)b.L.near.size()); },
         [](const BatchMol &b) { return !b.dframe; }},
        {&A.d_near, [](const BatchMol &b) { return items_near_d((int)b.L.near.size()); },
         [](const BatchMol &b) { return b.dframe; }},
    };
    std::vector<std::pair<size_t, size_t>> offs;  // (slot offset, prefix offset) per spec
    std::vector<int> sizes;
    for (Spec &sp : specs) {
      std::vector<int> slots, prefix(1, 0);
      for (int m = 0; m < n; ++m) {
        const BatchMol &b = *mols[m];
        if (!sp.member(b)) continue;
        slots.push_back(b.slot);
        prefix.push_back(prefix.back() + sp.count(b));
      }
      size_t so, po;
      void *hs = up_.add(4 * std::max<size_t>(slots.size(), 1), so);
      std::memcpy(hs, slots.data(), 4 * slots.size());
      void *hp = up_.add(4 * prefix.size(), po);
      std::memcpy(hp, prefix.data(), 4 * prefix.size());
      offs.push_back({so, po});
      sp.L->n = (int)slots.size();
      sp.L->total = prefix.back();
    }
    size_t eo = 0;
    if (with_eig) {
      for (int m = 0; m < n; ++m) A.buckets[mols[m]->np].push_back(m);
      size_t total = 0;
      for (auto &kv : A.buckets) total += kv.second.size() * ((size_t)kv.first * kv.first + kv.first);
      if (total > arena_cap) {
        if (arena) CUDA_OK(cudaFreeAsync(arena, st_));
        arena_cap = total + total / 4;
        CUDA_OK(cudaMallocAsync((void **)&arena, 8 * arena_cap, st_));
      }
      A.eig_h.resize(n);
      double *p = arena;
      for (auto &kv : A.buckets) {
        const int np = kv.first, cnt = (int)kv.second.size();
        double *in = p, *w = p + (size_t)cnt * np * np;
        for (int i = 0; i < cnt; ++i) {
          EigSlot &e = A.eig_h[kv.second[i]];
          e.in = in + (size_t)i * np * np;
          e.eps = w + (size_t)i * np;
          e.ldv = np;
          e.pad_ = 0;
        }
        p += (size_t)cnt * ((size_t)np * np + np);
      }
      void *he = up_.add(sizeof(EigSlot) * std::max(n, 1), eo);
      std::memcpy(he, A.eig_h.data(), sizeof(EigSlot) * n);
    }
    char *dev = up_.commit(st_);
    for (size_t k = 0; k < specs.size(); ++k) {
      specs[k].L->slot = (const int *)(dev + offs[k].first);
      specs[k].L->prefix = (const int *)(dev + offs[k].second);
    }
    if (with_eig) A.eig = (const EigSlot *)(dev + eo);
    for (const BatchMol *b : mols) A.max_atoms = std::max(A.max_atoms, b->m.n);
    return A;
  }

  // Eigendecomposition of every bucket matrix (eigenvalues ascending; with `vectors`,
  // eigenvector k in row k, in place): one batched call per bucket size, or one
  // divide-and-conquer call per matrix for the large sizes.
  // Eigensolves of the bucket matrices with order >= min_np. Orders from 512 go to the
  // side streams; when min_np > 0 the caller joins them (join_side) after queuing its own
  // work on the main stream.
  void eigensolve(const Lists &A, bool vectors = true, int min_np = 0) {
    for (auto &kv : A.buckets) {
      if (kv.first < min_np) continue;
      // the batched routine is faster with vectors than without at these sizes; the
      // divide-and-conquer one saves its back-transformation when only values are needed
      const cusolverEigMode_t jobz =
          (vectors || kv.first < 512) ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
      const int np = kv.first, cnt = (int)kv.second.size();
      double *in = A.eig_h[kv.second[0]].in, *w = A.eig_h[kv.second[0]].eps;
      if ((size_t)cnt > info_cap_) {
        if (info_) CUDA_OK(cudaFreeAsync(info_, st_));
        info_cap_ = cnt * 2;
        CUDA_OK(cudaMallocAsync((void **)&info_, sizeof(int) * info_cap_, st_));
      }
      if (np >= 512) {
        // divide and conquer per matrix, spread over the side streams so that several run
        // at once (one alone leaves most of the GPU idle)
        int lwork = 0;
        SOLVER_OK(cusolverDnDsyevd_bufferSize(solver_, jobz, CUBLAS_FILL_MODE_LOWER, np, in, np, w, &lwork));
        const size_t wd = sizeof(double) * (size_t)lwork;
        CUDA_OK(cudaEventRecord(fork_, st_));
        const int used = std::min(cnt, kSide);
        for (int k = 0; k < used; ++k) {
          Side &sd = side_[k];
          CUDA_OK(cudaStreamWaitEvent(sd.st, fork_, 0));
          if (wd > sd.cap) {
            if (sd.work) CUDA_OK(cudaFreeAsync(sd.work, sd.st));
            sd.cap = wd + wd / 4;
            CUDA_OK(cudaMallocAsync(&sd.work, sd.cap, sd.st));
          }
        }
        for (int i = 0; i < cnt; ++i) {
          const EigSlot &e = A.eig_h[kv.second[i]];
          Side &sd = side_[i % used];
          SOLVER_OK(cusolverDnDsyevd(sd.solver, jobz, CUBLAS_FILL_MODE_LOWER, np, e.in, np, e.eps, (double *)sd.work,
                                     lwork, sd.info));
        }
        side_used_ = std::max(side_used_, used);
        if (min_np == 0) join_side();
        continue;
      }
      size_t wd = 0, wh = 0;
      SOLVER_OK(cusolverDnXsyevBatched_bufferSize(solver_, sparams_, jobz, CUBLAS_FILL_MODE_LOWER, np, CUDA_R_64F, in,
                                                  np, CUDA_R_64F, w, CUDA_R_64F, &wd, &wh, cnt));
      if (wd > work_cap_) {
        if (work_) CUDA_OK(cudaFreeAsync(work_, st_));
        work_cap_ = wd + wd / 4;
        CUDA_OK(cudaMallocAsync(&work_, work_cap_, st_));
      }
      if (wh > host_work_.size()) host_work_.resize(wh);
      SOLVER_OK(cusolverDnXsyevBatched(solver_, sparams_, jobz, CUBLAS_FILL_MODE_LOWER, np, CUDA_R_64F, in, np,
                                       CUDA_R_64F, w, CUDA_R_64F, work_, work_cap_,
                                       host_work_.empty() ? nullptr : host_work_.data(), wh, info_, cnt));
    }
  }

  // Lanczos-narrowed SP2 intervals for the molecules of list set L (vectors in shared memory).
  void launch_b_lanczos(const Lists &L, const std::vector<BatchMol *> &mols) {
    int nmax = 0;
    for (const BatchMol *b : mols) nmax = std::max(nmax, std::min(b->L.nao, kLzMaxOrder));
    if (nmax < 2 * kLzSteps) return;
    const size_t smem = sizeof(double) * (3 * (size_t)nmax + 33);
    if (smem > lz_smem_) {
      CUDA_OK(cudaFuncSetAttribute(k_b_lanczos, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      lz_smem_ = smem;
    }
    k_b_lanczos<<<L.mol.n, 1024, smem, st_>>>(L.mol, desc_, ctl_);
    note_launch();
  }

  // The main stream waits for the side streams' eigensolves.
  void join_side() {
    for (int k = 0; k < side_used_; ++k) {
      CUDA_OK(cudaEventRecord(side_[k].done, side_[k].st));
      CUDA_OK(cudaStreamWaitEvent(st_, side_[k].done, 0));
    }
    side_used_ = 0;
  }

  // Final Fock and energy, corrections, reported orbitals and per-atom outputs of the
  // finished molecules, one packed read-back, the results on the host; then the
  // molecules' device memory is freed.
  void retire(std::vector<BatchMol *> &R) {
    Lists A = lists(R, true);
    const int n = A.mol.n;
    bool vectors = false;
    for (const BatchMol *b : R) vectors = vectors || b->o.want_matrices;
    finish_scf(A, R);
    {
      // reported orbitals: eigenvectors of the last extrapolated Fock, or of the final
      // Fock when a level shift was active (scf.rs:1299-1305)
      Stage s_(st_, "batch_orbitals");
      k_b_to_bucket<<<dim3(n, kBucketBlocks), RB, 0, st_>>>(A.mol, desc_, ctl_, A.eig, 2);
      if (vectors) {
        eigensolve(A, true);
      } else {
        // Energies only. Orders from kLeanEig up: the library's divide and conquer, one
        // matrix per side stream; below: all at once through the cluster tridiagonalisation
        // (the top-left nao x nao block of each bucket matrix) on this stream, meanwhile.
        eigensolve(A, false, kLeanEig);
        std::vector<EigvalsRequest> req;
        for (auto &kv : A.buckets)
          if (kv.first < kLeanEig)
            for (int m : kv.second) req.push_back({A.eig_h[m].in, R[m]->L.nao, A.eig_h[m].ldv, A.eig_h[m].eps});
        eigvals_device(st_, req, eig_scr_);
        join_side();
      }
      k_b_save_orbitals<<<n, RB, 0, st_>>>(A.mol, desc_, A.eig);
      note_launch(2);
    }
    finish_outputs(R, A, vectors);
  }

  // Final Fock and energy, corrections and per-atom outputs (the SCF's last step of the
  // finished molecules), on the main stream.
  void finish_scf(const Lists &A, const std::vector<BatchMol *> &R) {
    const int n = A.mol.n;
    Stage s_(st_, "batch_finish");
    launch_b_fock(st_, A.mol, A.rows, A.near, A.atoms, desc_, ctl_, *P_, 1);
    // the final electronic energy as the reference's two folds (the final Fock is in X)
    queue_energy_folds(A, R, fold_retire_up_, 1);
    k_b_fold_energy<<<(n + 127) / 128, 128, 0, st_>>>(n, A.mol.slot, ctl_);
    note_launch();
    launch_b_corrections(st_, A.mol, A.pairs, desc_, ctl_, method_, A.max_atoms);
    k_b_atom_out<<<n, 128, 0, st_>>>(A.mol, desc_, *P_);
    note_launch();
  }

  // Retirement without returned matrices, first half: the SCF's last step, the reported
  // Fock into the retirement buckets, and the eigenvalue solves queued off the main stream
  // (orders from kLeanEig: dsyevd on the side streams, on the nao x nao block of each
  // bucket; below: the cluster kernel on eig_st_), writing straight into each molecule's
  // eps_out. The next SCF step of the other molecules overlaps them; retire_end finishes.
  void retire_begin(std::vector<BatchMol *> &R) {
    Lists A = lists(R, true, nullptr, true);
    const int n = A.mol.n;
    finish_scf(A, R);
    {
      Stage s_(st_, "batch_orbitals");
      k_b_to_bucket<<<dim3(n, kBucketBlocks), RB, 0, st_>>>(A.mol, desc_, ctl_, A.eig, 2);
      note_launch();
    }
    CUDA_OK(cudaEventRecord(fork_, st_));
    std::vector<EigvalsRequest> small;
    for (auto &kv : A.buckets) {
      const int np = kv.first;
      if (np < kLeanEig) {
        for (int m : kv.second) small.push_back({A.eig_h[m].in, R[m]->L.nao, np, R[m]->d.eps_out});
        continue;
      }
      int lwork = 0;
      SOLVER_OK(cusolverDnDsyevd_bufferSize(solver_, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER, np,
                                            A.eig_h[kv.second[0]].in, np, A.eig_h[kv.second[0]].eps, &lwork));
      const size_t wd = sizeof(double) * (size_t)lwork;
      for (size_t i = 0; i < kv.second.size(); ++i) {
        const int m = kv.second[i];
        Side &sd = side_[rside_ % kSide];
        ++rside_;
        CUDA_OK(cudaStreamWaitEvent(sd.st, fork_, 0));
        if (wd > sd.cap) {
          if (sd.work) CUDA_OK(cudaFreeAsync(sd.work, sd.st));
          sd.cap = wd + wd / 4;
          CUDA_OK(cudaMallocAsync(&sd.work, sd.cap, sd.st));
        }
        SOLVER_OK(cusolverDnDsyevd(sd.solver, CUSOLVER_EIG_MODE_NOVECTOR, CUBLAS_FILL_MODE_LOWER, R[m]->L.nao,
                                   A.eig_h[m].in, np, R[m]->d.eps_out, (double *)sd.work, lwork, sd.info));
      }
    }
    if (!small.empty()) {
      CUDA_OK(cudaStreamWaitEvent(eig_st_, fork_, 0));
      Stage s_(eig_st_, "batch_orbitals_side");
      eigvals_device(eig_st_, small, eig_scr_);
    }
    // the lists' pinned and device buffers are reused by the next step's lists
    CUDA_OK(cudaStreamSynchronize(st_));
    retiring_ = R;
  }

  // Second half: the main stream waits for the eigenvalue solves, then the packed outputs
  // and the results. Returns the retired molecules.
  std::vector<BatchMol *> retire_end() {
    std::vector<BatchMol *> R;
    R.swap(retiring_);
    for (int k = 0; k < kSide; ++k) {
      CUDA_OK(cudaEventRecord(side_[k].done, side_[k].st));
      CUDA_OK(cudaStreamWaitEvent(st_, side_[k].done, 0));
    }
    CUDA_OK(cudaEventRecord(eig_done_, eig_st_));
    CUDA_OK(cudaStreamWaitEvent(st_, eig_done_, 0));
    Lists A = lists(R, false);
    finish_outputs(R, A, false);
    return R;
  }

  // Packed read-back of the retired molecules' outputs, their results on the host, and
  // the release of their device memory.
  void finish_outputs(std::vector<BatchMol *> &R, const Lists &A, bool vectors) {
    const int n = A.mol.n;
    std::vector<long long> off(n + 1, 0);
    for (int m = 0; m < n; ++m)
      off[m + 1] = off[m] + kOutScalars + R[m]->L.nao + (long long)kAtomOut * R[m]->m.n;
    ptr_up_.begin();
    size_t oo;
    void *ho = ptr_up_.add(sizeof(long long) * off.size(), oo);
    std::memcpy(ho, off.data(), sizeof(long long) * off.size());
    const long long *doff = (const long long *)(ptr_up_.commit(st_) + oo);
    const size_t total = (size_t)off[n];
    if (total > out_cap_) {
      if (out_d_) CUDA_OK(cudaFreeAsync(out_d_, st_));
      out_cap_ = total + total / 4;
      CUDA_OK(cudaMallocAsync((void **)&out_d_, 8 * out_cap_, st_));
    }
    k_b_gather_out<<<n, 128, 0, st_>>>(A.mol, desc_, ctl_, doff, out_d_);
    note_launch();
    double *host = (double *)pinned_stage(8 * total);
    CUDA_OK(cudaMemcpyAsync(host, out_d_, 8 * total, cudaMemcpyDeviceToHost, st_));
    CUDA_OK(cudaStreamSynchronize(st_));
    std::vector<std::vector<double>> V(n), Pd(n);
    if (vectors) {
      for (int m = 0; m < n; ++m) {
        BatchMol &b = *R[m];
        const double *o = host + off[m];
        if (!b.o.want_matrices || o[2] == 0.0) continue;
        const size_t nn = (size_t)b.L.nao * b.L.nao;
        V[m].resize(nn);
        Pd[m].resize(nn);
        CUDA_OK(cudaMemcpyAsync(V[m].data(), b.d.V_out, 8 * nn, cudaMemcpyDeviceToHost, st_));
        const double *Pnow = ((int)o[0] % 2 == 0) ? b.d.P : b.d.Pn;  // P and P' swap every iteration
        CUDA_OK(cudaMemcpyAsync(Pd[m].data(), Pnow, 8 * nn, cudaMemcpyDeviceToHost, st_));
      }
      CUDA_OK(cudaStreamSynchronize(st_));
    }
    // nuclear gradients of the converged molecules that asked for one, at their final density,
    // before their device memory goes (closed_form_gradient, src/gradient.rs:500-561)
    for (int m = 0; m < n; ++m) {
      BatchMol &b = *R[m];
      const double *o = host + off[m];
      if (!b.grad_out || o[2] == 0.0) continue;
      GradGeometry g{};
      g.n_atoms = b.d.g.n_atoms;
      g.nao = b.d.g.nao;
      g.n_near = b.d.g.n_near;
      g.z = b.d.g.z;
      g.aoff = b.d.g.aoff;
      g.xyz = b.d.g.xyz;
      g.near_mask = b.d.g.near_mask;
      g.np = b.d.g.np;
      g.Pt = ((int)o[0] % 2 == 0) ? b.d.P : b.d.Pn;  // P and P' swap every iteration
      g.Ps = nullptr;
      try {
        const std::vector<double> gr =
            geometry_gradient(st_, *P_, g, b.dframe, method_, b.o.smooth_dispersion, true,
                              std::find(b.m.z.begin(), b.m.z.end(), 14) != b.m.z.end());
        std::memcpy(b.grad_out, gr.data(), sizeof(double) * gr.size());
      } catch (const Failure &f) {
        b.grad_status = f.code;
        b.grad_error = f.msg;
      }
    }
    parallel_for(n, [&](int m) {
      BatchMol &b = *R[m];
      const double *o = host + off[m];
      const int nao = b.L.nao;
      ResultParts rp;
      rp.iterations = (int)o[0];
      rp.density_error = o[1];
      rp.converged = o[2] != 0.0;
      rp.electronic_ev = o[3];
      rp.core_ev = o[4];
      for (int k = 0; k < 5; ++k) rp.corr[k] = o[5 + k];
      rp.n_occ = b.n_occ;
      rp.fp32_iterations = (int)o[11];
      rp.eps_a.assign(o + kOutScalars, o + kOutScalars + nao);
      const double *ao = o + kOutScalars + nao;
      std::vector<double> pops(b.m.n);
      for (int a = 0; a < b.m.n; ++a) pops[a] = ao[(size_t)kAtomOut * a];
      try {
        fill_result(&b.result, b.m, b.L, *b.ps, b.o, rp, pops, [&](int a, int i, int j) {
          const int k = atom_out_index(i, j);
          return k < 0 ? 0.0 : ao[(size_t)kAtomOut * a + k];
        });
        if (b.o.want_matrices) {
          b.result.density = host_vec(Pd[m]);
          std::vector<double> Cm((size_t)nao * nao);
          for (int i = 0; i < nao; ++i)
            for (int k = 0; k < nao; ++k) Cm[(size_t)i * nao + k] = V[m][(size_t)k * nao + i];
          b.result.mo_coeff = host_vec(Cm);
        }
        b.status = b.grad_status;
        b.error = b.grad_error;
      } catch (const Failure &f) {
        b.status = f.code;
        b.error = f.msg;
      } catch (const std::exception &e) {
        b.status = PM7_ERR_INVALID_INPUT;
        b.error = e.what();
      }
    });
    for (BatchMol *b : R) release(*b);
  }

  DeviceContext &ctx_;
  int method_;
  const ParamSet &ps_;
  const DeviceParams *P_ = nullptr;
  cudaStream_t st_ = nullptr;
  cusolverDnHandle_t solver_ = nullptr;
  cusolverDnParams_t sparams_ = nullptr;
  MolDesc *desc_ = nullptr;
  MolCtl *ctl_ = nullptr;
  int cap_ = 0;
  std::vector<int> free_slots_;
  std::vector<BatchMol *> active_;
  size_t bytes_in_use_ = 0;
  ListUpload up_, up_fallback_, up_sp2_, up_sp32_, ptr_up_, fold_build_up_, fold_retire_up_;
  void *fold_scr_ = nullptr;  // records of the reference-order sums
  size_t fold_cap_ = 0;
  char *pin_ = nullptr;
  size_t pin_cap_ = 0;
  double *out_d_ = nullptr;
  size_t out_cap_ = 0;
  unsigned char *maps_ = nullptr;      // 2 CUtensorMap (128 B each) per slot
  std::vector<unsigned char> map_stage_;
  int *err32_ = nullptr;               // set by the tcgen05 squaring when a wait expired
  // side streams for the large eigendecompositions
  static constexpr int kSide = 4;
  struct Side {
    cudaStream_t st = nullptr;
    cusolverDnHandle_t solver = nullptr;
    cudaEvent_t done = nullptr;
    void *work = nullptr;
    size_t cap = 0;
    int *info = nullptr;
  };
  Side side_[kSide];
  cudaEvent_t fork_ = nullptr;
  double *arena_ = nullptr;
  size_t arena_cap_ = 0;
  EigvalsScratch eig_scr_;  // eigenvalue solves at retirement
  std::vector<BatchMol *> retiring_;  // retirement eigensolves in flight (retire_begin)
  double *rarena_ = nullptr;          // their bucket matrices
  size_t rarena_cap_ = 0;
  cudaStream_t eig_st_ = nullptr;     // the cluster eigenvalue kernel of retirements
  cudaEvent_t eig_done_ = nullptr;
  unsigned rside_ = 0;                // round robin over the side streams
  int side_used_ = 0;       // side streams with queued eigensolves not yet joined
  size_t lz_smem_ = 48 * 1024;  // dynamic shared memory k_b_lanczos is set up for
  // Eigenvalues alone at retirement: the cluster kernel for every order it takes (it runs
  // asynchronously beside the next SCF step; cuSOLVER's dsyevd held the host thread for the
  // whole solve of each large molecule, ~1 s per 600 requests of the served stream).
  static constexpr int kLeanEig = kTriMaxN + 1;
  void *work_ = nullptr;
  size_t work_cap_ = 0;
  std::vector<char> host_work_;
  int *info_ = nullptr;
  size_t info_cap_ = 0;
  unsigned char *flags_h_ = nullptr, *flags_d_ = nullptr;
  int sp2_min_nao_ = 96;  // SP2 from this many basis functions up
  long long sp2_fallbacks_ = 0;
  double phase_s_[kPhases] = {0};
};

// HBM budget for a batch: the caller's max_memory_mb when given, else 80% of free memory.
static size_t batch_budget(int64_t mb) {
  if (mb >= 0) return (size_t)mb << 20;
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return (size_t)8 << 30;
  return fr / 10 * 8;
}

// Runs a closed batch: molecules are admitted as memory allows and iterated together;
// open-shell requests take the single-molecule path.
static void run_batch_impl(int n, const pm7_molecule *mols, const pm7_params *params, const pm7_options *opts,
                           pm7_result *results, pm7_status *status, double *const *gradients = nullptr) {
  if (n < 0 || (n > 0 && (!mols || !opts || !results || !status || !params)))
    throw Failure{PM7_ERR_INVALID_INPUT, "null argument"};
  if (n == 0) return;
  const auto t_start = std::chrono::steady_clock::now();
  const int method = *reinterpret_cast<const int *>(params);
  const int device = opts[0].device;
  BatchRunner runner(device, method);
  std::vector<std::unique_ptr<BatchMol>> items(n);
  std::vector<BatchMol *> pending;
  std::vector<pm7_status> prep(n, PM7_OK);
  // host preparation (validation, layout, pair lists) on all host cores
  parallel_for(n, [&](int i) {
    try {
      items[i] = runner.prepare(to_molecule(&mols[i]), opts[i]);
    } catch (const Failure &f) {
      prep[i] = f.code;
    } catch (const std::exception &) {
      prep[i] = PM7_ERR_INVALID_INPUT;
    }
  });
  for (int i = 0; i < n; ++i) {
    std::memset(&results[i], 0, sizeof(pm7_result));
    status[i] = prep[i];
    if (!items[i]) continue;
    if (!BatchRunner::batchable(*items[i])) {
      status[i] = gradients ? pm7_gradient(&mols[i], params, &opts[i], &results[i], gradients[i], nullptr)
                            : pm7_run(&mols[i], params, &opts[i], &results[i]);
      items[i].reset();
      continue;
    }
    if (gradients) items[i]->grad_out = gradients[i];
    pending.push_back(items[i].get());
  }
  const auto t_prep = std::chrono::steady_clock::now();
  const size_t budget = batch_budget(opts[0].max_memory_mb);
  size_t next = 0;
  double t_admit = 0.0, t_iter = 0.0;
  int n_iter = 0;
  while (next < pending.size() || runner.busy()) {
    std::vector<BatchMol *> admit;
    size_t used = runner.bytes_in_use();
    while (next < pending.size() && (used + pending[next]->bytes <= budget || (runner.active_count() == 0 && admit.empty()))) {
      used += pending[next]->bytes;
      admit.push_back(pending[next++]);
    }
    const auto a0 = std::chrono::steady_clock::now();
    runner.admit(admit);
    const auto a1 = std::chrono::steady_clock::now();
    runner.iterate();
    const auto a2 = std::chrono::steady_clock::now();
    t_admit += std::chrono::duration<double>(a1 - a0).count();
    t_iter += std::chrono::duration<double>(a2 - a1).count();
    ++n_iter;
  }
  if (std::getenv("PM7_BATCH_TRACE")) {
    std::fprintf(stderr, "batch: %d molecules, prepare %.3f s, admit %.3f s, %d iterations %.3f s, sp2 fallbacks %lld\n",
                 n, std::chrono::duration<double>(t_prep - t_start).count(), t_admit, n_iter, t_iter,
                 runner.sp2_fallbacks());
    std::fprintf(stderr, "batch iterations (host wall, s):");
    for (int k = 0; k < BatchRunner::kPhases; ++k)
      std::fprintf(stderr, " %s %.3f", BatchRunner::phase_name(k), runner.phase_seconds(k));
    std::fprintf(stderr, "\n");
  }
  for (int i = 0; i < n; ++i)
    if (items[i]) {
      results[i] = items[i]->result;
      status[i] = items[i]->status;
    }
}

// ===========================================================================
// serving engine: a worker thread runs the batch loop over a request queue
// ===========================================================================
struct EngineRequest {
  uint64_t ticket;
  std::unique_ptr<BatchMol> mol;
  pm7_status status = PM7_OK;
  std::string error;
  pm7_result result{};
  bool done = false;
  std::chrono::steady_clock::time_point t_submit, t_done;
};

}  // namespace pm7

struct pm7_engine {
  int device = 0, method = 0;
  size_t budget = 0;
  int max_active = 0;
  std::unique_ptr<pm7::BatchRunner> runner;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<pm7::EngineRequest *> queue;
  std::deque<pm7::EngineRequest *> single;  // open-shell requests: the pm7_run path, own thread
  std::unordered_map<uint64_t, std::unique_ptr<pm7::EngineRequest>> requests;
  std::unordered_map<pm7::BatchMol *, pm7::EngineRequest *> by_mol;
  uint64_t next_ticket = 1;
  // admission record: requests admitted, most requests resident at once, most bytes resident
  int64_t admitted = 0, peak_active = 0, peak_bytes = 0;
  bool stop = false;
  std::string worker_error;
  std::thread worker, single_worker;
};

namespace pm7 {

// Requests the batch does not take (open shells, forced UHF) run one at a time through
// pm7_run / pm7_gradient on a second worker thread, on the device context's own stream, so
// they proceed beside the batch's SCF steps instead of being refused.
static void engine_single_loop(pm7_engine *E) {
  const pm7_params *params = nullptr;
  const pm7_status ps = pm7_params_load(E->method, &params);
  for (;;) {
    EngineRequest *r = nullptr;
    {
      std::unique_lock<std::mutex> lk(E->mu);
      E->cv.wait(lk, [&] { return E->stop || !E->single.empty(); });
      if (E->single.empty()) break;  // stopping, nothing left
      r = E->single.front();
      E->single.pop_front();
    }
    BatchMol &b = *r->mol;
    std::vector<uint8_t> z(b.m.z.begin(), b.m.z.end());
    const pm7_molecule mol{b.m.n, z.data(), b.m.xyz.data()};
    pm7_options o = b.o;
    o.device = E->device;
    o.initial_density = b.init_density.empty() ? nullptr : b.init_density.data();
    o.initial_spin_density = b.init_spin.empty() ? nullptr : b.init_spin.data();
    pm7_result res{};
    pm7_status st = ps;
    std::string err = ps == PM7_OK ? "" : g_last_error;
    if (ps == PM7_OK) {
      st = b.grad_out ? pm7_gradient(&mol, params, &o, &res, b.grad_out, nullptr) : pm7_run(&mol, params, &o, &res);
      err = st == PM7_OK ? "" : g_last_error;
    }
    std::lock_guard<std::mutex> lk(E->mu);
    r->status = st;
    r->error = err;
    r->result = res;
    r->done = true;
    r->t_done = std::chrono::steady_clock::now();
    E->done_cv.notify_all();
  }
}

static void engine_loop(pm7_engine *E) {
  try {
    CUDA_OK(cudaSetDevice(E->device));
    E->runner = std::make_unique<BatchRunner>(E->device, E->method);
    for (;;) {
      std::vector<BatchMol *> admit;
      {
        std::unique_lock<std::mutex> lk(E->mu);
        E->cv.wait(lk, [&] { return E->stop || !E->queue.empty() || E->runner->busy(); });
        if (E->stop && !E->runner->busy()) break;
        size_t used = E->runner->bytes_in_use();
        int active = E->runner->active_count();
        while (!E->queue.empty()) {
          EngineRequest *r = E->queue.front();
          const bool fits = used + r->mol->bytes <= E->budget && (E->max_active <= 0 || active < E->max_active);
          if (!fits && !(active == 0 && admit.empty())) break;
          E->queue.pop_front();
          used += r->mol->bytes;
          ++active;
          admit.push_back(r->mol.get());
          E->by_mol[r->mol.get()] = r;
        }
        E->admitted += (int64_t)admit.size();
        E->peak_active = std::max<int64_t>(E->peak_active, active);
        E->peak_bytes = std::max<int64_t>(E->peak_bytes, (int64_t)used);
      }
      E->runner->admit(admit);
      std::vector<BatchMol *> fin = E->runner->iterate();
      if (!fin.empty()) {
        std::lock_guard<std::mutex> lk(E->mu);
        const auto now = std::chrono::steady_clock::now();
        for (BatchMol *b : fin) {
          EngineRequest *r = E->by_mol[b];
          E->by_mol.erase(b);
          r->status = b->status;
          r->error = b->error;
          r->result = b->result;
          r->done = true;
          r->t_done = now;
        }
        E->done_cv.notify_all();
      }
    }
  } catch (const Failure &f) {
    std::lock_guard<std::mutex> lk(E->mu);
    E->worker_error = f.msg;
    for (auto &kv : E->requests)
      if (!kv.second->done) {
        kv.second->status = f.code;
        kv.second->error = f.msg;
        kv.second->done = true;
      }
    E->done_cv.notify_all();
  }
}

}  // namespace pm7

using namespace pm7;

extern "C" {

pm7_status pm7_run_batch(int32_t n_molecules, const pm7_molecule *molecules, const pm7_params *params,
                         const pm7_options *options, pm7_result *results, pm7_status *statuses) {
  try {
    run_batch_impl(n_molecules, molecules, params, options, results, statuses);
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

pm7_status pm7_run_batch_gradient(int32_t n_molecules, const pm7_molecule *molecules, const pm7_params *params,
                                  const pm7_options *options, pm7_result *results, pm7_status *statuses,
                                  double *const *gradients) {
  try {
    if (n_molecules > 0 && !gradients) throw Failure{PM7_ERR_INVALID_INPUT, "null gradient array"};
    for (int i = 0; i < n_molecules; ++i)
      if (!gradients[i]) throw Failure{PM7_ERR_INVALID_INPUT, "null gradient buffer for molecule " + std::to_string(i)};
    run_batch_impl(n_molecules, molecules, params, options, results, statuses, gradients);
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

pm7_status pm7_batch_partition(int32_t n_molecules, const pm7_molecule *molecules, int32_t method, int32_t n_ranks,
                               int32_t *rank_of, double *rank_cost) {
  try {
    if (n_molecules < 0 || n_ranks < 1 || (n_molecules > 0 && (!molecules || !rank_of)))
      throw Failure{PM7_ERR_INVALID_INPUT, "pm7_batch_partition: bad counts or null arrays"};
    if (method < 0 || method > 4) throw Failure{PM7_ERR_INVALID_INPUT, "unknown PM7 method"};
    const ParamSet &ps = param_set(method);
    std::vector<double> cost(n_molecules);
    for (int i = 0; i < n_molecules; ++i) {
      const pm7_molecule &m = molecules[i];
      if (m.n_atoms < 0 || (m.n_atoms > 0 && !m.z))
        throw Failure{PM7_ERR_INVALID_INPUT, "pm7_batch_partition: molecule " + std::to_string(i) + " is malformed"};
      double nao = 0;
      for (int a = 0; a < m.n_atoms; ++a) {
        const ElementRec *e = ps.element(m.z[a]);
        nao += e ? e->n_orb : 1;
      }
      const double pairs = 0.5 * (double)m.n_atoms * (double)(m.n_atoms - 1 > 0 ? m.n_atoms - 1 : 0);
      cost[i] = 2.0e5 + nao * nao * nao + 1.0e3 * pairs;
    }
    std::vector<int> order(n_molecules);
    for (int i = 0; i < n_molecules; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<double> load(n_ranks, 0.0);
    for (int i : order) {
      int best = 0;
      for (int r = 1; r < n_ranks; ++r)
        if (load[r] < load[best]) best = r;
      rank_of[i] = best;
      load[best] += cost[i];
    }
    if (rank_cost)
      for (int r = 0; r < n_ranks; ++r) rank_cost[r] = load[r];
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    return f.code;
  }
}

void pm7_engine_config_default(pm7_engine_config *c) {
  if (!c) return;
  c->device = 0;
  c->method = 0;
  c->hbm_budget_mb = -1;
  c->max_active = 0;
}

pm7_status pm7_engine_create(const pm7_engine_config *config, pm7_engine **out) {
  if (!config || !out) return PM7_ERR_INVALID_INPUT;
  try {
    if (config->method < 0 || config->method > 4) throw Failure{PM7_ERR_INVALID_INPUT, "unknown PM7 method"};
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
      throw Failure{PM7_ERR_CUDA, "no CUDA device is available; this engine has no CPU fallback"};
    if (config->device < 0 || config->device >= count) throw Failure{PM7_ERR_CUDA, "invalid CUDA device ordinal"};
    CUDA_OK(cudaSetDevice(config->device));
    auto *E = new pm7_engine();
    E->device = config->device;
    E->method = config->method;
    E->budget = batch_budget(config->hbm_budget_mb);
    E->max_active = config->max_active;
    E->worker = std::thread(engine_loop, E);
    E->single_worker = std::thread(engine_single_loop, E);
    *out = E;
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    return f.code;
  }
}

static pm7_status engine_submit(pm7_engine *E, const pm7_molecule *molecule, const pm7_options *options,
                                double *gradient, uint64_t *ticket) {
  if (!E || !molecule || !options || !ticket) return PM7_ERR_INVALID_INPUT;
  try {
    auto r = std::make_unique<EngineRequest>();
    r->t_submit = std::chrono::steady_clock::now();
    // the runner is created by the worker thread; wait (bounded) until it exists
    for (int spin = 0; spin < 20000; ++spin) {
      {
        std::lock_guard<std::mutex> g(E->mu);
        if (E->runner || !E->worker_error.empty()) break;
      }
      std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    BatchRunner *runner = nullptr;
    {
      std::lock_guard<std::mutex> g(E->mu);
      if (!E->runner) throw Failure{PM7_ERR_CUDA, E->worker_error.empty() ? "engine not ready" : E->worker_error};
      runner = E->runner.get();
    }
    // host preparation (validation, layout, pair lists) outside the engine's lock: it reads
    // only the runner's fixed parameters, and the worker keeps admitting and iterating meanwhile
    EngineRequest *raw = r.get();
    bool batch = false;
    try {
      r->mol = runner->prepare(to_molecule(molecule), *options);
      r->mol->grad_out = gradient;
      batch = BatchRunner::batchable(*r->mol);
    } catch (const Failure &f) {
      raw->status = f.code;
      raw->error = f.msg;
      raw->done = true;
    }
    std::lock_guard<std::mutex> g(E->mu);
    r->ticket = E->next_ticket++;
    *ticket = r->ticket;
    if (!raw->done) (batch ? E->queue : E->single).push_back(raw);
    E->requests[raw->ticket] = std::move(r);
    E->cv.notify_all();
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    return f.code;
  }
}

pm7_status pm7_engine_submit(pm7_engine *E, const pm7_molecule *molecule, const pm7_options *options,
                             uint64_t *ticket) {
  return engine_submit(E, molecule, options, nullptr, ticket);
}

pm7_status pm7_engine_submit_gradient(pm7_engine *E, const pm7_molecule *molecule, const pm7_options *options,
                                      double *gradient, uint64_t *ticket) {
  if (!gradient) {
    g_last_error = "null gradient buffer";
    return PM7_ERR_INVALID_INPUT;
  }
  return engine_submit(E, molecule, options, gradient, ticket);
}

pm7_status pm7_engine_poll(pm7_engine *E, uint64_t ticket, int32_t wait, int32_t *done, pm7_result *result,
                           double *latency_ms) {
  if (!E || !done) return PM7_ERR_INVALID_INPUT;
  std::unique_lock<std::mutex> lk(E->mu);
  auto it = E->requests.find(ticket);
  if (it == E->requests.end()) {
    g_last_error = "unknown ticket";
    return PM7_ERR_INVALID_INPUT;
  }
  EngineRequest *r = it->second.get();
  if (wait) E->done_cv.wait(lk, [&] { return r->done; });
  *done = r->done ? 1 : 0;
  if (!r->done) return PM7_OK;
  const pm7_status s = r->status;
  if (latency_ms)
    *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  if (result) *result = r->result;
  else pm7_result_free(&r->result);
  g_last_error = r->error;
  E->requests.erase(it);
  return s;
}

pm7_status pm7_engine_stats(pm7_engine *E, int64_t out[4]) {
  if (!E || !out) return PM7_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(E->mu);
  out[0] = E->admitted;
  out[1] = E->peak_active;
  out[2] = E->peak_bytes;
  out[3] = (int64_t)E->budget;
  return PM7_OK;
}

pm7_status pm7_engine_destroy(pm7_engine *E) {
  if (!E) return PM7_ERR_INVALID_INPUT;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    E->stop = true;
    E->cv.notify_all();
  }
  if (E->worker.joinable()) E->worker.join();
  if (E->single_worker.joinable()) E->single_worker.join();
  if (std::getenv("PM7_BATCH_TRACE") && E->runner) {
    std::fprintf(stderr, "engine: %lld requests, peak %lld resident; iterations (host wall, s):", (long long)E->admitted,
                 (long long)E->peak_active);
    for (int k = 0; k < pm7::BatchRunner::kPhases; ++k)
      std::fprintf(stderr, " %s %.3f", pm7::BatchRunner::phase_name(k), E->runner->phase_seconds(k));
    std::fprintf(stderr, "\n");
  }
  for (auto &kv : E->requests) pm7_result_free(&kv.second->result);
  E->runner.reset();
  delete E;
  return PM7_OK;
}

}  // extern "C"
