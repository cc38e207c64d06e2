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
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <unordered_map>
#include <functional>

#include "batch.hpp"
#include "common.cuh"
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
}

// Core-core energy of each molecule: its pair-sweep partials in fixed order.
__global__ void __launch_bounds__(RB) k_b_cc_sum(BatchList L, const MolDesc *__restrict__ D, MolCtl *__restrict__ C) {
  const int slot = L.slot[blockIdx.x];
  const MolDesc &d = D[slot];
  const size_t np = (size_t)d.g.n_atoms * d.cc_nx;
  double v[1] = {0.0};
  for (size_t i = threadIdx.x; i < np; i += RB) v[0] += d.cc_partial[i];
  block_sum_n<1>(v);
  if (threadIdx.x == 0) C[slot].core_core = d.g.n_atoms >= 2 ? v[0] : 0.0;
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

// E_el = 1/2 sum P (H + F) (scf.rs:1237); in the SCF loop also D_slot = P.
__global__ void __launch_bounds__(RB) k_b_energy(BatchList L, const MolDesc *__restrict__ D, MolCtl *__restrict__ C,
                                                 int final_pass) {
  const int slot = L.slot[blockIdx.x];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  const size_t nn = mol_nn(d);
  const double *F = final_pass ? d.X : hist_F(d, c.slot);
  double *Dc = final_pass ? nullptr : hist_D(d, c.slot);
  double v[1] = {0.0};
  for (size_t i = threadIdx.x; i < nn; i += RB) {
    const double p = d.P[i];
    v[0] += p * (d.H[i] + F[i]);
    if (Dc) Dc[i] = p;
  }
  block_sum_n<1>(v);
  if (threadIdx.x == 0) {
    if (final_pass) c.e_final = 0.5 * v[0];
    else c.e_elec = 0.5 * v[0];
  }
}

// E_slot = X - X^T with X = F P, and |E|^2 (scf.rs:1148-1156).
__global__ void __launch_bounds__(RB) k_b_antisym(BatchList L, const MolDesc *__restrict__ D, MolCtl *__restrict__ C) {
  const int slot = L.slot[blockIdx.x];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  const int n = d.g.nao;
  const size_t nn = (size_t)n * n;
  double *E = hist_E(d, c.slot);
  double v[1] = {0.0};
  for (size_t i = threadIdx.x; i < nn; i += RB) {
    const size_t r = i / n, col = i - r * n;
    const double e = d.X[i] - d.X[col * n + r];
    E[i] = e;
    v[0] += e * e;
  }
  block_sum_n<1>(v);
  if (threadIdx.x == 0) c.err2 = v[0];
}

// Inner products of the new history entry with the older ones (chronological):
// ee[i] = <E_i, E_new>, ee[k] = <E_new, E_new>; df_row[j] = <D_new, F_j>, df_row[k] =
// <D_new, F_new>; df_col[i] = <D_i, F_new>.
__global__ void __launch_bounds__(RB) k_b_dots(BatchList L, const MolDesc *__restrict__ D, MolCtl *__restrict__ C) {
  const int slot = L.slot[blockIdx.x];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  const size_t nn = mol_nn(d);
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
  for (size_t e = threadIdx.x; e < nn; e += RB) {
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
  if (threadIdx.x == 0) {
    for (int i = 0; i < k; ++i) {
      c.ee[i] = v[i];
      c.df_row[i] = v[kHist + 1 + i];
      c.df_col[i] = v[2 * kHist + 2 + i];
    }
    c.ee[k] = v[kHist];
    c.df_row[k] = v[2 * kHist + 1];
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
__global__ void k_b_control(int n, const int *__restrict__ slots, MolCtl *__restrict__ C) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  MolCtl &c = C[slots[m]];
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

// Extrapolated Fock sum_i c_i F_i + shift (I - P/2) (src = 0), or the final Fock X
// (src = 1), written into the molecule's padded bucket matrix.
__global__ void __launch_bounds__(RB) k_b_to_bucket(BatchList L, const MolDesc *__restrict__ D,
                                                    const MolCtl *__restrict__ C, const EigSlot *__restrict__ E,
                                                    int src) {
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const MolCtl &c = C[slot];
  const int n = d.g.nao, np = E[m].ldv;
  double *out = E[m].in;
  const double *Fs[kHist];
  for (int i = 0; i < kHist; ++i) Fs[i] = hist_F(d, i < c.ncoef ? c.csrc[i] : 0);
  const size_t len = (size_t)np * np;
  for (size_t e = threadIdx.x; e < len; e += RB) {
    const int r = (int)(e / np), col = (int)(e - (size_t)r * np);
    double v;
    if (r < n && col < n) {
      const size_t ij = (size_t)r * n + col;
      if (src == 1) {
        v = d.X[ij];
      } else {
        v = 0.0;
        for (int i = 0; i < c.ncoef; ++i) v += c.coef[i] * Fs[i][ij];
        if (c.shift > 0.0) {
          const double q = d.P[ij] * 0.5;
          v += c.shift * ((r == col) ? 1.0 - q : -q);
        }
      }
    } else {
      v = r == col ? kPad : 0.0;
    }
    out[e] = v;
  }
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

// Density step, convergence test (scf.rs:1274-1287), stall guard, P <- P'; a molecule
// that converged with no level shift keeps this iteration's orbitals.
__global__ void __launch_bounds__(RB) k_b_converge(BatchList L, MolDesc *__restrict__ D, MolCtl *__restrict__ C,
                                                   const EigSlot *__restrict__ E, unsigned char *__restrict__ flags) {
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  const int n = d.g.nao;
  const size_t nn = (size_t)n * n;
  double v[1] = {0.0};
  for (size_t i = threadIdx.x; i < nn; i += RB) {
    const double t = d.Pn[i] - d.P[i];
    v[0] += t * t;
  }
  block_sum_n<1>(v);
  __shared__ int s_save;
  if (threadIdx.x == 0) {
    const double dp = sqrt(v[0] / (double)(nn > 0 ? nn : 1));
    c.dp = dp;
    const double de = fabs(c.e_elec - c.e_old);
    double *t = d.P;
    d.P = d.Pn;
    d.Pn = t;
    c.e_old = c.e_elec;
    const bool residual_ok = c.shift == 0.0 && sqrt(c.err2) < 1.0e-7;
    if (c.iter > 0 && de < c.e_tol && (dp < c.p_tol || residual_ok)) {
      c.converged = 1;
      c.done = 1;
    } else {
      guard_update(c, dp, c.e_elec);
    }
    c.iter += 1;
    if (!c.done && c.iter >= c.max_scf) c.done = 1;
    flags[m] = (unsigned char)c.done;
    s_save = c.converged && c.shift == 0.0;
  }
  __syncthreads();
  if (s_save) {
    const int ld = E[m].ldv;
    for (int i = threadIdx.x; i < n; i += RB) d.eps_out[i] = E[m].eps[i];
    if (d.want_matrices)
      for (size_t e = threadIdx.x; e < nn; e += RB) {
        const size_t r = e / n, col = e - r * n;
        d.V_out[e] = E[m].in[r * ld + col];
      }
  }
}

// Orbitals of the final Fock (level-shifted molecules) from the bucket output.
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
  // device state
  int slot = -1;
  char *base = nullptr;
  size_t bytes = 0;
  MolDesc d{};
  int np = 0;  // bucket matrix size
  // outcome
  pm7_status status = PM7_OK;
  std::string error;
  pm7_result result{};
  double t_admit = 0.0;
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

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
  d.cc_partial = (double *)take(8 * (size_t)n * gx);
  d.eps_out = (double *)take(8 * (size_t)nao);
  d.V_out = b.o.want_matrices ? (double *)take(8 * nn) : nullptr;
  d.atom_out = (double *)take(8 * (size_t)kAtomOut * n);
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
  d.n_occ = b.n_occ;
  d.dframe = b.dframe;
  d.cc_nx = gx;
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
  }
  ~BatchRunner() {
    cudaSetDevice(ctx_.device);
    cudaStreamSynchronize(st_);
    for (auto &kv : active_) release(*kv);
    if (desc_) cudaFree(desc_);
    if (ctl_) cudaFree(ctl_);
    if (arena_) cudaFree(arena_);
    if (work_) cudaFree(work_);
    if (flags_h_) cudaFreeHost(flags_h_);
    if (flags_d_) cudaFree(flags_d_);
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
    b->bytes = mol_layout(*b, nullptr);
    b->np = bucket_size(b->L.nao);
    if (o.initial_density) {
      const size_t nn = (size_t)b->L.nao * b->L.nao;
      b->init_density.assign(o.initial_density, o.initial_density + nn);
    }
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
  int active_count() const { return (int)active_.size(); }

  // Allocate, upload and build the integrals of the given molecules (one launch per
  // build phase for all of them); they join the next iteration.
  void admit(std::vector<BatchMol *> &in) {
    if (in.empty()) return;
    CUDA_OK(cudaSetDevice(ctx_.device));
    for (BatchMol *b : in) {
      b->slot = take_slot();
      CUDA_OK(cudaMallocAsync((void **)&b->base, b->bytes, st_));
      mol_layout(*b, b->base);
      std::vector<char> img = upload_image(*b);
      size_t start, bytes;
      upload_span(*b, start, bytes);
      staging_.emplace_back(std::move(img));
      CUDA_OK(cudaMemcpyAsync(b->base + start, staging_.back().data(), staging_.back().size(),
                              cudaMemcpyHostToDevice, st_));
      if (!b->init_density.empty())
        CUDA_OK(cudaMemcpyAsync(b->d.Pn, b->init_density.data(), 8 * b->init_density.size(), cudaMemcpyHostToDevice,
                                st_));
      bytes_in_use_ += b->bytes;
    }
    // descriptors and control records
    for (BatchMol *b : in) {
      CUDA_OK(cudaMemcpyAsync(desc_ + b->slot, &b->d, sizeof(MolDesc), cudaMemcpyHostToDevice, st_));
      MolCtl c;
      std::memset(&c, 0, sizeof c);
      c.max_scf = b->o.max_scf;
      c.accel = (b->o.use_diis && b->o.accelerator != PM7_ACCEL_NONE) ? (b->o.accelerator == PM7_ACCEL_CDIIS ? 2 : 1) : 0;
      c.e_tol = b->o.e_tol;
      c.p_tol = b->o.p_tol;
      c.adiis_switch = b->o.adiis_switch;
      c.shift_floor = b->o.level_shift;
      c.shift = b->o.level_shift;
      ctl_stage_.push_back(c);
      CUDA_OK(cudaMemcpyAsync(ctl_ + b->slot, &ctl_stage_.back(), sizeof(MolCtl), cudaMemcpyHostToDevice, st_));
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
      k_b_cc_sum<<<A.mol.n, RB, 0, st_>>>(A.mol, desc_, ctl_);
      note_launch();
    }
    CUDA_OK(cudaStreamSynchronize(st_));
    CUDA_OK(cudaGetLastError());
    staging_.clear();
    ctl_stage_.clear();
    for (BatchMol *b : in) active_.push_back(b);
  }

  // One SCF iteration of every active molecule. Returns the molecules that finished
  // (their results filled, device memory released).
  std::vector<BatchMol *> iterate() {
    std::vector<BatchMol *> finished;
    if (active_.empty()) return finished;
    CUDA_OK(cudaSetDevice(ctx_.device));
    Lists A = lists(active_, true);
    const int n = A.mol.n;
    {
      Stage s_(st_, "batch_fock");
      k_b_push<<<(n + 127) / 128, 128, 0, st_>>>(n, A.mol.slot, ctl_);
      note_launch();
      launch_b_fock(st_, A.mol, A.rows, A.near, A.atoms, desc_, ctl_, *P_, 0);
      k_b_energy<<<n, RB, 0, st_>>>(A.mol, desc_, ctl_, 0);
      note_launch();
    }
    {
      Stage s_(st_, "batch_commutator");
      launch_b_gemm(st_, A.gfull, desc_, ctl_, A.eig, 0);
      k_b_antisym<<<n, RB, 0, st_>>>(A.mol, desc_, ctl_);
      note_launch();
    }
    {
      Stage s_(st_, "batch_diis");
      k_b_dots<<<n, RB, 0, st_>>>(A.mol, desc_, ctl_);
      k_b_control<<<(n + 63) / 64, 64, 0, st_>>>(n, A.mol.slot, ctl_);
      k_b_to_bucket<<<n, RB, 0, st_>>>(A.mol, desc_, ctl_, A.eig, 0);
      note_launch(3);
    }
    {
      Stage s_(st_, "batch_eigensolve");
      eigensolve(A);
    }
    {
      Stage s_(st_, "batch_density");
      launch_b_gemm(st_, A.glow, desc_, ctl_, A.eig, 1);
      k_b_converge<<<n, RB, 0, st_>>>(A.mol, desc_, ctl_, A.eig, flags_d_);
      note_launch();
    }
    CUDA_OK(cudaMemcpyAsync(flags_h_, flags_d_, n, cudaMemcpyDeviceToHost, st_));
    CUDA_OK(cudaStreamSynchronize(st_));
    CUDA_OK(cudaGetLastError());
    std::vector<BatchMol *> keep;
    for (int m = 0; m < n; ++m) (flags_h_[m] ? finished : keep).push_back(active_[m]);
    active_.swap(keep);
    if (!finished.empty()) retire(finished);
    return finished;
  }

 private:
  struct Lists {
    BatchList mol, rows, near, atoms, gfull, glow, sp_pairs, d_pairs, sp_near, d_near, pairs;
    const EigSlot *eig = nullptr;
    std::vector<EigSlot> eig_h;
    std::map<int, std::vector<int>> buckets;  // np -> list positions
    int max_atoms = 0;
  };

  int take_slot() {
    if (free_slots_.empty()) grow(std::max(cap_ * 2, 256));
    const int s = free_slots_.back();
    free_slots_.pop_back();
    return s;
  }

  void grow(int cap) {
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
    CUDA_OK(cudaMallocHost((void **)&flags_h_, cap));
    CUDA_OK(cudaMalloc((void **)&flags_d_, cap));
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
  Lists lists(const std::vector<BatchMol *> &mols, bool with_eig) {
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
        {&A.near, [](const BatchMol &b) { return items_near_chunks((int)b.L.near.size()); }, all},
        {&A.atoms, [](const BatchMol &b) { return b.m.n; }, all},
        {&A.gfull, [](const BatchMol &b) { return items_gemm_full(b.L.nao); }, all},
        {&A.glow, [](const BatchMol &b) { return items_gemm_lower(b.L.nao); }, all},
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
      if (total > arena_cap_) {
        if (arena_) CUDA_OK(cudaFreeAsync(arena_, st_));
        arena_cap_ = total + total / 4;
        CUDA_OK(cudaMallocAsync((void **)&arena_, 8 * arena_cap_, st_));
      }
      A.eig_h.resize(n);
      double *p = arena_;
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

  // One batched eigensolve per bucket size (eigenvalues ascending, vectors in place).
  void eigensolve(const Lists &A) {
    for (auto &kv : A.buckets) {
      const int np = kv.first, cnt = (int)kv.second.size();
      double *in = A.eig_h[kv.second[0]].in, *w = A.eig_h[kv.second[0]].eps;
      size_t wd = 0, wh = 0;
      SOLVER_OK(cusolverDnXsyevBatched_bufferSize(solver_, sparams_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                                  np, CUDA_R_64F, in, np, CUDA_R_64F, w, CUDA_R_64F, &wd, &wh, cnt));
      if (wd > work_cap_) {
        if (work_) CUDA_OK(cudaFreeAsync(work_, st_));
        work_cap_ = wd + wd / 4;
        CUDA_OK(cudaMallocAsync(&work_, work_cap_, st_));
      }
      if (wh > host_work_.size()) host_work_.resize(wh);
      if ((size_t)cnt > info_cap_) {
        if (info_) CUDA_OK(cudaFreeAsync(info_, st_));
        info_cap_ = cnt * 2;
        CUDA_OK(cudaMallocAsync((void **)&info_, sizeof(int) * info_cap_, st_));
      }
      SOLVER_OK(cusolverDnXsyevBatched(solver_, sparams_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, np,
                                       CUDA_R_64F, in, np, CUDA_R_64F, w, CUDA_R_64F, work_, work_cap_,
                                       host_work_.empty() ? nullptr : host_work_.data(), wh, info_, cnt));
    }
  }

  // Final Fock and energy, corrections, orbitals of level-shifted solves, the per-atom
  // outputs, and the results on the host; then the molecules' device memory is freed.
  void retire(std::vector<BatchMol *> &R) {
    Lists A = lists(R, false);
    const int n = A.mol.n;
    {
      Stage s_(st_, "batch_finish");
      launch_b_fock(st_, A.mol, A.rows, A.near, A.atoms, desc_, ctl_, *P_, 1);
      k_b_energy<<<n, RB, 0, st_>>>(A.mol, desc_, ctl_, 1);
      note_launch();
      launch_b_corrections(st_, A.mol, A.pairs, desc_, ctl_, method_, A.max_atoms);
      k_b_atom_out<<<n, 128, 0, st_>>>(A.mol, desc_, *P_);
      note_launch();
    }
    std::vector<MolCtl> ctl(n);
    for (int m = 0; m < n; ++m)
      CUDA_OK(cudaMemcpyAsync(&ctl[m], ctl_ + R[m]->slot, sizeof(MolCtl), cudaMemcpyDeviceToHost, st_));
    CUDA_OK(cudaStreamSynchronize(st_));
    // level-shifted solves report the orbitals of the final Fock (scf.rs:1299-1305)
    std::vector<BatchMol *> shifted;
    for (int m = 0; m < n; ++m)
      if (ctl[m].converged && ctl[m].shift > 0.0) shifted.push_back(R[m]);
    if (!shifted.empty()) {
      Lists S = lists(shifted, true);
      k_b_to_bucket<<<S.mol.n, RB, 0, st_>>>(S.mol, desc_, ctl_, S.eig, 1);
      eigensolve(S);
      k_b_save_orbitals<<<S.mol.n, RB, 0, st_>>>(S.mol, desc_, S.eig);
      note_launch(2);
    }
    std::vector<std::vector<double>> atom(n), eps(n), V(n), Pd(n);
    for (int m = 0; m < n; ++m) {
      BatchMol &b = *R[m];
      const size_t nao = b.L.nao, nn = nao * nao;
      atom[m].resize((size_t)kAtomOut * b.m.n);
      eps[m].resize(nao);
      CUDA_OK(cudaMemcpyAsync(atom[m].data(), b.d.atom_out, 8 * atom[m].size(), cudaMemcpyDeviceToHost, st_));
      CUDA_OK(cudaMemcpyAsync(eps[m].data(), b.d.eps_out, 8 * nao, cudaMemcpyDeviceToHost, st_));
      if (b.o.want_matrices && ctl[m].converged) {
        V[m].resize(nn);
        Pd[m].resize(nn);
        CUDA_OK(cudaMemcpyAsync(V[m].data(), b.d.V_out, 8 * nn, cudaMemcpyDeviceToHost, st_));
        const double *Pnow = (ctl[m].iter % 2 == 0) ? b.d.P : b.d.Pn;
        CUDA_OK(cudaMemcpyAsync(Pd[m].data(), Pnow, 8 * nn, cudaMemcpyDeviceToHost, st_));
      }
    }
    CUDA_OK(cudaStreamSynchronize(st_));
    for (int m = 0; m < n; ++m) {
      BatchMol &b = *R[m];
      const MolCtl &c = ctl[m];
      ResultParts rp;
      rp.iterations = c.iter;
      rp.density_error = c.dp;
      rp.converged = c.converged != 0;
      rp.electronic_ev = c.e_final;
      rp.core_ev = c.core_core;
      for (int k = 0; k < 5; ++k) rp.corr[k] = c.corr[k];
      rp.n_occ = b.n_occ;
      rp.eps_a = eps[m];
      std::vector<double> pops(b.m.n);
      for (int a = 0; a < b.m.n; ++a) pops[a] = atom[m][(size_t)kAtomOut * a];
      const std::vector<double> &ao = atom[m];
      try {
        fill_result(&b.result, b.m, b.L, *b.ps, b.o, rp, pops, [&](int a, int i, int j) {
          const int k = atom_out_index(i, j);
          return k < 0 ? 0.0 : ao[(size_t)kAtomOut * a + k];
        });
        if (b.o.want_matrices) {
          const int nao = b.L.nao;
          b.result.density = host_vec(Pd[m]);
          std::vector<double> C((size_t)nao * nao);
          for (int i = 0; i < nao; ++i)
            for (int k = 0; k < nao; ++k) C[(size_t)i * nao + k] = V[m][(size_t)k * nao + i];
          b.result.mo_coeff = host_vec(C);
        }
        b.status = PM7_OK;
      } catch (const Failure &f) {
        b.status = f.code;
        b.error = f.msg;
      }
      release(b);
    }
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
  ListUpload up_, ptr_up_;
  std::deque<std::vector<char>> staging_;
  std::deque<MolCtl> ctl_stage_;
  double *arena_ = nullptr;
  size_t arena_cap_ = 0;
  void *work_ = nullptr;
  size_t work_cap_ = 0;
  std::vector<char> host_work_;
  int *info_ = nullptr;
  size_t info_cap_ = 0;
  unsigned char *flags_h_ = nullptr, *flags_d_ = nullptr;
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
                           pm7_result *results, pm7_status *status) {
  if (n < 0 || (n > 0 && (!mols || !opts || !results || !status || !params)))
    throw Failure{PM7_ERR_INVALID_INPUT, "null argument"};
  if (n == 0) return;
  const int method = *reinterpret_cast<const int *>(params);
  const int device = opts[0].device;
  BatchRunner runner(device, method);
  std::vector<std::unique_ptr<BatchMol>> items(n);
  std::vector<BatchMol *> pending;
  for (int i = 0; i < n; ++i) {
    std::memset(&results[i], 0, sizeof(pm7_result));
    status[i] = PM7_OK;
    try {
      items[i] = runner.prepare(to_molecule(&mols[i]), opts[i]);
      if (!BatchRunner::batchable(*items[i])) {
        status[i] = pm7_run(&mols[i], params, &opts[i], &results[i]);
        items[i].reset();
        continue;
      }
      pending.push_back(items[i].get());
    } catch (const Failure &f) {
      status[i] = f.code;
      items[i].reset();
    }
  }
  const size_t budget = batch_budget(opts[0].max_memory_mb);
  size_t next = 0;
  while (next < pending.size() || runner.active_count() > 0) {
    std::vector<BatchMol *> admit;
    size_t used = runner.bytes_in_use();
    while (next < pending.size() && (used + pending[next]->bytes <= budget || (runner.active_count() == 0 && admit.empty()))) {
      used += pending[next]->bytes;
      admit.push_back(pending[next++]);
    }
    runner.admit(admit);
    runner.iterate();
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
  std::unordered_map<uint64_t, std::unique_ptr<pm7::EngineRequest>> requests;
  std::unordered_map<pm7::BatchMol *, pm7::EngineRequest *> by_mol;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::string worker_error;
  std::thread worker;
};

namespace pm7 {

static void engine_loop(pm7_engine *E) {
  try {
    CUDA_OK(cudaSetDevice(E->device));
    E->runner = std::make_unique<BatchRunner>(E->device, E->method);
    for (;;) {
      std::vector<BatchMol *> admit;
      {
        std::unique_lock<std::mutex> lk(E->mu);
        E->cv.wait(lk, [&] { return E->stop || !E->queue.empty() || E->runner->active_count() > 0; });
        if (E->stop && E->runner->active_count() == 0) break;
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
    *out = E;
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    return f.code;
  }
}

pm7_status pm7_engine_submit(pm7_engine *E, const pm7_molecule *molecule, const pm7_options *options,
                             uint64_t *ticket) {
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
    std::lock_guard<std::mutex> g(E->mu);
    if (!E->runner) throw Failure{PM7_ERR_CUDA, E->worker_error.empty() ? "engine not ready" : E->worker_error};
    r->ticket = E->next_ticket++;
    *ticket = r->ticket;
    EngineRequest *raw = r.get();
    try {
      r->mol = E->runner->prepare(to_molecule(molecule), *options);
      if (!BatchRunner::batchable(*r->mol))
        throw Failure{PM7_ERR_UNSUPPORTED, "the serving engine runs closed-shell RHF requests; use pm7_run"};
      E->queue.push_back(raw);
    } catch (const Failure &f) {
      raw->status = f.code;
      raw->error = f.msg;
      raw->done = true;
    }
    E->requests[raw->ticket] = std::move(r);
    E->cv.notify_all();
    g_last_error.clear();
    return PM7_OK;
  } catch (const Failure &f) {
    g_last_error = f.msg;
    return f.code;
  }
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

pm7_status pm7_engine_destroy(pm7_engine *E) {
  if (!E) return PM7_ERR_INVALID_INPUT;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    E->stop = true;
    E->cv.notify_all();
  }
  if (E->worker.joinable()) E->worker.join();
  for (auto &kv : E->requests) pm7_result_free(&kv.second->result);
  E->runner.reset();
  delete E;
  return PM7_OK;
}

}  // extern "C"
