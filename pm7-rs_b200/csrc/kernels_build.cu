// One-time device build of a molecule: resonance (beta*S) blocks and core-core
// energies over all atom pairs, the stored two-electron blocks of the near pairs
// (r < 7 Angstrom), and the diagonal blocks of the core Hamiltonian.
//
// Follows pm7-rs src/hamiltonian.rs:310-638 (build_core_generic, molecular path)
// and src/repulsion.rs:16-36,164-263 (core_core_energy).
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.hpp"
#include "core_repulsion.cuh"
#include "nddo_sp.cuh"
#include "batch.hpp"

namespace pm7 {

__device__ __forceinline__ double beta_of(const ElementRec &e, int orb) {
  return orb == 0 ? e.beta_s : (orb <= 3 ? e.beta_p : e.beta_d);
}

// One pair u < v (v may be out of range): beta*S off-diagonal blocks of H; returns the
// core-core energy of the pair (0 when v is not a partner).
__device__ __forceinline__ double pair_sp_elem(int n_atoms, const int *__restrict__ z, const double *__restrict__ xyz,
                                               const int *__restrict__ aoff, int nao, const DeviceParams &P,
                                               double *__restrict__ H, int *status, int u, int v) {
  double ecc = 0.0;
  if (v > u && v < n_atoms) {
    const ElementRec &eu = P.elements[z[u]];
    const ElementRec &ev = P.elements[z[v]];
    // heavier-first ordering (hamiltonian.rs:388-392)
    const bool keep = eu.n_orb >= ev.n_orb;
    const int a = keep ? u : v, b = keep ? v : u;
    const ElementRec &ea = keep ? eu : ev;
    const ElementRec &eb = keep ? ev : eu;
    const double dx = xyz[3 * b] - xyz[3 * a], dy = xyz[3 * b + 1] - xyz[3 * a + 1], dz = xyz[3 * b + 2] - xyz[3 * a + 2];
    double S[4][4];
    if (!d_overlap_sp(ea, eb, dx, dy, dz, S, P.tab)) {
      if (status) atomicOr(status, 1);
    } else {
      const int oa = aoff[a], ob = aoff[b];
      for (int i = 0; i < ea.n_orb && i < 4; ++i) {
        const double bi = beta_of(ea, i);
        for (int j = 0; j < eb.n_orb && j < 4; ++j) {
          const double val = 0.5 * (bi + beta_of(eb, j)) * S[i][j];
          H[(size_t)(oa + i) * nao + ob + j] = val;
          H[(size_t)(ob + j) * nao + oa + i] = val;
        }
      }
    }
    ecc = pair_core_energy(P, eu, ev, sqrt((xyz[3 * v] - xyz[3 * u]) * (xyz[3 * v] - xyz[3 * u]) +
                                           (xyz[3 * v + 1] - xyz[3 * u + 1]) * (xyz[3 * v + 1] - xyz[3 * u + 1]) +
                                           (xyz[3 * v + 2] - xyz[3 * u + 2]) * (xyz[3 * v + 2] - xyz[3 * u + 2])));
  }
  return ecc;
}

// All pairs u < v: beta*S off-diagonal blocks of H and the core-core energy of each pair,
// written to cc_terms[pair_index(u, v)] (pair order, for the reference-order sum).
// Grid: (ceil(N/128), N), block 128; blockIdx.y = u.
__global__ void k_pairs_all(int n_atoms, const int *__restrict__ z, const double *__restrict__ xyz,
                            const int *__restrict__ aoff, int nao, DeviceParams P, double *__restrict__ H,
                            double *__restrict__ cc_terms, int *__restrict__ status) {
  const int u = blockIdx.y, v = blockIdx.x * blockDim.x + threadIdx.x;
  const double ecc = pair_sp_elem(n_atoms, z, xyz, aoff, nao, P, H, status, u, v);
  if (v > u && v < n_atoms) cc_terms[pair_index(n_atoms, u, v)] = ecc;
}

// Batched: item = (atom u, column block) of one molecule; each pair's core-core energy to
// cc_terms in pair order.
__global__ void k_b_pairs_all(BatchList L, const MolDesc *__restrict__ D, DeviceParams P) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const MolDesc &d = D[L.slot[m]];
  const int local = item - L.prefix[m];
  const int u = local / d.cc_nx, bx = local - u * d.cc_nx;
  const int v = bx * blockDim.x + threadIdx.x;
  const double ecc = pair_sp_elem(d.g.n_atoms, d.g.z, d.g.xyz, d.g.aoff, d.g.nao, P, d.H, nullptr, u, v);
  if (v > u && v < d.g.n_atoms) d.cc_terms[pair_index(d.g.n_atoms, u, v)] = ecc;
}

// Near pairs: store w in (u,v) orientation and the packed electron-core blocks of
// both atoms (integrals.rs:186-271 for the sp kernel). One thread per pair.
__device__ __forceinline__ void near_sp_pair(const int *__restrict__ z, const double *__restrict__ xyz,
                                             const NearPair q, const DeviceParams &P, double *__restrict__ w,
                                             double *__restrict__ ecore, int *status) {
  const ElementRec &eu = P.elements[z[q.u]];
  const ElementRec &ev = P.elements[z[q.v]];
  if (eu.n_orb == 9 || ev.n_orb == 9) {
    if (status) atomicOr(status, 2);
    return;
  }
  const bool keep = eu.n_orb >= ev.n_orb;
  const int a = keep ? q.u : q.v, b = keep ? q.v : q.u;
  const ElementRec &ea = keep ? eu : ev;
  const ElementRec &eb = keep ? ev : eu;
  const double dx = xyz[3 * b] - xyz[3 * a], dy = xyz[3 * b + 1] - xyz[3 * a + 1], dz = xyz[3 * b + 2] - xyz[3 * a + 2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double inv = 1.0 / r;
  double rot[3][3];
  d_rotation_to_x(-(dx * inv), -(dy * inv), -(dz * inv), rot);
  const bool ha = ea.n_orb >= 4, hb = eb.n_orb >= 4;
  double *wp = w + q.woff;
  double *e_a = ecore + (keep ? q.eoff_u : q.eoff_v);
  double *e_b = ecore + (keep ? q.eoff_v : q.eoff_u);
  if (!ha && !hb) {
    const double aee = (ea.rho0 + eb.rho0) * (ea.rho0 + eb.rho0);
    double cf, pt;
    d_feather(r, cf, pt);
    const double ee = (1.0 / sqrt(r * r + aee)) * kEv * cf + pt * (1.0 - cf);
    wp[0] = ee;
    e_a[0] = ee * (-eb.core);
    e_b[0] = ee * (-ea.core);
    return;
  }
  if (ha && !hb) {
    double ri[4];
    d_local_xh(ea, eb, r, ri);
    double wxh[10];
    wxh[0] = ri[0];
    for (int k = 0; k < 3; ++k) wxh[dpack(k + 1, 0)] = ri[1] * rot[0][k];
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l <= k; ++l)
        wxh[dpack(k + 1, l + 1)] =
            ri[2] * (rot[0][k] * rot[0][l]) + ri[3] * (rot[1][k] * rot[1][l] + rot[2][k] * rot[2][l]);
    // (u,v) orientation: heavy atom a is u when kept, otherwise v -- a 10x1 or 1x10 block,
    // stored identically because one dimension is 1.
    for (int k = 0; k < 10; ++k) {
      wp[k] = wxh[k];
      e_a[k] = wxh[k] * (-eb.core);
    }
    e_b[0] = wxh[0] * (-ea.core);
    return;
  }
  double ri[22];
  d_local_xx(ea, eb, r, ri);
  int pi = 0;
  for (int kk = 0; kk < 4; ++kk)
    for (int ll = 0; ll <= kk; ++ll, ++pi) {
      int pj = 0;
      for (int mm = 0; mm < 4; ++mm)
        for (int nn = 0; nn <= mm; ++nn, ++pj) {
          const double val = d_rotate_xx_elem(ri, rot, kk, ll, mm, nn);
          if (keep) wp[pi * 10 + pj] = val;
          else wp[pj * 10 + pi] = val;
          if (pj == 0) e_a[pi] = val * (-eb.core);
          if (pi == 0) e_b[pj] = val * (-ea.core);
        }
    }
}

__global__ void k_near_integrals(int n_near, const int *__restrict__ z, const double *__restrict__ xyz,
                                 const NearPair *__restrict__ np, DeviceParams P, double *__restrict__ w,
                                 double *__restrict__ ecore, int *__restrict__ status) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_near) return;
  near_sp_pair(z, xyz, np[p], P, w, ecore, status);
}

// Batched: item = a chunk of 128 near pairs of one molecule.
__global__ void k_b_near_integrals(BatchList L, const MolDesc *__restrict__ D, DeviceParams P) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const MolDesc &d = D[L.slot[m]];
  const int p = (item - L.prefix[m]) * 128 + threadIdx.x;
  if (p >= d.g.n_near) return;
  near_sp_pair(d.g.z, d.g.xyz, d.g.np[p], P, d.w, d.ecore, nullptr);
}

// Diagonal atom blocks of H_core: U on the diagonal plus the electron-core
// attraction of every other atom. Near partners contribute their stored packed
// blocks (summed in partner order); every other atom is beyond the 7 Angstrom
// feather range, where the attraction is exactly the point charge -Z_B * EV / r on
// the diagonal (integrals.rs:540-574). One block per atom.
constexpr int HDIAG_THREADS = 128;
__device__ __forceinline__ void hcore_diag_block(int A, int n_atoms, const int *__restrict__ z,
                                                 const double *__restrict__ xyz, const int *__restrict__ aoff,
                                                 const int *__restrict__ csr_start, const int2 *__restrict__ csr,
                                                 const NearPair *__restrict__ np, const double *__restrict__ ecore,
                                                 const unsigned char *__restrict__ near_mask, const DeviceParams &P,
                                                 int nao, double *__restrict__ H) {
  const ElementRec &e = P.elements[z[A]];
  const int no = e.n_orb, off = aoff[A];
  if (no == 0) return;
  const int npk = no * (no + 1) / 2;
  __shared__ double s_far;
  __shared__ double acc[45];
  const double xa = xyz[3 * A], ya = xyz[3 * A + 1], za = xyz[3 * A + 2];
  const unsigned char *mask = near_mask + (size_t)A * n_atoms;
  double far = 0.0;
  for (int B = threadIdx.x; B < n_atoms; B += HDIAG_THREADS) {
    if (B == A || mask[B]) continue;
    const double dx = xyz[3 * B] - xa, dy = xyz[3 * B + 1] - ya, dz = xyz[3 * B + 2] - za;
    far += -P.elements[z[B]].core * ((1.0 / sqrt(dx * dx + dy * dy + dz * dz)) * kEv);
  }
  far = block_sum<HDIAG_THREADS>(far);
  if (threadIdx.x == 0) s_far = far;
  const int c0 = csr_start[A], c1 = csr_start[A + 1];
  for (int k = threadIdx.x; k < npk; k += HDIAG_THREADS) {
    double a = 0.0;
    for (int c = c0; c < c1; ++c) {
      const NearPair q = np[csr[c].y];
      a += ecore[(q.u == A ? q.eoff_u : q.eoff_v) + k];
    }
    acc[k] = a;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < npk; idx += HDIAG_THREADS) {
    int mu = 0;
    while ((mu + 1) * (mu + 2) / 2 <= idx) ++mu;
    const int nu = idx - mu * (mu + 1) / 2;
    double v = acc[idx];
    if (mu == nu) v += (mu == 0 ? e.u_ss : (mu <= 3 ? e.u_pp : e.u_dd)) + s_far;
    H[(size_t)(off + mu) * nao + off + nu] = v;
    H[(size_t)(off + nu) * nao + off + mu] = v;
  }
}

__global__ void __launch_bounds__(HDIAG_THREADS) k_hcore_diag(int n_atoms, const int *__restrict__ z,
                                                              const double *__restrict__ xyz,
                                                              const int *__restrict__ aoff,
                                                              const int *__restrict__ csr_start,
                                                              const int2 *__restrict__ csr,
                                                              const NearPair *__restrict__ np,
                                                              const double *__restrict__ ecore,
                                                              const unsigned char *__restrict__ near_mask,
                                                              DeviceParams P, int nao, double *__restrict__ H) {
  hcore_diag_block(blockIdx.x, n_atoms, z, xyz, aoff, csr_start, csr, np, ecore, near_mask, P, nao, H);
}

// Batched: item = an atom of one molecule.
__global__ void __launch_bounds__(HDIAG_THREADS) k_b_hcore_diag(BatchList L, const MolDesc *__restrict__ D,
                                                                DeviceParams P) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const MolDesc &d = D[L.slot[m]];
  hcore_diag_block(item - L.prefix[m], d.g.n_atoms, d.g.z, d.g.xyz, d.g.aoff, d.g.csr_start, d.g.csr, d.g.np,
                   d.ecore, d.g.near_mask, P, d.g.nao, d.H);
}

// ---- host launchers ------------------------------------------------------

void launch_pairs_all(cudaStream_t st, int n_atoms, const int *z, const double *xyz, const int *aoff, int nao,
                      const DeviceParams &P, double *H, double *cc_terms, int *status) {
  if (n_atoms < 2) return;
  dim3 grid((n_atoms + 127) / 128, n_atoms);
  k_pairs_all<<<grid, 128, 0, st>>>(n_atoms, z, xyz, aoff, nao, P, H, cc_terms, status);
  note_launch();
}


void launch_near_integrals(cudaStream_t st, int n_near, const int *z, const double *xyz, const NearPair *np,
                           const DeviceParams &P, double *w, double *ecore, int *status) {
  if (n_near == 0) return;
  k_near_integrals<<<(n_near + 127) / 128, 128, 0, st>>>(n_near, z, xyz, np, P, w, ecore, status);
  note_launch();
}

void launch_hcore_diag(cudaStream_t st, int n_atoms, const int *z, const double *xyz, const int *aoff,
                       const int *csr_start, const int2 *csr, const NearPair *np, const double *ecore,
                       const unsigned char *near_mask, const DeviceParams &P, int nao, double *H) {
  k_hcore_diag<<<n_atoms, HDIAG_THREADS, 0, st>>>(n_atoms, z, xyz, aoff, csr_start, csr, np, ecore, near_mask, P,
                                                  nao, H);
  note_launch();
}

void launch_b_pairs_all(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P) {
  if (L.total <= 0) return;
  k_b_pairs_all<<<L.total, 128, 0, st>>>(L, D, P);
  note_launch();
}

void launch_b_near_integrals(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P) {
  if (L.total <= 0) return;
  k_b_near_integrals<<<L.total, 128, 0, st>>>(L, D, P);
  note_launch();
}

void launch_b_hcore_diag(cudaStream_t st, const BatchList &L, const MolDesc *D, const DeviceParams &P) {
  if (L.total <= 0) return;
  k_b_hcore_diag<<<L.total, HDIAG_THREADS, 0, st>>>(L, D, P);
  note_launch();
}

}  // namespace pm7

namespace pm7 {

// One pair's blocks in the (i, j) orientation with n_orb(i) >= n_orb(j), for the
// stage entry point: w (npair_i x npair_j), e1b/e2a (9x9) and the overlap (9x9).
__global__ void k_stage_pair(DeviceParams P, int zi, int zj, double dx, double dy, double dz, double *w,
                             double *e1b, double *e2a, double *s, int *np_out, int *status) {
  const ElementRec &ea = P.elements[zi];
  const ElementRec &eb = P.elements[zj];
  for (int k = 0; k < 81; ++k) e1b[k] = e2a[k] = s[k] = 0.0;
  double S[4][4];
  if (!d_overlap_sp(ea, eb, dx, dy, dz, S, P.tab)) {
    *status = 1;
    return;
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) s[i * 9 + j] = (i < ea.n_orb && j < eb.n_orb) ? S[i][j] : S[i][j];
  const double r = sqrt(dx * dx + dy * dy + dz * dz), inv = 1.0 / r;
  double rot[3][3];
  d_rotation_to_x(-(dx * inv), -(dy * inv), -(dz * inv), rot);
  const bool ha = ea.n_orb >= 4, hb = eb.n_orb >= 4;
  if (!ha && !hb) {
    double cf, pt;
    d_feather(r, cf, pt);
    const double ee = (1.0 / sqrt(r * r + (ea.rho0 + eb.rho0) * (ea.rho0 + eb.rho0))) * kEv * cf + pt * (1.0 - cf);
    w[0] = ee;
    e1b[0] = ee * (-eb.core);
    e2a[0] = ee * (-ea.core);
    np_out[0] = np_out[1] = 1;
    return;
  }
  if (ha && !hb) {
    double ri[4];
    d_local_xh(ea, eb, r, ri);
    w[0] = ri[0];
    for (int k = 0; k < 3; ++k) w[dpack(k + 1, 0)] = ri[1] * rot[0][k];
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l <= k; ++l)
        w[dpack(k + 1, l + 1)] = ri[2] * (rot[0][k] * rot[0][l]) + ri[3] * (rot[1][k] * rot[1][l] + rot[2][k] * rot[2][l]);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) e1b[a * 9 + b] = w[dpack(a, b)] * (-eb.core);
    e2a[0] = w[0] * (-ea.core);
    np_out[0] = 10;
    np_out[1] = 1;
    return;
  }
  double ri[22];
  d_local_xx(ea, eb, r, ri);
  int pi = 0;
  for (int kk = 0; kk < 4; ++kk)
    for (int ll = 0; ll <= kk; ++ll, ++pi) {
      int pj = 0;
      for (int mm = 0; mm < 4; ++mm)
        for (int nn = 0; nn <= mm; ++nn, ++pj) w[pi * 10 + pj] = d_rotate_xx_elem(ri, rot, kk, ll, mm, nn);
    }
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      e1b[a * 9 + b] = w[dpack(a, b) * 10] * (-eb.core);
      e2a[a * 9 + b] = w[dpack(a, b)] * (-ea.core);
    }
  np_out[0] = np_out[1] = 10;
}

void launch_stage_pair(cudaStream_t st, const DeviceParams &P, int zi, int zj, const double d[3], double *w,
                       double *e1b, double *e2a, double *s, int *np_out, int *status) {
  k_stage_pair<<<1, 1, 0, st>>>(P, zi, zj, d[0], d[1], d[2], w, e1b, e2a, s, np_out, status);
  note_launch();
}

}  // namespace pm7
