// Device Fock build F = H + J(P_tot) - K(P_spin), molecular path.
//
// Follows pm7-rs src/fock.rs:149-418 (build_fock_spin_x, no exchange cutoff). Every
// element of F is written by exactly one kernel, so the three kernels need no atomics
// and give the same bits on every run:
//   * k_fock_far   - off-diagonal atom blocks of pairs beyond the 7 Angstrom feather
//                    range, where (mu nu|la si) = delta_mu,nu delta_la,si EV/r and the
//                    exchange block is -P_spin * EV/r (integrals.rs:540-574);
//   * k_fock_near  - off-diagonal blocks of the near pairs from their stored integrals,
//                    plus each pair's packed Coulomb contributions to both atoms;
//   * k_fock_atom  - diagonal atom blocks: one-centre terms, the near Coulomb
//                    contributions in partner order, and the far point-charge Coulomb.
// The kernels are templated on R, the type of the density and the stored integrals they read
// and of their sums: double for every FP64 cycle, float for the early cycles of the mixed
// precision mode (the output F, H, the far potential and the populations stay double).
#include <cuda_runtime.h>

#include "common.cuh"
#include "batch.hpp"
#include "kernels.hpp"
#include "autotune.hpp"
#include "nddo_sp.cuh"

namespace pm7 {

__global__ void k_atom_pop(int n_atoms, const int *__restrict__ aoff, const int *__restrict__ z, DeviceParams P,
                           int nao, const double *__restrict__ Pm, double *__restrict__ pop) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= n_atoms) return;
  const int off = aoff[A], no = P.elements[z[A]].n_orb;
  double s = 0.0;
  for (int k = 0; k < no; ++k) s += Pm[(size_t)(off + k) * nao + off + k];
  pop[A] = s;
}

// The atom-diagonal density blocks, 9 x 9 per atom (n_orb x n_orb used), for the reported
// dipole's hybrid terms without reading the whole density back.
__global__ void k_atom_blocks(int n_atoms, const int *__restrict__ aoff, const int *__restrict__ z, DeviceParams P,
                              int nao, const double *__restrict__ Pm, double *__restrict__ out) {
  const int A = blockIdx.x;
  const int off = aoff[A], no = P.elements[z[A]].n_orb;
  for (int e = threadIdx.x; e < 81; e += blockDim.x) {
    const int i = e / 9, j = e % 9;
    out[(size_t)A * 81 + e] = (i < no && j < no) ? Pm[(size_t)(off + i) * nao + off + j] : 0.0;
  }
}

template <typename R>
__device__ __forceinline__ void fock_far_elem(const FockGeometry &g, const double *__restrict__ H,
                                              const R *__restrict__ Ps, double s_scale, double *__restrict__ F,
                                              int i, int j) {
  const int A = g.ao_atom[i], B = g.ao_atom[j];
  if (A == B || g.near_mask[(size_t)A * g.n_atoms + B]) return;
  double v;
  if (g.gfar) {
    v = g.gfar[(size_t)A * g.n_atoms + B];
  } else {
    const double dx = g.xyz[3 * B] - g.xyz[3 * A], dy = g.xyz[3 * B + 1] - g.xyz[3 * A + 1],
                 dz = g.xyz[3 * B + 2] - g.xyz[3 * A + 2];
    v = (1.0 / sqrt(dx * dx + dy * dy + dz * dz)) * kEv;
  }
  const size_t ij = (size_t)i * g.nao + j;
  F[ij] = H[ij] - (double)((R)s_scale * Ps[ij] * (R)v);
}

template <typename R>
__global__ void k_fock_far(FockGeometry g, const double *__restrict__ H, const R *__restrict__ Ps,
                           double s_scale, double *__restrict__ F) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nao || j >= g.nao) return;
  fock_far_elem<R>(g, H, Ps, s_scale, F, i, j);
}

// One near pair's Fock terms, a group of G lanes per pair: lanes over the pair's outputs —
// the exchange block F_uv (n_u x n_v elements), then the packed Coulomb partials of u from
// P_vv and of v from P_uu (summed per atom by the atom kernel). Every output is one lane's
// sum in a fixed order, so the result does not depend on G or the block size. `wstore` is the
// w store in type R (g.w itself for double).
template <int G, typename R = double>
__device__ __forceinline__ void fock_near_pair(const FockGeometry &g, const DeviceParams &P,
                                               const double *__restrict__ H, const R *__restrict__ Pt,
                                               const R *__restrict__ Ps, double s_scale,
                                               double *__restrict__ F, double *__restrict__ jbuf, int p, int lane,
                                               const R *__restrict__ wstore) {
  const NearPair q = g.np[p];
  const int nu_ = P.elements[g.z[q.u]].n_orb, nv = P.elements[g.z[q.v]].n_orb;
  const int ou = g.aoff[q.u], ov = g.aoff[q.v], nao = g.nao;
  const int npv = nv * (nv + 1) / 2, npu = nu_ * (nu_ + 1) / 2;
  const R *w = wstore + q.woff;
  const int nx = nu_ * nv, total = nx + npu + npv;
  for (int t = lane; t < total; t += G) {
    if (t < nx) {  // exchange element (mu, la)
      const int mu = t / nv, la = t - mu * nv;
      R acc = 0;
      for (int nu = 0; nu < nu_; ++nu) {
        const R *row = w + dpack(mu, nu) * npv;
        for (int si = 0; si < nv; ++si) acc += Ps[(size_t)(ou + nu) * nao + ov + si] * row[dpack(la, si)];
      }
      const double kv = -(double)(acc * (R)s_scale);
      const size_t e1 = (size_t)(ou + mu) * nao + ov + la, e2 = (size_t)(ov + la) * nao + ou + mu;
      F[e1] = H[e1] + kv;
      F[e2] = H[e2] + kv;
    } else if (t < nx + npu) {  // Coulomb on u from P_vv, packed element k = (mu >= nu)
      const int k = t - nx;
      int mu = 0;
      while ((mu + 1) * (mu + 2) / 2 <= k) ++mu;
      const R *row = w + k * npv;
      R acc = 0;
      for (int la = 0; la < nv; ++la)
        for (int si = 0; si < nv; ++si) acc += Pt[(size_t)(ov + la) * nao + ov + si] * row[dpack(la, si)];
      jbuf[q.eoff_u + k] = (double)acc;
    } else {  // Coulomb on v from P_uu, packed element col
      const int col = t - nx - npu;
      R acc = 0;
      for (int mu = 0; mu < nu_; ++mu)
        for (int nu = 0; nu < nu_; ++nu) acc += Pt[(size_t)(ou + mu) * nao + ou + nu] * w[dpack(mu, nu) * npv + col];
      jbuf[q.eoff_v + col] = (double)acc;
    }
  }
}

// A block of T threads per 128 near pairs (pairs 128 b .. 128 b + 127), in groups of G lanes
// that take a pair at a time. (G, T) is an autotuned launch shape with identical results:
// whole warps suit the 9-orbital pairs, narrow groups the hydrogen-rich sp pairs (3 to 36
// outputs each).
template <int G, int T, typename R = double>
__global__ void __launch_bounds__(T, 1) k_fock_near(FockGeometry g, DeviceParams P, const double *__restrict__ H,
                                                    const R *__restrict__ Pt, const R *__restrict__ Ps,
                                                    double s_scale, double *__restrict__ F,
                                                    double *__restrict__ jbuf, const R *__restrict__ w) {
  constexpr int NG = T / G;
  static_assert(128 % NG == 0, "groups per block must divide 128");
  const int lane = threadIdx.x % G, grp = threadIdx.x / G;
  for (int r = 0; r < 128 / NG; ++r) {
    const int p = blockIdx.x * 128 + grp + NG * r;
    if (p < g.n_near) fock_near_pair<G, R>(g, P, H, Pt, Ps, s_scale, F, jbuf, p, lane, w);
  }
}

// The near-pair launch shapes, X(variant, G lanes per pair, T threads per block).
#define PM7_NEAR_SHAPES(X) X(0, 32, 1024) X(1, 32, 256) X(2, 8, 256) X(3, 4, 128) X(4, 1, 128)
constexpr int kNearVariants = 5;

// One-centre two-electron integral (a b | c d) of an sp atom (fock.rs:69-107).
__device__ __forceinline__ double oc_sp(int a, int b, int c, int d, const ElementRec &e) {
  if (a == b && c == d) {
    if (a == 0 && c == 0) return e.g_ss;
    if (a == 0 || c == 0) return e.g_sp;
    return a == c ? e.g_pp : e.g_p2;
  }
  const int ba = a < b ? a : b, bb = a < b ? b : a, kc = c < d ? c : d, kd = c < d ? d : c;
  if (ba == 0 && bb != 0 && kc == 0 && kd != 0 && bb == kd) return e.h_sp;
  if (ba != 0 && bb != 0 && ba != bb && ba == kc && bb == kd) return 0.5 * (e.g_pp - e.g_p2);
  return 0.0;
}

// One group of G lanes per atom: the far point-charge Coulomb (32 partial sums over partner
// atoms, B = v, v + 32, ..., combined by a fixed xor tree; with G < 32 each lane holds 32/G of
// the partials and does the upper tree levels in registers, so every G gives the same bits),
// the near Coulomb partials summed in partner order (lanes over packed elements), then the
// one-centre terms and the assembly of the atom's diagonal block (lanes over its elements).
// `jacc` is the group's 45 doubles of shared memory; `gmask` the group's lanes. No block-wide
// barrier.
template <int G, typename R = double>
__device__ __forceinline__ void fock_atom_group(const FockGeometry &g, const DeviceParams &P,
                                                const double *__restrict__ H, const R *__restrict__ Pt,
                                                const R *__restrict__ Ps, double s_scale,
                                                const double *__restrict__ pop, const double *__restrict__ jbuf,
                                                double *__restrict__ F, int A, double *jacc, int lane,
                                                unsigned gmask) {
  constexpr int V = 32 / G;
  const ElementRec &e = P.elements[g.z[A]];
  const int no = e.n_orb, off = g.aoff[A], nao = g.nao;
  if (no == 0) return;
  const int npk = no * (no + 1) / 2;
  const double xa = g.xyz[3 * A], ya = g.xyz[3 * A + 1], za = g.xyz[3 * A + 2];
  const unsigned char *mask = g.near_mask + (size_t)A * g.n_atoms;
  double part[V];
#pragma unroll
  for (int k = 0; k < V; ++k) part[k] = 0.0;
  if (g.gfar) {
    // gfar is exactly 0 for A itself and its near partners and populations are >= 0, so those
    // terms add +0.0 and change no partial: no branch, independent loads
    const double *grow = g.gfar + (size_t)A * g.n_atoms;
#pragma unroll 2
    for (int B0 = 0; B0 < g.n_atoms; B0 += 32) {
#pragma unroll
      for (int k = 0; k < V; ++k) {
        const int B = B0 + lane + G * k;  // partial v = lane + G k
        if (B < g.n_atoms) part[k] += grow[B] * pop[B];
      }
    }
  } else {
    for (int B0 = 0; B0 < g.n_atoms; B0 += 32) {
#pragma unroll
      for (int k = 0; k < V; ++k) {
        const int B = B0 + lane + G * k;  // partial v = lane + G k
        if (B >= g.n_atoms || B == A || mask[B]) continue;
        const double dx = g.xyz[3 * B] - xa, dy = g.xyz[3 * B + 1] - ya, dz = g.xyz[3 * B + 2] - za;
        part[k] += ((1.0 / sqrt(dx * dx + dy * dy + dz * dz)) * kEv) * pop[B];
      }
    }
  }
  // xor tree over the 32 partials: levels o >= G pair partials of one lane, o < G cross lanes
#pragma unroll
  for (int o = 16; o >= G; o >>= 1) {
    double t[V];
#pragma unroll
    for (int k = 0; k < V; ++k) t[k] = part[k] + part[k ^ (o / G)];
#pragma unroll
    for (int k = 0; k < V; ++k) part[k] = t[k];
  }
  double far = part[0];
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) far += __shfl_xor_sync(gmask, far, o, G);
  const int c0 = g.csr_start[A], c1 = g.csr_start[A + 1];
  for (int k = lane; k < npk; k += G) {
    double acc = 0.0;
    if (g.csr_eoff) {  // one independent load per partner
      for (int c = c0; c < c1; ++c) acc += jbuf[g.csr_eoff[c] + k];
    } else {
      for (int c = c0; c < c1; ++c) {
        const NearPair q = g.np[g.csr[c].y];
        acc += jbuf[(q.u == A ? q.eoff_u : q.eoff_v) + k];
      }
    }
    jacc[k] = acc;
  }
  __syncwarp(gmask);
  const double *oc = (no == 9 && e.onecenter_slot >= 0) ? P.onecenter + (size_t)e.onecenter_slot * 2025 : nullptr;
  for (int idx = lane; idx < no * no; idx += G) {
    const int mu = idx / no, nu = idx - mu * no;
    R acc = 0;
    for (int la = 0; la < no; ++la)
      for (int si = 0; si < no; ++si) {
        const R pt = Pt[(size_t)(off + la) * nao + off + si];
        const R ps = (R)s_scale * Ps[(size_t)(off + la) * nao + off + si];
        if (oc) {
          acc += pt * (R)oc[dpack(mu, nu) * 45 + dpack(la, si)];
          acc -= ps * (R)oc[dpack(mu, la) * 45 + dpack(nu, si)];
        } else {
          acc += pt * (R)oc_sp(mu, nu, la, si, e);
          acc -= ps * (R)oc_sp(mu, la, nu, si, e);
        }
      }
    double v = (double)acc + jacc[dpack(mu, nu)];
    if (mu == nu) v += far;
    const size_t ij = (size_t)(off + mu) * nao + off + nu;
    F[ij] = H[ij] + v;
  }
}

// The lanes of this thread's aligned group of G within its warp.
template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) return 0xffffffffu;
  else return ((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1));
}

// A block of T threads, T/G atoms (a group of G lanes each).
template <int G, int T, typename R = double>
__global__ void __launch_bounds__(T) k_fock_atom(FockGeometry g, DeviceParams P, const double *__restrict__ H,
                                                 const R *__restrict__ Pt, const R *__restrict__ Ps,
                                                 double s_scale, const double *__restrict__ pop,
                                                 const double *__restrict__ jbuf, double *__restrict__ F) {
  constexpr int NG = T / G;
  __shared__ double jacc[NG][45];
  const int grp = threadIdx.x / G;
  const int A = blockIdx.x * NG + grp;
  if (A < g.n_atoms)
    fock_atom_group<G, R>(g, P, H, Pt, Ps, s_scale, pop, jbuf, F, A, jacc[grp], threadIdx.x % G, group_mask<G>());
}

// The atom launch shapes, X(variant, G lanes per atom, T threads per block).
#define PM7_ATOM_SHAPES(X) X(0, 32, 256) X(1, 8, 256) X(2, 4, 128)
constexpr int kAtomVariants = 3;

// ---- batched Fock (RHF: P_spin = P/2) ----------------------------------------------

__device__ __forceinline__ double *fock_target(const MolDesc &d, const MolCtl &c, int final_pass) {
  return final_pass ? d.X : hist_F(d, c.slot);
}

// Per molecule: atom populations of P.
__global__ void k_b_atom_pop(BatchList L, const MolDesc *__restrict__ D, DeviceParams P) {
  const MolDesc &d = D[L.slot[blockIdx.x]];
  for (int A = threadIdx.x; A < d.g.n_atoms; A += blockDim.x) {
    const int off = d.g.aoff[A], no = P.elements[d.g.z[A]].n_orb;
    double s = 0.0;
    for (int k = 0; k < no; ++k) s += d.P[(size_t)(off + k) * d.g.nao + off + k];
    d.pop[A] = s;
  }
}

// The FP32 build's inputs, item = 8 rows of one molecule (the far kernel's items): rows of the
// density as float and a 1/items share of the w store (on the guess iteration only, whose
// build is always FP32 in mixed precision); item 0 marks the ring slot this iteration's Fock
// matrix goes to as built in FP32 or not.
__global__ void __launch_bounds__(256) k_b_fock32_inputs(BatchList L, const MolDesc *__restrict__ D,
                                                         MolCtl *__restrict__ C) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  const int q = item - L.prefix[m], nq = L.prefix[m + 1] - L.prefix[m];
  const bool f32 = fock32_now(d, c);
  if (q == 0 && threadIdx.x == 0) {  // nothing in this launch reads f32_slots
    if (f32) c.f32_slots |= 1 << c.slot;
    else c.f32_slots &= ~(1 << c.slot);
  }
  if (!f32) return;
  const size_t n = d.g.nao, e0 = (size_t)q * 8 * n, e1 = min(e0 + 8 * n, n * n);
  for (size_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) d.P32[e] = (float)d.P[e];
  if (c.iter == 0) {
    const size_t w0 = d.w_len * q / nq, w1 = d.w_len * (q + 1) / nq;
    for (size_t e = w0 + threadIdx.x; e < w1; e += blockDim.x) d.w32[e] = (float)d.g.w[e];
  }
}

// Item = 8 rows of one molecule's matrix (warp per row, lanes over columns).
__global__ void __launch_bounds__(256) k_b_fock_far(BatchList L, const MolDesc *__restrict__ D,
                                                    const MolCtl *__restrict__ C, int final_pass) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const int i = (item - L.prefix[m]) * 8 + (threadIdx.x >> 5);
  if (i >= d.g.nao) return;
  double *F = fock_target(d, C[slot], final_pass);
  if (!final_pass && fock32_now(d, C[slot])) {
    for (int j = threadIdx.x & 31; j < d.g.nao; j += 32) fock_far_elem<float>(d.g, d.H, d.P32, 0.5, F, i, j);
  } else {
    for (int j = threadIdx.x & 31; j < d.g.nao; j += 32) fock_far_elem<double>(d.g, d.H, d.P, 0.5, F, i, j);
  }
}

// Item = 128 near pairs of one molecule (groups of G lanes, a pair per group at a time).
template <int G, int T>
__global__ void __launch_bounds__(T, 1) k_b_fock_near(BatchList L, const MolDesc *__restrict__ D,
                                                      const MolCtl *__restrict__ C, DeviceParams P, int final_pass) {
  constexpr int NG = T / G;
  static_assert(128 % NG == 0, "groups per block must divide 128");
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const int lane = threadIdx.x % G, grp = threadIdx.x / G;
  double *F = fock_target(d, C[slot], final_pass);
  const bool f32 = !final_pass && fock32_now(d, C[slot]);
  for (int r = 0; r < 128 / NG; ++r) {
    const int p = (item - L.prefix[m]) * 128 + grp + NG * r;
    if (p >= d.g.n_near) continue;
    if (f32) fock_near_pair<G, float>(d.g, P, d.H, d.P32, d.P32, 0.5, F, d.jbuf, p, lane, d.w32);
    else fock_near_pair<G>(d.g, P, d.H, d.P, d.P, 0.5, F, d.jbuf, p, lane, d.g.w);
  }
}

// Item = an atom of one molecule (a group of G lanes per item, T/G per block).
template <int G, int T>
__global__ void __launch_bounds__(T) k_b_fock_atom(BatchList L, const MolDesc *__restrict__ D,
                                                   const MolCtl *__restrict__ C, DeviceParams P, int final_pass) {
  constexpr int NG = T / G;
  __shared__ double jacc[NG][45];
  const int grp = threadIdx.x / G;
  const int item = blockIdx.x * NG + grp;
  if (item >= L.total) return;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  double *F = fock_target(d, C[slot], final_pass);
  if (!final_pass && fock32_now(d, C[slot]))
    fock_atom_group<G, float>(d.g, P, d.H, d.P32, d.P32, 0.5, d.pop, d.jbuf, F, item - L.prefix[m], jacc[grp],
                              threadIdx.x % G, group_mask<G>());
  else
    fock_atom_group<G>(d.g, P, d.H, d.P, d.P, 0.5, d.pop, d.jbuf, F, item - L.prefix[m], jacc[grp],
                       threadIdx.x % G, group_mask<G>());
}

// Size bucket of an autotune key: the next power of two above n.
static int pow2_bucket(int n) { return n <= 0 ? 1 : 1 << (32 - __builtin_clz((unsigned)n)); }

void launch_b_fock(cudaStream_t st, const BatchList &Lmol, const BatchList &Lrows, const BatchList &Lnear,
                   const BatchList &Latoms, const MolDesc *D, const MolCtl *C, const DeviceParams &P, int final_pass) {
  if (Lmol.n <= 0) return;
  k_b_atom_pop<<<Lmol.n, 128, 0, st>>>(Lmol, D, P);
  note_launch();
  if (!final_pass && Lrows.total > 0) {
    k_b_fock32_inputs<<<Lrows.total, 256, 0, st>>>(Lrows, D, const_cast<MolCtl *>(C));
    note_launch();
  }
  if (Lrows.total > 0) k_b_fock_far<<<Lrows.total, 256, 0, st>>>(Lrows, D, C, final_pass);
  note_launch();
  if (Lnear.total > 0)
    autotune(st, "b_fock_near|items" + std::to_string(pow2_bucket(Lnear.total)), kNearVariants, [&](int v) {
      switch (v) {
#define PM7_LAUNCH(i, G, T) \
  case i: k_b_fock_near<G, T><<<Lnear.total, T, 0, st>>>(Lnear, D, C, P, final_pass); break;
        PM7_NEAR_SHAPES(PM7_LAUNCH)
#undef PM7_LAUNCH
      }
      note_launch();
    });
  if (Latoms.total > 0)
    autotune(st, "b_fock_atom|items" + std::to_string(pow2_bucket(Latoms.total)), kAtomVariants, [&](int v) {
      switch (v) {
#define PM7_LAUNCH(i, G, T) \
  case i: k_b_fock_atom<G, T><<<(Latoms.total + T / G - 1) / (T / G), T, 0, st>>>(Latoms, D, C, P, final_pass); break;
        PM7_ATOM_SHAPES(PM7_LAUNCH)
#undef PM7_LAUNCH
      }
      note_launch();
    });
}

// Thread per (A, B): EV / r_AB for far pairs, 0 for A == B and near pairs. Grid (ceil(N/128), N).
__global__ void k_far_coulomb(int n, const double *__restrict__ xyz, const unsigned char *__restrict__ near_mask,
                              double *__restrict__ gfar) {
  const int A = blockIdx.y, B = blockIdx.x * blockDim.x + threadIdx.x;
  if (B >= n) return;
  double v = 0.0;
  if (A != B && !near_mask[(size_t)A * n + B]) {
    const double dx = xyz[3 * B] - xyz[3 * A], dy = xyz[3 * B + 1] - xyz[3 * A + 1], dz = xyz[3 * B + 2] - xyz[3 * A + 2];
    v = (1.0 / sqrt(dx * dx + dy * dy + dz * dz)) * kEv;
  }
  gfar[(size_t)A * n + B] = v;
}

void launch_far_coulomb(cudaStream_t st, int n, const double *xyz, const unsigned char *near_mask, double *gfar) {
  if (n <= 0) return;
  k_far_coulomb<<<dim3((n + 127) / 128, n), 128, 0, st>>>(n, xyz, near_mask, gfar);
  note_launch();
}

void launch_atom_blocks(cudaStream_t st, int n_atoms, const int *aoff, const int *z, const DeviceParams &P, int nao,
                        const double *Pm, double *out) {
  if (n_atoms <= 0) return;
  k_atom_blocks<<<n_atoms, 96, 0, st>>>(n_atoms, aoff, z, P, nao, Pm, out);
  note_launch();
}

void launch_atom_pop(cudaStream_t st, int n_atoms, const int *aoff, const int *z, const DeviceParams &P, int nao,
                     const double *Pm, double *pop) {
  k_atom_pop<<<(n_atoms + 127) / 128, 128, 0, st>>>(n_atoms, aoff, z, P, nao, Pm, pop);
  note_launch();
}

void launch_fock(cudaStream_t st, const FockGeometry &g, const DeviceParams &P, const double *H, const double *Pt,
                 const double *Ps, double s_scale, double *F, double *pop, double *jbuf) {
  launch_atom_pop(st, g.n_atoms, g.aoff, g.z, P, g.nao, Pt, pop);
  dim3 blk(32, 8), grd((g.nao + 31) / 32, (g.nao + 7) / 8);
  k_fock_far<double><<<grd, blk, 0, st>>>(g, H, Ps, s_scale, F);
  note_launch();
  if (g.n_near > 0) {
    const int blocks = (g.n_near + 127) / 128;
    autotune(st, "fock_near|pairs" + std::to_string(pow2_bucket(g.n_near)), kNearVariants, [&](int v) {
      switch (v) {
#define PM7_LAUNCH(i, G, T) \
  case i: k_fock_near<G, T><<<blocks, T, 0, st>>>(g, P, H, Pt, Ps, s_scale, F, jbuf, g.w); break;
        PM7_NEAR_SHAPES(PM7_LAUNCH)
#undef PM7_LAUNCH
      }
      note_launch();
    });
  }
  autotune(st, "fock_atom|atoms" + std::to_string(pow2_bucket(g.n_atoms)), kAtomVariants, [&](int v) {
    switch (v) {
#define PM7_LAUNCH(i, G, T) \
  case i: k_fock_atom<G, T><<<(g.n_atoms + T / G - 1) / (T / G), T, 0, st>>>(g, P, H, Pt, Ps, s_scale, pop, jbuf, F); break;
      PM7_ATOM_SHAPES(PM7_LAUNCH)
#undef PM7_LAUNCH
    }
    note_launch();
  });
}

__global__ void k_to_float(size_t n, const double *__restrict__ src, float *__restrict__ dst) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    dst[e] = (float)src[e];
}

void launch_to_float(cudaStream_t st, size_t n, const double *src, float *dst) {
  if (n == 0) return;
  const size_t blocks = std::min<size_t>((n + 255) / 256, 148 * 8);
  k_to_float<<<(unsigned)blocks, 256, 0, st>>>(n, src, dst);
  note_launch();
}

// The FP32 build: one launch shape each (near pairs in groups of 8 lanes, atoms a warp each);
// the populations come from the double density Pt64.
void launch_fock32(cudaStream_t st, const FockGeometry &g, const DeviceParams &P, const double *H,
                   const double *Pt64, const float *Pt, const float *Ps, double s_scale, double *F, double *pop,
                   double *jbuf, const float *w) {
  launch_atom_pop(st, g.n_atoms, g.aoff, g.z, P, g.nao, Pt64, pop);
  dim3 blk(32, 8), grd((g.nao + 31) / 32, (g.nao + 7) / 8);
  k_fock_far<float><<<grd, blk, 0, st>>>(g, H, Ps, s_scale, F);
  note_launch();
  if (g.n_near > 0) {
    k_fock_near<8, 256, float><<<(g.n_near + 127) / 128, 256, 0, st>>>(g, P, H, Pt, Ps, s_scale, F, jbuf, w);
    note_launch();
  }
  k_fock_atom<32, 256, float><<<(g.n_atoms + 7) / 8, 256, 0, st>>>(g, P, H, Pt, Ps, s_scale, pop, jbuf, F);
  note_launch();
}

}  // namespace pm7
