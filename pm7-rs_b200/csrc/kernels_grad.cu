// Nuclear gradient at a fixed density, sp frame, and the per-atom sums (both frames).
//
// Follows pm7-rs src/gradient.rs:1082-1247 (pair terms), src/repulsion.rs (core-core) and the
// scatter of :1240-1246 (the pair's force added to b, subtracted from a, partners in order).
// The stencil and the pair functional are described in gradient.cuh.
#include <cuda_runtime.h>

#include "common.cuh"
#include "core_repulsion.cuh"
#include "gradient.cuh"
#include "kernels.hpp"
#include "nddo_sp.cuh"

namespace pm7 {
namespace {

// Every pair u < v and stencil point s: core-core, beta*S and (beyond the feather range) the
// point-charge terms. Grid (ceil((N - 1) * 12 / 128), N), blockIdx.y = u.
__global__ void k_grad_pairs_sp(GradGeometry g, DeviceParams P) {
  const int u = blockIdx.y;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = u + 1 + t / kStencil, s = t % kStencil;
  if (v >= g.n_atoms) return;
  const StencilPair q = stencil_pair(g, P, u, v, s);
  const ElementRec &ea = P.elements[g.z[q.a]];
  const ElementRec &eb = P.elements[g.z[q.b]];
  double E = pair_core_energy(P, ea, eb, q.r);
  double S[4][4];
  if (!d_overlap_sp(ea, eb, q.d[0], q.d[1], q.d[2], S, P.tab)) {
    atomicOr(g.status, 1);
  } else {
    const int oa = g.aoff[q.a], ob = g.aoff[q.b];
    for (int i = 0; i < ea.n_orb && i < 4; ++i)
      for (int j = 0; j < eb.n_orb && j < 4; ++j)
        E += g.Pt[(size_t)(oa + i) * g.nao + ob + j] * (grad_beta(ea, i) + grad_beta(eb, j)) * S[i][j];
  }
  if (!g.near_mask[(size_t)u * g.n_atoms + v])
    E += ((1.0 / q.r) * kEv) * far_bracket(g, g.aoff[q.a], ea.n_orb, g.aoff[q.b], eb.n_orb, ea.core, eb.core);
  g.E[tri_index(g.n_atoms, u, v) * kStencil + s] = E;
}

// Near pair p and stencil point s (thread per item): the two-electron and electron-core terms
// of the sp kernel (integrals.rs:186-538 with e1b = -Z_b w[mu nu, ss], e2a = -Z_a w[ss, la si]),
// added to the pair's stencil energy.
__global__ void k_grad_near_sp(GradGeometry g, DeviceParams P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = t / kStencil, s = t % kStencil;
  if (p >= g.n_near) return;
  const NearPair np = g.np[p];
  const int u = np.u < np.v ? np.u : np.v, v = np.u < np.v ? np.v : np.u;
  const StencilPair q = stencil_pair(g, P, u, v, s);
  const ElementRec &ea = P.elements[g.z[q.a]];
  const ElementRec &eb = P.elements[g.z[q.b]];
  if (ea.n_orb == 9 || eb.n_orb == 9) {
    atomicOr(g.status, 2);
    return;
  }
  const int oa = g.aoff[q.a], ob = g.aoff[q.b];
  const double r = q.r, inv = 1.0 / r;
  const bool ha = ea.n_orb >= 4, hb = eb.n_orb >= 4;
  // a sparkle (no orbitals; b, the lighter side, when there is one) holds no density: only its
  // core's attraction on a's electrons (e1b) remains, and its density block is never read
  const bool a_orb = ea.n_orb > 0, b_orb = eb.n_orb > 0;
  double E = 0.0;
  if (!ha && !hb) {
    const double aee = (ea.rho0 + eb.rho0) * (ea.rho0 + eb.rho0);
    double cf, pt;
    d_feather(r, cf, pt);
    const double ee = (1.0 / sqrt(r * r + aee)) * kEv * cf + pt * (1.0 - cf);
    double c = 0.0;
    if (a_orb && b_orb) c += two_e_coef(g, oa, ob, 0, 0, 0, 0);
    if (a_orb) c -= eb.core * ecore_coef(g, oa, 0, 0);
    if (b_orb) c -= ea.core * ecore_coef(g, ob, 0, 0);
    E = ee * c;
  } else {
    double rot[3][3];
    d_rotation_to_x(-(q.d[0] * inv), -(q.d[1] * inv), -(q.d[2] * inv), rot);
    if (ha && !hb) {
      double ri[4];
      d_local_xh(ea, eb, r, ri);
      for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu <= mu; ++nu) {
          double val;
          if (mu == 0) val = ri[0];
          else if (nu == 0) val = ri[1] * rot[0][mu - 1];
          else
            val = ri[2] * (rot[0][mu - 1] * rot[0][nu - 1]) +
                  ri[3] * (rot[1][mu - 1] * rot[1][nu - 1] + rot[2][mu - 1] * rot[2][nu - 1]);
          double c = (b_orb ? two_e_coef(g, oa, ob, mu, nu, 0, 0) : 0.0) - eb.core * ecore_coef(g, oa, mu, nu);
          if (mu == 0 && b_orb) c -= ea.core * ecore_coef(g, ob, 0, 0);
          E += c * val;
        }
    } else {
      double ri[22];
      d_local_xx(ea, eb, r, ri);
      for (int kk = 0; kk < 4; ++kk)
        for (int ll = 0; ll <= kk; ++ll)
          for (int mm = 0; mm < 4; ++mm)
            for (int nn = 0; nn <= mm; ++nn) {
              const double val = d_rotate_xx_elem(ri, rot, kk, ll, mm, nn);
              double c = two_e_coef(g, oa, ob, kk, ll, mm, nn);
              if (mm == 0) c -= eb.core * ecore_coef(g, oa, kk, ll);
              if (kk == 0) c -= ea.core * ecore_coef(g, ob, mm, nn);
              E += c * val;
            }
    }
  }
  g.E[tri_index(g.n_atoms, u, v) * kStencil + s] += E;
}

// A warp per atom A: the derivative of every pair (A, B) from its stencil energies, + for A = v
// (the displaced atom of the pair) and - for A = u; lanes over partners, fixed xor tree.
__global__ void k_grad_atoms(GradGeometry g, double *__restrict__ grad) {
  const int A = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (A >= g.n_atoms) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int B = lane; B < g.n_atoms; B += 32) {
    if (B == A) continue;
    const int u = A < B ? A : B, v = A < B ? B : A;
    const double *e = g.E + tri_index(g.n_atoms, u, v) * kStencil;
    const double sg = A == v ? 1.0 : -1.0;
    for (int k = 0; k < 3; ++k) acc[k] += sg * stencil_derivative(e + 4 * k, kGradStep);
  }
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  }
  if (lane == 0)
    for (int k = 0; k < 3; ++k) grad[3 * A + k] = acc[k];
}

__global__ void k_grad_add(int n3, double scale, const double *__restrict__ extra, double *__restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) grad[i] += scale * extra[i];
}

}  // namespace

void launch_grad_pairs_sp(cudaStream_t st, const GradGeometry &g, const DeviceParams &P) {
  if (g.n_atoms < 2) return;
  const dim3 grid((unsigned)(((size_t)(g.n_atoms - 1) * kStencil + 127) / 128), (unsigned)g.n_atoms);
  k_grad_pairs_sp<<<grid, 128, 0, st>>>(g, P);
  note_launch();
}

void launch_grad_near_sp(cudaStream_t st, const GradGeometry &g, const DeviceParams &P) {
  if (g.n_near <= 0) return;
  const size_t items = (size_t)g.n_near * kStencil;
  k_grad_near_sp<<<(unsigned)((items + 127) / 128), 128, 0, st>>>(g, P);
  note_launch();
}

void launch_grad_atoms(cudaStream_t st, const GradGeometry &g, double *grad) {
  if (g.n_atoms <= 0) return;
  k_grad_atoms<<<(g.n_atoms + 3) / 4, 128, 0, st>>>(g, grad);
  note_launch();
}

void launch_grad_add(cudaStream_t st, int n, double scale, const double *extra, double *grad) {
  if (n <= 0) return;
  k_grad_add<<<(3 * n + 127) / 128, 128, 0, st>>>(3 * n, scale, extra, grad);
  note_launch();
}

}  // namespace pm7
