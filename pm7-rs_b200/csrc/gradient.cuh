// Nuclear gradient at a fixed density (Hellmann-Feynman), shared pieces of the pair kernels.
//
// Follows pm7-rs src/gradient.rs:1082-1247 (electronic_gradient_generic, molecular path) and
// :1372-1500 (the spin-resolved form): every atom pair (a, b), heavier first, contributes
//   E_ab(d) = sum_ij P_ab (beta_i + beta_j) S_ij(d) + sum P_aa e1b(d) + sum P_bb e2a(d)
//           + sum_{mu nu la si} [P_aa(mu nu) P_bb(la si) - sum_s P^s_ab(mu la) P^s_ab(nu si)] w(d)
// plus its core-core energy (src/repulsion.rs), d = R_b - R_a, with the density held fixed;
// the pair's force is dE_ab/dd, added to b and subtracted from a. The reference takes dE_ab/dd
// by forward-mode dual numbers through the integral kernels; here E_ab is evaluated by the same
// device integral kernels as the SCF build at 12 displaced separations (d + t h e_k, t = +-1,
// +-2, h = 1e-3 Bohr) and differentiated by the five-point central difference
//   dE/dd_k = (8 [E(+h) - E(-h)] - [E(+2h) - E(-2h)]) / (12 h),
// whose truncation error (h^4 / 30 times the fifth derivative) and rounding error (~ eps E / h)
// are both near 1e-11 relative for these integrals. Contracting with P before differencing
// keeps one scalar per stencil point instead of every integral's derivative.
//
// The spin terms use P^a = (P + S) / 2 and P^b = (P - S) / 2 (S the spin density; zero for a
// closed shell), so sum_s P^s P^s' = (P P' + S S') / 2.
#pragma once

#include <cuda_runtime.h>

#include "device_params.hpp"
#include "kernels.hpp"

namespace pm7 {

constexpr double kGradStep = 1.0e-3;  // Bohr
constexpr int kStencil = 12;          // 3 axes x {+h, -h, +2h, -2h}

// Displacement of stencil point s (axis s / 4; multiples +1, -1, +2, -2 of h).
__host__ __device__ inline void stencil_offset(int s, double h, double o[3]) {
  const int j = s & 3;
  const double t = (j == 0) ? 1.0 : (j == 1 ? -1.0 : (j == 2 ? 2.0 : -2.0));
  o[0] = o[1] = o[2] = 0.0;
  o[s >> 2] = t * h;
}

// Five-point derivative from the four stencil energies of one axis.
__host__ __device__ inline double stencil_derivative(const double *e4, double h) {
  return (8.0 * (e4[0] - e4[1]) - (e4[2] - e4[3])) / (12.0 * h);
}

// Derivative at 0 from energies at -2h, -h, 0, +h, +2h that may hold a jump or kink (the
// post-SCF corrections' hard switches): with all four one-step differences on one smooth curve
// (both third differences below `tol`, about h^3 times the third derivative for a smooth f)
// the five-point formula; else a second-order formula on points free of the break: the
// one-sided formula of a side whose second difference is under half the other's (the side the
// break is not on, giving the derivative of the branch 0 lies on); for a break at 0 itself
// (both outer second differences below 1% of the middle one: a switch the geometry sits on,
// as at a symmetric tie) the right-hand branch; otherwise (breaks on both sides) the central
// difference on +-h. The factor-2 margins keep rounding from tipping a choice.
__host__ __device__ inline double robust_derivative(double em2, double em1, double e0, double ep1, double ep2, double h,
                                                    double tol) {
  const double d0 = em1 - em2, d1 = e0 - em1, d2 = ep1 - e0, d3 = ep2 - ep1;
  const double t1 = (d2 - d1) - (d1 - d0), t2 = (d3 - d2) - (d2 - d1);
  if (fabs(t1) <= tol && fabs(t2) <= tol) return (8.0 * (ep1 - em1) - (ep2 - em2)) / (12.0 * h);
  const double sl = fabs(d1 - d0), sr = fabs(d3 - d2), sm = fabs(d2 - d1);
  const double left = (3.0 * e0 - 4.0 * em1 + em2) / (2.0 * h), right = (-3.0 * e0 + 4.0 * ep1 - ep2) / (2.0 * h);
  if (fmax(sl, sr) < 0.01 * sm) return right;  // the break is at 0
  if (sl < 0.5 * sr) return left;
  if (sr < 0.5 * sl) return right;
  return (ep1 - em1) / (2.0 * h);
}

// Index of the pair u < v in the row-major upper triangle of an n-atom molecule.
__host__ __device__ inline size_t tri_index(int n, int u, int v) {
  return (size_t)u * (size_t)n - (size_t)u * (size_t)(u + 1) / 2 + (size_t)(v - u - 1);
}

// What the pair kernels read and write. E holds kStencil energies per pair u < v: the pair's
// fixed-density energy with R_v displaced by stencil point s.
struct GradGeometry {
  int n_atoms, nao, n_near;
  const int *z, *aoff;
  const double *xyz;
  const unsigned char *near_mask;  // n_atoms^2, 1 for pairs closer than the feather range
  const NearPair *np;
  const double *Pt, *Ps;  // total and spin density (Ps null for a closed shell)
  double *E;
  int *status;
};

__device__ __forceinline__ double grad_beta(const ElementRec &e, int orb) {
  return orb == 0 ? e.beta_s : (orb <= 3 ? e.beta_p : e.beta_d);
}

// The two-electron coefficient of the packed pair (mu >= nu on a, la >= si on b): the sum over
// the orderings of both index pairs of P_aa P_bb - (P_ab P_ab + S_ab S_ab) / 2.
__device__ inline double two_e_coef(const GradGeometry &g, int oa, int ob, int mu, int nu, int la, int si) {
  const size_t n = (size_t)g.nao;
  const double mi = mu == nu ? 1.0 : 2.0, mj = la == si ? 1.0 : 2.0;
  const double coul = (mi * mj) * (g.Pt[(oa + mu) * n + oa + nu] * g.Pt[(ob + la) * n + ob + si]);
  double x = 0.0;
  for (int o1 = 0; o1 < (mu == nu ? 1 : 2); ++o1) {
    const int m1 = o1 ? nu : mu, n1 = o1 ? mu : nu;
    for (int o2 = 0; o2 < (la == si ? 1 : 2); ++o2) {
      const int l2 = o2 ? si : la, s2 = o2 ? la : si;
      const size_t e1 = (oa + m1) * n + ob + l2, e2 = (oa + n1) * n + ob + s2;
      x += g.Pt[e1] * g.Pt[e2];
      if (g.Ps) x += g.Ps[e1] * g.Ps[e2];
    }
  }
  return coul - 0.5 * x;
}

// The electron-core coefficient of the packed element (mu >= nu) of an atom block at offset o.
__device__ __forceinline__ double ecore_coef(const GradGeometry &g, int o, int mu, int nu) {
  return (mu == nu ? 1.0 : 2.0) * g.Pt[(size_t)(o + mu) * g.nao + o + nu];
}

// A pair beyond the feather range, where every integral is the point charge EV / r
// (src/integrals.rs:540-574): its energy is EV / r times this bracket,
// -Z_b pop_a - Z_a pop_b + pop_a pop_b - sum_{mu in a, la in b} (P_ab^2 + S_ab^2) / 2.
__device__ inline double far_bracket(const GradGeometry &g, int oa, int na, int ob, int nb, double za, double zb) {
  const size_t n = (size_t)g.nao;
  double pa = 0.0, pb = 0.0, x = 0.0;
  for (int k = 0; k < na; ++k) pa += g.Pt[(oa + k) * n + oa + k];
  for (int k = 0; k < nb; ++k) pb += g.Pt[(ob + k) * n + ob + k];
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      const size_t e = (oa + i) * n + ob + j;
      x += g.Pt[e] * g.Pt[e];
      if (g.Ps) x += g.Ps[e] * g.Ps[e];
    }
  return -zb * pa - za * pb + pa * pb - 0.5 * x;
}

// Ordered pair of stencil point s: a (heavier first, as the SCF build orders it), b, and the
// displaced separation d_ab = R_b - R_a with R_v moved by the stencil offset.
struct StencilPair {
  int a, b;
  bool keep;  // a == u
  double d[3], r;
};

__device__ __forceinline__ StencilPair stencil_pair(const GradGeometry &g, const DeviceParams &P, int u, int v, int s) {
  StencilPair q;
  const ElementRec &eu = P.elements[g.z[u]];
  const ElementRec &ev = P.elements[g.z[v]];
  q.keep = eu.n_orb >= ev.n_orb;
  q.a = q.keep ? u : v;
  q.b = q.keep ? v : u;
  double o[3];
  stencil_offset(s, kGradStep, o);
  const double sg = q.keep ? 1.0 : -1.0;
  for (int k = 0; k < 3; ++k) q.d[k] = sg * ((g.xyz[3 * v + k] - g.xyz[3 * u + k]) + o[k]);
  q.r = sqrt(q.d[0] * q.d[0] + q.d[1] * q.d[1] + q.d[2] * q.d[2]);
  return q;
}

// Launchers (kernels_grad.cu for the sp frame and the atom sums, kernels_d.cu for the MNDO/d
// frame). Each pair kernel writes (all pairs) or adds (near pairs) g.E.
void launch_grad_pairs_sp(cudaStream_t st, const GradGeometry &g, const DeviceParams &P);
void launch_grad_near_sp(cudaStream_t st, const GradGeometry &g, const DeviceParams &P);
void launch_grad_pairs_d(cudaStream_t st, const GradGeometry &g, const DeviceParams &P);
void launch_grad_near_d(cudaStream_t st, const GradGeometry &g, const DeviceParams &P);
// grad[3A + k] = sum over partners B (ascending) of the pair derivatives, eV/Bohr.
void launch_grad_atoms(cudaStream_t st, const GradGeometry &g, double *grad);
// grad[3A + k] += scale * extra[3A + k]
void launch_grad_add(cudaStream_t st, int n, double scale, const double *extra, double *grad);

// Correction-energy gradient (kcal/mol per Bohr) by five-point differences of the correction
// energy (kernels_corr.cu): the pair terms pair by pair, the many-body terms over displaced
// copies of the geometry (`copies` per pass, >= 1). `work` holds
// corrections_gradient_work(n, copies, smooth) doubles, `energies` 12 n + 1.
size_t corrections_gradient_work(int n_atoms, int copies, int smooth);
// `any_si`: whether the molecule holds silicon (without it the Si-O-H term is zero).
void launch_corrections_gradient(cudaStream_t st, int n_atoms, const int *z, const double *xyz, int method, int smooth,
                                 int any_si, int copies, double *work, double *energies, double *grad);

}  // namespace pm7
