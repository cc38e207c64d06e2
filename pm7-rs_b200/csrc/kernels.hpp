// Host-callable launchers of the engine's CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "device_params.hpp"

namespace pm7 {

// Counts kernels launched by this library (read through pm7_launch_count()).
void note_launch(int kernels = 1);

// An atom pair closer than the 7 Angstrom feather range, whose two-electron block is
// stored. u < v; w is npair(u) x npair(v) row-major at `woff`; the packed per-atom
// blocks (electron-core attraction, then the Coulomb scratch of the Fock build) of
// u and v start at eoff_u / eoff_v.
struct NearPair {
  int32_t u, v;
  int64_t woff;
  int32_t eoff_u, eoff_v;
};

// ---- build (kernels_build.cu) ----
// cc_terms: the N(N-1)/2 pair core-core energies in pair order (u < v, row by row), for
// the reference-order sum.
void launch_pairs_all(cudaStream_t st, int n_atoms, const int *z, const double *xyz, const int *aoff, int nao,
                      const DeviceParams &P, double *H, double *cc_terms, int *status);
// Position of pair (u, v), u < v, in the pair order of `core_core_energy` (src/repulsion.rs:19-22).
__host__ __device__ inline size_t pair_index(int n, int u, int v) {
  return (size_t)u * (2 * (size_t)n - u - 1) / 2 + (size_t)(v - u - 1);
}
void launch_near_integrals(cudaStream_t st, int n_near, const int *z, const double *xyz, const NearPair *np,
                           const DeviceParams &P, double *w, double *ecore, int *status);
void launch_hcore_diag(cudaStream_t st, int n_atoms, const int *z, const double *xyz, const int *aoff,
                       const int *csr_start, const int2 *csr, const NearPair *np, const double *ecore,
                       const unsigned char *near_mask, const DeviceParams &P, int nao, double *H);

// ---- MNDO/d frame (kernels_d.cu): used for every pair of a molecule with a d-shell atom ----
// beta*S blocks from the general Slater overlaps, plus core-core partials (as launch_pairs_all).
void launch_pairs_all_d(cudaStream_t st, int n_atoms, const int *z, const double *xyz, const int *aoff, int nao,
                        const DeviceParams &P, double *H, double *cc_terms);
// Near-pair w blocks and packed electron-core blocks (as launch_near_integrals), one warp per pair.
void launch_near_integrals_d(cudaStream_t st, int n_near, const int *z, const double *xyz, const NearPair *np,
                             const DeviceParams &P, double *w, double *ecore);
// One pair in the (i, j) orientation, n_orb(i) >= n_orb(j): w, e1b, e2a, S (9x9), np_out[2].
void launch_stage_pair_d(cudaStream_t st, const DeviceParams &P, int zi, int zj, const double d[3], double *w,
                         double *e1b, double *e2a, double *s, int *np_out);

// ---- Fock build (kernels_fock.cu) ----
struct FockGeometry {
  int n_atoms, nao, n_near;
  const int *z, *aoff, *ao_atom;
  const double *xyz;
  const unsigned char *near_mask;  // n_atoms^2
  const NearPair *np;
  const int *csr_start;
  const int2 *csr;  // (partner atom, near-pair index), sorted by partner
  const int *csr_eoff;  // per csr entry: offset of the row atom's packed partials in jbuf (or null)
  const double *w;
  // n_atoms^2: EV / r of every pair beyond the feather range (0 for an atom with itself and
  // for near pairs), precomputed once per molecule; null to evaluate it in the Fock kernels
  const double *gfar;
};
// EV / r of the far pairs into gfar (n x n), the same expression the Fock kernels evaluate.
void launch_far_coulomb(cudaStream_t st, int n_atoms, const double *xyz, const unsigned char *near_mask,
                        double *gfar);
// F = H + J(Pt) - K(s * Ps). `pop` (n_atoms) and `jbuf` (packed, like ecore) are scratch.
void launch_fock(cudaStream_t st, const FockGeometry &g, const DeviceParams &P, const double *H, const double *Pt,
                 const double *Ps, double s_scale, double *F, double *pop, double *jbuf);
// The same F with the density and the stored integrals read as float (Pt, Ps, w: float copies)
// and summed in FP32; populations from the double density Pt64. For early mixed-precision cycles.
void launch_fock32(cudaStream_t st, const FockGeometry &g, const DeviceParams &P, const double *H,
                   const double *Pt64, const float *Pt, const float *Ps, double s_scale, double *F, double *pop,
                   double *jbuf, const float *w);
// dst[i] = (float)src[i], i < n.
void launch_to_float(cudaStream_t st, size_t n, const double *src, float *dst);

// ---- dense algebra (kernels_dense.cu) ----
// C[M x N] = alpha * A^T B, A: K x M row-major (lda), B: K x N row-major (ldb), C row-major (ldc). FP64 DMMA.
// Sets the DMMA GEMM kernels' shared-memory attributes on the current device (idempotent).
void prepare_gemm_kernels();
void launch_gemm_tn(cudaStream_t st, int M, int N, int K, double alpha, const double *A, int lda, const double *B,
                    int ldb, double *C, int ldc);
// P = w * V^T V for the first k rows of V (n columns, row stride ldv); symmetric output.
void launch_density(cudaStream_t st, int n, int k, double w, const double *V, int ldv, double *P);
// E = X - X^T, partial sums of E*E into `partials` (returns the partial count).
size_t launch_antisym(cudaStream_t st, int n, const double *X, double *E, double *partials);
// partials of sum(a*b) (returns the count).
size_t launch_dot(cudaStream_t st, size_t len, const double *a, const double *b, double *partials);
// partials of sum(P*(H+F)).
size_t launch_energy(cudaStream_t st, size_t len, const double *P, const double *H, const double *F,
                     double *partials);
// partials of sum((a-b)^2).
size_t launch_sqdiff(cudaStream_t st, size_t len, const double *a, const double *b, double *partials);
// out = sum_i c[i] * X[i] (+ shift*(I - Pd/occ)); coefficients in device memory.
void launch_combine(cudaStream_t st, int n, int k, const double *const *X, const double *c, const double *Pd,
                    double occ, double shift, double *out);
// Many dot products <X_i, Y_j> in one pass: out[i*ny + j] partials; see kernels_dense.cu.
void launch_dot_many(cudaStream_t st, size_t len, int nx, const double *const *X, int ny, const double *const *Y,
                     double *out_partials, int n_blocks);
void launch_reduce_rows(cudaStream_t st, const double *partials, int n_rows, int n_cols, double *out);
void launch_sum(cudaStream_t st, const double *partials, size_t n, double *out);
void launch_transpose(cudaStream_t st, int n, const double *in, double *out);
void launch_scale(cudaStream_t st, size_t len, double s, const double *in, double *out);
void launch_axpby(cudaStream_t st, size_t len, double a, const double *x, double b, const double *y, double *out);
void launch_set_diag(cudaStream_t st, int n, const double *diag, double *M);
void launch_atom_pop(cudaStream_t st, int n_atoms, const int *aoff, const int *z, const DeviceParams &P,
                     int nao, const double *Pm, double *pop);
// out[81 a + 9 i + j] = Pm of atom a's diagonal block (i, j < n_orb; 0 elsewhere).
void launch_atom_blocks(cudaStream_t st, int n_atoms, const int *aoff, const int *z, const DeviceParams &P, int nao,
                        const double *Pm, double *out);

// ---- reference-order sums (kernels_seqsum.cu) ----
// The exact value of the left-to-right fold s = ((-0 + t_0) + t_1) + ... over t_i = a[i]
// (b null) or t_i = fl(a[i] * b[i]) (no fused multiply-add), written to *out: bit for
// bit what a serial loop gives, computed in parallel. Up to four sums per launch.
struct SeqSumJob {
  const double *a, *b;
  size_t n;
  double *out;  // device
};
struct SeqSumBatch {
  SeqSumJob job[4];
  int count;
};
size_t seqsum_chunks(size_t n);  // work units of one sum of n terms
size_t seqsum_scratch_bytes(size_t n_max, int jobs);
void launch_seqsum(cudaStream_t st, const SeqSumBatch &B, void *scratch);
// Many sums from a device table: first[j] = sum over earlier jobs of seqsum_chunks(n),
// first[count] = total_chunks (device array of count + 1).
size_t seqsum_table_scratch_bytes(long long total_chunks);
void launch_seqsum_table(cudaStream_t st, const SeqSumJob *jobs, const long long *first, int count,
                         long long total_chunks, void *scratch);

// ---- Jacobi eigensolver (kernels_jacobi.cu): one block per matrix of order <= kJacobiMax ----
constexpr int kJacobiMax = 112;  // largest order: two n x (n + 1) tiles fit in shared memory
constexpr int kJacobiThreads = 512;
struct JacobiJob {
  double *slot;   // np x np: the symmetric matrix in, its eigenvectors (rows, ascending) out
  double *eps;    // np eigenvalues out (padding rows get `pad`)
  double *basis;  // np x np: the previous eigenvectors (rows), used when warm, updated
  int *info;      // 0 solved; 1 off-diagonal part still above 1e-12 of the diagonal after the
                  // last sweep; 2 non-finite
  int n, np;
};
size_t jacobi_smem(int n);
void prepare_jacobi_eigen(int max_n);  // shared-memory attribute on the current device
void launch_jacobi_eigen(cudaStream_t st, const JacobiJob *jobs, int count, int max_n, int warm, double pad);

// ---- corrections (kernels_corr.cu) ----
// out[0] dispersion, out[1] H-bond, out[2] C#C, out[3] Si-O-H, out[4] PM7-HH (kcal/mol).
void launch_corrections(cudaStream_t st, int n_atoms, const int *z, const double *xyz, int method, int smooth,
                        double *scratch, size_t scratch_len, double *out);
size_t corrections_scratch(int n_atoms);

}  // namespace pm7

namespace pm7 {
void launch_stage_pair(cudaStream_t st, const DeviceParams &P, int zi, int zj, const double d[3], double *w,
                       double *e1b, double *e2a, double *s, int *np_out, int *status);
}

namespace pm7 {
// Device-side SP2 control: every step kernel gets its step index and does nothing once
// an earlier step has stopped the purification (state[kSp2Stop] = that step), so steps
// can be queued in chunks without a host round trip per step.
enum Sp2State {
  kSp2TrX = 0, kSp2TrX2 = 1, kSp2Square = 2, kSp2Err = 3,  // traces, branch, tr X - tr X^2
  kSp2Stop = 4,                                            // step at which it stopped (1e9: running)
  kSp2Ok = 5,                                              // 1: converged, 0: failed
  kSp2Ring = 6,                                            // errors of the last three steps
  kSp2Parts = 9,                                           // trace partials of the current iterate
  kSp2Len = 12
};
// Stopping rule of one purification: converged when |err| <= tol_done, or at the rounding
// floor when |err| < tol_floor and no smaller than two steps before; failed on a
// non-finite error or after max_steps.
struct Sp2Rule {
  double tol_done, tol_floor;
  int max_steps;
};
}

namespace pm7 {
// FP64-accuracy SP2 squarings on the tcgen05 integer tensor cores (kernels_i8.cu): the
// iterate in fp64 (n x n) and as eight int8 digit planes (sp2_i8_digit_bytes(n) bytes, rows of
// sp2_i8_ld(n) bytes) whose two tensor maps (128-byte opaque CUtensorMap each) come from
// make_digit_maps. launch_sp2_step_i8 is the fused step of launch_sp2_step (same state, step
// and partial protocol) reading x_in and its planes, writing x_out and its planes; `error`:
// 1 a pipeline wait expired, 2 an element left the digits' range. launch_sp2_digits splits X
// into planes (step < 0: unconditionally; else only while that step is active).
int sp2_i8_ld(int n);
size_t sp2_i8_digit_bytes(int n);
int sp2_i8_tiles(int n);
bool make_digit_maps(const int8_t *dig, int n, void *map_a, void *map_b);
void prepare_i8_kernels();
void launch_sp2_digits(cudaStream_t st, int n, const double *X, int8_t *dig, const double *state, int step,
                       int *error);
void launch_sp2_step_i8(cudaStream_t st, int n, const void *map_a, const void *map_b, const double *x_in,
                        double *x_out, int8_t *dig_out, double *state, double *parts, int step, int *error);
}  // namespace pm7

namespace pm7 {
// FP32-accuracy (3xTF32) symmetric squaring on tcgen05 (kernels_tf32.cu). Matrices are
// ld x ld fp32, ld a multiple of 32, zero padded beyond n; the maps come from
// make_square_map (an opaque 128-byte CUtensorMap each).
bool make_square_map(const float *base, int ld, void *map_out);
// Sets the tcgen05 kernels' shared-memory attributes on the current device (idempotent).
void prepare_tf32_kernels();
size_t square_tf32x3_smem();
// state/step: as the fp64 SP2 steps (state may be null: always runs). drill != 0: the failure
// drill, the copy producer withholds every copy so each pipeline wait runs out its time limit
// and the kernel sets *error and returns.
void launch_square_tf32x3(cudaStream_t st, int n, int ld, const void *map_hi, const void *map_lo, float *C,
                          int *error, const double *state = nullptr, int step = 0, int drill = 0);
// C = A B for symmetric A, B given as split tensor maps (all 128x128 tiles, no mirror).
void launch_product_tf32x3(cudaStream_t st, int n, int ld, const void *a_hi, const void *a_lo, const void *b_hi,
                           const void *b_lo, float *C, int *error);
void launch_split_tf32(cudaStream_t st, int n, int ld, const double *X, float *hi, float *lo);
void launch_widen(cudaStream_t st, int n, int ld, const float *C32, double *C);
// The fp32 SP2 iteration: start, traces (fp64 sums), update with re-split, density.
void launch_sp2_init32(cudaStream_t st, int n, int ld, const double *F, const double *bounds, float *X, float *hi,
                       float *lo);
void launch_sp2_trace32(cudaStream_t st, int n, int ld, const float *X, const float *X2, double n_occ, double *state,
                        int step, Sp2Rule rule);
void launch_sp2_update32(cudaStream_t st, int n, int ld, float *X, const float *X2, const double *state, float *hi,
                         float *lo, int step);
void launch_sp2_density32(cudaStream_t st, int n, int ld, const float *X, double w, double *P);
}

namespace pm7 {
// SP2 purification building blocks (kernels_dense.cu).
void launch_gershgorin(cudaStream_t st, int n, const double *F, double *scratch, double *bounds);
void launch_sp2_init(cudaStream_t st, int n, const double *F, const double *bounds, double *X);
// Lanczos refinement of the SP2 interval in bounds[0..1] (which holds the Gershgorin one):
// kLzSteps steps on F, workspace lanczos_doubles(n). Matrices below 2 kLzSteps keep the
// Gershgorin interval.
constexpr int kLzSteps = 16;
size_t lanczos_doubles(int n);
void launch_lanczos_bounds(cudaStream_t st, int n, const double *F, double *lz, double *bounds);
void launch_sp2_reset(cudaStream_t st, double *state);
void launch_sp2_square(cudaStream_t st, int n, const double *X, double *X2, const double *state, int step);
void launch_sp2_trace(cudaStream_t st, int n, const double *X, const double *X2, double n_occ, double *state, int step,
                      Sp2Rule rule);
void launch_sp2_update(cudaStream_t st, int n, double *X, const double *X2, const double *state, int step);
// The fused SP2 iteration on a ping-pong pair: launch_sp2_norms gives the starting iterate's
// trace partials; per step, launch_sp2_decide turns the current partials into the branch and
// the stopping rule, and launch_sp2_step writes the next iterate Y = X^2 or 2X - X^2 (the
// squaring's epilogue applies the branch) with its own partials. `parts` holds
// sp2_parts_doubles(n) doubles.
size_t sp2_parts_doubles(int n);
void launch_sp2_norms(cudaStream_t st, int n, const double *X, double *state, double *parts);
void launch_sp2_decide(cudaStream_t st, double n_occ, double *state, const double *parts, int step, Sp2Rule rule);
void launch_sp2_step(cudaStream_t st, int n, const double *X, double *Y, double *state, double *parts, int step);
}

namespace pm7 {
// Eigenvalues of symmetric matrices, no eigenvectors (kernels_eig.cu): Householder
// tridiagonalisation with one thread-block cluster per matrix, then Sturm multisection.
constexpr int kTriPanel = 32;       // reflectors per panel
constexpr int kTriMaxCluster = 16;  // CTAs per matrix at most
constexpr int kTriMaxN = 4096;      // largest order accepted

struct EigvalsTask {
  const double *src;  // n x n symmetric, row-major, leading dimension ld; read only
  double *a;          // workspace (eigvals_task_layout): n x n copy, panel vectors, ...
  double *V, *W;      // panel vectors of all rows, n x kTriPanel each
  double *vec, *part; // e^2 (n); Gershgorin interval and pivot floor (3)
  double *d, *e;      // the tridiagonal matrix
  double *eps;        // n eigenvalues, ascending (output)
  int n, ld;
};

// Doubles of workspace one task of order n needs; eigvals_task_layout carves it.
size_t eigvals_work_doubles(int n);
void eigvals_task_layout(EigvalsTask &t, double *work);
// CTAs per matrix for order n (1 .. 16; 8 at most where 16-CTA clusters cannot run).
int tridiag_cluster_size(int n);
// Whether order n runs here (order and the per-CTA shared memory it needs); larger
// matrices go to the library eigensolver.
bool eigvals_supported(int n);
// All tasks share one cluster size; prefix[t] = sum of the orders of tasks before t,
// total = sum of all orders (device arrays / values). Returns the launch status.
cudaError_t launch_eigvals(cudaStream_t st, const EigvalsTask *tasks, int n_tasks, int cluster, int max_n,
                           const int *prefix, int total);
}
