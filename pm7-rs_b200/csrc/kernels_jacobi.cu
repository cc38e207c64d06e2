// Cyclic Jacobi eigensolver in shared memory, one thread block per symmetric matrix of
// order n <= kJacobiMax, eigenvectors and eigenvalues. Used wherever a matrix that small is
// diagonalised on the SCF path: the plain SCF of a small molecule, the batch's small
// molecules and the divide-and-conquer subsystems; it replaces, for those orders,
// `symmetric_eigen` (pm7-rs src/linalg.rs:231-278, faer's self_adjoint_eigen).
//
// A Fock matrix changes little from one SCF iteration to the next, so the previous
// iteration's eigenvectors W nearly diagonalise it: with `warm` the kernel forms W F W^T and
// runs parallel cyclic Jacobi sweeps (round-robin pairing, n'/2 disjoint rotations per round,
// the classical rotation of Golub & Van Loan, sym.schur2) on that, which converges in a few
// sweeps, and accumulates the rotations into W; cold, it starts from the identity. Sweeps
// stop when the off-diagonal part falls below 1e-15 of the diagonal (Frobenius norms), or
// after kJacSweeps; the job's info word then says whether it converged. Eigenvalues are
// sorted ascending (ties by index) and the eigenvectors written as rows of the np x np slot
// (zero padding; padding eigenvalues `pad`).
#include <cuda_runtime.h>

#include <cmath>

#include "engine_internal.hpp"
#include "kernels.hpp"

namespace pm7 {
namespace {

__device__ __forceinline__ double jac_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block sum in a fixed order (warps, then warp 0 over the warp sums); result in thread 0.
__device__ double block_sum(double v, double *sh) {
  v = jac_warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    t = jac_warp_sum(t);
  }
  __syncthreads();
  return t;
}

constexpr int kJacSweeps = 24;


__global__ void __launch_bounds__(kJacobiThreads) k_jacobi(const JacobiJob *__restrict__ jobs, int warm, double pad) {
  extern __shared__ double jsm[];
  __shared__ double cc[kJacobiMax / 2 + 1], ss[kJacobiMax / 2 + 1], red[32];
  __shared__ int pp[kJacobiMax / 2 + 1], qq[kJacobiMax / 2 + 1], rk[kJacobiMax], inv[kJacobiMax];
  __shared__ int done;
  const JacobiJob jb = jobs[blockIdx.x];
  const int n = jb.n, np = jb.np, ld = n + 1;
  if (n <= 0 || n > kJacobiMax) return;
  double *A = jsm, *W = jsm + (size_t)n * ld;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, k = e % n;
    W[i * ld + k] = warm ? jb.basis[(size_t)i * np + k] : (i == k ? 1.0 : 0.0);
  }
  __syncthreads();
  if (warm) {
    // T = F W^T (F read from the slot) into A, then W T back into the slot
    for (int e = tid; e < n * n; e += nt) {
      const int k = e / n, j = e % n;
      const double *f = jb.slot + (size_t)k * np;
      double t = 0.0;
      for (int l = 0; l < n; ++l) t += f[l] * W[j * ld + l];
      A[k * ld + j] = t;
    }
    __syncthreads();
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e % n;
      double t = 0.0;
      for (int k = 0; k < n; ++k) t += W[i * ld + k] * A[k * ld + j];
      jb.slot[(size_t)i * np + j] = t;
    }
    __syncthreads();
  }
  for (int e = tid; e < n * n; e += nt) {  // symmetric part
    const int i = e / n, j = e % n;
    A[i * ld + j] = 0.5 * (jb.slot[(size_t)i * np + j] + jb.slot[(size_t)j * np + i]);
  }
  __syncthreads();
  const int m = (n % 2 == 0) ? n - 1 : n;  // rotating indices 1..m around the fixed index 0
  const int half = (m + 1) / 2;            // rotations per round
  for (int sweep = 0; sweep < kJacSweeps; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e % n;
      const double v = A[i * ld + j];
      if (i == j) dia += v * v;
      else off += v * v;
    }
    off = block_sum(off, red);
    dia = block_sum(dia, red);
    if (tid == 0) done = !(off > 1.0e-30 * dia);
    __syncthreads();
    if (done) break;
    for (int r = 0; r < m; ++r) {
      for (int k = tid; k < half; k += nt) {
        int p = k == 0 ? 0 : (r + k) % m + 1, q = k == 0 ? r + 1 : (r - k + m) % m + 1;
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, s = 0.0;
        if (q < n) {  // index n is the odd order's idle slot
          const double apq = A[p * ld + q];
          if (apq != 0.0) {
            const double tau = (A[q * ld + q] - A[p * ld + p]) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        pp[k] = p;
        qq[k] = q;
        cc[k] = c;
        ss[k] = s;
      }
      __syncthreads();
      for (int e = tid; e < half * n; e += nt) {  // A <- A J
        const int k = e / n, i = e % n, p = pp[k], q = qq[k];
        if (q >= n) continue;
        const double ap = A[i * ld + p], aq = A[i * ld + q];
        A[i * ld + p] = cc[k] * ap - ss[k] * aq;
        A[i * ld + q] = ss[k] * ap + cc[k] * aq;
      }
      __syncthreads();
      for (int e = tid; e < half * n; e += nt) {  // A <- J^T A, W <- J^T W
        const int k = e / n, j = e % n, p = pp[k], q = qq[k];
        if (q >= n) continue;
        const double ap = A[p * ld + j], aq = A[q * ld + j];
        A[p * ld + j] = cc[k] * ap - ss[k] * aq;
        A[q * ld + j] = ss[k] * ap + cc[k] * aq;
        const double wp = W[p * ld + j], wq = W[q * ld + j];
        W[p * ld + j] = cc[k] * wp - ss[k] * wq;
        W[q * ld + j] = ss[k] * wp + cc[k] * wq;
      }
      __syncthreads();
    }
  }
  {
    // convergence and finiteness of what is handed on
    double off = 0.0, dia = 0.0;
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e % n;
      const double v = A[i * ld + j];
      if (i == j) dia += v * v;
      else off += v * v;
    }
    off = block_sum(off, red);
    dia = block_sum(dia, red);
    if (tid == 0) *jb.info = !(isfinite(off) && isfinite(dia)) ? 2 : (off > 1.0e-24 * dia ? 1 : 0);
  }
  for (int i = tid; i < n; i += nt) {  // a total order (NaN last), so the ranks are a permutation
    const double vi = A[i * ld + i], v = vi == vi ? vi : INFINITY;
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const double uj = A[j * ld + j], u = uj == uj ? uj : INFINITY;
      r += (u < v) || (u == v && j < i);
    }
    rk[i] = r;
  }
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    inv[rk[i]] = i;
    jb.eps[rk[i]] = A[i * ld + i];
  }
  for (int i = n + tid; i < np; i += nt) jb.eps[i] = pad;
  __syncthreads();
  for (int e = tid; e < np * np; e += nt) {
    const int r = e / np, k = e % np;
    const double v = (r < n && k < n) ? W[inv[r] * ld + k] : 0.0;
    jb.slot[e] = v;
    jb.basis[e] = v;
  }
}

}  // namespace

size_t jacobi_smem(int n) { return sizeof(double) * 2 * (size_t)n * (n + 1); }

void prepare_jacobi_eigen(int max_n) {
  CUDA_OK(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)jacobi_smem(max_n)));
}

void launch_jacobi_eigen(cudaStream_t st, const JacobiJob *jobs, int count, int max_n, int warm, double pad) {
  if (count <= 0) return;
  k_jacobi<<<(unsigned)count, kJacobiThreads, jacobi_smem(max_n), st>>>(jobs, warm, pad);
  note_launch();
}

}  // namespace pm7
