// Eigenvalues of symmetric matrices without eigenvectors, many matrices per launch.
//
// The reported MO energies and HOMO/LUMO (pm7-rs src/scf.rs:757-823) need the spectrum of
// the final Fock matrix; the reference takes it from a full eigendecomposition
// (src/linalg.rs:231-278). When no orbitals are returned, only eigenvalues are needed:
//
//  1. k_tridiag: Householder reduction to tridiagonal form, one thread-block cluster
//     of C CTAs per matrix (C = 1 .. 16 by size). Blocked as LAPACK's dsytrd/dlatrd
//     (lower): panels of 32 reflectors whose two-sided update is applied to the trailing
//     matrix once per panel; inside a panel the symmetric matrix-vector product uses the
//     panel-start matrix corrected by the panel's V and W. Rows are dealt cyclically to
//     the CTAs and every matrix row is read and written only by its owner, so the only
//     cross-CTA traffic is the vectors v, p, the current column and fixed per-CTA partial
//     sums, synchronised by hardware cluster barriers (three per column, two per panel).
//  2. k_tri_eigs: all eigenvalues of the tridiagonal matrices, one warp per eigenvalue:
//     multisection on the Sturm count (32 points per round, the interval shrinking 33x
//     per round) until the bracket is a few ulps wide.
//
// Every sum is taken in a fixed order (fixed warp-shuffle trees, partials summed by CTA
// rank), so results are bitwise reproducible for equal input.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "kernels.hpp"

namespace cg = cooperative_groups;

namespace pm7 {

namespace {
constexpr int NB = kTriPanel;          // reflectors per panel
constexpr int THREADS = 1024;          // per CTA
constexpr int WARPS = THREADS / 32;
constexpr int SV = NB + 4;             // shared row stride of the own rows' V and W
constexpr int TT = 64, TLD = 68;       // trailing-update tile edge and its shared row stride
// per-CTA partial slots: [0] sigma, [1] p.v, [2 .. 2+2NB) V^T v and W^T v
constexpr int P_SIG = 0, P_PTV = 1, P_YZ = 2, P_LEN = 2 + 2 * NB;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of one value per thread over the CTA, fixed order; the result in every thread.
__device__ __forceinline__ double block_sum(double v, double *red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double s = lane < WARPS ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0) red[WARPS] = s;
  }
  __syncthreads();
  return red[WARPS];
}

__device__ __forceinline__ void dmma16x8x8(double *d, const double *a, const double *b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Shared-memory plan of one CTA (doubles): the gathered v (nmax), the own rows' V and W
// panels (rmax x SV each), the own rows' v, p, current column and captured next column
// (rmax each), this CTA's partial sums, row j of V and W, V^T v | W^T v, the reduction
// scratch and one trailing-update tile.
struct TriSmem {
  double *vs, *Vs, *Ws, *vl, *pl, *cl, *cn, *pt, *rowj, *yz, *red, *tB;
  __host__ __device__ static size_t doubles(int nmax, int rmax) {
    return (size_t)nmax + 2 * (size_t)rmax * SV + 4 * (size_t)rmax + P_LEN + 4 * NB + (WARPS + 2) + TT * TLD;
  }
  __device__ TriSmem(double *sm, int nmax, int rmax) {
    vs = sm;
    Vs = vs + nmax;
    Ws = Vs + (size_t)rmax * SV;
    vl = Ws + (size_t)rmax * SV;
    pl = vl + rmax;
    cl = pl + rmax;
    cn = cl + rmax;
    pt = cn + rmax;
    rowj = pt + P_LEN;
    yz = rowj + 2 * NB;
    red = yz + 2 * NB;
    tB = red + WARPS + 2;
  }
};
}  // namespace

// Rows are dealt cyclically: CTA r of C owns rows i = r + m C, m = 0 .. cnt-1 (local
// index m). Everything a CTA keeps per own row lives in its shared memory; another CTA
// reads it through distributed shared memory (cluster.map_shared_rank). Matrix rows are
// read and written only by their owner, in global memory (L2-resident at these sizes).
__global__ void __launch_bounds__(THREADS, 1) k_tridiag(const EigvalsTask *__restrict__ tasks, int C, int nmax,
                                                         int rmax) {
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const EigvalsTask T = tasks[blockIdx.x / C];
  const int n = T.n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  extern __shared__ __align__(16) double sm[];
  const TriSmem S(sm, nmax, rmax);
  double *a = T.a;
  const int cnt = n > r ? (n - r + C - 1) / C : 0;  // own rows
  auto m_of = [&](int i0) { return i0 <= r ? 0 : (i0 - r + C - 1) / C; };  // first own local row >= i0
  // sum over the cluster of partial slot `slot`: lane q reads CTA q's value (fixed tree)
  auto part_sum = [&](int slot) {
    double v = 0.0;
    if (lane < C) v = cluster.map_shared_rank(S.pt, lane)[slot];
    return warp_sum(v);
  };

  for (int m = warp; m < cnt; m += WARPS) {
    const int i = r + m * C;
    for (int k = lane; k < n; k += 32) a[(size_t)i * n + k] = T.src[(size_t)i * T.ld + k];
  }

  double tau_prev = 0.0;
  for (int j0 = 0; j0 < n - 1; j0 += NB) {
    const int jb = min(NB, n - 1 - j0);
    for (int jj = 0; jj < jb; ++jj) {
      const int j = j0 + jj;
      // ---- A: finish W[., jj-1]; column j corrected by the panel so far
      double gamma = 0.0;
      if (jj > 0) {
        gamma = -0.5 * tau_prev * part_sum(P_PTV);
        for (int m = m_of(j) + tid; m < cnt; m += THREADS) S.Ws[m * SV + jj - 1] = S.pl[m] + gamma * S.vl[m];
      }
      if (tid < jj) {
        const int oj = j % C, mj = j / C;
        S.rowj[tid] = cluster.map_shared_rank(S.Vs, oj)[mj * SV + tid];
        S.rowj[NB + tid] = tid == jj - 1
                               ? cluster.map_shared_rank(S.pl, oj)[mj] + gamma * cluster.map_shared_rank(S.vl, oj)[mj]
                               : cluster.map_shared_rank(S.Ws, oj)[mj * SV + tid];
      }
      __syncthreads();
      double sig = 0.0;
      for (int m = m_of(j) + warp; m < cnt; m += WARPS) {
        const int i = r + m * C;
        double s = 0.0;
        if (lane < jj) s = S.Vs[m * SV + lane] * S.rowj[NB + lane] + S.Ws[m * SV + lane] * S.rowj[lane];
        s = warp_sum(s);
        if (lane == 0) {
          const double col = (jj == 0 ? a[(size_t)i * n + j] : S.cn[m]) - s;
          if (i == j) {
            T.d[j] = col;
          } else {
            S.cl[m] = col;
            if (i >= j + 2) sig += col * col;
          }
        }
      }
      sig = block_sum(sig, S.red);
      if (tid == 0) S.pt[P_SIG] = sig;
      cluster.sync();
      // ---- B: the reflector H = I - tau v v^T with v[j+1] = 1 (LAPACK dlarfg)
      const double sigma = part_sum(P_SIG);
      const double alpha = cluster.map_shared_rank(S.cl, (j + 1) % C)[(j + 1) / C];
      double tau = 0.0, beta = alpha, scale = 0.0;
      if (sigma > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
        tau = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
      }
      if (r == 0 && tid == 0) T.e[j] = beta;
      for (int m = m_of(j + 1) + tid; m < cnt; m += THREADS) {
        const double v = r + m * C == j + 1 ? 1.0 : S.cl[m] * scale;
        S.vl[m] = v;
        S.Vs[m * SV + jj] = v;
      }
      __syncthreads();
      for (int q = warp; q < 2 * jj; q += WARPS) {  // one warp per V^T v / W^T v entry
        const double *M = q < jj ? S.Vs : S.Ws;
        const int c = q < jj ? q : q - jj;
        double s = 0.0;
        for (int m = m_of(j + 1) + lane; m < cnt; m += 32) s += M[m * SV + c] * S.vl[m];
        s = warp_sum(s);
        if (lane == 0) S.pt[P_YZ + q] = s;
      }
      cluster.sync();
      // ---- C: p = tau (A - V W^T - W V^T) v over the trailing rows
      for (int k = j + 1 + tid; k < n; k += THREADS) S.vs[k] = cluster.map_shared_rank(S.vl, k % C)[k / C];
      for (int q = warp; q < 2 * jj; q += WARPS) {
        const double s = part_sum(P_YZ + q);
        if (lane == 0) S.yz[q] = s;
      }
      __syncthreads();
      double ptv = 0.0;
      for (int m = m_of(j + 1) + warp; m < cnt; m += WARPS) {
        const int i = r + m * C;
        const double *ai = a + (size_t)i * n;
        if (lane == 0) S.cn[m] = ai[j + 1];  // the next column of this row, for its step A
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, s5 = 0.0, s6 = 0.0, s7 = 0.0;
        int k = j + 1 + lane;
        for (; k + 224 < n; k += 256) {
          const double x0 = ai[k], x1 = ai[k + 32], x2 = ai[k + 64], x3 = ai[k + 96];
          const double x4 = ai[k + 128], x5 = ai[k + 160], x6 = ai[k + 192], x7 = ai[k + 224];
          s0 += x0 * S.vs[k];
          s1 += x1 * S.vs[k + 32];
          s2 += x2 * S.vs[k + 64];
          s3 += x3 * S.vs[k + 96];
          s4 += x4 * S.vs[k + 128];
          s5 += x5 * S.vs[k + 160];
          s6 += x6 * S.vs[k + 192];
          s7 += x7 * S.vs[k + 224];
        }
        for (; k < n; k += 32) s0 += ai[k] * S.vs[k];
        double s = ((s0 + s1) + (s2 + s3)) + ((s4 + s5) + (s6 + s7));
        if (lane < jj) s -= S.Vs[m * SV + lane] * S.yz[jj + lane] + S.Ws[m * SV + lane] * S.yz[lane];
        s = warp_sum(s);
        if (lane == 0) {
          const double p = tau * s;
          S.pl[m] = p;
          ptv += p * S.vl[m];
        }
      }
      ptv = block_sum(ptv, S.red);
      if (tid == 0) S.pt[P_PTV] = ptv;
      cluster.sync();
      tau_prev = tau;
    }
    // ---- end of panel: last W column; own V and W rows to global for everyone's update
    const int t0 = j0 + jb, mt = m_of(t0);
    {
      const double gamma = -0.5 * tau_prev * part_sum(P_PTV);
      for (int m = mt + tid; m < cnt; m += THREADS) S.Ws[m * SV + jb - 1] = S.pl[m] + gamma * S.vl[m];
    }
    __syncthreads();
    for (int e = tid; e < (cnt - mt) * NB; e += THREADS) {
      const int m = mt + e / NB, c = e % NB;
      const size_t i = (size_t)(r + m * C);
      T.V[i * NB + c] = c < jb ? S.Vs[m * SV + c] : 0.0;
      T.W[i * NB + c] = c < jb ? S.Ws[m * SV + c] : 0.0;
    }
    cluster.sync();
    // A -= V W^T + W V^T on own rows x columns >= t0, per 64 x 64 tile on FP64 tensor cores:
    // D = [V_i | W_i] [W_k | V_k]^T (inner dimension 2 NB, zero past jb).
    const int fm = (warp >> 3) * 16, fn = (warp & 7) * 8, g = lane >> 2, t = lane & 3;
    for (int mb = mt; mb < cnt; mb += TT) {
      for (int kb = t0; kb < n; kb += TT) {
        __syncthreads();  // previous tile consumed
        for (int e = tid; e < TT * 2 * NB; e += THREADS) {
          const int q = e / (2 * NB), c = e % (2 * NB), k = kb + q;
          double v = 0.0;
          if (k < n) v = c < NB ? __ldcg(T.W + (size_t)k * NB + c) : __ldcg(T.V + (size_t)k * NB + c - NB);
          S.tB[q * TLD + c] = v;
        }
        __syncthreads();
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        const int m0 = mb + fm + g, m1 = m0 + 8;
#pragma unroll
        for (int c0 = 0; c0 < 2 * NB; c0 += 8) {
          const double *P = c0 < NB ? S.Vs : S.Ws;
          const int cc = (c0 % NB) + t;
          const bool k0 = cc < jb, k1 = cc + 4 < jb;
          const double av[4] = {m0 < cnt && k0 ? P[m0 * SV + cc] : 0.0, m1 < cnt && k0 ? P[m1 * SV + cc] : 0.0,
                                m0 < cnt && k1 ? P[m0 * SV + cc + 4] : 0.0, m1 < cnt && k1 ? P[m1 * SV + cc + 4] : 0.0};
          const double bv[2] = {S.tB[(fn + g) * TLD + c0 + t], S.tB[(fn + g) * TLD + c0 + t + 4]};
          dmma16x8x8(acc, av, bv);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int m = mb + fm + g + (q >> 1) * 8, k = kb + fn + 2 * t + (q & 1);
          if (m < cnt && k < n) a[(size_t)(r + m * C) * n + k] -= acc[q];
        }
      }
    }
  }
  if (r == (n - 1) % C && tid == 0) T.d[n - 1] = a[(size_t)(n - 1) * n + n - 1];
  cluster.sync();
  // Gershgorin interval, pivot floor and squared off-diagonal for the Sturm counts
  if (r == 0) {
    double lo = 1e300, hi = -1e300, emax = 0.0;
    for (int i = tid; i < n; i += THREADS) {
      const double el = i > 0 ? fabs(__ldcg(T.e + i - 1)) : 0.0, er = i < n - 1 ? fabs(__ldcg(T.e + i)) : 0.0;
      const double di = __ldcg(T.d + i);
      lo = fmin(lo, di - el - er);
      hi = fmax(hi, di + el + er);
      emax = fmax(emax, er * er);
      if (i < n - 1) T.vec[i] = __ldcg(T.e + i) * __ldcg(T.e + i);  // e^2
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    }
    __syncthreads();
    if (lane == 0) {
      S.tB[warp] = lo;
      S.tB[WARPS + warp] = hi;
      S.tB[2 * WARPS + warp] = emax;
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < WARPS; ++w) {
        lo = fmin(lo, S.tB[w]);
        hi = fmax(hi, S.tB[WARPS + w]);
        emax = fmax(emax, S.tB[2 * WARPS + w]);
      }
      const double tnorm = fmax(fabs(lo), fabs(hi));
      const double pivmin = 2.2250738585072014e-308 * fmax(1.0, emax) * 16.0;
      const double pad = 2.1 * n * 2.220446049250313e-16 * tnorm + 4.0 * pivmin;
      T.part[0] = lo - pad;
      T.part[1] = hi + pad;
      T.part[2] = pivmin;
    }
  }
}

// Number of eigenvalues of the tridiagonal (d, e^2) below x (Sturm count with a pivot
// floor, LAPACK dlaebz's recurrence).
__device__ __forceinline__ int sturm_count(const double *__restrict__ d, const double *__restrict__ e2, int n, double x,
                                           double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int c = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    c += q < 0.0;
  }
  return c;
}

// One warp per eigenvalue; item w of the launch is eigenvalue w - prefix[t] of task t.
__global__ void __launch_bounds__(256) k_tri_eigs(const EigvalsTask *__restrict__ tasks,
                                                  const int *__restrict__ prefix, int n_tasks, int total) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= total) return;
  int lo_t = 0, hi_t = n_tasks - 1;
  while (lo_t < hi_t) {
    const int mid = (lo_t + hi_t + 1) >> 1;
    if (prefix[mid] <= w) lo_t = mid;
    else hi_t = mid - 1;
  }
  const EigvalsTask &T = tasks[lo_t];
  const int k = w - prefix[lo_t], n = T.n;
  const double *d = T.d, *e2 = T.vec;
  double lo = T.part[0], hi = T.part[1];
  const double pivmin = T.part[2];
  for (int round = 0; round < 40; ++round) {
    const double tol = 4.0 * 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)) + pivmin;
    if (hi - lo <= tol) break;
    const double x = lo + (hi - lo) * (double)(lane + 1) * (1.0 / 33.0);
    const int cnt = sturm_count(d, e2, n, x, pivmin);
    const unsigned above = __ballot_sync(0xffffffffu, cnt > k);
    const int f = above ? __ffs(above) - 1 : 32;
    const double xl = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
    const double xh = __shfl_sync(0xffffffffu, x, f < 32 ? f : 31);
    if (f > 0) lo = xl;
    if (f < 32) hi = xh;
  }
  if (lane == 0) T.eps[k] = 0.5 * (lo + hi);
}

constexpr int kSmemMax = 232448;  // opt-in shared memory per CTA on sm_100a (227 KB)

static int cluster_cap() {
  static std::mutex mu;
  static int cap[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 8;
  std::lock_guard<std::mutex> lock(mu);
  if (cap[dev] == 0) {
    // attributes are per device: set them with the device current
    cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemMax);
    // 16-CTA clusters are a non-portable size: use them only where they can be scheduled
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = kSmemMax;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 16;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    const cudaError_t err = cudaOccupancyMaxActiveClusters(&clusters, k_tridiag, &cfg);
    if (err != cudaSuccess) cudaGetLastError();
    cap[dev] = (err == cudaSuccess && clusters > 0) ? 16 : 8;
  }
  return cap[dev];
}

static size_t smem_bytes(int nmax, int C) {
  const int rmax = (nmax + C - 1) / C;
  return sizeof(double) * TriSmem::doubles(nmax, rmax);
}

int tridiag_cluster_size(int n) {
  const int cap = cluster_cap();
  int c = 1;
  while (c < cap && c * 128 <= n) c *= 2;
  return c;
}

bool eigvals_supported(int n) {
  return n >= 1 && n <= kTriMaxN && smem_bytes(n, tridiag_cluster_size(n)) <= (size_t)kSmemMax;
}

size_t eigvals_work_doubles(int n) { return (size_t)n * n + 2 * (size_t)n * NB + 3 * (size_t)n + 8; }

void eigvals_task_layout(EigvalsTask &t, double *work) {
  const size_t n = t.n;
  t.a = work;
  t.V = t.a + n * n;
  t.W = t.V + n * NB;
  t.vec = t.W + n * NB;  // e^2 for the Sturm counts
  t.d = t.vec + n;
  t.e = t.d + n;
  t.part = t.e + n;      // Gershgorin interval and pivot floor
}

cudaError_t launch_eigvals(cudaStream_t st, const EigvalsTask *tasks, int n_tasks, int cluster, int max_n,
                           const int *prefix, int total) {
  if (n_tasks <= 0) return cudaSuccess;
  const size_t smem = smem_bytes(max_n, cluster);
  if (max_n > kTriMaxN || cluster < 1 || cluster > kTriMaxCluster || smem > (size_t)kSmemMax)
    return cudaErrorInvalidValue;
  cluster_cap();  // attributes set once per device
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n_tasks * cluster);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cluster;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const int rmax = (max_n + cluster - 1) / cluster;
  cudaError_t err = cudaLaunchKernelEx(&cfg, k_tridiag, tasks, cluster, max_n, rmax);
  note_launch();
  if (err != cudaSuccess) return err;
  const int threads = 256, warps_per_block = threads / 32;
  k_tri_eigs<<<(total + warps_per_block - 1) / warps_per_block, threads, 0, st>>>(tasks, prefix, n_tasks, total);
  note_launch();
  return cudaGetLastError();
}

}  // namespace pm7
