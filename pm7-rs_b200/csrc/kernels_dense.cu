// Dense FP64 algebra of the SCF loop: the tensor-core contractions (density
// P = w V_occ^T V_occ and the DIIS commutator F P) and the HBM-bound reductions
// around them. All reductions write fixed per-block partials that are summed in a
// fixed order, so results are bitwise reproducible.
#include <algorithm>
#include <cuda_runtime.h>

#include "common.cuh"
#include "batch.hpp"
#include "kernels.hpp"
#include "autotune.hpp"

namespace pm7 {

// ---------------------------------------------------------------------------
// FP64 tensor-core GEMM, C = alpha * A^T * B (A: K x M, B: K x N, both row-major).
// DMMA (mma.sync .f64, here the m16n8k8 shape) is the FP64 tensor-core instruction on
// sm_100a; tcgen05 has no FP64 kind. Block tiles BM x BN x 16 over 4 warps, a
// three-stage cp.async ring in dynamic shared memory. Shared rows are BM + 4 (BN + 4)
// doubles long, so the fragment loads of a half-warp (4 k-rows x 4 columns) hit 16
// distinct bank pairs; tiles move in 16-byte copies when the leading dimensions are
// even and the bases 16-byte aligned, else in 8-byte copies. Out-of-range elements are
// zero-filled by the copy itself, so K and M/N edges need no separate masking.
// Two shapes: 64x64 (warp tile 32x32, four CTAs per SM) for full products, and 128x64
// (warp tile 64x32, two CTAs per SM) over an enumerated lower triangle for symmetric
// ones, whose fewer, larger tiles fill the SMs more evenly at nao ~ 2,000.
// ---------------------------------------------------------------------------
namespace {
constexpr int BK = 16, STAGES = 3;
constexpr int BM = 64, BN = 64;  // full-product tile (also the batched kernel's)

template <int TBM, int TBN, int TBK = BK, int TST = STAGES>
struct GemmShape {
  static constexpr int LA = TBM + 4, LB = TBN + 4;
  static constexpr int STAGE = TBK * (LA + LB);         // doubles per stage
  static constexpr int SMEM = TST * STAGE * 8;          // bytes
};
constexpr int GEMM_SMEM = GemmShape<64, 64>::SMEM;       // 52,224 bytes
constexpr int SYM_BM = 128, SYM_BN = 64;
constexpr int SYM_SMEM = GemmShape<SYM_BM, SYM_BN>::SMEM;  // 76,800 bytes
constexpr int SYM_SMEM_K32 = GemmShape<SYM_BM, SYM_BN, 32, 2>::SMEM;  // 102,400 bytes: 32-deep slabs, two stages

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int bytes = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
// 16-byte copy of `bytes` (0, 8 or 16) source bytes, the rest of the 16 zero-filled
__device__ __forceinline__ void cp_async16(double *smem, const double *gmem, int bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D(16x8) += A(16x8) B(8x8), fragments as the PTX ISA lays out .f64 m16n8k8:
// a0 (g, t) a1 (g+8, t) a2 (g, t+4) a3 (g+8, t+4); b0 (t, g) b1 (t+4, g);
// d0 (g, 2t) d1 (g, 2t+1) d2 (g+8, 2t) d3 (g+8, 2t+1), g = lane/4, t = lane%4.
__device__ __forceinline__ void dmma16x8x8(double *d, const double *a, const double *b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// One k-slab (TBK rows) of the A and B tiles into shared memory, 128 threads.
template <int TBM, int TBN, bool VEC, int TBK = BK, int TST = STAGES>
__device__ __forceinline__ void load_stage(double *sA, double *sB, int k0, int m0, int n0, int M, int N, int K,
                                           const double *__restrict__ A, int lda, const double *__restrict__ B,
                                           int ldb) {
  using S = GemmShape<TBM, TBN, TBK, TST>;
  const int tid = threadIdx.x;
  if (VEC) {
#pragma unroll
    for (int e = tid; e < TBK * TBM / 2; e += 128) {
      const int row = e / (TBM / 2), col = (e % (TBM / 2)) * 2, kr = k0 + row;
      const int r = kr < K ? min(max(M - (m0 + col), 0), 2) * 8 : 0;
      cp_async16(sA + row * S::LA + col, r ? A + (size_t)kr * lda + m0 + col : A, r);
    }
#pragma unroll
    for (int e = tid; e < TBK * TBN / 2; e += 128) {
      const int row = e / (TBN / 2), col = (e % (TBN / 2)) * 2, kr = k0 + row;
      const int r = kr < K ? min(max(N - (n0 + col), 0), 2) * 8 : 0;
      cp_async16(sB + row * S::LB + col, r ? B + (size_t)kr * ldb + n0 + col : B, r);
    }
  } else {
#pragma unroll
    for (int e = tid; e < TBK * TBM; e += 128) {
      const int row = e / TBM, col = e % TBM, kr = k0 + row;
      const bool p = kr < K && (m0 + col) < M;
      cp_async8(sA + row * S::LA + col, p ? A + (size_t)kr * lda + m0 + col : A, p);
    }
#pragma unroll
    for (int e = tid; e < TBK * TBN; e += 128) {
      const int row = e / TBN, col = e % TBN, kr = k0 + row;
      const bool p = kr < K && (n0 + col) < N;
      cp_async8(sB + row * S::LB + col, p ? B + (size_t)kr * ldb + n0 + col : B, p);
    }
  }
}
}  // namespace

// The fused SP2 step in a symmetric product's epilogue: with `x` (the squared matrix
// itself, row stride lda), each written element becomes y = X^2 (square) or 2X - X^2, and
// tr Y and |Y|_F^2 (off-diagonal elements counted twice: Y is symmetric) are summed per
// 64 x 64 block (R, C), R >= C, of the lower triangle into parts[2 b], parts[2 b + 1],
// b = R (R + 1) / 2 + C. The order of those sums depends on the element coordinates alone
// (per row over its 32-column warp span in fragment order, the four lanes of a row by a
// fixed shuffle tree, the two spans, then the block's rows in ascending order), so every
// tile shape gives the same bits.
struct Sp2Fuse {
  const double *x;  // null: a plain product
  bool square;
  double *parts;
  double scale;     // written elements are scale * y (2: the final iterate becomes the density)
};

// One TBM x TBN tile, 4 warps as 2 x 2 of (TBM/2) x (TBN/2). sym != 0: only elements
// with m >= n are written, each also mirrored to (n, m), so the output is exactly
// symmetric (P = w V^T V and X X).
template <int TBM, int TBN, bool VEC, int TBK = BK, int TST = STAGES>
__device__ __forceinline__ void gemm_tile_impl(double *smem, int bm, int bn, int M, int N, int K, double alpha,
                                               const double *__restrict__ A, int lda, const double *__restrict__ B,
                                               int ldb, double *__restrict__ C, int ldc, int sym,
                                               const Sp2Fuse &fuse = Sp2Fuse{nullptr, false, nullptr, 1.0}) {
  using S = GemmShape<TBM, TBN, TBK, TST>;
  constexpr int TM = TBM / 2, TN = TBN / 2, FM = TM / 16, FN = TN / 8;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = bm * TBM, n0 = bn * TBN;
  double acc[FM][FN][4];
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

  const int ktiles = (K + TBK - 1) / TBK;
#pragma unroll
  for (int s = 0; s < TST - 1; ++s) {
    if (s < ktiles) {
      double *st = smem + s * S::STAGE;
      load_stage<TBM, TBN, VEC, TBK, TST>(st, st + TBK * S::LA, s * TBK, m0, n0, M, N, K, A, lda, B, ldb);
    }
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<TST - 2>();  // tile kt has landed (this thread's copies)
    __syncthreads();           // ... everyone's, and stage (kt - 1) % TST is free
    const int pf = kt + TST - 1;
    if (pf < ktiles) {
      double *st = smem + (pf % TST) * S::STAGE;
      load_stage<TBM, TBN, VEC, TBK, TST>(st, st + TBK * S::LA, pf * TBK, m0, n0, M, N, K, A, lda, B, ldb);
    }
    cp_async_commit();
    const double *sA = smem + (kt % TST) * S::STAGE;
    const double *sB = sA + TBK * S::LA;
#pragma unroll
    for (int kk = 0; kk < TBK; kk += 8) {
      double a[FM][4], b[FN][2];
#pragma unroll
      for (int i = 0; i < FM; ++i) {
        const double *pa = sA + (kk + t) * S::LA + wm * TM + i * 16 + g;
        a[i][0] = pa[0];
        a[i][1] = pa[8];
        a[i][2] = pa[4 * S::LA];
        a[i][3] = pa[4 * S::LA + 8];
      }
#pragma unroll
      for (int j = 0; j < FN; ++j) {
        const double *pb = sB + (kk + t) * S::LB + wn * TN + j * 8 + g;
        b[j][0] = pb[0];
        b[j][1] = pb[4 * S::LB];
      }
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) dmma16x8x8(acc[i][j], a[i], b[j]);
    }
  }
  cp_async_wait<0>();
  double rtr[FM][2], rsq[FM][2];  // fused step: this thread's part of each of its rows
#pragma unroll
  for (int i = 0; i < FM; ++i) rtr[i][0] = rtr[i][1] = rsq[i][0] = rsq[i][1] = 0.0;
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm * TM + i * 16 + g + (q >> 1) * 8;
        const int n = n0 + wn * TN + j * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        double v = alpha * acc[i][j][q];
        if (!sym) {
          C[(size_t)m * ldc + n] = v;
        } else if (m >= n) {
          if (fuse.x) {
            if (!fuse.square) v = 2.0 * fuse.x[(size_t)m * lda + n] - v;
            if (m == n) {
              rtr[i][q >> 1] += v;
              rsq[i][q >> 1] += v * v;
            } else {
              rsq[i][q >> 1] += 2.0 * (v * v);
            }
          }
          if (fuse.x) v *= fuse.scale;
          C[(size_t)m * ldc + n] = v;
          C[(size_t)n * ldc + m] = v;
        }
      }
  if (fuse.x) {
    static_assert(TN == 32 && TBN == 64, "the fused SP2 sums assume 32-column warp spans of 64-column tiles");
    // the four lanes of a row (t = 0..3) by a fixed tree
#pragma unroll
    for (int i = 0; i < FM; ++i)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int o = 1; o <= 2; o <<= 1) {
          rtr[i][h] += __shfl_xor_sync(0xffffffffu, rtr[i][h], o);
          rsq[i][h] += __shfl_xor_sync(0xffffffffu, rsq[i][h], o);
        }
    __syncthreads();  // the pipeline's shared memory is free again
    double *row_tr = smem, *row_sq = smem + 2 * TBM;  // [span][row of the tile]
    if (t == 0)
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wm * TM + i * 16 + g + 8 * h;
          row_tr[wn * TBM + r] = rtr[i][h];
          row_sq[wn * TBM + r] = rsq[i][h];
        }
    __syncthreads();
    constexpr int NB = TBM / 64;
    if (tid < NB) {
      const int R = m0 / 64 + tid, Cb = n0 / 64;
      if (R >= Cb) {
        double a = 0.0, b = 0.0;
        for (int r = 64 * tid; r < 64 * tid + 64; ++r) {
          a += row_tr[r] + row_tr[TBM + r];
          b += row_sq[r] + row_sq[TBM + r];
        }
        const size_t blk = (size_t)R * (R + 1) / 2 + Cb;
        fuse.parts[2 * blk] = a;
        fuse.parts[2 * blk + 1] = b;
      }
    }
  }
}

__device__ __forceinline__ bool gemm_vec_ok(const double *A, int lda, const double *B, int ldb) {
  return ((lda | ldb) & 1) == 0 && ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) == 0;
}

template <int TBM, int TBN, int TBK = BK, int TST = STAGES>
__device__ __forceinline__ void gemm_tile_t(double *smem, int bm, int bn, int M, int N, int K, double alpha,
                                            const double *__restrict__ A, int lda, const double *__restrict__ B,
                                            int ldb, double *__restrict__ C, int ldc, int sym,
                                            const Sp2Fuse &fuse = Sp2Fuse{nullptr, false, nullptr, 1.0}) {
  if (gemm_vec_ok(A, lda, B, ldb))
    gemm_tile_impl<TBM, TBN, true, TBK, TST>(smem, bm, bn, M, N, K, alpha, A, lda, B, ldb, C, ldc, sym, fuse);
  else
    gemm_tile_impl<TBM, TBN, false, TBK, TST>(smem, bm, bn, M, N, K, alpha, A, lda, B, ldb, C, ldc, sym, fuse);
}

__device__ __forceinline__ void gemm_tile(double *smem, int bm, int bn, int M, int N, int K, double alpha,
                                          const double *__restrict__ A, int lda, const double *__restrict__ B, int ldb,
                                          double *__restrict__ C, int ldc, int sym) {
  gemm_tile_t<BM, BN>(smem, bm, bn, M, N, K, alpha, A, lda, B, ldb, C, ldc, sym);
}

__global__ void __launch_bounds__(128, 4) k_gemm_tn(int M, int N, int K, double alpha, const double *__restrict__ A,
                                                    int lda, const double *__restrict__ B, int ldb,
                                                    double *__restrict__ C, int ldc) {
  extern __shared__ __align__(16) double gemm_smem[];
  gemm_tile(gemm_smem, blockIdx.y, blockIdx.x, M, N, K, alpha, A, lda, B, ldb, C, ldc, 0);
}

// Number of SYM_BM x SYM_BN tiles that hold elements with m >= n of an n x n product.
static inline int sym_tiles(int n) {
  const int rows = (n + SYM_BM - 1) / SYM_BM, cols = (n + SYM_BN - 1) / SYM_BN;
  int t = 0;
  for (int r = 0; r < rows; ++r) t += std::min(((r + 1) * SYM_BM + SYM_BN - 1) / SYM_BN, cols);
  return t;
}

// The fused SP2 step of a symmetric n x n product (launch_sp2_step): parts != null makes
// the tiles apply the update chosen in state[kSp2Square] and write the 64 x 64 block trace
// partials; the first CTA records their count in state[kSp2Parts].
__device__ __forceinline__ Sp2Fuse sp2_fuse(int n, const double *x, double *state, double *parts) {
  if (!parts) return Sp2Fuse{nullptr, false, nullptr, 1.0};
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int t64 = (n + 63) / 64;
    state[kSp2Parts] = (double)(t64 * (t64 + 1) / 2);
  }
  return Sp2Fuse{x, state[kSp2Square] != 0.0, parts, 1.0};
}

// Symmetric n x n product on 64x64 tiles of the lower triangle (four CTAs per SM): more,
// smaller tiles than k_gemm_sym, the faster shape when 128x64 tiles leave SMs idle.
__global__ void __launch_bounds__(128, 4) k_gemm_sym64(int n, int K, double alpha, const double *__restrict__ A,
                                                       int lda, const double *__restrict__ B, int ldb,
                                                       double *__restrict__ C, int ldc, double *__restrict__ sp2,
                                                       int step, double *__restrict__ parts) {
  extern __shared__ __align__(16) double gemm_smem[];
  if (!sp2_active(sp2, step)) return;
  int t = blockIdx.x, r = 0;
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  gemm_tile_t<BM, BN>(gemm_smem, r, t - r * (r + 1) / 2, n, n, K, alpha, A, lda, B, ldb, C, ldc, 1,
                      sp2_fuse(n, A, sp2, parts));
}

// Symmetric n x n product over the enumerated lower-triangle tiles (row block r holds
// column blocks 0 .. ceil((r+1) SYM_BM / SYM_BN) - 1); K slabs of TBK rows, TST stages.
template <int TBK, int TST>
__global__ void __launch_bounds__(128, 2) k_gemm_sym(int n, int K, double alpha, const double *__restrict__ A,
                                                     int lda, const double *__restrict__ B, int ldb,
                                                     double *__restrict__ C, int ldc, double *__restrict__ sp2,
                                                     int step, double *__restrict__ parts) {
  extern __shared__ __align__(16) double gemm_smem[];
  if (!sp2_active(sp2, step)) return;  // an SP2 step after the purification stopped
  const int cols = (n + SYM_BN - 1) / SYM_BN;
  int t = blockIdx.x, r = 0;
  for (;; ++r) {
    const int nc = min(((r + 1) * SYM_BM + SYM_BN - 1) / SYM_BN, cols);
    if (t < nc) break;
    t -= nc;
  }
  gemm_tile_t<SYM_BM, SYM_BN, TBK, TST>(gemm_smem, r, t, n, n, K, alpha, A, lda, B, ldb, C, ldc, 1,
                                        sp2_fuse(n, A, sp2, parts));
}

// Grouped over molecules: item = one 64x64 tile of one molecule's product.
// op 0: X = F_slot P (F symmetric, so F^T P = F P), all tiles.
// op 1: Pn = 2 V_occ^T V_occ from this iteration's eigenvectors, lower tiles mirrored.
__global__ void __launch_bounds__(128, 4) k_b_gemm(BatchList L, const MolDesc *__restrict__ D,
                                                const MolCtl *__restrict__ Cc, const EigSlot *__restrict__ E, int op) {
  extern __shared__ __align__(16) double gemm_smem[];
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  const int n = d.g.nao, tiles = (n + BM - 1) / BM;
  const int local = item - L.prefix[m];
  if (op == 0) {
    const int bm = local / tiles, bn = local - bm * tiles;
    gemm_tile(gemm_smem, bm, bn, n, n, n, 1.0, hist_F(d, Cc[slot].slot), n, d.P, n, d.X, n, 0);
  } else {
    int bm = 0;
    while ((bm + 1) * (bm + 2) / 2 <= local) ++bm;
    const int bn = local - bm * (bm + 1) / 2;
    if (op == 1) {
      gemm_tile(gemm_smem, bm, bn, n, n, d.n_occ, 2.0, E[m].in, E[m].ldv, E[m].in, E[m].ldv, d.Pn, n, 1);
    } else if (op == 2) {
      if (Cc[slot].sp2_state == 0) gemm_tile(gemm_smem, bm, bn, n, n, n, 1.0, d.X, n, d.X, n, d.Pn, n, 1);
    } else {
      // the fused SP2 step on the (X, Pn) ping-pong pair: step k (decided just before by
      // k_b_sp2_decide64) reads its iterate from X for even k, from Pn for odd k, and writes
      // the next one, updated, to the other; the 64 x 64 tiles' trace partials go to part.
      // When the step is the last (converged), an iterate landing in Pn is written as the
      // density 2 X right away (one landing in X is doubled into Pn after the steps).
      const MolCtl &c = Cc[slot];
      if (!c.sp2_apply) return;
      const int k = c.sp2_steps - 1;
      const double *cur = (k % 2 == 0) ? d.X : d.Pn;
      double *dst = (k % 2 == 0) ? d.Pn : d.X;
      const double scale = (c.sp2_state == 1 && dst == d.Pn) ? 2.0 : 1.0;
      gemm_tile_t<BM, BN>(gemm_smem, bm, bn, n, n, n, 1.0, cur, n, cur, n, dst, n, 1,
                          Sp2Fuse{cur, c.sp2_square != 0, d.part, scale});
    }
  }
}

// Opt the GEMM kernels in to more than 48 KB of dynamic shared memory (once per device).
static void gemm_smem_attr() {
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaFuncSetAttribute(k_gemm_tn, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM);
  cudaFuncSetAttribute(k_gemm_sym<BK, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, SYM_SMEM);
  cudaFuncSetAttribute(k_gemm_sym<32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SYM_SMEM_K32);
  cudaFuncSetAttribute(k_gemm_sym64, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM);
  cudaFuncSetAttribute(k_b_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM);
  done[dev] = true;
}

void prepare_gemm_kernels() { gemm_smem_attr(); }

void launch_b_gemm(cudaStream_t st, const BatchList &L, const MolDesc *D, const MolCtl *C, const EigSlot *E, int op) {
  if (L.total <= 0) return;
  gemm_smem_attr();
  k_b_gemm<<<L.total, 128, GEMM_SMEM, st>>>(L, D, C, E, op);
  note_launch();
}

void launch_gemm_tn(cudaStream_t st, int M, int N, int K, double alpha, const double *A, int lda, const double *B,
                    int ldb, double *C, int ldc) {
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  gemm_smem_attr();
  k_gemm_tn<<<grid, 128, GEMM_SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, C, ldc);
  note_launch();
}

// Symmetric product C = alpha A^T B (n x n, inner dimension K) on the tile shape the
// autotuner picked for this size: 0 = 128x64 (k_gemm_sym, 16-deep slabs, three stages),
// 1 = 64x64 (k_gemm_sym64), 2 = 128x64 with 32-deep slabs in two stages. All give the same
// bits: every element is the same chain of DMMA steps over k in the same order. With
// `parts` the product is the fused SP2 step (sp2_fuse).
static void launch_sym(cudaStream_t st, const char *what, int n, int K, double alpha, const double *A, int lda,
                       const double *B, int ldb, double *C, int ldc, double *sp2, int step, double *parts = nullptr) {
  gemm_smem_attr();
  const int bucket = ((n + 255) / 256) * 256;
  autotune(st, std::string(what) + "|n" + std::to_string(bucket), 3, [&](int v) {
    if (v == 0) {
      k_gemm_sym<BK, STAGES><<<sym_tiles(n), 128, SYM_SMEM, st>>>(n, K, alpha, A, lda, B, ldb, C, ldc, sp2, step,
                                                                  parts);
    } else if (v == 1) {
      const int t = (n + BM - 1) / BM;
      k_gemm_sym64<<<t * (t + 1) / 2, 128, GEMM_SMEM, st>>>(n, K, alpha, A, lda, B, ldb, C, ldc, sp2, step, parts);
    } else {
      k_gemm_sym<32, 2><<<sym_tiles(n), 128, SYM_SMEM_K32, st>>>(n, K, alpha, A, lda, B, ldb, C, ldc, sp2, step,
                                                                  parts);
    }
    note_launch();
  });
}

size_t sp2_parts_doubles(int n) {
  const int t = (n + BM - 1) / BM;
  return 2 * (size_t)std::max(std::max(sym_tiles(n), t * (t + 1) / 2), 296) + 8;
}

void launch_density(cudaStream_t st, int n, int k, double w, const double *V, int ldv, double *P) {
  if (k == 0) {
    cudaMemsetAsync(P, 0, sizeof(double) * (size_t)n * n, st);
    return;
  }
  launch_sym(st, "density_sym", n, k, w, V, ldv, V, ldv, P, n, nullptr, 0);
}

// ---------------------------------------------------------------------------
// Reductions with fixed partial layouts.
// ---------------------------------------------------------------------------
constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs
constexpr int RED_THREADS = 256;

__global__ void __launch_bounds__(RED_THREADS) k_dot(size_t len, const double *__restrict__ a,
                                                     const double *__restrict__ b, double *__restrict__ partials) {
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * RED_THREADS + threadIdx.x; i < len; i += (size_t)gridDim.x * RED_THREADS)
    s += a[i] * b[i];
  s = block_sum<RED_THREADS>(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RED_THREADS) k_energy(size_t len, const double *__restrict__ P,
                                                        const double *__restrict__ H, const double *__restrict__ F,
                                                        double *__restrict__ partials) {
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * RED_THREADS + threadIdx.x; i < len; i += (size_t)gridDim.x * RED_THREADS)
    s += P[i] * (H[i] + F[i]);
  s = block_sum<RED_THREADS>(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(RED_THREADS) k_sqdiff(size_t len, const double *__restrict__ a,
                                                        const double *__restrict__ b, double *__restrict__ partials) {
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * RED_THREADS + threadIdx.x; i < len; i += (size_t)gridDim.x * RED_THREADS) {
    const double d = a[i] - b[i];
    s += d * d;
  }
  s = block_sum<RED_THREADS>(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

size_t launch_dot(cudaStream_t st, size_t len, const double *a, const double *b, double *partials) {
  k_dot<<<RED_BLOCKS, RED_THREADS, 0, st>>>(len, a, b, partials);
  note_launch();
  return RED_BLOCKS;
}
size_t launch_energy(cudaStream_t st, size_t len, const double *P, const double *H, const double *F,
                     double *partials) {
  k_energy<<<RED_BLOCKS, RED_THREADS, 0, st>>>(len, P, H, F, partials);
  note_launch();
  return RED_BLOCKS;
}
size_t launch_sqdiff(cudaStream_t st, size_t len, const double *a, const double *b, double *partials) {
  k_sqdiff<<<RED_BLOCKS, RED_THREADS, 0, st>>>(len, a, b, partials);
  note_launch();
  return RED_BLOCKS;
}

__global__ void k_sum(const double *__restrict__ in, size_t n, double *__restrict__ out) {
  double s = 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) s += in[i];
  s = block_sum<256>(s);
  if (threadIdx.x == 0) *out = s;
}
void launch_sum(cudaStream_t st, const double *partials, size_t n, double *out) {
  k_sum<<<1, 256, 0, st>>>(partials, n, out);
  note_launch();
}

// E = X - X^T via 32x32 shared tiles; partial sums of E^2 per block.
__global__ void k_antisym(int n, const double *__restrict__ X, double *__restrict__ E, double *__restrict__ partials) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int i = bx + r, j = by + tx;  // transposed tile source
    tile[r][tx] = (i < n && j < n) ? X[(size_t)i * n + j] : 0.0;
  }
  __syncthreads();
  double s = 0.0;
  for (int r = ty; r < 32; r += 8) {
    const int i = by + r, j = bx + tx;
    if (i < n && j < n) {
      const double e = X[(size_t)i * n + j] - tile[tx][r];
      E[(size_t)i * n + j] = e;
      s += e * e;
    }
  }
  // block of 256 threads
  s = block_sum<256>(s);
  if (tx == 0 && ty == 0) partials[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
}
size_t launch_antisym(cudaStream_t st, int n, const double *X, double *E, double *partials) {
  dim3 grid((n + 31) / 32, (n + 31) / 32), blk(32, 8);
  k_antisym<<<grid, blk, 0, st>>>(n, X, E, partials);
  note_launch();
  return (size_t)grid.x * grid.y;
}

__global__ void k_transpose(int n, const double *__restrict__ in, double *__restrict__ out) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = by + r, j = bx + threadIdx.x;
    if (i < n && j < n) tile[r][threadIdx.x] = in[(size_t)i * n + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = bx + r, j = by + threadIdx.x;
    if (i < n && j < n) out[(size_t)i * n + j] = tile[threadIdx.x][r];
  }
}
void launch_transpose(cudaStream_t st, int n, const double *in, double *out) {
  dim3 grid((n + 31) / 32, (n + 31) / 32), blk(32, 8);
  k_transpose<<<grid, blk, 0, st>>>(n, in, out);
  note_launch();
}

// out = sum_i c_i X_i + shift * (delta_ij - Pd_ij / occ)
__global__ void k_combine(int n, int k, const double *const *__restrict__ X, const double *__restrict__ c,
                          const double *__restrict__ Pd, double inv_occ, double shift, double *__restrict__ out) {
  const size_t len = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int i = 0; i < k; ++i) v += c[i] * X[i][e];
    if (shift > 0.0) {
      const size_t row = e / n, col = e - row * n;
      const double q = Pd[e] * inv_occ;
      v += shift * ((row == col) ? 1.0 - q : -q);
    }
    out[e] = v;
  }
}
void launch_combine(cudaStream_t st, int n, int k, const double *const *X, const double *c, const double *Pd,
                    double occ, double shift, double *out) {
  k_combine<<<RED_BLOCKS * 2, 256, 0, st>>>(n, k, X, c, Pd, 1.0 / occ, shift, out);
  note_launch();
}

// Dot products of one X with NY vectors Y_j in one sweep, accumulators in registers;
// partials laid out [block][j].
template <int NY>
__global__ void __launch_bounds__(256) k_dot_row(size_t len, const double *const *__restrict__ Xp,
                                                 const double *const *__restrict__ Yp, double *__restrict__ out) {
  const double *x = Xp[0];
  const double *y[NY];
#pragma unroll
  for (int j = 0; j < NY; ++j) y[j] = Yp[j];
  double acc[NY];
#pragma unroll
  for (int j = 0; j < NY; ++j) acc[j] = 0.0;
  for (size_t e = (size_t)blockIdx.x * 256 + threadIdx.x; e < len; e += (size_t)gridDim.x * 256) {
    const double xv = x[e];
#pragma unroll
    for (int j = 0; j < NY; ++j) acc[j] += xv * y[j][e];
  }
#pragma unroll
  for (int j = 0; j < NY; ++j) {
    const double s = block_sum<256>(acc[j]);
    if (threadIdx.x == 0) out[(size_t)blockIdx.x * NY + j] = s;
  }
}

void launch_dot_many(cudaStream_t st, size_t len, int nx, const double *const *X, int ny, const double *const *Y,
                     double *out_partials, int n_blocks) {
  (void)nx;  // one X per sweep
  switch (ny) {
#define DOT_CASE(k) \
  case k: k_dot_row<k><<<n_blocks, 256, 0, st>>>(len, X, Y, out_partials); break;
    DOT_CASE(1) DOT_CASE(2) DOT_CASE(3) DOT_CASE(4) DOT_CASE(5) DOT_CASE(6) DOT_CASE(7) DOT_CASE(8) DOT_CASE(9)
#undef DOT_CASE
    default: return;
  }
  note_launch();
}

// out[c] = sum over rows of partials[row * n_cols + c]
__global__ void k_reduce_rows(const double *__restrict__ partials, int n_rows, int n_cols, double *__restrict__ out) {
  const int c = blockIdx.x;
  double s = 0.0;
  for (int r = threadIdx.x; r < n_rows; r += 256) s += partials[(size_t)r * n_cols + c];
  s = block_sum<256>(s);
  if (threadIdx.x == 0) out[c] = s;
}
void launch_reduce_rows(cudaStream_t st, const double *partials, int n_rows, int n_cols, double *out) {
  k_reduce_rows<<<n_cols, 256, 0, st>>>(partials, n_rows, n_cols, out);
  note_launch();
}

__global__ void k_scale(size_t len, double s, const double *__restrict__ in, double *__restrict__ out) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x)
    out[e] = s * in[e];
}
void launch_scale(cudaStream_t st, size_t len, double s, const double *in, double *out) {
  k_scale<<<RED_BLOCKS * 2, 256, 0, st>>>(len, s, in, out);
  note_launch();
}

__global__ void k_axpby(size_t len, double a, const double *__restrict__ x, double b, const double *__restrict__ y,
                        double *__restrict__ out) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x)
    out[e] = a * x[e] + b * y[e];
}
void launch_axpby(cudaStream_t st, size_t len, double a, const double *x, double b, const double *y, double *out) {
  k_axpby<<<RED_BLOCKS * 2, 256, 0, st>>>(len, a, x, b, y, out);
  note_launch();
}

__global__ void k_set_diag(int n, const double *__restrict__ d, double *__restrict__ M) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) M[(size_t)i * n + i] = d[i];
}
void launch_set_diag(cudaStream_t st, int n, const double *diag, double *M) {
  cudaMemsetAsync(M, 0, sizeof(double) * (size_t)n * n, st);
  k_set_diag<<<(n + 255) / 256, 256, 0, st>>>(n, diag, M);
  note_launch();
}

}  // namespace pm7

namespace pm7 {

// ---------------------------------------------------------------------------
// SP2 density-matrix purification (second-order spectral projection): the aufbau
// projector onto the n_occ lowest eigenvectors of a symmetric F from matrix squarings
// on the FP64 tensor cores, without an eigendecomposition.
// ---------------------------------------------------------------------------

// Gershgorin bounds of each row: lo = F_ii - sum_j!=i |F_ij|, hi = F_ii + sum_j!=i |F_ij|;
// block-reduced into partial min / max.
__global__ void k_gershgorin(int n, const double *__restrict__ F, double *__restrict__ part_lo,
                             double *__restrict__ part_hi) {
  __shared__ double slo[8], shi[8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double lo = 1.0e300, hi = -1.0e300;
  for (int row = blockIdx.x * 8 + warp; row < n; row += gridDim.x * 8) {
    double off = 0.0;
    const double *r = F + (size_t)row * n;
    for (int j = lane; j < n; j += 32)
      if (j != row) off += fabs(r[j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) off += __shfl_down_sync(0xffffffffu, off, o);
    if (lane == 0) {
      lo = fmin(lo, r[row] - off);
      hi = fmax(hi, r[row] + off);
    }
  }
  if (lane == 0) {
    slo[warp] = lo;
    shi[warp] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) {
      lo = fmin(lo, slo[w]);
      hi = fmax(hi, shi[w]);
    }
    part_lo[blockIdx.x] = lo;
    part_hi[blockIdx.x] = hi;
  }
}

// bounds[0] = min, bounds[1] = max over the partials.
__global__ void k_minmax(int m, const double *__restrict__ lo, const double *__restrict__ hi, double *bounds) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 1.0e300, b = -1.0e300;
  for (int i = 0; i < m; ++i) {
    a = fmin(a, lo[i]);
    b = fmax(b, hi[i]);
  }
  // widen the interval so no level starts on 0 or 1 (fixed points of both SP2 maps)
  const double pad = 1.0e-3 * (b - a) + 1.0e-6;
  bounds[0] = a - pad;
  bounds[1] = b + pad;
}

// ---------------------------------------------------------------------------
// Tighter SP2 bounds: Lanczos (no reorthogonalisation) for the extreme eigenvalues of F.
// Gershgorin discs can be far wider than the spectrum (at 2,000 basis functions -43..+31 eV
// against -32..+9 eV), and every doubling of the bound interval costs SP2 about one more
// squaring. 16 Lanczos steps put the extreme Ritz values within ~1% of the range; the
// interval handed to SP2 is [theta_min - 2% R, theta_max + 4% R] (R = theta_max -
// theta_min) inside the Gershgorin interval, widened like the latter. A purification that
// then fails its acceptance checks is redone on the Gershgorin interval.
// ---------------------------------------------------------------------------
// lz layout (doubles): V (3 n: v_{j-1}, v_j, v_{j+1} by j mod 3) | w (n) | alpha (kLzSteps) |
// beta (kLzSteps + 1) | per-row partials of w . v_j (n)

// v_0: a fixed, dense, normalised start vector.
__global__ void k_lz_init(int n, double *__restrict__ lz) {
  double *V = lz, *beta = lz + 4 * (size_t)n + kLzSteps;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = 1.0 + 0.5 * sin(0.7 * i);
    V[i] = v;
    s += v * v;
  }
  s = block_sum<1024>(s);
  __shared__ double inv;
  if (threadIdx.x == 0) inv = 1.0 / sqrt(s);
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) V[i] *= inv;
  if (threadIdx.x == 0) beta[0] = 0.0;
}

// w = F v_j and the per-row products w_i v_j,i (summed by k_lz_step). One 256-thread block
// per row, each lane with up to 8 predicated loads in flight per pass, so the matrix streams
// from L2 at bandwidth rather than at one load latency per element.
__global__ void __launch_bounds__(256) k_lz_matvec(int n, int j, const double *__restrict__ F, double *__restrict__ lz) {
  const double *v = lz + (size_t)(j % 3) * n;
  double *w = lz + 3 * (size_t)n;
  double *part = lz + 4 * (size_t)n + 2 * kLzSteps + 1;
  const int i = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double *fi = F + (size_t)i * n;
  double acc = 0.0;
  for (int base = threadIdx.x; base < n; base += 2048) {
    double x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = base + 256 * u;
      x[u] = k < n ? fi[k] * v[k] : 0.0;
    }
    acc += ((x[0] + x[1]) + (x[2] + x[3])) + ((x[4] + x[5]) + (x[6] + x[7]));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[8];
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double wi = ((red[0] + red[1]) + (red[2] + red[3])) + ((red[4] + red[5]) + (red[6] + red[7]));
    w[i] = wi;
    part[i] = wi * v[i];
  }
}

// alpha_j = w . v_j; w -= alpha_j v_j + beta_j v_{j-1}; beta_{j+1} = |w|; v_{j+1} = w / beta_{j+1}.
__global__ void __launch_bounds__(1024) k_lz_step(int n, int j, double *__restrict__ lz) {
  double *V = lz, *w = lz + 3 * (size_t)n;
  double *alpha = lz + 4 * (size_t)n, *beta = alpha + kLzSteps, *part = beta + kLzSteps + 1;
  const double *vj = V + (size_t)(j % 3) * n, *vp = V + (size_t)((j + 2) % 3) * n;
  double *vn = V + (size_t)((j + 1) % 3) * n;
  __shared__ double a_s, b_s;
  double a = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) a += part[q];
  a = block_sum<1024>(a);
  if (threadIdx.x == 0) a_s = a;
  __syncthreads();
  a = a_s;
  const double bj = j > 0 ? beta[j] : 0.0;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = w[i] - a * vj[i] - (j > 0 ? bj * vp[i] : 0.0);  // no v_{-1}
    w[i] = x;
    s += x * x;
  }
  s = block_sum<1024>(s);
  if (threadIdx.x == 0) {
    b_s = sqrt(s);
    alpha[j] = a;
    beta[j + 1] = b_s;
  }
  __syncthreads();
  const double inv = b_s > 1.0e-280 ? 1.0 / b_s : 0.0;  // an invariant subspace: v stops
  for (int i = threadIdx.x; i < n; i += blockDim.x) vn[i] = w[i] * inv;
}

// Extreme eigenvalues of the Lanczos tridiagonal T (bisection on its Sturm count) and the
// SP2 interval, inside the Gershgorin one already in bounds[0..1].
__device__ int lz_count(const double *a, const double *b, int m, double x) {
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
// One warp: 32-point multisection on the Sturm count (lanes evaluate 32 interior points, a
// ballot keeps the sub-interval holding the wanted eigenvalue; 12 rounds shrink the Gershgorin
// interval of T by 33^12, to the rounding floor).
__device__ double lz_extreme(const double *a, const double *b, int m, double lo, double hi, int target, int lane) {
  for (int it = 0; it < 12; ++it) {
    const double x = lo + (hi - lo) * (double)(lane + 1) / 33.0;
    const unsigned hit = __ballot_sync(0xffffffffu, lz_count(a, b, m, x) >= target);
    const double xl = __shfl_sync(0xffffffffu, x, hit ? __ffs(hit) - 1 : 31);
    if (hit) {
      const int f = __ffs(hit) - 1;
      const double xp = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
      hi = xl;
      if (f > 0) lo = xp;
    } else {
      lo = xl;
    }
  }
  return hi;
}

__global__ void k_lz_bounds(int n, const double *__restrict__ lz, double *__restrict__ bounds) {
  if (blockIdx.x != 0) return;
  const int lane = threadIdx.x & 31;
  const double *a = lz + 4 * (size_t)n, *b = a + kLzSteps;
  const int m = kLzSteps;
  double g_lo = 1.0e300, g_hi = -1.0e300;
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? fabs(b[i]) : 0.0) + (i + 1 < m ? fabs(b[i + 1]) : 0.0);
    g_lo = fmin(g_lo, a[i] - r);
    g_hi = fmax(g_hi, a[i] + r);
  }
  const double tmin = lz_extreme(a, b, m, g_lo, g_hi, 1, lane);  // smallest: count(x) >= 1
  const double tmax = lz_extreme(a, b, m, g_lo, g_hi, m, lane);  // largest: count(x) >= m
  if (lane != 0) return;
  const double R = tmax - tmin;
  if (!(R > 0.0) || !isfinite(R)) return;  // keep the Gershgorin interval
  double elo = fmax(tmin - 0.02 * R, bounds[0]), ehi = fmin(tmax + 0.04 * R, bounds[1]);
  const double pad = 1.0e-3 * (ehi - elo) + 1.0e-6;
  bounds[0] = fmax(elo - pad, bounds[0]);
  bounds[1] = fmin(ehi + pad, bounds[1]);
}

// X = (emax I - F) / (emax - emin): spectrum mapped into [0, 1], occupied levels near 1.
__global__ void k_sp2_init(int n, const double *__restrict__ F, const double *__restrict__ bounds,
                           double *__restrict__ X) {
  const double emin = bounds[0], emax = bounds[1];
  const double inv = 1.0 / (emax - emin);
  const size_t len = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / n, j = e - i * n;
    X[e] = ((i == j ? emax : 0.0) - F[e]) * inv;
  }
}

// Traces of X and X^2 and the SP2 branch: state[0] = tr X, state[1] = tr X^2,
// state[2] = 1 when squaring brings the trace closer to n_occ, state[3] = tr X - tr X^2;
// then the stopping rule.
__global__ void k_sp2_trace(int n, const double *__restrict__ X, const double *__restrict__ X2, double n_occ,
                            double *__restrict__ state, int step, Sp2Rule rule) {
  if (!sp2_active(state, step)) return;
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a += X[(size_t)i * n + i];
    b += X2[(size_t)i * n + i];
  }
  a = block_sum<256>(a);
  b = block_sum<256>(b);
  if (threadIdx.x == 0) {
    state[kSp2TrX] = a;
    state[kSp2TrX2] = b;
    state[kSp2Square] = fabs(b - n_occ) < fabs(2.0 * a - b - n_occ) ? 1.0 : 0.0;
    state[kSp2Err] = a - b;
    sp2_control(state, step, a - b, rule);
  }
}

// X <- X^2 or 2X - X^2 according to state[2].
__global__ void k_sp2_update(size_t len, double *__restrict__ X, const double *__restrict__ X2,
                             const double *__restrict__ state, int step) {
  if (!sp2_active(state, step)) return;
  const bool square = state[kSp2Square] != 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x)
    X[e] = square ? X2[e] : 2.0 * X[e] - X2[e];
}

// tr X and |X|_F^2 (= tr X^2 for symmetric X) of the starting iterate, per-block partials in
// the layout of the fused step's (parts[2 b], parts[2 b + 1]); the count to state[kSp2Parts].
__global__ void k_sp2_norms(int n, const double *__restrict__ X, double *__restrict__ state,
                            double *__restrict__ parts) {
  const size_t len = (size_t)n * n;
  double tr = 0.0, sq = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const double v = X[e];
    sq += v * v;
    if (e % (n + 1) == 0) tr += v;
  }
  tr = block_sum<256>(tr);
  sq = block_sum<256>(sq);
  if (threadIdx.x == 0) {
    parts[2 * blockIdx.x] = tr;
    parts[2 * blockIdx.x + 1] = sq;
    if (blockIdx.x == 0) state[kSp2Parts] = (double)gridDim.x;
  }
}

// The SP2 decision of step `step` from the current iterate's trace partials (the fused
// step's epilogue, or k_sp2_norms for the first): tr X, tr X^2 = |X|_F^2, the branch
// (square when it brings the trace closer to n_occ) and the stopping rule on tr X - tr X^2.
__global__ void k_sp2_decide(double n_occ, double *__restrict__ state, const double *__restrict__ parts, int step,
                             Sp2Rule rule) {
  if (!sp2_active(state, step)) return;
  const int count = (int)state[kSp2Parts];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    a += parts[2 * i];
    b += parts[2 * i + 1];
  }
  a = block_sum<256>(a);
  b = block_sum<256>(b);
  if (threadIdx.x == 0) {
    state[kSp2TrX] = a;
    state[kSp2TrX2] = b;
    state[kSp2Square] = fabs(b - n_occ) < fabs(2.0 * a - b - n_occ) ? 1.0 : 0.0;
    state[kSp2Err] = a - b;
    sp2_control(state, step, a - b, rule);
  }
}

__global__ void k_sp2_reset(double *state) {
  const int i = threadIdx.x;
  if (i < kSp2Len) state[i] = i == kSp2Stop ? 1.0e9 : 0.0;
}

void launch_gershgorin(cudaStream_t st, int n, const double *F, double *scratch, double *bounds) {
  const int blocks = 296;
  k_gershgorin<<<blocks, 256, 0, st>>>(n, F, scratch, scratch + blocks);
  note_launch();
  k_minmax<<<1, 32, 0, st>>>(blocks, scratch, scratch + blocks, bounds);
  note_launch();
}

void launch_sp2_init(cudaStream_t st, int n, const double *F, const double *bounds, double *X) {
  k_sp2_init<<<RED_BLOCKS * 2, 256, 0, st>>>(n, F, bounds, X);
  note_launch();
}

size_t lanczos_doubles(int n) { return 5 * (size_t)n + 2 * kLzSteps + 1; }

void launch_lanczos_bounds(cudaStream_t st, int n, const double *F, double *lz, double *bounds) {
  if (n < 2 * kLzSteps) return;  // small matrices: the Gershgorin interval
  k_lz_init<<<1, 1024, 0, st>>>(n, lz);
  note_launch();
  for (int j = 0; j < kLzSteps; ++j) {
    k_lz_matvec<<<n, 256, 0, st>>>(n, j, F, lz);
    k_lz_step<<<1, 1024, 0, st>>>(n, j, lz);
    note_launch(2);
  }
  k_lz_bounds<<<1, 32, 0, st>>>(n, lz, bounds);
  note_launch();
}

void launch_sp2_reset(cudaStream_t st, double *state) {
  k_sp2_reset<<<1, 32, 0, st>>>(state);
  note_launch();
}

void launch_sp2_square(cudaStream_t st, int n, const double *X, double *X2, const double *state, int step) {
  launch_sym(st, "sp2_square", n, n, 1.0, X, n, X, n, X2, n, const_cast<double *>(state), step);
}

void launch_sp2_step(cudaStream_t st, int n, const double *X, double *Y, double *state, double *parts, int step) {
  launch_sym(st, "sp2_square", n, n, 1.0, X, n, X, n, Y, n, state, step, parts);
}

void launch_sp2_norms(cudaStream_t st, int n, const double *X, double *state, double *parts) {
  k_sp2_norms<<<296, 256, 0, st>>>(n, X, state, parts);
  note_launch();
}

void launch_sp2_decide(cudaStream_t st, double n_occ, double *state, const double *parts, int step, Sp2Rule rule) {
  k_sp2_decide<<<1, 256, 0, st>>>(n_occ, state, parts, step, rule);
  note_launch();
}

void launch_sp2_trace(cudaStream_t st, int n, const double *X, const double *X2, double n_occ, double *state, int step,
                      Sp2Rule rule) {
  k_sp2_trace<<<1, 256, 0, st>>>(n, X, X2, n_occ, state, step, rule);
  note_launch();
}

void launch_sp2_update(cudaStream_t st, int n, double *X, const double *X2, const double *state, int step) {
  k_sp2_update<<<RED_BLOCKS * 2, 256, 0, st>>>((size_t)n * n, X, X2, state, step);
  note_launch();
}

}  // namespace pm7
