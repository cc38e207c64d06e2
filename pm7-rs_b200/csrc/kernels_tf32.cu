// FP32-accuracy products of symmetric matrices on the 5th-generation tensor cores (tcgen05,
// kind::tf32) for the mixed-precision SCF cycles: the SP2 squaring C = X X and the DIIS
// commutator product F P.
//
// X is stored split as X = Xhi + Xlo with Xhi = tf32(X) and Xlo = X - Xhi (both fp32
// arrays, row-major, leading dimension ld, zero padded to ld); the product is accumulated
// in fp32 in tensor memory as Xhi Xhi + Xhi Xlo + Xlo Xhi (the "3xTF32" split, about fp32
// accuracy). X is symmetric, so C = X X^T: both operands are row blocks of X, K-major.
//
// One CTA per 128x128 lower tile of C (the upper tiles are mirrored). Warp 0 lane 0 feeds
// a 3-stage shared-memory ring with TMA (cp.async.bulk.tensor, 128-byte swizzle, no
// multicast); warp 1 lane 0 issues tcgen05.mma (M=128, N=128, K=8) into a 128-column TMEM
// accumulator and releases each stage with tcgen05.commit; all four warps read the
// accumulator back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and
// store it. Every mbarrier wait has a time limit (1 s); on expiry the CTA records an error,
// stops issuing, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "kernels.hpp"
#include "tcgen05.cuh"

namespace pm7 {
namespace {

constexpr int TM = 128, TN = 128, TK = 32, STAGES = 3;
constexpr int TILE_BYTES = TM * TK * 4;            // 16 KB: 128 rows x 32 fp32 (128 B per row)
constexpr int STAGE_BYTES = 4 * TILE_BYTES;        // Ahi, Alo, Bhi, Blo
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;  // + alignment slack + barriers

using namespace tc;

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, 8-row groups 1024 B
// apart (SBO), version 1 (tcgen05), base offset 0 (stage buffers are 1024-byte aligned).
__device__ __forceinline__ uint64_t smem_desc(const void *tile) {
  const uint32_t addr = smem_u32(tile);
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;               // stride byte offset
  d |= (uint64_t)1 << 46;                         // version
  d |= (uint64_t)2 << 61;                         // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::tf32: fp32 accumulate, TF32 A and B, both K-major, N=128, M=128.
constexpr uint32_t kIdesc = (1u << 4)              // c_format F32
                            | (2u << 7)            // a_format TF32
                            | (2u << 10)           // b_format TF32
                            | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}


// One 128x128 tile (bm, bn) of C = A B for symmetric A, B (so B's columns are its rows:
// both operands K-major row blocks). `smem_raw` is the CTA's dynamic shared memory
// (SMEM_BYTES); a_hi / a_lo and b_hi / b_lo the tensor maps of the split operands. With
// `mirror` (the squaring, A = B, lower tiles bm >= bn only) each element of the lower
// triangle is written with its mirror; without, the tile is written as it is.
__device__ __forceinline__ void product_tile(int bm, int bn, const CUtensorMap *a_hi, const CUtensorMap *a_lo,
                                             const CUtensorMap *b_hi, const CUtensorMap *b_lo, bool mirror, int n,
                                             int ld, float *__restrict__ C, int *__restrict__ error,
                                             unsigned char *smem_raw, bool withhold_copies = false) {
  // stage buffers on a 1024-byte boundary (128-byte swizzle atoms)
  unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int m0 = bm * TM, n0 = bn * TN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ktiles = (ld + TK - 1) / TK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // producer: TMA ring
    for (int kt = 0; kt < ktiles; ++kt) {
      const int s = kt % STAGES;
      if (kt >= STAGES && !mbar_wait(&empty[s], (uint32_t)((kt / STAGES - 1) & 1), abort_flag)) break;
      unsigned char *st = smem + s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      if (withhold_copies) continue;  // failure drill: the stage never fills, every wait runs out
      const int k0 = kt * TK;
      tma_load_2d(st + 0 * TILE_BYTES, a_hi, &full[s], k0, m0);
      tma_load_2d(st + 1 * TILE_BYTES, a_lo, &full[s], k0, m0);
      tma_load_2d(st + 2 * TILE_BYTES, b_hi, &full[s], k0, n0);
      tma_load_2d(st + 3 * TILE_BYTES, b_lo, &full[s], k0, n0);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    bool ok = true;
    for (int kt = 0; kt < ktiles && ok; ++kt) {
      const int s = kt % STAGES;
      if (!mbar_wait(&full[s], (uint32_t)((kt / STAGES) & 1), abort_flag)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      unsigned char *st = smem + s * STAGE_BYTES;
      const uint64_t ahi = smem_desc(st), alo = smem_desc(st + TILE_BYTES);
      const uint64_t bhi = smem_desc(st + 2 * TILE_BYTES), blo = smem_desc(st + 3 * TILE_BYTES);
#pragma unroll
      for (int j = 0; j < TK / 8; ++j) {
        const uint64_t off = (uint64_t)(j * 2);  // 8 fp32 = 32 bytes = 2 units of 16 bytes
        mma_tf32(tmem, ahi + off, bhi + off, (kt > 0 || j > 0) ? 1u : 0u);
        mma_tf32(tmem, ahi + off, blo + off, 1u);
        mma_tf32(tmem, alo + off, bhi + off, 1u);
      }
      mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
    }
    if (ok) mma_commit(done);  // the accumulator is final once every MMA completed
    else *abort_flag = 1;
  }
  __syncwarp();
  // epilogue: all four warps
  const bool ok = mbar_wait(done, 0u, abort_flag);
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (ok) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll
    for (int c = 0; c < TN / 32; ++c) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
            "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int col = n0 + c * 32 + q;
        if (row >= n || col >= n) continue;
        const float v = __uint_as_float(r[q]);
        if (!mirror) {
          C[(size_t)row * ld + col] = v;
        } else if (row >= col) {  // lower triangle, each element once, and its mirror
          C[(size_t)row * ld + col] = v;
          C[(size_t)col * ld + row] = v;
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(error, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
}

__device__ __forceinline__ void lower_tile(int t, int &bm, int &bn) {
  int m = 0;
  while ((m + 1) * (m + 2) / 2 <= t) ++m;
  bm = m;
  bn = t - m * (m + 1) / 2;
}

__global__ void __launch_bounds__(128) k_square_tf32x3(const __grid_constant__ CUtensorMap map_hi,
                                                       const __grid_constant__ CUtensorMap map_lo, int n, int ld,
                                                       float *__restrict__ C, int *__restrict__ error,
                                                       const double *__restrict__ sp2, int step, int drill) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // an SP2 step after the purification stopped: the whole CTA leaves before any barrier,
  // tensor-memory or copy set-up
  if (!sp2_active(sp2, step)) return;
  int bm, bn;
  lower_tile(blockIdx.x, bm, bn);
  product_tile(bm, bn, &map_hi, &map_lo, &map_hi, &map_lo, true, n, ld, C, error, smem_raw, drill != 0);
}

// C = A B of two symmetric split operands, every 128x128 tile (the DIIS commutator F P of
// the fp32 cycles).
__global__ void __launch_bounds__(128) k_product_tf32x3(const __grid_constant__ CUtensorMap a_hi,
                                                        const __grid_constant__ CUtensorMap a_lo,
                                                        const __grid_constant__ CUtensorMap b_hi,
                                                        const __grid_constant__ CUtensorMap b_lo, int n, int ld,
                                                        float *__restrict__ C, int *__restrict__ error) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int t = (n + TM - 1) / TM;
  product_tile(blockIdx.x / t, blockIdx.x % t, &a_hi, &a_lo, &b_hi, &b_lo, false, n, ld, C, error, smem_raw);
}

}  // namespace

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
TensorMapEncodeFn tensor_map_encode_fn() {
  static TensorMapEncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<TensorMapEncodeFn>(p);
  });
  return fn;
}

// Tensor map of an ld x ld fp32 row-major matrix with 32 x 128 boxes, 128-byte swizzle.
bool make_square_map(const float *base, int ld, void *map_out) {
  TensorMapEncodeFn fn = tensor_map_encode_fn();
  if (!fn || ld % 32 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)ld};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  const cuuint32_t box[2] = {TK, TM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(reinterpret_cast<CUtensorMap *>(map_out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        const_cast<float *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

size_t square_tf32x3_smem() { return SMEM_BYTES; }

void launch_product_tf32x3(cudaStream_t st, int n, int ld, const void *a_hi, const void *a_lo, const void *b_hi,
                           const void *b_lo, float *C, int *error) {
  prepare_tf32_kernels();
  const int t = (n + TM - 1) / TM;
  k_product_tf32x3<<<t * t, 128, SMEM_BYTES, st>>>(
      *reinterpret_cast<const CUtensorMap *>(a_hi), *reinterpret_cast<const CUtensorMap *>(a_lo),
      *reinterpret_cast<const CUtensorMap *>(b_hi), *reinterpret_cast<const CUtensorMap *>(b_lo), n, ld, C, error);
  note_launch();
}

void launch_square_tf32x3(cudaStream_t st, int n, int ld, const void *map_hi, const void *map_lo, float *C,
                          int *error, const double *state, int step, int drill) {
  prepare_tf32_kernels();
  const int t = (n + TM - 1) / TM;
  k_square_tf32x3<<<t * (t + 1) / 2, 128, SMEM_BYTES, st>>>(*reinterpret_cast<const CUtensorMap *>(map_hi),
                                                            *reinterpret_cast<const CUtensorMap *>(map_lo), n, ld, C,
                                                            error, state, step, drill);
  note_launch();
}

}  // namespace pm7

namespace pm7 {
namespace {

// fp64 n x n -> fp32 split pair (hi = tf32 rounding, lo = remainder), ld x ld, zero padded.
__global__ void k_split_tf32(int n, int ld, const double *__restrict__ X, float *__restrict__ hi,
                             float *__restrict__ lo) {
  const size_t len = (size_t)ld * ld;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / ld, j = e - i * ld;
    float h = 0.0f, l = 0.0f;
    if (i < (size_t)n && j < (size_t)n) {
      const float x = (float)X[i * n + j];
      uint32_t t;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(x));
      h = __uint_as_float(t);
      l = x - h;
    }
    hi[e] = h;
    lo[e] = l;
  }
}

__global__ void k_widen(int n, int ld, const float *__restrict__ C32, double *__restrict__ C) {
  const size_t len = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / n, j = e - i * n;
    C[e] = (double)C32[i * ld + j];
  }
}

}  // namespace

void launch_split_tf32(cudaStream_t st, int n, int ld, const double *X, float *hi, float *lo) {
  k_split_tf32<<<1184, 256, 0, st>>>(n, ld, X, hi, lo);
  note_launch();
}

void launch_widen(cudaStream_t st, int n, int ld, const float *C32, double *C) {
  k_widen<<<1184, 256, 0, st>>>(n, ld, C32, C);
  note_launch();
}

}  // namespace pm7

// ---- the fp32 SP2 iteration around the tcgen05 squaring ------------------------------
namespace pm7 {
namespace {

__device__ __forceinline__ void split_store(float x, float *hi, float *lo, size_t e) {
  uint32_t t;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(x));
  const float h = __uint_as_float(t);
  hi[e] = h;
  lo[e] = x - h;
}

// X = (emax I - F) / (emax - emin) in fp32 (ld x ld, padding untouched) and its split.
__global__ void k_sp2_init32(int n, int ld, const double *__restrict__ F, const double *__restrict__ bounds,
                             float *__restrict__ X, float *__restrict__ hi, float *__restrict__ lo) {
  const double emin = bounds[0], emax = bounds[1], inv = 1.0 / (emax - emin);
  const size_t len = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / n, j = e - i * n, q = i * ld + j;
    const float x = (float)(((i == j ? emax : 0.0) - F[e]) * inv);
    X[q] = x;
    split_store(x, hi, lo, q);
  }
}

// state[0] = tr X, state[1] = tr X^2 (fp64 sums), state[2] = SP2 branch, state[3] = tr X - tr X^2.
__global__ void k_sp2_trace32(int n, int ld, const float *__restrict__ X, const float *__restrict__ X2, double n_occ,
                              double *__restrict__ state, int step, Sp2Rule rule) {
  if (!sp2_active(state, step)) return;
  __shared__ double sa[8], sb[8];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) {
    a += (double)X[(size_t)i * ld + i];
    b += (double)X2[(size_t)i * ld + i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    sb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = 0.0;
    b = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += sa[w];
      b += sb[w];
    }
    state[0] = a;
    state[1] = b;
    state[2] = fabs(b - n_occ) < fabs(2.0 * a - b - n_occ) ? 1.0 : 0.0;
    state[3] = a - b;
    sp2_control(state, step, a - b, rule);
  }
}

// X <- X^2 or 2X - X^2 by state[2], and its split.
__global__ void k_sp2_update32(int n, int ld, float *__restrict__ X, const float *__restrict__ X2,
                               const double *__restrict__ state, float *__restrict__ hi, float *__restrict__ lo,
                               int step) {
  if (!sp2_active(state, step)) return;
  const bool square = state[2] != 0.0;
  const size_t len = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / n, j = e - i * n, q = i * ld + j;
    const float x2 = X2[q];
    const float x = square ? x2 : 2.0f * X[q] - x2;
    X[q] = x;
    split_store(x, hi, lo, q);
  }
}

// P = w X (fp64 n x n from the fp32 iterate).
__global__ void k_sp2_density32(int n, int ld, const float *__restrict__ X, double w, double *__restrict__ P) {
  const size_t len = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = e / n, j = e - i * n;
    P[e] = w * (double)X[i * ld + j];
  }
}

}  // namespace

void launch_sp2_init32(cudaStream_t st, int n, int ld, const double *F, const double *bounds, float *X, float *hi,
                       float *lo) {
  k_sp2_init32<<<1184, 256, 0, st>>>(n, ld, F, bounds, X, hi, lo);
  note_launch();
}
void launch_sp2_trace32(cudaStream_t st, int n, int ld, const float *X, const float *X2, double n_occ, double *state,
                        int step, Sp2Rule rule) {
  k_sp2_trace32<<<1, 256, 0, st>>>(n, ld, X, X2, n_occ, state, step, rule);
  note_launch();
}
void launch_sp2_update32(cudaStream_t st, int n, int ld, float *X, const float *X2, const double *state, float *hi,
                         float *lo, int step) {
  k_sp2_update32<<<1184, 256, 0, st>>>(n, ld, X, X2, state, hi, lo, step);
  note_launch();
}
void launch_sp2_density32(cudaStream_t st, int n, int ld, const float *X, double w, double *P) {
  k_sp2_density32<<<1184, 256, 0, st>>>(n, ld, X, w, P);
  note_launch();
}

}  // namespace pm7

// ---- batched mixed precision -------------------------------------------------------
#include "batch.hpp"

namespace pm7 {
namespace {

// Grouped squaring: item = (molecule, lower 128x128 tile) of the molecules whose fp32
// purification is still running; each molecule's tensor maps are maps[2 slot], maps[2 slot + 1].
__global__ void __launch_bounds__(128) k_b_square_tf32x3(BatchList L, const MolDesc *__restrict__ D,
                                                         const MolCtl *__restrict__ Cc,
                                                         const CUtensorMap *__restrict__ maps, int *error) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const int slot = L.slot[m];
  if (Cc[slot].sp2_state != 0) return;
  int bm, bn;
  lower_tile(item - L.prefix[m], bm, bn);
  const MolDesc &d = D[slot];
  product_tile(bm, bn, &maps[2 * slot], &maps[2 * slot + 1], &maps[2 * slot], &maps[2 * slot + 1], true, d.g.nao,
               d.ld32, d.C32, error, smem_raw);
}

// X32 = fp32 of the (fp64) SP2 start X, and its split. Item = a chunk.
__global__ void __launch_bounds__(256) k_b_to32(BatchList L, const MolDesc *__restrict__ D) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const int n = d.g.nao, ld = d.ld32;
  for (size_t e = r.e0 + threadIdx.x; e < r.e1; e += 256) {
    const size_t i = e / n, j = e - i * n, q = i * ld + j;
    const float x = (float)d.X[e];
    d.X32[q] = x;
    split_store(x, d.hi32, d.lo32, q);
  }
}

// One fp32 SP2 decision (block per molecule): as the fp64 one, with the fp32 rounding
// floor (idempotency error stalls below 1e-2 n_occ) and trace tolerance (1e-2 n_occ).
__global__ void __launch_bounds__(256) k_b_sp2_decide32(BatchList L, const MolDesc *__restrict__ D,
                                                        MolCtl *__restrict__ C, unsigned char *__restrict__ flags) {
  const int m = blockIdx.x;
  const int slot = L.slot[m];
  const MolDesc &d = D[slot];
  MolCtl &c = C[slot];
  if (c.sp2_state != 0) {
    if (threadIdx.x == 0) c.sp2_apply = 0;
    return;
  }
  const int n = d.g.nao, ld = d.ld32;
  __shared__ double sa[8], sb[8];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) {
    a += (double)d.X32[(size_t)i * ld + i];
    b += (double)d.C32[(size_t)i * ld + i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    sb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = 0.0;
    b = 0.0;
    for (int w = 0; w < 8; ++w) {
      a += sa[w];
      b += sb[w];
    }
    const double nocc = (double)d.n_occ, scale = fmax(1.0, nocc);
    c.sp2_square = fabs(b - nocc) < fabs(2.0 * a - b - nocc) ? 1 : 0;
    const double e = a - b;
    const int k = c.sp2_steps;
    int state = 0;
    if (!isfinite(e)) {
      state = 2;
    } else if (fabs(e) <= 1.0e-6 * scale) {
      state = 1;
    } else if (k >= 2 && fabs(e) < 1.0e-2 * scale && fabs(e) >= fabs(c.sp2_err[(k + 1) % 3])) {
      state = 1;  // at the fp32 rounding floor
    } else if (k + 1 >= 100) {
      state = 2;
    }
    if (state == 1 && fabs(a - nocc) > 1.0e-2 * scale) state = 2;
    c.sp2_err[k % 3] = e;
    c.sp2_steps = k + 1;
    c.sp2_state = state;
    c.sp2_apply = 1;
    flags[m] = (unsigned char)state;
  }
}

// X32 <- X^2 or 2X - X^2 and its split for the molecules decided this step; Pn = 2 X
// (fp64) for those that finished. Item = a chunk.
__global__ void __launch_bounds__(256) k_b_sp2_apply32(BatchList L, const MolDesc *__restrict__ D,
                                                       const MolCtl *__restrict__ C) {
  const ChunkRef r = chunk_ref(L, D, blockIdx.x);
  const MolDesc &d = D[r.slot];
  const MolCtl &c = C[r.slot];
  if (!c.sp2_apply) return;
  const bool sq = c.sp2_square != 0, fin = c.sp2_state == 1;
  const int n = d.g.nao, ld = d.ld32;
  for (size_t e = r.e0 + threadIdx.x; e < r.e1; e += 256) {
    const size_t i = e / n, j = e - i * n, q = i * ld + j;
    const float x2 = d.C32[q];
    const float x = sq ? x2 : 2.0f * d.X32[q] - x2;
    d.X32[q] = x;
    split_store(x, d.hi32, d.lo32, q);
    if (fin) d.Pn[e] = 2.0 * (double)x;
  }
}

}  // namespace

// The tcgen05 kernels' dynamic shared memory limit, once per device (kernel attributes are
// per device). Called by every launcher and by the batched engine before any graph capture.
void prepare_tf32_kernels() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaFuncSetAttribute(k_square_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  cudaFuncSetAttribute(k_product_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  cudaFuncSetAttribute(k_b_square_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  done[dev] = true;
}

void launch_b_square_tf32x3(cudaStream_t st, const BatchList &L, const MolDesc *D, const MolCtl *C, const void *maps,
                            int *error) {
  if (L.total <= 0) return;
  prepare_tf32_kernels();
  k_b_square_tf32x3<<<L.total, 128, SMEM_BYTES, st>>>(L, D, C, reinterpret_cast<const CUtensorMap *>(maps), error);
  note_launch();
}

void launch_b_to32(cudaStream_t st, const BatchList &L, const MolDesc *D) {
  if (L.total <= 0) return;
  k_b_to32<<<L.total, 256, 0, st>>>(L, D);
  note_launch();
}

void launch_b_sp2_decide32(cudaStream_t st, const BatchList &L, const MolDesc *D, MolCtl *C, unsigned char *flags) {
  if (L.n <= 0) return;
  k_b_sp2_decide32<<<L.n, 256, 0, st>>>(L, D, C, flags);
  note_launch();
}

void launch_b_sp2_apply32(cudaStream_t st, const BatchList &L, const MolDesc *D, const MolCtl *C) {
  if (L.total <= 0) return;
  k_b_sp2_apply32<<<L.total, 256, 0, st>>>(L, D, C);
  note_launch();
}

}  // namespace pm7
