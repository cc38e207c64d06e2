// FP64-accuracy SP2 squarings on the tcgen05 integer tensor cores (kind::i8).
//
// An SP2 iterate X is symmetric with its spectrum in [0, 1] (to the interval's margins), so
// every element lies in [-1, 1]. It is held, besides its fp64 copy, as eight int8 digit
// planes in fixed point, x = 2^-6 (a_0 + 2^-7 (a_1 + ... + 2^-7 a_7)) + r with |r| <= 2^-56;
// the split is exact in fp64 (each step scales by a power of two and subtracts the nearest
// integer) and every digit lies in [-64, 64]. The product is then
//   X X = 2^-12 sum_g 2^-7g G_g,   G_g = sum_{i + j = g} A_i A_j^T   (g = 0 .. 7),
// each G_g an exact int32 sum of int8 products (|G_g| <= 8 * 4096 * n), the terms with
// i + j > 7 (below 2^-56 per product element) dropped: the Ozaki-scheme emulation of an fp64
// product with fixed-point splits. The error of one squaring is ~1e-17 n in the largest
// element, about that of an fp64 GEMM.
//
// Tiles of 128 x 64 over the lower triangle (the upper part mirrored), walked by a persistent
// CTA per SM with specialised warps. A producer lane feeds a 3-stage ring with two 3-D TMA loads
// per stage (the eight planes of the A row block and of the B row block, 32 bytes of K each,
// 32-byte swizzle, no multicast); an MMA lane issues the 36 digit-pair MMAs of each stage
// (M = 128, N = 64, K = 32) into eight 64-column int32 accumulators in TMEM (all 512 columns,
// G_g at column 64 g); four epilogue warps combine the accumulators in fp64 (Horner over g)
// into a staging tile, release TMEM for the CTA's next tile, and apply the fused SP2 step while
// that tile's MMAs run: X_{k+1} = X_k^2 or 2 X_k - X_k^2 by the step's decision, written in
// fp64 with its mirror (coalesced), and the tile's share of tr X_{k+1} and |X_{k+1}|_F^2 for
// the next decision. A separate elementwise kernel then splits X_{k+1} into its digit planes
// (integer arithmetic, every SM busy). Every mbarrier wait has a time limit.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "common.cuh"
#include "kernels.hpp"
#include "tcgen05.cuh"

namespace pm7 {
namespace {
using namespace tc;

constexpr int kDigits = 8;               // int8 planes per element
constexpr int IM = 128, IN = 64;         // tile rows, columns
constexpr int kTmemCols = kDigits * IN;  // eight 64-column accumulators
constexpr int LDT = IN + 1;              // staging row stride (doubles)

// The stage geometry for KS bytes of K per stage (32: 32-byte swizzle, 3 stages of 48 KB), and
// the CTA's shared memory: the stages, the epilogue's fp64 staging tile (its own, so that the
// next tile's loads proceed during the epilogue), the partials, the barriers and the alignment
// slack.
template <int KS>
struct I8Stage {
  static constexpr int STAGES = 3;
  static constexpr int A_PLANE = IM * KS, B_PLANE = IN * KS;
  static constexpr int BYTES = kDigits * (A_PLANE + B_PLANE);
  static constexpr int SMEM = STAGES * BYTES + IM * LDT * 8 + 64 + (2 * STAGES + 2) * 8 + 16 + 1024;
  static_assert(SMEM <= 227 * 1024, "one CTA per SM within the shared-memory limit");
};

// Shared-memory matrix descriptor: K-major operand with KS-byte rows and the matching swizzle
// (8-row groups 8 KS bytes apart), version 1; the plane bases are 1024-byte aligned.
template <int KS>
__device__ __forceinline__ uint64_t desc_swz(const void *tile) {
  const uint32_t addr = smem_u32(tile);
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);           // start address
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((8 * KS) >> 4) << 32;            // stride byte offset
  d |= (uint64_t)1 << 46;                          // version
  d |= (uint64_t)(KS == 32 ? 6 : 4) << 61;         // SWIZZLE_32B / SWIZZLE_64B
  return d;
}

// Instruction descriptor, kind::i8: s32 accumulate, signed 8-bit A and B, both K-major, N = 64, M = 128.
constexpr uint32_t kIdescI8 = (2u << 4)    // c_format S32
                              | (1u << 7)  // a_format signed 8-bit
                              | (1u << 10) // b_format signed 8-bit
                              | ((uint32_t)(IN >> 3) << 17) | ((uint32_t)(IM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdescI8), "r"(accumulate));
}

// The digits of x (see the file header) by integer arithmetic: x rounded to a multiple of
// 2^-55 (a 64-bit fixed-point integer, exact scaling), then balanced base-128 digits from the
// lowest (each in [-64, 63], the remainder divided exactly by 128), the first digit what is
// left (|a_0| <= 127 for |x| < 1.98). False, with zero digits, beyond that range or for a
// non-finite x.
__device__ __forceinline__ bool split_digits(double x, int8_t (&a)[kDigits]) {
  if (!(fabs(x) < 1.98)) {
#pragma unroll
    for (int p = 0; p < kDigits; ++p) a[p] = 0;
    return false;
  }
  long long v = __double2ll_rn(x * 36028797018963968.0);  // x 2^55
#pragma unroll
  for (int p = kDigits - 1; p >= 1; --p) {
    const long long d = ((v + 64) & 127) - 64;
    a[p] = (int8_t)d;
    v = (v - d) >> 7;
  }
  a[0] = (int8_t)v;
  return true;
}

// Lower tiles of 128 x 64: row block r holds column blocks 0 .. min(2r + 1, tn - 1).
__host__ __device__ __forceinline__ int i8_tile_count(int n) {
  const int tm = (n + IM - 1) / IM, tn = (n + IN - 1) / IN;
  int t = 0;
  for (int r = 0; r < tm; ++r) t += 2 * r + 2 < tn ? 2 * r + 2 : tn;
  return t;
}
__device__ __forceinline__ void i8_tile(int t, int n, int &bm, int &bn) {
  const int tn = (n + IN - 1) / IN;
  int r = 0;
  for (;;) {
    const int c = 2 * r + 2 < tn ? 2 * r + 2 : tn;
    if (t < c) break;
    t -= c;
    ++r;
  }
  bm = r;
  bn = t;
}

// Persistent fused SP2 steps (see the file header) into x_out (fp64; its digit planes follow
// from k_sp2_digits). One CTA per SM walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// with specialised warps: warp 4 lane 0 feeds the TMA ring (running ahead into the next tile),
// warp 5 lane 0 issues the MMAs and owns the TMEM allocation, warps 0-3 (TMEM lane quarters
// 0-3) are the epilogue. The eight accumulators fill the 512 TMEM columns, so the epilogue first
// drains them into the fp64 staging tile and releases TMEM (tmem_empty), and only then applies
// the SP2 update and stores, while the MMAs of the CTA's next tile already run. `map_a` /
// `map_b` are the input digit planes' 3-D tensor maps with 128- and 64-row boxes. The step does
// nothing once an earlier step has stopped the purification.
template <int KS>
__global__ void __launch_bounds__(192, 1) k_sp2_step_i8(const __grid_constant__ CUtensorMap map_a,
                                                        const __grid_constant__ CUtensorMap map_b, int n,
                                                        const double *__restrict__ x_in, double *__restrict__ x_out,
                                                        double *__restrict__ state, int step,
                                                        double *__restrict__ parts, int *__restrict__ error) {
  using G = I8Stage<KS>;
  constexpr int ISTAGES = G::STAGES, I_STAGE = G::BYTES, A_PLANE = G::A_PLANE, B_PLANE = G::B_PLANE;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  if (!sp2_active(state, step)) return;  // the whole CTA, before any barrier or TMEM set-up
  const int tiles = i8_tile_count(n);
  const bool square = state[kSp2Square] != 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) state[kSp2Parts] = (double)tiles;

  unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  double *T = reinterpret_cast<double *>(smem + ISTAGES * I_STAGE);  // epilogue staging, IM x LDT
  double *red = T + IM * LDT;
  uint64_t *full = reinterpret_cast<uint64_t *>(red + 8);
  uint64_t *empty = full + ISTAGES;
  uint64_t *tmem_full = empty + ISTAGES;
  uint64_t *tmem_empty = tmem_full + 1;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tmem_empty + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ktiles = (n + KS - 1) / KS;

  if (threadIdx.x == 0) {
    for (int s = 0; s < ISTAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tmem_full, 1);
    mbar_init(tmem_empty, 4);  // one arrival per epilogue warp
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    if (lane == 0) {  // producer: the TMA ring over all of this CTA's tiles
      int g = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        int bm, bn;
        i8_tile(t, n, bm, bn);
        for (int kt = 0; kt < ktiles; ++kt, ++g) {
          const int s = g % ISTAGES;
          if (g >= ISTAGES && !mbar_wait(&empty[s], (uint32_t)((g / ISTAGES - 1) & 1), abort_flag)) {
            ok = false;
            break;
          }
          unsigned char *st = smem + s * I_STAGE;
          mbar_expect_tx(&full[s], I_STAGE);
          tma_load_3d(st, &map_a, &full[s], kt * KS, bm * IM, 0);
          tma_load_3d(st + kDigits * A_PLANE, &map_b, &full[s], kt * KS, bn * IN, 0);
        }
      }
    }
  } else if (warp == 5) {
    if (lane == 0) {  // MMA issuer: digit pairs (i, j), i + j <= 7, into accumulator i + j
      int g = 0, u = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++u) {
        // the epilogue has drained the previous tile's accumulators
        if (u > 0 && !mbar_wait(tmem_empty, (uint32_t)((u - 1) & 1), abort_flag)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        for (int kt = 0; kt < ktiles; ++kt, ++g) {
          const int s = g % ISTAGES;
          if (!mbar_wait(&full[s], (uint32_t)((g / ISTAGES) & 1), abort_flag)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          unsigned char *st = smem + s * I_STAGE;
          // plane and K offsets go into the descriptors' start-address field (16-byte units;
          // the stage lies below 256 KB, so the 14-bit field does not carry)
          const uint64_t da = desc_swz<KS>(st), db = desc_swz<KS>(st + kDigits * A_PLANE);
#pragma unroll
          for (int ks = 0; ks < KS / 32; ++ks) {  // K = 32 bytes per MMA: start address + 32 ks bytes
            const uint64_t koff = (uint64_t)(2 * ks);
#pragma unroll
            for (int i = 0; i < kDigits; ++i) {
              const uint64_t a = da + (uint64_t)((i * A_PLANE) >> 4) + koff;
#pragma unroll
              for (int j = 0; j + i < kDigits; ++j)
                mma_i8(tmem + (uint32_t)((i + j) * IN), a, db + (uint64_t)((j * B_PLANE) >> 4) + koff,
                       (kt > 0 || ks > 0 || i > 0) ? 1u : 0u);
            }
          }
          mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
        }
        if (ok) mma_commit(tmem_full);  // the tile's accumulators are final once its MMAs completed
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // epilogue, warps 0-3: warp w reads TMEM lanes 32 w .. 32 w + 31 = tile rows
    int u = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++u) {
      int bm, bn;
      i8_tile(t, n, bm, bn);
      const int m0 = bm * IM, n0 = bn * IN;
      const bool ok = mbar_wait(tmem_full, (uint32_t)(u & 1), abort_flag);
      asm volatile("bar.sync 1, 128;" ::: "memory");  // every epilogue thread has its verdict
      if (!ok || *abort_flag) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      // accumulators -> X_k^2 tile in fp64 (Horner over g), thread = tile row
#pragma unroll 1
      for (int h = 0; h < IN / 32; ++h) {
        double acc[32];
        uint32_t r[32];
        tmem_ld32(tmem, warp, (kDigits - 1) * IN + 32 * h, r);
#pragma unroll
        for (int q = 0; q < 32; ++q) acc[q] = (double)(int)r[q];
#pragma unroll 1
        for (int g = kDigits - 2; g >= 0; --g) {
          tmem_ld32(tmem, warp, g * IN + 32 * h, r);
#pragma unroll
          for (int q = 0; q < 32; ++q) acc[q] = (double)(int)r[q] + acc[q] * 0.0078125;  // 2^-7
        }
#pragma unroll
        for (int q = 0; q < 32; ++q) T[(warp * 32 + lane) * LDT + 32 * h + q] = acc[q] * 0.000244140625;  // 2^-12
      }
      // TMEM is free for the next tile's MMAs
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(tmem_empty)) : "memory");
      asm volatile("bar.sync 1, 128;" ::: "memory");  // the staging tile is complete
      // the tile's lower-triangle elements (row >= column), thread = column c of a 64-row half;
      // X_k read 8 rows at a time; the new value goes back into the staging for the mirror
      double tr = 0.0, fro = 0.0;
      const int c = threadIdx.x & (IN - 1), i_lo = (threadIdx.x / IN) * (IM / 2), gc = n0 + c;
      for (int i0 = i_lo; i0 < i_lo + IM / 2; i0 += 8) {
        double xo[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int gr = m0 + i0 + v;
          const bool live = !square && gr < n && gc < n && gr >= gc;
          xo[v] = live ? __ldg(x_in + (size_t)gr * n + gc) : 0.0;
        }
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int i = i0 + v, gr = m0 + i;
          if (gr >= n || gc >= n || gr < gc) continue;
          const double y = T[i * LDT + c];
          const double x = square ? y : 2.0 * xo[v] - y;
          T[i * LDT + c] = x;
          x_out[(size_t)gr * n + gc] = x;
          if (gr == gc) {
            tr += x;
            fro += x * x;
          } else {
            fro += 2.0 * x * x;
          }
        }
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      // the mirror (column block n0 .. n0 + 63 as rows), thread = column m0 + threadIdx.x
      const int mc = m0 + threadIdx.x;
      for (int j = 0; j < IN; ++j) {
        const int gr = n0 + j;
        if (gr >= n || mc >= n || mc <= gr) continue;
        x_out[(size_t)gr * n + mc] = T[threadIdx.x * LDT + j];
      }
      // the tile's partials, summed in a fixed order
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        tr += __shfl_down_sync(0xffffffffu, tr, o);
        fro += __shfl_down_sync(0xffffffffu, fro, o);
      }
      if (lane == 0) {
        red[2 * warp] = tr;
        red[2 * warp + 1] = fro;
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");  // partials written, staging reads done
      if (threadIdx.x == 0) {
        parts[2 * t] = (red[0] + red[2]) + (red[4] + red[6]);
        parts[2 * t + 1] = (red[1] + red[3]) + (red[5] + red[7]);
      }
    }
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(error, 1);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 5) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// The digit planes (plane p at dig + p plane, rows of ld8 bytes) of an n x n fp64 matrix: the
// start iterate, and the output of each step (skipped, like the step, once the purification
// has stopped; step < 0: always). Grid (ceil(n / 1024), n): a thread takes four columns of one
// row and stores each plane's four digits as one 32-bit word (ld8 is a multiple of 16, so the
// words stay inside the row's padding).
__global__ void __launch_bounds__(256) k_sp2_digits(int n, int ld8, const double *__restrict__ X,
                                                    int8_t *__restrict__ dig, const double *__restrict__ state,
                                                    int step, int *__restrict__ error) {
  if (step >= 0 && !sp2_active(state, step)) return;
  const int row = blockIdx.y, c0 = (blockIdx.x * 256 + threadIdx.x) * 4;
  if (c0 >= n) return;
  const size_t plane = (size_t)n * ld8;
  const double *xr = X + (size_t)row * n;
  uint32_t word[kDigits];
#pragma unroll
  for (int p = 0; p < kDigits; ++p) word[p] = 0u;
  bool good = true;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int8_t a[kDigits];
    if (c0 + q < n) {
      good = split_digits(xr[c0 + q], a) && good;
    } else {
#pragma unroll
      for (int p = 0; p < kDigits; ++p) a[p] = 0;
    }
#pragma unroll
    for (int p = 0; p < kDigits; ++p) word[p] |= (uint32_t)(uint8_t)a[p] << (8 * q);
  }
  int8_t *base = dig + (size_t)row * ld8 + c0;
#pragma unroll
  for (int p = 0; p < kDigits; ++p) *reinterpret_cast<uint32_t *>(base + (size_t)p * plane) = word[p];
  if (!good) atomicExch(error, 2);
}

}  // namespace

// K bytes per pipeline stage (32-byte swizzle): with the epilogue's own staging tile, three
// 48 KB stages fit beside it.
constexpr int kKStage = 32;

// CTAs of the persistent step: one per SM (or per tile, when there are fewer tiles).
static int i8_grid(int tiles) {
  static std::mutex mu;
  static int sms[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int c;
  {
    std::lock_guard<std::mutex> lock(mu);
    int &slot = sms[dev & 63];
    if (slot == 0 && cudaDeviceGetAttribute(&slot, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) slot = 148;
    c = slot;
  }
  return tiles < c ? tiles : c;
}

int sp2_i8_ld(int n) { return ((n + 15) / 16) * 16; }
size_t sp2_i8_digit_bytes(int n) { return (size_t)kDigits * n * sp2_i8_ld(n); }
int sp2_i8_tiles(int n) { return i8_tile_count(n); }

// The two tensor maps of a digit-plane set: 3-D (column, row, plane) over n x n bytes per
// plane, boxes of 32 columns x 128 (A) or 64 (B) rows x 8 planes, 32-byte swizzle; columns
// and rows beyond n read as zero.
bool make_digit_maps(const int8_t *dig, int n, void *map_a, void *map_b) {
  TensorMapEncodeFn fn = tensor_map_encode_fn();
  const int ld8 = sp2_i8_ld(n);
  if (!fn || n < 1 || (reinterpret_cast<uintptr_t>(dig) & 15) != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)kDigits};
  const cuuint64_t strides[2] = {(cuuint64_t)ld8, (cuuint64_t)ld8 * n};
  const cuuint32_t estr[3] = {1, 1, 1};
  const cuuint32_t ks = (cuuint32_t)kKStage;
  const cuuint32_t box_a[3] = {ks, IM, kDigits}, box_b[3] = {ks, IN, kDigits};
  void *maps[2] = {map_a, map_b};
  const cuuint32_t *boxes[2] = {box_a, box_b};
  for (int k = 0; k < 2; ++k) {
    const CUresult r = fn(reinterpret_cast<CUtensorMap *>(maps[k]),
                          CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<int8_t *>(dig), dims, strides, boxes[k], estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, ks == 32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
  }
  return true;
}

void prepare_i8_kernels() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaFuncSetAttribute(k_sp2_step_i8<kKStage>, cudaFuncAttributeMaxDynamicSharedMemorySize, I8Stage<kKStage>::SMEM);
  done[dev] = true;
}

void launch_sp2_digits(cudaStream_t st, int n, const double *X, int8_t *dig, const double *state, int step,
                       int *error) {
  k_sp2_digits<<<dim3((n + 1023) / 1024, n), 256, 0, st>>>(n, sp2_i8_ld(n), X, dig, state, step, error);
  note_launch();
}

void launch_sp2_step_i8(cudaStream_t st, int n, const void *map_a, const void *map_b, const double *x_in,
                        double *x_out, int8_t *dig_out, double *state, double *parts, int step, int *error) {
  prepare_i8_kernels();
  const CUtensorMap &ma = *reinterpret_cast<const CUtensorMap *>(map_a);
  const CUtensorMap &mb = *reinterpret_cast<const CUtensorMap *>(map_b);
  k_sp2_step_i8<kKStage><<<i8_grid(i8_tile_count(n)), 192, I8Stage<kKStage>::SMEM, st>>>(
      ma, mb, n, x_in, x_out, state, step, parts, error);
  note_launch();
  launch_sp2_digits(st, n, x_out, dig_out, state, step, error);
}

}  // namespace pm7
