// Reference-order sums: the exact value of a left-to-right f64 accumulation
//
//     s = -0.0;  for i in 0..n: s = fl(s + t_i),   t_i = a_i  or  t_i = fl(a_i * b_i),
//
// which is what pm7-rs computes for its energies (`Matrix::frobenius_dot`,
// src/linalg.rs:138-141, and `core_core_energy`, src/repulsion.rs:16-36, are plain
// iterator folds). At a thousand atoms the rounding of such a fold is ~1e-5 kcal/mol of
// heat of formation (millions of terms on a running sum of ~5e6 eV), so a drop-in has to
// reproduce the fold itself, not a more accurate sum.
//
// The fold is evaluated in parallel and exactly. While the running sum S stays in one
// binade [2^(k-1), 2^k), every S is a multiple of u = 2^(k-53) and fl(S + t) =
// S + u * rne(t / u): the sum of a run of terms is S + u * (sum of integers), where the
// integers depend on the terms alone. So
//   1. chunk sums (any order) and their prefix give an estimate of S at each chunk start;
//   2. each 256-term sub-block of a chunk rounds its terms to the grid of its estimated
//      start and keeps the integer total and the lowest and highest integer prefix, and the
//      chunk keeps the same summary of itself when its sub-blocks share one grid;
//   3. one warp walks the chunks in order with the true S: a summary is applied in one step
//      when S really is in the binade it assumed and every running value stays strictly
//      inside it (checked exactly in integers). A chunk whose summary does not apply is
//      taken sub-block by sub-block; a sub-block whose summary does not apply either is
//      recomputed on the grid of the true S, and added term by term when it still leaves
//      the binade, holds a tie (t / u exactly half an integer, where the parity of S
//      decides), a non-finite or a huge term.
// A running value that stays inside [2^(k-1) + u, 2^k - u] was rounded on the grid u (the
// exact sum it rounds was in the binade too), so every step of this is exact and the
// result is the fold's bits for any input.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "kernels.hpp"

namespace pm7 {

namespace {

constexpr int kSsThreads = 512;
constexpr int kSsPerThread = 8;
constexpr int kSsChunk = kSsThreads * kSsPerThread;  // terms per chunk
constexpr int kSsSub = 256;                          // terms per sub-block of the walk (32 lanes x 8)
constexpr double kSsHuge = 1125899906842624.0;       // 2^50: larger grid multiples go term by term

constexpr int kSsSubs = kSsChunk / kSsSub;            // sub-blocks per chunk (one warp each)

// Integer summary of a run of terms on one grid: total, lowest and highest inclusive
// prefix, the binade exponent k of the grid (frexp convention), and a flag when the run
// cannot be applied in one step (a tie, a non-finite or huge term, no usable estimate).
struct RunRec {
  long long total, lo, hi;
  int k, flag;
};

struct ChunkRec {
  double csum;  // approximate chunk sum
  double est;   // approximate running sum before the chunk
  RunRec run;   // the whole chunk on one grid (flagged when its sub-blocks need different grids)
  RunRec sub[kSsSubs];  // each sub-block on the grid of its own estimated start
};

__device__ __forceinline__ double ss_term(const double *__restrict__ a, const double *__restrict__ b, size_t i) {
  return b ? __dmul_rn(a[i], b[i]) : a[i];
}

// Grid integer of t on the grid 2^(k-53); false when t is not finite, too large for the
// integer path, or exactly half-way (ties depend on the parity of the running sum).
__device__ __forceinline__ bool ss_grid(double t, int k, long long &n) {
  const double q = scalbn(t, 53 - k);
  if (!(fabs(q) <= kSsHuge)) return false;
  const double r = rint(q);
  if (fabs(q - r) == 0.5) return false;
  n = (long long)r;
  return true;
}

// Whether S (nonzero, finite, normal) sits in a binade, which (k), and its grid integer.
__device__ __forceinline__ bool ss_binade(double S, int &k, long long &I) {
  if (!(S != 0.0) || !isfinite(S) || fabs(S) < 1.0e-290) return false;
  frexp(S, &k);
  I = (long long)scalbn(S, 53 - k);
  return true;
}

// Whether every running value I + p, p in [lo, hi], keeps the sign of I and stays strictly
// inside the binade: |I + p| in [2^52 + 1, 2^53 - 1].
__device__ __forceinline__ bool ss_inside(long long I, long long lo, long long hi) {
  const long long a = 4503599627370497LL, b = 9007199254740991LL;  // 2^52 + 1, 2^53 - 1
  if (I > 0) return I + lo >= a && I + hi <= b;
  return I + hi <= -a && I + lo >= -b;
}

// The jobs of one launch: up to four inline (kernel parameters, nothing to upload) or a
// device table; first[j] is job j's first chunk, first[count] the total.
struct SsJobs {
  const SeqSumJob *table;
  const long long *first;
  SeqSumJob inl[4];
  long long inl_first[5];
  int count;
};

__device__ __forceinline__ const SeqSumJob &ss_job(const SsJobs &J, int j) { return J.table ? J.table[j] : J.inl[j]; }
__device__ __forceinline__ long long ss_first(const SsJobs &J, int j) { return J.table ? J.first[j] : J.inl_first[j]; }

// The job that owns global chunk c (the last job whose first chunk is <= c).
__device__ __forceinline__ int ss_owner(const SsJobs &J, long long c) {
  int lo = 0, hi = J.count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ss_first(J, mid) <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Pass 1: approximate chunk sums. One block per chunk (all jobs' chunks in one grid).
__global__ void __launch_bounds__(kSsThreads) k_ss_chunks(SsJobs J, ChunkRec *__restrict__ recs) {
  const long long c = blockIdx.x;
  const int j = ss_owner(J, c);
  const SeqSumJob &Jb = ss_job(J, j);
  const size_t base = (size_t)(c - ss_first(J, j)) * kSsChunk;
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < kSsPerThread; ++t) {
    const size_t i = base + (size_t)t * kSsThreads + threadIdx.x;
    if (i < Jb.n) s += ss_term(Jb.a, Jb.b, i);
  }
  __shared__ double part[kSsThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kSsThreads / 32; ++w) t += part[w];
    recs[c].csum = t;
  }
}

// Pass 2: exclusive prefix of each job's chunk sums (one block per job; approximate is
// enough: it only chooses the grid the chunk's integers are taken on).
constexpr int kSsScan = 256;
__global__ void __launch_bounds__(kSsScan) k_ss_scan(SsJobs J, ChunkRec *__restrict__ recs) {
  const long long c0 = ss_first(J, blockIdx.x);
  const int nchunks = (int)(ss_first(J, blockIdx.x + 1) - c0);
  ChunkRec *r = recs + c0;
  const int per = (nchunks + kSsScan - 1) / kSsScan;
  const int beg = min(nchunks, (int)threadIdx.x * per), end = min(nchunks, beg + per);
  double local = 0.0;
  for (int c = beg; c < end; ++c) local += r[c].csum;
  __shared__ double scan[kSsScan];
  scan[threadIdx.x] = local;
  __syncthreads();
  for (int o = 1; o < kSsScan; o <<= 1) {
    const double v = threadIdx.x >= (unsigned)o ? scan[threadIdx.x - o] : 0.0;
    __syncthreads();
    scan[threadIdx.x] += v;
    __syncthreads();
  }
  double run = scan[threadIdx.x] - local;
  for (int c = beg; c < end; ++c) {
    r[c].est = run;
    run += r[c].csum;
  }
}

// Pass 3: grid integers. Warp w of the chunk's block takes sub-block w (256 terms, 8 per
// lane); each sub-block is summarised on the grid of its own estimated start (the chunk's
// estimate plus the approximate sums of the sub-blocks before it), and the chunk as a whole
// when every sub-block chose the same grid.
__global__ void __launch_bounds__(kSsThreads) k_ss_ints(SsJobs J, ChunkRec *__restrict__ recs) {
  const long long c = blockIdx.x;
  const int j = ss_owner(J, c);
  const SeqSumJob &Jb = ss_job(J, j);
  ChunkRec &R = recs[c];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t beg = (size_t)(c - ss_first(J, j)) * kSsChunk + (size_t)warp * kSsSub;
  const size_t mine = beg + (size_t)lane * kSsPerThread;
  double t[kSsPerThread];
  double part = 0.0;
#pragma unroll
  for (int q = 0; q < kSsPerThread; ++q) {
    t[q] = mine + q < Jb.n ? ss_term(Jb.a, Jb.b, mine + q) : 0.0;
    part += t[q];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  __shared__ double sub_sum[kSsSubs];
  __shared__ RunRec sub_rec[kSsSubs];
  if (lane == 0) sub_sum[warp] = part;
  __syncthreads();
  double est = R.est;
  for (int w = 0; w < warp; ++w) est += sub_sum[w];
  int k = 0;
  bool ok = est != 0.0 && isfinite(est) && fabs(est) >= 1.0e-290;
  if (ok) frexp(est, &k);
  long long pre = 0, lo = LLONG_MAX, hi = LLONG_MIN;
#pragma unroll
  for (int q = 0; q < kSsPerThread; ++q)
    if (mine + q < Jb.n && ok) {
      long long v = 0;
      ok = ss_grid(t[q], k, v);
      pre += v;
      lo = min(lo, pre);
      hi = max(hi, pre);
    }
  ok = __all_sync(0xffffffffu, ok);
  long long inc = pre;  // inclusive scan of the lane totals
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lo != LLONG_MAX) {
    lo += inc - pre;
    hi += inc - pre;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const long long total = __shfl_sync(0xffffffffu, inc, 31);
  if (lane == 0) {
    const RunRec r{total, lo, hi, k, ok ? 0 : 1};
    sub_rec[warp] = r;
    R.sub[warp] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // the chunk on one grid: the sub-blocks' summaries chained, when they share the grid
    RunRec all{0, LLONG_MAX, LLONG_MIN, sub_rec[0].k, 0};
    for (int w = 0; w < kSsSubs; ++w) {
      const RunRec &r = sub_rec[w];
      if (r.flag || r.k != all.k) {
        all.flag = 1;
        break;
      }
      if (r.lo != LLONG_MAX) {
        all.lo = min(all.lo, all.total + r.lo);
        all.hi = max(all.hi, all.total + r.hi);
      }
      all.total += r.total;
    }
    R.run = all;
  }
}

// One sub-block (at most 256 terms from `beg`) added to S by the whole warp; S is the
// same in every lane before and after.
__device__ double ss_subblock(double S, const SeqSumJob &J, size_t beg, size_t end, int lane) {
  double t[kSsPerThread];
  const size_t mine = beg + (size_t)lane * kSsPerThread;
#pragma unroll
  for (int j = 0; j < kSsPerThread; ++j) t[j] = mine + j < end ? ss_term(J.a, J.b, mine + j) : 0.0;
  int k = 0;
  long long I = 0;
  bool ok = ss_binade(S, k, I);
  long long pre = 0, lo = LLONG_MAX, hi = LLONG_MIN;
  if (ok) {
#pragma unroll
    for (int j = 0; j < kSsPerThread; ++j)
      if (mine + j < end) {
        long long q = 0;
        if (!ss_grid(t[j], k, q)) ok = false;
        pre += q;
        lo = min(lo, pre);
        hi = max(hi, pre);
      }
  }
  ok = __all_sync(0xffffffffu, ok);
  if (ok) {
    long long inc = pre;  // inclusive scan of the lane totals
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    const long long off = inc - pre;
    if (lo != LLONG_MAX) {
      lo += off;
      hi += off;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const long long total = __shfl_sync(0xffffffffu, inc, 31);
    if (lo == LLONG_MAX || ss_inside(I, lo, hi)) return scalbn((double)(I + total), k - 53);
  }
  // term by term, in order (every lane adds the same values)
  for (int src = 0; src < 32; ++src)
#pragma unroll
    for (int j = 0; j < kSsPerThread; ++j) {
      const double v = __shfl_sync(0xffffffffu, t[j], src);
      if (beg + (size_t)src * kSsPerThread + j < end) S = S + v;
    }
  return S;
}

// Whether a run summary applies at S, and S after it (exact: an integer below 2^53 times a
// power of two).
__device__ __forceinline__ bool ss_apply(double &S, const RunRec &r) {
  int ks = 0;
  long long I = 0;
  if (r.flag || !ss_binade(S, ks, I) || ks != r.k) return false;
  if (r.lo != LLONG_MAX && !ss_inside(I, r.lo, r.hi)) return false;
  S = scalbn((double)(I + r.total), ks - 53);
  return true;
}

// Pass 4: the ordered walk, one warp per job. A chunk whose one-grid summary does not apply
// at the true running sum is taken sub-block by sub-block; a sub-block whose summary does
// not apply either is recomputed on the grid of the true sum or added term by term.
__global__ void __launch_bounds__(32) k_ss_walk(SsJobs J, const ChunkRec *__restrict__ recs) {
  const SeqSumJob &Jb = ss_job(J, blockIdx.x);
  const int lane = threadIdx.x;
  const long long c0 = ss_first(J, blockIdx.x);
  const size_t nchunks = (size_t)(ss_first(J, blockIdx.x + 1) - c0);
  const ChunkRec *r = recs + c0;
  double S = -0.0;
  for (size_t c = 0; c < nchunks; ++c) {
    // every lane reads the same summary (one broadcast load)
    const RunRec run = r[c].run;
    if (ss_apply(S, run)) continue;
    RunRec sub{0, 0, 0, 0, 1};
    if (lane < kSsSubs) sub = r[c].sub[lane];
    const size_t beg = c * (size_t)kSsChunk;
    for (int w = 0; w < kSsSubs; ++w) {
      const size_t sb = beg + (size_t)w * kSsSub;
      if (sb >= Jb.n) break;
      RunRec rw;
      rw.total = __shfl_sync(0xffffffffu, sub.total, w);
      rw.lo = __shfl_sync(0xffffffffu, sub.lo, w);
      rw.hi = __shfl_sync(0xffffffffu, sub.hi, w);
      rw.k = __shfl_sync(0xffffffffu, sub.k, w);
      rw.flag = __shfl_sync(0xffffffffu, sub.flag, w);
      if (ss_apply(S, rw)) continue;
      S = ss_subblock(S, Jb, sb, min(Jb.n, sb + kSsSub), lane);
    }
  }
  if (lane == 0) *Jb.out = S;
}

void ss_launch(cudaStream_t st, const SsJobs &J, long long total_chunks, void *scratch) {
  if (J.count <= 0) return;
  ChunkRec *recs = static_cast<ChunkRec *>(scratch);
  if (total_chunks > 0) {
    k_ss_chunks<<<(unsigned)total_chunks, kSsThreads, 0, st>>>(J, recs);
    k_ss_scan<<<J.count, kSsScan, 0, st>>>(J, recs);
    k_ss_ints<<<(unsigned)total_chunks, kSsThreads, 0, st>>>(J, recs);
    note_launch(3);
  }
  k_ss_walk<<<J.count, 32, 0, st>>>(J, recs);
  note_launch(1);
}

}  // namespace

size_t seqsum_chunks(size_t n) { return (n + kSsChunk - 1) / kSsChunk; }

size_t seqsum_scratch_bytes(size_t n_max, int jobs) {
  const size_t c = seqsum_chunks(n_max) * (size_t)(jobs > 0 ? jobs : 1);
  return sizeof(ChunkRec) * (c > 0 ? c : 1);
}

size_t seqsum_table_scratch_bytes(long long total_chunks) {
  return sizeof(ChunkRec) * (size_t)(total_chunks > 0 ? total_chunks : 1);
}

void launch_seqsum(cudaStream_t st, const SeqSumBatch &B, void *scratch) {
  SsJobs J{};
  J.count = B.count;
  long long c = 0;
  for (int j = 0; j < B.count; ++j) {
    J.inl[j] = B.job[j];
    J.inl_first[j] = c;
    c += (long long)seqsum_chunks(B.job[j].n);
  }
  J.inl_first[B.count] = c;
  ss_launch(st, J, c, scratch);
}

void launch_seqsum_table(cudaStream_t st, const SeqSumJob *jobs, const long long *first, int count,
                         long long total_chunks, void *scratch) {
  SsJobs J{};
  J.table = jobs;
  J.first = first;
  J.count = count;
  ss_launch(st, J, total_chunks, scratch);
}

}  // namespace pm7
