// kernels_read.cu -- read-out kernels: probabilities, marginals, sampling,
// amplitude gather, Pauli expectations.  Every reduction is deterministic:
// per-block partial sums in a fixed tree order, then a fixed-order combine,
// all in FP64 whatever the state precision.
#include <algorithm>

#include "common.cuh"
#include "read.h"

namespace ket {

namespace {

template <typename R>
__device__ __forceinline__ double pref(const typename Vec2<R>::T* a, uint64_t i) {
  typename Vec2<R>::T v = a[i];
  return norm2_ref(v.x, v.y);
}

// ------------------------------------------------------------------ sums
template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_norm_partial(const typename Vec2<R>::T* a, uint64_t N, uint64_t chunk,
                                                     double* partial) {
  __shared__ double red[32];
  uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  double acc = 0.0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) acc += pref<R>(a, i);
  double t = block_sum<NT>(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// Fixed-order sum of n partials (one block): thread t sums a strided subset
// sequentially, then a block tree.
template <int NT>
__global__ void __launch_bounds__(NT) k_sum(const double* partial, uint64_t n, double* out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (uint64_t i = threadIdx.x; i < n; i += NT) acc += partial[i];
  double t = block_sum<NT>(acc, red);
  if (threadIdx.x == 0) *out = t;
}

// out[j] = sum over blocks b of partial[b*stride + j], in block order.
__global__ void k_sum_columns(const double* partial, uint64_t nblocks, int width, double* out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= width) return;
  double acc = 0.0;
  for (uint64_t b = 0; b < nblocks; b++) acc += partial[b * width + j];
  out[j] = acc;
}

// ------------------------------------------------------------------ state comparison
// Per block: sum of conj(a_i) b_i (re, im) and max |a_i - b_i|, all in FP64.
template <typename RA, typename RB, int NT>
__global__ void __launch_bounds__(NT) k_compare(const typename Vec2<RA>::T* a, const typename Vec2<RB>::T* b,
                                                uint64_t N, uint64_t chunk, double* partial) {
  __shared__ double red[32];
  uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  double sr = 0.0, si = 0.0, mx = 0.0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) {
    const typename Vec2<RA>::T u = a[i];
    const typename Vec2<RB>::T v = b[i];
    const double ur = u.x, ui = u.y, vr = v.x, vi = v.y;
    sr += ur * vr + ui * vi;
    si += ur * vi - ui * vr;
    const double dr = ur - vr, di = ui - vi;
    mx = fmax(mx, sqrt(dr * dr + di * di));
  }
  const double tr = block_sum<NT>(sr, red);
  const double ti = block_sum<NT>(si, red);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < NT / 32; w++) m = fmax(m, red[w]);
    partial[3 * blockIdx.x] = tr;
    partial[3 * blockIdx.x + 1] = ti;
    partial[3 * blockIdx.x + 2] = m;
  }
}

// Fixed-order combine of the block partials (one thread).
__global__ void k_compare_combine(const double* partial, uint64_t nb, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double r = 0.0, i = 0.0, m = 0.0;
  for (uint64_t b = 0; b < nb; b++) {
    r += partial[3 * b];
    i += partial[3 * b + 1];
    m = fmax(m, partial[3 * b + 2]);
  }
  out[0] = r;
  out[1] = i;
  out[2] = m;
}

// ------------------------------------------------------------------ probabilities
template <typename R>
__global__ void k_probs_dense(const typename Vec2<R>::T* a, uint64_t off, uint64_t cnt, double thr, double* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
    double p = pref<R>(a, off + i);
    out[i] = p > thr ? p : 0.0;
  }
}

template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_count_kept(const typename Vec2<R>::T* a, uint64_t N, uint64_t chunk, double thr,
                                                   uint64_t* counts) {
  __shared__ unsigned long long red;
  if (threadIdx.x == 0) red = 0;
  __syncthreads();
  uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  unsigned long long c = 0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) c += pref<R>(a, i) > thr ? 1 : 0;
  atomicAdd(&red, c);  // integer: order does not matter
  __syncthreads();
  if (threadIdx.x == 0) counts[blockIdx.x] = red;
}

// Compaction preserving ascending index order within each chunk.
template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_compact_kept(const typename Vec2<R>::T* a, uint64_t N, uint64_t chunk, double thr,
                                                     const uint64_t* offsets, uint64_t cap, uint64_t* oidx, double* op) {
  __shared__ uint32_t wsum[NT / 32];
  __shared__ uint64_t running;
  if (threadIdx.x == 0) running = offsets[blockIdx.x];
  __syncthreads();
  uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (uint64_t s = lo; s < hi; s += NT) {
    uint64_t i = s + threadIdx.x;
    double p = 0.0;
    bool keep = false;
    if (i < hi) { p = pref<R>(a, i); keep = p > thr; }
    uint32_t bal = __ballot_sync(0xffffffffu, keep);
    uint32_t before = __popc(bal & ((1u << lane) - 1));
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    uint64_t wbase = running;
    for (int j = 0; j < w; j++) wbase += wsum[j];
    if (keep) {
      uint64_t pos = wbase + before;
      if (pos < cap) { oidx[pos] = i; op[pos] = p; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t t = 0;
      for (int j = 0; j < NT / 32; j++) t += wsum[j];
      running += t;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ marginals
// P(q = 1) for every qubit: per-block partials [block][n].
template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_marginals(const typename Vec2<R>::T* a, int n, uint64_t chunk, double* partial) {
  __shared__ double red[32];
  uint64_t N = uint64_t(1) << n;
  uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  double acc[KET_MAX_QUBITS];
#pragma unroll
  for (int q = 0; q < KET_MAX_QUBITS; q++) acc[q] = 0.0;
  for (uint64_t i = lo + threadIdx.x; i < hi; i += NT) {
    double p = pref<R>(a, i);
#pragma unroll
    for (int q = 0; q < KET_MAX_QUBITS; q++)
      if (q < n && ((i >> q) & 1)) acc[q] += p;
  }
#pragma unroll
  for (int q = 0; q < KET_MAX_QUBITS; q++) {
    if (q < n) {  // uniform across the block
      double t = block_sum<NT>(acc[q], red);
      if (threadIdx.x == 0) partial[blockIdx.x * (uint64_t)n + q] = t;
    }
  }
}

// Joint distribution of m qubits.  Block b covers indices [b*2^c, (b+1)*2^c).
// Thread u walks the in-chunk bin combination u over the other in-chunk bits
// in ascending order; the out-of-chunk bin bits are fixed by the block.
template <typename R>
__global__ void k_marginal_dist(const typename Vec2<R>::T* a, int c, MarginalSpec spec, double* partial) {
  uint64_t base = (uint64_t)blockIdx.x << c;
  uint64_t chunkmask = (c >= 64) ? ~uint64_t(0) : ((uint64_t(1) << c) - 1);
  uint64_t inmask = spec.mask & chunkmask;
  uint64_t other = chunkmask & ~inmask;
  int nin = __popcll(inmask);
  uint32_t width = 1u << spec.m;
  // out-of-chunk bin bits from the block base
  uint32_t outbin = 0;
  for (int k = 0; k < spec.m; k++)
    if (spec.q[k] >= c && ((base >> spec.q[k]) & 1)) outbin |= 1u << k;
  for (uint32_t u = threadIdx.x; u < (1u << nin); u += blockDim.x) {
    // scatter u over inmask
    uint64_t ubits = 0;
    {
      uint64_t msk = inmask;
      uint32_t uu = u;
      while (msk) {
        uint64_t low = msk & (~msk + 1);
        if (uu & 1) ubits |= low;
        uu >>= 1;
        msk ^= low;
      }
    }
    double acc = 0.0;
    uint64_t x = 0;
    do {
      acc += pref<R>(a, base | ubits | x);
      x = (x - other) & other;
    } while (x != 0);
    uint32_t bin = outbin;
    for (int k = 0; k < spec.m; k++)
      if (spec.q[k] < c && ((ubits >> spec.q[k]) & 1)) bin |= 1u << k;
    partial[(uint64_t)blockIdx.x * width + bin] = acc;
  }
}

// ------------------------------------------------------------------ sampling
// The sampling CDF is the reference's running FP64 sum over kept entries in
// ascending index order, rounded after every addition (circuit.ts:3429-3436),
// reproduced bit for bit at every state size.  It is kept as checkpoints:
// ck[k] = the running sum before entry 32k, ck[nk] = the total.  A draw finds
// its 32-entry sub-chunk by binary search over ck and finishes with the
// reference's own FP64 additions from ck[k].
//
// While the running sum s stays in one binade [2^(e-1), 2^e), every value it
// takes is a multiple of u = 2^(e-53): s = S u with S an integer in
// [2^52, 2^53).  Adding p rounds to the nearest multiple of u, so
// s + p = (S + d) u with d = round(p / u) -- an increment that does not
// depend on s, except when p / u lies exactly halfway (the tie goes to the
// even S + d) or when S + d reaches 2^53 (the sum leaves the binade and rounds
// on the next grid).  A run of entries inside one binade is therefore an
// integer prefix sum of the d's.  Five kernels build the checkpoints:
//   k_cdf_block_sums    per block of 4096 entries, the plain sum of the kept
//                       p's and the first and last kept index;
//   k_cdf_block_prefix  an approximate exclusive prefix of those sums -- it
//                       only guesses the binade each block starts in -- and
//                       the first and last kept index of the state;
//   k_cdf_block_d       per block, in the guessed binade, the d's, their sum D
//                       and their exclusive prefix at every 32-entry
//                       sub-chunk; a block holding a tie or an oversized d, or
//                       with nothing kept before it, is marked unclean;
//   k_cdf_walk          one CTA carries the exact running sum across windows
//                       of blocks.  A block is taken whole when nothing in it
//                       is kept, or when it is clean in the binade the exact
//                       sum is in and S + D stays below 2^53 -- its integer
//                       prefix is then exact.  Any other block runs entry by
//                       entry (cdf_exact_range): integer prefix sums up to the
//                       next tie or crossing, which takes the FP64 addition
//                       itself;
//   k_cdf_fill          the checkpoints of the blocks taken whole, from their
//                       exact start and the sub-chunk prefixes.
// Only blocks holding a binade crossing, a tie or the first kept entry run
// entry by entry: a crossing happens about once per doubling of s.
constexpr int kCdfThreads = 1024;
constexpr int kCdfPer = 4;                          // entries per thread per chunk
constexpr int kCdfChunk = kCdfThreads * kCdfPer;    // 4096
constexpr int kCdfBlock = 4096;                     // entries per block
constexpr int kCdfSub = 32;                         // entries per checkpoint
constexpr int kCdfSubPerBlock = kCdfBlock / kCdfSub;
constexpr int kCdfWalkPer = 4;                      // blocks per walker thread per window
constexpr long long kTwo52 = 4503599627370496ll;
constexpr long long kTwo53 = 9007199254740992ll;
static_assert(kCdfChunk == kCdfBlock, "an entry-by-entry block is one chunk");

enum : int { kBlkUnclean = 0, kBlkClean = 1, kBlkEmpty = 2, kBlkExact = 3 };

// Inclusive block scan of v over NT threads; `wsum` holds 32 partials.
template <int NT, typename T>
__device__ __forceinline__ T block_scan_incl(T v, T* wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) wsum[w] = v;
  __syncthreads();
  if (w == 0) {
    T x = lane < NT / 32 ? wsum[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    wsum[lane] = x;
  }
  __syncthreads();
  const T r = v + (w > 0 ? wsum[w - 1] : T(0));
  __syncthreads();  // wsum is reused by the next scan
  return r;
}

// Block minimum of v over NT threads; every thread gets it.
template <int NT>
__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long* wred) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) wred[w] = v;
  __syncthreads();
  if (w == 0) {
    unsigned long long x = lane < NT / 32 ? wred[lane] : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) wred[32] = x;
  }
  __syncthreads();
  const unsigned long long r = wred[32];
  __syncthreads();
  return r;
}

// The kept probability of entry i: p when p > thr, else +0.0 (adds nothing).
template <typename R>
__device__ __forceinline__ double kept_p(const typename Vec2<R>::T* a, uint64_t i, double thr) {
  const double p = pref<R>(a, i);
  return p > thr ? p : 0.0;
}

template <typename R>
__global__ void __launch_bounds__(256) k_cdf_block_sums(const typename Vec2<R>::T* a, uint64_t N, double thr,
                                                        double* bsum, unsigned long long* bfirst,
                                                        unsigned long long* blast) {
  __shared__ double red[32];
  __shared__ unsigned long long wred[33];
  const uint64_t lo = (uint64_t)blockIdx.x * kCdfBlock;
  double acc = 0.0;
  unsigned long long f = ~0ull, l = ~0ull;  // l holds ~index, so the minimum is the largest index
#pragma unroll 4
  for (int k = 0; k < kCdfBlock / 256; k++) {
    const uint64_t i = lo + (uint64_t)k * 256 + threadIdx.x;
    if (i < N) {
      const double p = pref<R>(a, i);
      if (p > thr) {
        acc += p;
        if (f == ~0ull) f = i;
        l = ~(unsigned long long)i;
      }
    }
  }
  const double t = block_sum<256>(acc, red);
  f = block_min_u64<256>(f, wred);
  l = block_min_u64<256>(l, wred);
  if (threadIdx.x == 0) {
    bsum[blockIdx.x] = t;
    bfirst[blockIdx.x] = f;
    blast[blockIdx.x] = l;
  }
}

// bsum[0..nb) -> its exclusive prefix, bsum[nb] = the total; fl[0] = the
// first kept index, fl[1] = the last (~0: nothing kept).
__global__ void __launch_bounds__(kCdfThreads) k_cdf_block_prefix(double* bsum, const unsigned long long* bfirst,
                                                                  const unsigned long long* blast, uint64_t nb,
                                                                  unsigned long long* fl) {
  __shared__ double wsd[32];
  __shared__ unsigned long long wred[33];
  const uint64_t per = (nb + kCdfThreads - 1) / kCdfThreads;
  const uint64_t lo = min(nb, (uint64_t)threadIdx.x * per), hi = min(nb, lo + per);
  double t = 0.0;
  unsigned long long f = ~0ull, l = ~0ull;
  for (uint64_t b = lo; b < hi; b++) {
    t += bsum[b];
    f = min(f, bfirst[b]);
    l = min(l, blast[b]);
  }
  const double incl = block_scan_incl<kCdfThreads>(t, wsd);
  double x = incl - t;
  for (uint64_t b = lo; b < hi; b++) {
    const double v = bsum[b];
    bsum[b] = x;
    x += v;
  }
  f = block_min_u64<kCdfThreads>(f, wred);
  l = block_min_u64<kCdfThreads>(l, wred);
  if (threadIdx.x == kCdfThreads - 1) bsum[nb] = incl;
  if (threadIdx.x == 0) {
    fl[0] = f;
    fl[1] = l == ~0ull ? ~0ull : ~l;
  }
}

// Warp w handles sub-chunks 16w .. 16w + 15; lane l reads entry 32j + l of
// sub-chunk j, so every load is 32 consecutive amplitudes.
template <typename R>
__global__ void __launch_bounds__(256) k_cdf_block_d(const typename Vec2<R>::T* a, uint64_t N, double thr,
                                                     const double* bstart_approx, long long* ckd, long long* bd,
                                                     int* bst, int* be) {
  static_assert(kCdfSubPerBlock == 8 * 16, "8 warps of 16 sub-chunks");
  __shared__ long long wsum[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint64_t b = blockIdx.x, lo = b * kCdfBlock;
  const double A = bstart_approx[b];
  int e = 0;
  if (A > 0.0) frexp(A, &e);
  const bool guess = A > 0.0;
  bool pos = false, bad = false;
  long long mine = 0;  // lane k < 16: the d-sum of sub-chunk 16w + k
#pragma unroll 4
  for (int k = 0; k < 16; k++) {
    const uint64_t i = lo + (uint64_t)(16 * w + k) * kCdfSub + lane;
    const double p = i < N ? kept_p<R>(a, i, thr) : 0.0;
    pos |= p > 0.0;
    long long d = 0;
    if (guess) {
      const double q = ldexp(p, 53 - e);  // p / u, exact
      if (q >= 4503599627370496.0) bad = true;  // 2^52: S + d would leave the binade
      else if (q - floor(q) == 0.5) bad = true;   // a tie: the rounding depends on S
      else d = (long long)rint(q);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == k) mine = d;
  }
  const bool any_pos = __syncthreads_or(pos);
  const bool any_bad = __syncthreads_or(bad);
  // a sub-chunk sum is below 2^57; clamped at 2^53 the block total stays exact
  // below 2^53 and cannot overflow
  const long long v = lane < 16 ? (mine < kTwo53 ? mine : kTwo53) : 0;
  const long long incl = block_scan_incl<256>(v, wsum);
  __shared__ long long total;
  if (threadIdx.x == 255) total = incl;
  __syncthreads();
  const uint64_t j = 16 * w + lane;
  if (lane < 16 && lo + j * kCdfSub < N) ckd[b * kCdfSubPerBlock + j] = incl - v;
  if (threadIdx.x == 0) {
    int st;
    if (!any_pos) st = kBlkEmpty;
    else if (!guess || any_bad || total >= kTwo53) st = kBlkUnclean;
    else st = kBlkClean;
    bst[b] = st;
    be[b] = e;
    bd[b] = total;
  }
}

// The running sum over entries [lo, hi) (hi - lo <= kCdfChunk) in the
// reference's rounding, from the exact sum *s_io before lo.  Writes the
// checkpoints ck[(i + 1) / 32] for entries i with (i + 1) % 32 == 0 and
// i + 1 < hi, and leaves the sum after entry hi - 1 in *s_io.  Called by the
// whole CTA of kCdfThreads threads.
template <typename R>
__device__ void cdf_exact_range(const typename Vec2<R>::T* a, uint64_t lo, uint64_t hi, double thr, double* ck,
                                double* s_io, unsigned long long* c_io, long long* wsum, unsigned long long* wred) {
  const int tid = threadIdx.x;
  const unsigned long long NONE = ~0ull;
  if (tid == 0) *c_io = lo;
  __syncthreads();
  for (;;) {
    const uint64_t c = *c_io;
    const double s = *s_io;
    if (c >= hi) break;
    // this thread's entries c + kCdfPer*tid + k
    const uint64_t i0 = c + (uint64_t)kCdfPer * tid;
    double pv[kCdfPer];
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) pv[k] = i0 + k < hi ? kept_p<R>(a, i0 + k, thr) : 0.0;
    if (s == 0.0) {
      // before the first positive kept entry the sum is +0.0; that entry sets
      // it exactly
      unsigned long long f = NONE;
#pragma unroll
      for (int k = 0; k < kCdfPer; k++)
        if (f == NONE && pv[k] > 0.0) f = i0 + k;
      f = block_min_u64<kCdfThreads>(f, wred);
      const uint64_t z = f == NONE ? hi : f;
#pragma unroll
      for (int k = 0; k < kCdfPer; k++) {
        const uint64_t i = i0 + k;
        if (i < z && ((i + 1) & (kCdfSub - 1)) == 0 && i + 1 < hi) ck[(i + 1) / kCdfSub] = 0.0;
      }
      if (tid == 0) {
        if (f != NONE) {
          const double sn = 0.0 + kept_p<R>(a, f, thr);
          if (((f + 1) & (kCdfSub - 1)) == 0 && f + 1 < hi) ck[(f + 1) / kCdfSub] = sn;
          *s_io = sn;
          *c_io = f + 1;
        } else {
          *c_io = hi;
        }
      }
      __syncthreads();
      continue;
    }
    // s in [2^(e-1), 2^e): u = 2^(e-53), S = s / u
    int e;
    frexp(s, &e);
    const long long S0 = (long long)ldexp(s, 53 - e);
    unsigned long long special = NONE;  // first entry that is a tie or crosses for sure
    long long d[kCdfPer];
    long long tsum = 0;
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) {
      const uint64_t i = i0 + k;
      d[k] = 0;
      if (i >= hi) continue;
      const double q = ldexp(pv[k], 53 - e);  // p / u, exact
      if (q >= 9007199254740992.0) {          // 2^53: the sum leaves the binade
        if (special == NONE) special = i;
        continue;
      }
      if (q - floor(q) == 0.5) {              // a tie: the rounding depends on S
        if (special == NONE) special = i;
        continue;
      }
      if (special == NONE) {
        d[k] = (long long)rint(q);
        tsum += d[k];
      }
    }
    special = block_min_u64<kCdfThreads>(special, wred);
    // entries at or after the first special one do not count in the scan
    if (special != NONE) {
      tsum = 0;
#pragma unroll
      for (int k = 0; k < kCdfPer; k++)
        if (i0 + k < special) tsum += d[k];
    }
    const long long incl = block_scan_incl<kCdfThreads>(tsum, wsum);
    long long Sr = S0 + incl - tsum;  // S before this thread's first entry
    unsigned long long cross = NONE;  // first entry whose sum reaches 2^53 u
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) {
      const uint64_t i = i0 + k;
      if (i >= hi || i >= special) break;
      const long long Sn = Sr + d[k];
      if (Sn >= kTwo53) { cross = i; break; }
      Sr = Sn;
    }
    cross = block_min_u64<kCdfThreads>(cross, wred);
    const uint64_t lim = c + (uint64_t)kCdfChunk < hi ? c + (uint64_t)kCdfChunk : hi;
    uint64_t stop = special < cross ? (uint64_t)special : (uint64_t)cross;
    if (stop > lim) stop = lim;
    // the exact sums of the entries before `stop`
    Sr = S0 + incl - tsum;
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) {
      const uint64_t i = i0 + k;
      if (i >= stop) break;
      Sr += d[k];
      const double v = ldexp((double)Sr, e - 53);
      if (((i + 1) & (kCdfSub - 1)) == 0 && i + 1 < hi) ck[(i + 1) / kCdfSub] = v;
      if (i + 1 == stop) *s_io = v;
    }
    __syncthreads();
    if (tid == 0) {
      double sp = *s_io;  // the sum before `stop` (s itself when stop == c)
      if (stop < lim) {
        // the special entry, by the reference's own FP64 addition
        sp = sp + kept_p<R>(a, stop, thr);
        if (((stop + 1) & (kCdfSub - 1)) == 0 && stop + 1 < hi) ck[(stop + 1) / kCdfSub] = sp;
        *s_io = sp;
        *c_io = stop + 1;
      } else {
        *c_io = stop;
      }
    }
    __syncthreads();
  }
}

template <typename R>
__global__ void __launch_bounds__(kCdfThreads) k_cdf_walk(const typename Vec2<R>::T* a, uint64_t N, double thr,
                                                          uint64_t nb, uint64_t nk, double* ck, const long long* bd,
                                                          int* bst, const int* be, double* bstart) {
  __shared__ long long wsum[32];
  __shared__ unsigned long long wred[33];
  __shared__ double s_sh;              // the exact running sum before block c
  __shared__ unsigned long long c_sh;  // the next block
  __shared__ unsigned long long x_sh;  // cdf_exact_range's position
  const int tid = threadIdx.x;
  const unsigned long long NONE = ~0ull;
  if (tid == 0) { s_sh = 0.0; c_sh = 0; }
  __syncthreads();
  for (;;) {
    const uint64_t c = c_sh;
    const double s = s_sh;
    if (c >= nb) break;
    int e = 0;
    long long S0 = 0;
    if (s > 0.0) {
      frexp(s, &e);
      S0 = (long long)ldexp(s, 53 - e);
    }
    // this thread's blocks c + kCdfWalkPer*tid + k
    const uint64_t b0 = c + (uint64_t)kCdfWalkPer * tid;
    long long dv[kCdfWalkPer];
    unsigned long long fail = NONE;  // first block that is not taken whole
#pragma unroll
    for (int k = 0; k < kCdfWalkPer; k++) {
      const uint64_t b = b0 + k;
      dv[k] = 0;
      if (b >= nb || fail != NONE) continue;
      const int st = bst[b];
      if (st == kBlkEmpty) continue;
      if (st == kBlkClean && s > 0.0 && be[b] == e) dv[k] = bd[b];
      else fail = b;
    }
    fail = block_min_u64<kCdfThreads>(fail, wred);
    long long tsum = 0;
#pragma unroll
    for (int k = 0; k < kCdfWalkPer; k++)
      if (b0 + k < fail) tsum += dv[k];
    const long long incl = block_scan_incl<kCdfThreads>(tsum, wsum);  // each D < 2^53: no overflow
    long long Sr = S0 + incl - tsum;
    unsigned long long cross = NONE;  // first block whose sum reaches 2^53 u
#pragma unroll
    for (int k = 0; k < kCdfWalkPer; k++) {
      const uint64_t b = b0 + k;
      if (b >= nb || b >= fail) break;
      if (Sr + dv[k] >= kTwo53) { cross = b; break; }
      Sr += dv[k];
    }
    cross = block_min_u64<kCdfThreads>(cross, wred);
    const uint64_t lim = c + (uint64_t)kCdfWalkPer * kCdfThreads < nb ? c + (uint64_t)kCdfWalkPer * kCdfThreads : nb;
    uint64_t stop = fail < cross ? (uint64_t)fail : (uint64_t)cross;
    if (stop > lim) stop = lim;
    // blocks before `stop` are taken whole
    Sr = S0 + incl - tsum;
#pragma unroll
    for (int k = 0; k < kCdfWalkPer; k++) {
      const uint64_t b = b0 + k;
      if (b >= stop) break;
      bstart[b] = s > 0.0 ? ldexp((double)Sr, e - 53) : 0.0;
      Sr += dv[k];
      if (b + 1 == stop) s_sh = s > 0.0 ? ldexp((double)Sr, e - 53) : 0.0;
    }
    __syncthreads();
    if (stop < lim) {
      // block `stop` entry by entry
      if (tid == 0) {
        const double sb = s_sh;
        bstart[stop] = sb;
        bst[stop] = kBlkExact;
        ck[stop * kCdfSubPerBlock] = sb;
      }
      const uint64_t lo = stop * kCdfBlock;
      const uint64_t hi = lo + kCdfBlock < N ? lo + kCdfBlock : N;
      cdf_exact_range<R>(a, lo, hi, thr, ck, &s_sh, &x_sh, wsum, wred);
      if (tid == 0) c_sh = stop + 1;
    } else if (tid == 0) {
      c_sh = stop;
    }
    __syncthreads();
  }
  if (tid == 0) ck[nk] = s_sh;
}

// Checkpoints of the blocks taken whole: the exact start plus the sub-chunk's
// d prefix, in the block's binade (ck holds the prefixes as integers until now).
__global__ void k_cdf_fill(double* ck, uint64_t nk, const int* bst, const int* be, const double* bstart) {
  long long* ckd = (long long*)ck;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nk; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = k / kCdfSubPerBlock;
    const int st = bst[b];
    if (st == kBlkEmpty) {
      ck[k] = bstart[b];
    } else if (st == kBlkClean) {
      const int e = be[b];
      const long long S = (long long)ldexp(bstart[b], 53 - e);
      ck[k] = ldexp((double)(S + ckd[k]), e - 53);
    }
  }
}

// One draw per thread: the first kept entry whose running sum is >= r, the
// last kept entry's sum taken as 1.0 (circuit.ts:3438-3451).  The host checks
// 0 <= r <= 1, so the walk ends inside one sub-chunk.
template <typename R>
__global__ void k_sample_ck(const typename Vec2<R>::T* a, uint64_t N, double thr, const double* ck, uint64_t nk,
                            const double* r, uint64_t shots, const unsigned long long* fl, uint64_t* out) {
  const uint64_t first = fl[0], last = fl[1];
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < shots; s += (uint64_t)gridDim.x * blockDim.x) {
    if (last == ~uint64_t(0)) { out[s] = 0; continue; }
    const double rv = r[s];
    if (ck[nk] < rv) { out[s] = last; continue; }
    uint64_t lo = 0, hi = nk;  // the first checkpoint >= r
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (ck[mid] < rv) lo = mid + 1; else hi = mid;
    }
    const uint64_t k = lo > 0 ? lo - 1 : 0;
    double acc = ck[k];
    uint64_t i = k * kCdfSub;
    if (i < first) i = first;
    uint64_t res = last;
    for (; i < last; i++) {
      const double p = pref<R>(a, i);
      if (p > thr) {
        acc = acc + p;
        if (acc >= rv) { res = i; break; }
      }
    }
    out[s] = res;
  }
}

// ------------------------------------------------------------------ gather, Pauli
template <typename R>
__global__ void k_gather(const typename Vec2<R>::T* a, const uint64_t* idx, uint64_t k, double* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x) {
    typename Vec2<R>::T v = a[idx[i]];
    out[2 * i] = (double)v.x;
    out[2 * i + 1] = (double)v.y;
  }
}

// <psi|P|psi> partials for a group of Pauli terms sharing the flip mask f:
// sum_y Re( psi_y * conj(psi_{y^f}) * i^nY ) * sum_t coeff_t (-1)^popc(y & zm_t).
template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_pauli_group(const typename Vec2<R>::T* a, uint64_t N, uint64_t chunk,
                                                    PauliGroup grp, double* partial) {
  __shared__ double red[32];
  uint64_t lo = blockIdx.x * chunk, hi = min(N, lo + chunk);
  double acc = 0.0;
  for (uint64_t y = lo + threadIdx.x; y < hi; y += NT) {
    typename Vec2<R>::T v = a[y], w = a[y ^ grp.flip];
    double vr = v.x, vi = v.y, wr = w.x, wi = -(double)w.y;  // conj(psi_{y^f})
    double pr = vr * wr - vi * wi, pi = vr * wi + vi * wr;
    double base;
    switch (grp.ny & 3) {
      case 0: base = pr; break;
      case 1: base = -pi; break;   // * i
      case 2: base = -pr; break;
      default: base = pi; break;   // * -i
    }
    double c = 0.0;
    for (int t = 0; t < grp.nterms; t++) c += (__popcll(y & grp.zm[t]) & 1) ? -grp.coeff[t] : grp.coeff[t];
    acc += base * c;
  }
  double t = block_sum<NT>(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

inline unsigned gridn(uint64_t work, int nt, int cap_per_sm = 16) {
  uint64_t b = (work + nt - 1) / nt;
  uint64_t cap = (uint64_t)num_sms() * cap_per_sm;
  return (unsigned)std::max<uint64_t>(1, std::min(b, cap));
}

}  // namespace

// ------------------------------------------------------------------ launchers
template <typename R>
static cudaError_t norm2_t(const void* amp, int n, double* scratch, double* out, cudaStream_t s) {
  const uint64_t N = uint64_t(1) << n;
  const uint64_t chunk = std::max<uint64_t>(N / 4096, 4096);
  const uint64_t nb = (N + chunk - 1) / chunk;
  k_norm_partial<R, 256><<<(unsigned)nb, 256, 0, s>>>((const typename Vec2<R>::T*)amp, N, chunk, scratch);
  k_sum<256><<<1, 256, 0, s>>>(scratch, nb, out);
  return cudaGetLastError();
}

cudaError_t launch_norm2(const void* amp, int n, int prec, double* scratch, double* out, cudaStream_t s) {
  return prec == KET_C64 ? norm2_t<float>(amp, n, scratch, out, s) : norm2_t<double>(amp, n, scratch, out, s);
}
size_t norm2_scratch(int n) { return 8 * 4096 + 64; }

template <typename R>
static cudaError_t probs_dense_t(const void* amp, uint64_t off, uint64_t cnt, double thr, double* out, cudaStream_t s) {
  k_probs_dense<R><<<gridn(cnt, 256), 256, 0, s>>>((const typename Vec2<R>::T*)amp, off, cnt, thr, out);
  return cudaGetLastError();
}
cudaError_t launch_probs_dense(const void* amp, int prec, uint64_t off, uint64_t cnt, double thr, double* out,
                               cudaStream_t s) {
  return prec == KET_C64 ? probs_dense_t<float>(amp, off, cnt, thr, out, s)
                         : probs_dense_t<double>(amp, off, cnt, thr, out, s);
}

uint64_t kept_chunk(int n) {
  uint64_t N = uint64_t(1) << n;
  return std::max<uint64_t>(N / 8192, 1024);
}
template <typename R>
static cudaError_t count_kept_t(const void* amp, int n, double thr, uint64_t* counts, cudaStream_t s) {
  uint64_t N = uint64_t(1) << n, chunk = kept_chunk(n), nb = (N + chunk - 1) / chunk;
  k_count_kept<R, 256><<<(unsigned)nb, 256, 0, s>>>((const typename Vec2<R>::T*)amp, N, chunk, thr, counts);
  return cudaGetLastError();
}
cudaError_t launch_count_kept(const void* amp, int n, int prec, double thr, uint64_t* counts, cudaStream_t s) {
  return prec == KET_C64 ? count_kept_t<float>(amp, n, thr, counts, s) : count_kept_t<double>(amp, n, thr, counts, s);
}
template <typename R>
static cudaError_t compact_t(const void* amp, int n, double thr, const uint64_t* offs, uint64_t cap, uint64_t* oi,
                             double* op, cudaStream_t s) {
  uint64_t N = uint64_t(1) << n, chunk = kept_chunk(n), nb = (N + chunk - 1) / chunk;
  k_compact_kept<R, 256><<<(unsigned)nb, 256, 0, s>>>((const typename Vec2<R>::T*)amp, N, chunk, thr, offs, cap, oi, op);
  return cudaGetLastError();
}
cudaError_t launch_compact_kept(const void* amp, int n, int prec, double thr, const uint64_t* offs, uint64_t cap,
                                uint64_t* oidx, double* op, cudaStream_t s) {
  return prec == KET_C64 ? compact_t<float>(amp, n, thr, offs, cap, oidx, op, s)
                         : compact_t<double>(amp, n, thr, offs, cap, oidx, op, s);
}

uint64_t marg_chunk(int n) {
  uint64_t N = uint64_t(1) << n;
  return std::max<uint64_t>(N / 2048, 256);
}
template <typename R>
static cudaError_t marginals_t(const void* amp, int n, double* partial, double* out, cudaStream_t s) {
  uint64_t N = uint64_t(1) << n, chunk = marg_chunk(n), nb = (N + chunk - 1) / chunk;
  k_marginals<R, 256><<<(unsigned)nb, 256, 0, s>>>((const typename Vec2<R>::T*)amp, n, chunk, partial);
  k_sum_columns<<<1, 64, 0, s>>>(partial, nb, n, out);
  return cudaGetLastError();
}
cudaError_t launch_marginals(const void* amp, int n, int prec, double* partial, double* out, cudaStream_t s) {
  return prec == KET_C64 ? marginals_t<float>(amp, n, partial, out, s) : marginals_t<double>(amp, n, partial, out, s);
}

int mdist_chunk_bits(int n, int m) { return std::min(n, std::max(20, m)); }
template <typename R>
static cudaError_t mdist_t(const void* amp, int n, const MarginalSpec& spec, double* partial, double* out,
                           cudaStream_t s) {
  int c = mdist_chunk_bits(n, spec.m);
  uint64_t nb = uint64_t(1) << (n - c);
  uint32_t width = 1u << spec.m;
  cudaMemsetAsync(partial, 0, sizeof(double) * nb * width, s);
  k_marginal_dist<R><<<(unsigned)nb, 1024, 0, s>>>((const typename Vec2<R>::T*)amp, c, spec, partial);
  k_sum_columns<<<(width + 255) / 256, 256, 0, s>>>(partial, nb, (int)width, out);
  return cudaGetLastError();
}
cudaError_t launch_marginal_dist(const void* amp, int n, int prec, const MarginalSpec& spec, double* partial,
                                 double* out, cudaStream_t s) {
  return prec == KET_C64 ? mdist_t<float>(amp, n, spec, partial, out, s) : mdist_t<double>(amp, n, spec, partial, out, s);
}

// Scratch layout of the sampler: nk + 1 checkpoints, then per block the
// approximate prefix (nb + 1), the first and last kept index, D, the exact
// start, the state and the binade; the state's first and last kept index.
struct CdfScratch {
  double* ck;
  double* bsum;
  unsigned long long* bfirst;
  unsigned long long* blast;
  long long* bd;
  double* bstart;
  int* bst;
  int* be;
  unsigned long long* fl;
  size_t bytes;
};
static CdfScratch cdf_scratch(int n, void* base) {
  const uint64_t N = uint64_t(1) << n;
  const uint64_t nk = (N + kCdfSub - 1) / kCdfSub, nb = (N + kCdfBlock - 1) / kCdfBlock;
  CdfScratch c;
  char* p = (char*)base;
  auto take = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~size_t(255);
    return (void*)r;
  };
  c.ck = (double*)take(8 * (nk + 1));
  c.bsum = (double*)take(8 * (nb + 1));
  c.bfirst = (unsigned long long*)take(8 * nb);
  c.blast = (unsigned long long*)take(8 * nb);
  c.bd = (long long*)take(8 * nb);
  c.bstart = (double*)take(8 * nb);
  c.bst = (int*)take(4 * nb);
  c.be = (int*)take(4 * nb);
  c.fl = (unsigned long long*)take(16);
  c.bytes = (size_t)(p - (char*)base);
  return c;
}

template <typename R>
static cudaError_t sample_t(const void* amp, int n, double thr, const double* r, uint64_t shots, void* scratch,
                            uint64_t* out, cudaStream_t s) {
  const typename Vec2<R>::T* a = (const typename Vec2<R>::T*)amp;
  const uint64_t N = uint64_t(1) << n;
  const uint64_t nk = (N + kCdfSub - 1) / kCdfSub, nb = (N + kCdfBlock - 1) / kCdfBlock;
  const CdfScratch c = cdf_scratch(n, scratch);
  k_cdf_block_sums<R><<<(unsigned)nb, 256, 0, s>>>(a, N, thr, c.bsum, c.bfirst, c.blast);
  k_cdf_block_prefix<<<1, kCdfThreads, 0, s>>>(c.bsum, c.bfirst, c.blast, nb, c.fl);
  k_cdf_block_d<R><<<(unsigned)nb, 256, 0, s>>>(a, N, thr, c.bsum, (long long*)c.ck, c.bd, c.bst, c.be);
  k_cdf_walk<R><<<1, kCdfThreads, 0, s>>>(a, N, thr, nb, nk, c.ck, c.bd, c.bst, c.be, c.bstart);
  k_cdf_fill<<<gridn(nk, 256), 256, 0, s>>>(c.ck, nk, c.bst, c.be, c.bstart);
  k_sample_ck<R><<<gridn(shots, 128), 128, 0, s>>>(a, N, thr, c.ck, nk, r, shots, c.fl, out);
  return cudaGetLastError();
}
size_t sample_scratch(int n) { return cdf_scratch(n, nullptr).bytes; }
int sample_launches() { return 6; }
cudaError_t launch_sample(const void* amp, int n, int prec, double thr, const double* r, uint64_t shots, void* scratch,
                          uint64_t* out, cudaStream_t s) {
  return prec == KET_C64 ? sample_t<float>(amp, n, thr, r, shots, scratch, out, s)
                         : sample_t<double>(amp, n, thr, r, shots, scratch, out, s);
}

cudaError_t launch_gather(const void* amp, int prec, const uint64_t* idx, uint64_t k, double* out, cudaStream_t s) {
  if (prec == KET_C64) k_gather<float><<<gridn(k, 256), 256, 0, s>>>((const float2*)amp, idx, k, out);
  else k_gather<double><<<gridn(k, 256), 256, 0, s>>>((const double2*)amp, idx, k, out);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t pauli_t(const void* amp, int n, const PauliGroup& g, double* partial, double* out, cudaStream_t s) {
  const uint64_t N = uint64_t(1) << n;
  const uint64_t chunk = std::max<uint64_t>(N / 4096, 2048);
  const uint64_t nb = (N + chunk - 1) / chunk;
  k_pauli_group<R, 256><<<(unsigned)nb, 256, 0, s>>>((const typename Vec2<R>::T*)amp, N, chunk, g, partial);
  k_sum<256><<<1, 256, 0, s>>>(partial, nb, out);
  return cudaGetLastError();
}
cudaError_t launch_pauli_group(const void* amp, int n, int prec, const PauliGroup& g, double* partial, double* out,
                               cudaStream_t s) {
  return prec == KET_C64 ? pauli_t<float>(amp, n, g, partial, out, s) : pauli_t<double>(amp, n, g, partial, out, s);
}
size_t pauli_scratch(int n) { return 8 * 4096 + 64; }

template <typename RA, typename RB>
static cudaError_t compare_t(const void* a, const void* b, int n, double* scratch, double* out, cudaStream_t s) {
  const uint64_t N = uint64_t(1) << n;
  const uint64_t chunk = std::max<uint64_t>(N / 4096, 4096);
  const uint64_t nb = (N + chunk - 1) / chunk;
  k_compare<RA, RB, 256><<<(unsigned)nb, 256, 0, s>>>((const typename Vec2<RA>::T*)a,
                                                      (const typename Vec2<RB>::T*)b, N, chunk, scratch);
  k_compare_combine<<<1, 32, 0, s>>>(scratch, nb, out);
  return cudaGetLastError();
}
cudaError_t launch_compare(const void* a, int pa, const void* b, int pb, int n, double* scratch, double* out,
                           cudaStream_t s) {
  if (pa == KET_C64 && pb == KET_C64) return compare_t<float, float>(a, b, n, scratch, out, s);
  if (pa == KET_C64) return compare_t<float, double>(a, b, n, scratch, out, s);
  if (pb == KET_C64) return compare_t<double, float>(a, b, n, scratch, out, s);
  return compare_t<double, double>(a, b, n, scratch, out, s);
}
size_t compare_scratch(int) { return 3 * 8 * 4096 + 64; }

}  // namespace ket
