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
// Exact reference order (small states): cum[i] = the running FP64 sum over
// kept entries in ascending index order, rounded after every addition as
// the reference's loop does (circuit.ts:3429-3436) -- computed in parallel,
// bit for bit.
//
// While the running sum s stays in one binade [2^(e-1), 2^e), every value it
// takes is a multiple of u = 2^(e-53), s = S u with S an integer in
// [2^52, 2^53).  Adding p then rounds to the nearest multiple of u, so
// s + p = (S + d) u with d = round(p / u) -- an increment that does not
// depend on s, except when p / u lies exactly halfway (the tie goes to the
// even S + d) or when S + d reaches 2^53 (the sum leaves the binade and
// rounds on the next grid).  So a chunk of entries is an integer prefix sum
// of the d's, done by the whole block, up to the first tie or binade
// crossing; thread 0 takes that one entry with the FP64 addition itself, and
// the next chunk starts after it.  Entries that are not kept add nothing.
// Before the first kept entry the sum is +0.0.  A binade is crossed about
// once per doubling of s, so the single-entry steps are few.
constexpr int kCdfThreads = 1024;
constexpr int kCdfPer = 4;                          // entries per thread per chunk
constexpr int kCdfChunk = kCdfThreads * kCdfPer;    // 4096

// Inclusive block scan of v (NT = kCdfThreads); `wsum` holds 32 partials.
__device__ __forceinline__ long long block_scan_incl(long long v, long long* wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) wsum[w] = v;
  __syncthreads();
  if (w == 0) {
    long long x = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    wsum[lane] = x;
  }
  __syncthreads();
  const long long r = v + (w > 0 ? wsum[w - 1] : 0);
  __syncthreads();  // wsum is reused by the next scan
  return r;
}

// Block minimum of v; every thread gets it.
__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long* wred) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) wred[w] = v;
  __syncthreads();
  if (w == 0) {
    unsigned long long x = wred[lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) wred[32] = x;
  }
  __syncthreads();
  const unsigned long long r = wred[32];
  __syncthreads();
  return r;
}

template <typename R>
__global__ void __launch_bounds__(kCdfThreads) k_cdf_sequential(const typename Vec2<R>::T* a, uint64_t N, double thr,
                                                                double* cum, uint64_t* last) {
  __shared__ long long wsum[32];
  __shared__ unsigned long long wred[33];
  __shared__ double s_sh;            // the running sum after entry c - 1 (exact)
  __shared__ unsigned long long c_sh;  // next entry
  const int tid = threadIdx.x;
  const uint64_t NONE = ~0ull;
  long long lk = -1;  // the last kept entry this thread loaded
  if (tid == 0) { s_sh = 0.0; c_sh = 0; }
  __syncthreads();
  for (;;) {
    const uint64_t c = c_sh;
    const double s = s_sh;
    if (c >= N) break;
    // this thread's entries c + kCdfPer*tid + k
    const uint64_t i0 = c + (uint64_t)kCdfPer * tid;
    double pv[kCdfPer];
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) {
      const uint64_t i = i0 + k;
      double p = -0.0;  // not kept (or past the end): adds nothing
      if (i < N) {
        const double q = pref<R>(a, i);
        if (q > thr) { p = q; lk = (long long)i; }
      }
      pv[k] = p;
    }
    if (s == 0.0) {
      // before the first kept entry the sum is +0.0; that entry sets it exactly
      unsigned long long f = NONE;
#pragma unroll
      for (int k = 0; k < kCdfPer; k++)
        if (f == NONE && i0 + k < N && __double_as_longlong(pv[k]) > 0) f = i0 + k;
      f = block_min_u64(f, wred);
#pragma unroll
      for (int k = 0; k < kCdfPer; k++) {
        const uint64_t i = i0 + k;
        if (i < N && i < f) cum[i] = 0.0;
      }
      if (tid == 0) {
        if (f != NONE) {
          const double p0 = pref<R>(a, f);
          s_sh = 0.0 + p0;
          cum[f] = s_sh;
          c_sh = f + 1;
        } else {
          c_sh = c + kCdfChunk;
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
      if (i >= N) continue;
      const double q = ldexp(pv[k], 53 - e);  // p / u, exact
      if (q >= 9007199254740992.0) {          // 2^53: the sum leaves the binade
        if (special == NONE) special = i;
        continue;
      }
      const double fl = floor(q);
      if (q - fl == 0.5) {                    // a tie: the rounding depends on S
        if (special == NONE) special = i;
        continue;
      }
      if (special == NONE) {
        d[k] = (long long)rint(q);
        tsum += d[k];
      }
    }
    special = block_min_u64(special, wred);
    // entries at or after the first special one do not count in the scan
    if (special != NONE && i0 >= special) tsum = 0;
    if (special != NONE && i0 < special) {
      tsum = 0;
#pragma unroll
      for (int k = 0; k < kCdfPer; k++)
        if (i0 + k < special) tsum += d[k];
    }
    const long long incl = block_scan_incl(tsum, wsum);
    long long Sr = S0 + incl - tsum;  // S before this thread's first entry
    unsigned long long cross = NONE;  // first entry whose sum reaches 2^53 u
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) {
      const uint64_t i = i0 + k;
      if (i >= N || (special != NONE && i >= special)) break;
      const long long Sn = Sr + d[k];
      if (Sn >= 9007199254740992ll) { cross = i; break; }
      Sr = Sn;
    }
    cross = block_min_u64(cross, wred);
    const uint64_t lim = c + (uint64_t)kCdfChunk < N ? c + (uint64_t)kCdfChunk : N;
    uint64_t stop = special < cross ? (uint64_t)special : (uint64_t)cross;
    if (stop > lim) stop = lim;
    // write the exact sums of the entries before `stop`
    Sr = S0 + incl - tsum;
#pragma unroll
    for (int k = 0; k < kCdfPer; k++) {
      const uint64_t i = i0 + k;
      if (i >= stop) break;
      Sr += d[k];
      cum[i] = ldexp((double)Sr, e - 53);
    }
    __syncthreads();
    if (tid == 0) {
      // the sum just before `stop`: the running S (all entries < stop are in range)
      double sp = s;
      if (stop > c) sp = cum[stop - 1];
      if (stop < lim) {
        // the special entry, by the reference's own FP64 addition
        const double q = pref<R>(a, stop);
        const double p = q > thr ? q : -0.0;
        sp = sp + p;
        cum[stop] = sp;
        c_sh = stop + 1;
      } else {
        c_sh = stop;
      }
      s_sh = sp;
    }
    __syncthreads();
  }
  // the last kept entry: the block's largest
  unsigned long long nl = lk < 0 ? NONE : ~(unsigned long long)lk;  // min of ~x is max of x
  nl = block_min_u64(nl, wred);
  const uint64_t l = nl == NONE ? NONE : ~nl;
  if (tid == 0) *last = l;
  __syncthreads();
  // the reference sets the last kept entry's cumP to 1.0; entries after it
  // are never kept, so the search treats them alike
  if (l != NONE)
    for (uint64_t i = l + tid; i < N; i += kCdfThreads) cum[i] = 1.0;
}

__global__ void k_sample_dense(const double* cum, uint64_t N, const double* r, uint64_t shots, const uint64_t* lastp,
                               uint64_t* out) {
  const uint64_t last = *lastp;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < shots; s += (uint64_t)gridDim.x * blockDim.x) {
    if (last == ~uint64_t(0)) { out[s] = 0; continue; }
    double rv = r[s];
    uint64_t lo = 0, hi = N - 1;
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if (cum[mid] < rv) lo = mid + 1; else hi = mid;
    }
    out[s] = lo;
  }
}

// Chunked CDF for large states: lane l of warp c sums sub-chunk (c*32 + l) of
// 32 entries sequentially; the warp then combines its 32 sub-chunk sums
// sequentially.  chunk_sum[c] and last_kept[c] are written.
template <typename R>
__global__ void k_chunk_sums(const typename Vec2<R>::T* a, uint64_t nchunks, double thr, double* chunk_sum,
                             uint64_t* last_kept) {
  uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nchunks) return;
  uint64_t base = warp * 1024 + (uint64_t)lane * 32;
  double s = 0.0;
  long long lk = -1;
  for (int j = 0; j < 32; j++) {
    double p = pref<R>(a, base + j);
    if (p > thr) { s += p; lk = (long long)(base + j); }
  }
  double tot = 0.0;
  long long l2 = -1;
  for (int j = 0; j < 32; j++) {
    double v = __shfl_sync(0xffffffffu, s, j);
    long long lj = __shfl_sync(0xffffffffu, lk, j);
    tot += v;
    if (lj >= 0) l2 = lj;
  }
  if (lane == 0) { chunk_sum[warp] = tot; last_kept[warp] = (uint64_t)l2; }
}

// Exclusive prefix E[0..nchunks] (sequential, one thread) and the last kept index.
__global__ void k_chunk_prefix(const double* chunk_sum, const uint64_t* last_kept, uint64_t nchunks, double* E,
                               uint64_t* last) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double acc = 0.0;
  uint64_t lk = ~uint64_t(0);
  for (uint64_t c = 0; c < nchunks; c++) {
    E[c] = acc;
    acc += chunk_sum[c];
    if (last_kept[c] != ~uint64_t(0)) lk = last_kept[c];
  }
  E[nchunks] = acc;
  *last = lk;
}

template <typename R>
__global__ void k_sample_chunked(const typename Vec2<R>::T* a, const double* E, uint64_t nchunks, double thr,
                                 const double* r, uint64_t shots, const uint64_t* lastp, uint64_t* out) {
  const uint64_t last = *lastp;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < shots; s += (uint64_t)gridDim.x * blockDim.x) {
    if (last == ~uint64_t(0)) { out[s] = 0; continue; }
    double rv = r[s];
    if (E[nchunks] < rv) { out[s] = last; continue; }  // the reference's last.cumP = 1.0
    uint64_t lo = 0, hi = nchunks - 1;                // first chunk c with E[c+1] >= r
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if (E[mid + 1] < rv) lo = mid + 1; else hi = mid;
    }
    const uint64_t c = lo;
    const double ec = E[c];
    uint64_t res = last;
    double W = 0.0;
    bool found = false;
    for (int sub = 0; sub < 32 && !found; sub++) {
      uint64_t b = c * 1024 + (uint64_t)sub * 32;
      double ps = 0.0;
      for (int j = 0; j < 32; j++) {
        double p = pref<R>(a, b + j);
        if (p > thr) ps += p;
      }
      double Wn = W + ps;
      if (ec + Wn >= rv) {
        double part = 0.0;
        for (int j = 0; j < 32; j++) {
          double p = pref<R>(a, b + j);
          if (p > thr) {
            part += p;
            if (ec + (W + part) >= rv) { res = b + j; found = true; break; }
          }
        }
      }
      W = Wn;
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

template <typename R>
static cudaError_t sample_t(const void* amp, int n, double thr, int seq_qubits, const double* r, uint64_t shots,
                            void* scratch, uint64_t* out, cudaStream_t s) {
  const typename Vec2<R>::T* a = (const typename Vec2<R>::T*)amp;
  const uint64_t N = uint64_t(1) << n;
  if (n <= seq_qubits || n < 10) {
    double* cum = (double*)scratch;
    uint64_t* last = (uint64_t*)(cum + N);
    k_cdf_sequential<R><<<1, kCdfThreads, 0, s>>>(a, N, thr, cum, last);
    k_sample_dense<<<gridn(shots, 256), 256, 0, s>>>(cum, N, r, shots, last, out);
  } else {
    const uint64_t nchunks = N / 1024;
    double* cs = (double*)scratch;
    uint64_t* lk = (uint64_t*)(cs + nchunks);
    double* E = (double*)(lk + nchunks);
    uint64_t* last = (uint64_t*)(E + nchunks + 1);
    k_chunk_sums<R><<<(unsigned)((nchunks * 32 + 255) / 256), 256, 0, s>>>(a, nchunks, thr, cs, lk);
    k_chunk_prefix<<<1, 32, 0, s>>>(cs, lk, nchunks, E, last);
    k_sample_chunked<R><<<gridn(shots, 128), 128, 0, s>>>(a, E, nchunks, thr, r, shots, last, out);
  }
  return cudaGetLastError();
}
size_t sample_scratch(int n, int seq_qubits) {
  uint64_t N = uint64_t(1) << n;
  if (n <= seq_qubits || n < 10) return 8 * N + 64;
  uint64_t nc = N / 1024;
  return 8 * (3 * nc + 8);
}
cudaError_t launch_sample(const void* amp, int n, int prec, double thr, int seq_qubits, const double* r, uint64_t shots,
                          void* scratch, uint64_t* out, cudaStream_t s) {
  return prec == KET_C64 ? sample_t<float>(amp, n, thr, seq_qubits, r, shots, scratch, out, s)
                         : sample_t<double>(amp, n, thr, seq_qubits, r, shots, scratch, out, s);
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
