// shots.cu -- run()'s per-shot path: mid-circuit measure / reset / if and
// stochastic Pauli noise (circuit.ts:55-83, :169-207, :289-304, :3455-3481).
//
// One device trajectory per shot.  The host walks the op list the way
// applyOps does and draws the reference's xorshift32 stream in the
// reference's order; every operation on the state runs on the device:
//   * runs of gates go through the fused engine (ket_apply_ops, with the
//     reference's per-gate pruning), with the Paulis that the noise draws
//     select spliced in right after their gate -- the draws never depend on
//     the state, so a run of noisy gates is still one engine call;
//   * measure and reset reduce P(q=1) on the device (k_prob_one, fixed-order
//     partial sums), the host compares it with its draw, and k_collapse
//     zeroes the other half and rescales the kept half in place by
//     1/sqrt(p) as collapseQubit does;
//   * the final readout is the sampling kernel with no probability
//     threshold: sampleSV walks every entry of its Map, and the engine's
//     pruned state holds exactly those entries as its nonzero amplitudes.
//     The sampler's running sum is sampleSV's, ascending index order and
//     rounding included; the in-shared-memory trajectories below walk chunk
//     sums and then one chunk, which differs from it only in rounding.
// The device state is the caller's ket_state, reset to |init> per shot.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "engine.h"
#include "launch.h"

using namespace ket;

namespace {

constexpr int KNT = 256;

// partial[b] = sum of |a_i|^2 over i with bit q set, for the b-th slice of
// the N/2 such indices (j -> i inserts a 1 at bit q).
template <typename R>
__global__ void __launch_bounds__(KNT) k_prob_one(const typename Vec2<R>::T* a, uint64_t half, int q, uint64_t chunk,
                                                  double* partial) {
  __shared__ double sh[KNT];
  const uint64_t lo = (uint64_t)blockIdx.x * chunk;
  const uint64_t hi = lo + chunk < half ? lo + chunk : half;
  const uint64_t low = (uint64_t(1) << q) - 1;
  double acc = 0.0;
  for (uint64_t j = lo + threadIdx.x; j < hi; j += KNT) {
    const uint64_t i = ((j & ~low) << 1) | (uint64_t(1) << q) | (j & low);
    const typename Vec2<R>::T v = a[i];
    const double re = (double)v.x, im = (double)v.y;
    acc += re * re + im * im;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = KNT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// out = the partials summed in index order (one thread: nb <= 4096).
__global__ void k_sum_in_order(const double* partial, int nb, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[b];
  *out = s;
}

// collapseQubit's projection: keep the amplitudes whose bit q equals the
// outcome, scaled by inv; zero the others.
template <typename R>
__global__ void k_collapse(typename Vec2<R>::T* a, uint64_t N, int q, int outcome, double inv) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    typename Vec2<R>::T v = a[i];
    if ((int)((i >> q) & 1) == outcome) {
      v.x = (R)((double)v.x * inv);
      v.y = (R)((double)v.y * inv);
    } else {
      v.x = (R)0;
      v.y = (R)0;
    }
    a[i] = v;
  }
}

#define TRY(x) do { int _rc = (x); if (_rc) return _rc; } while (0)

// ---------------------------------------------------------------- batched trajectories
// Small states (2^n amplitudes fit in shared memory) run one shot per CTA,
// many shots at a time.  Every thread keeps the same copy of the xorshift32
// state and makes the same draws, so a draw needs no communication; gate
// arithmetic rounds exactly as the reference's complex.ts does (products and
// sums each rounded, no fused multiply-add), pruning as accumulate() does.

enum { T_NOISE1 = 20, T_NOISE2 = 21 };

struct TOp {
  int32_t kind;  // ket_op_kind, or T_NOISE1 / T_NOISE2 (a dep1 / dep2 draw after the gate before it)
  int32_t q[4];  // gate qubits; MEASURE {q, cbit}; RESET {q}; IF {first bit, size, value, body length}
  int32_t mat;   // complex offset of the matrix in the matrix table (-1: none)
  int32_t k;     // UNITARY: qubit count
  int32_t pad;
};

struct cd { double re, im; };
__device__ __forceinline__ cd cmul_rn(cd a, cd b) {  // complex.ts mul
  return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
          __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ cd cadd_rn(cd a, cd b) { return {__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)}; }
__device__ __forceinline__ double norm2_rn(cd a) { return __dadd_rn(__dmul_rn(a.re, a.re), __dmul_rn(a.im, a.im)); }
__device__ __forceinline__ cd pruned(cd a) { return norm2_rn(a) < 1e-14 ? cd{0.0, 0.0} : a; }

template <typename V>
__device__ __forceinline__ cd ldc(const V* st, uint64_t i) { const V v = st[i]; return {(double)v.x, (double)v.y}; }
template <typename V>
__device__ __forceinline__ void stc(V* st, uint64_t i, cd a) {
  V v;
  v.x = (decltype(v.x))a.re;
  v.y = (decltype(v.y))a.im;
  st[i] = v;
}
__device__ __forceinline__ cd mat_at(const double* M, int64_t off, int i) {
  return {__ldg(M + 2 * (off + i)), __ldg(M + 2 * (off + i) + 1)};
}

// xorshift32 (circuit.ts:813-819), identical in every thread
__device__ __forceinline__ double tdraw(uint32_t& s) {
  s ^= s << 13;
  s ^= s >> 17;
  s ^= s << 5;
  return (double)s / 4294967296.0;
}

// 2x2 on target t; c >= 0: controlled on c, whose 0-entries pass through
// accumulate() and are pruned in place (applyControlled, statevector.ts:212-234)
template <typename V, int NT>
__device__ void t_apply2(V* st, int n, int t, int c, const double* M, int64_t off) {
  const cd g0 = mat_at(M, off, 0), g1 = mat_at(M, off, 1), g2 = mat_at(M, off, 2), g3 = mat_at(M, off, 3);
  const uint64_t half = uint64_t(1) << (n - 1);
  for (uint64_t j = threadIdx.x; j < half; j += NT) {
    const uint64_t i0 = insert0(j, t), i1 = i0 | (uint64_t(1) << t);
    const cd a0 = ldc(st, i0), a1 = ldc(st, i1);
    if (c >= 0 && !((i0 >> c) & 1)) {
      stc(st, i0, pruned(a0));
      stc(st, i1, pruned(a1));
      continue;
    }
    stc(st, i0, pruned(cadd_rn(cmul_rn(g0, a0), cmul_rn(g1, a1))));
    stc(st, i1, pruned(cadd_rn(cmul_rn(g2, a0), cmul_rn(g3, a1))));
  }
}

// X on t where all bits of cm are set (applyCNOT / applyToffoli: copies)
template <typename V, int NT>
__device__ void t_permx(V* st, int n, int t, uint64_t cm) {
  const uint64_t half = uint64_t(1) << (n - 1);
  for (uint64_t j = threadIdx.x; j < half; j += NT) {
    const uint64_t i0 = insert0(j, t), i1 = i0 | (uint64_t(1) << t);
    if ((i0 & cm) != cm) continue;
    const V v0 = st[i0];
    st[i0] = st[i1];
    st[i1] = v0;
  }
}

// swap bits a, b where all bits of cm are set (applySWAP / applyCSwap)
template <typename V, int NT>
__device__ void t_swap(V* st, int n, int a, int b, uint64_t cm) {
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  const uint64_t quarter = uint64_t(1) << (n - 2);
  for (uint64_t j = threadIdx.x; j < quarter; j += NT) {
    const uint64_t base = insert0(insert0(j, lo), hi);
    if ((base & cm) != cm) continue;
    const uint64_t x = base | (uint64_t(1) << a), y = base | (uint64_t(1) << b);
    const V v = st[x];
    st[x] = st[y];
    st[y] = v;
  }
}

// 4x4 on (a, b), a = MSB: [ctx, ctx|b, ctx|a, ctx|a|b] (applyTwo, statevector.ts:110-132)
template <typename V, int NT>
__device__ void t_apply4(V* st, int n, int a, int b, const double* M, int64_t off) {
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  const uint64_t quarter = uint64_t(1) << (n - 2);
  for (uint64_t j = threadIdx.x; j < quarter; j += NT) {
    const uint64_t base = insert0(insert0(j, lo), hi);
    const uint64_t idx[4] = {base, base | (uint64_t(1) << b), base | (uint64_t(1) << a),
                             base | (uint64_t(1) << a) | (uint64_t(1) << b)};
    cd x[4];
    for (int c = 0; c < 4; c++) x[c] = ldc(st, idx[c]);
    for (int r = 0; r < 4; r++) {
      cd out = {0.0, 0.0};
      for (int c = 0; c < 4; c++) out = cadd_rn(out, cmul_rn(mat_at(M, off, 4 * r + c), x[c]));
      stc(st, idx[r], pruned(out));
    }
  }
}

// applyCsrSwap (statevector.ts:177-207): sqrt(iSWAP) on (a, b) where c is set;
// every other entry passes through accumulate()
template <typename V, int NT>
__device__ void t_csrswap(V* st, int n, int c, int a, int b) {
  const double sq2 = 1.0 / 1.4142135623730951;  // 1 / Math.sqrt(2)
  const uint64_t quarter = uint64_t(1) << (n - 2);
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  for (uint64_t j = threadIdx.x; j < quarter; j += NT) {
    const uint64_t base = insert0(insert0(j, lo), hi);
    const uint64_t i00 = base, i01 = base | (uint64_t(1) << b), i10 = base | (uint64_t(1) << a),
                   i11 = i01 | (uint64_t(1) << a);
    const cd a00 = ldc(st, i00), a01 = ldc(st, i01), a10 = ldc(st, i10), a11 = ldc(st, i11);
    stc(st, i00, pruned(a00));
    stc(st, i11, pruned(a11));
    if (!((base >> c) & 1)) {
      stc(st, i01, pruned(a01));
      stc(st, i10, pruned(a10));
      continue;
    }
    stc(st, i01, pruned(cadd_rn(cmul_rn({sq2, 0.0}, a01), cmul_rn({0.0, sq2}, a10))));
    stc(st, i10, pruned(cadd_rn(cmul_rn({0.0, sq2}, a01), cmul_rn({sq2, 0.0}, a10))));
  }
}

// applyUnitary (statevector.ts:240-270): 2^k x 2^k on qs (qs[0] = MSB), k <= 4
template <typename V, int NT>
__device__ void t_applyk(V* st, int n, const int* qs, int k, const double* M, int64_t off) {
  int sorted[4];
  for (int i = 0; i < k; i++) sorted[i] = qs[i];
  for (int i = 1; i < k; i++)
    for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; j--) { const int w = sorted[j]; sorted[j] = sorted[j - 1]; sorted[j - 1] = w; }
  const int dim = 1 << k;
  const uint64_t groups = uint64_t(1) << (n - k);
  for (uint64_t j = threadIdx.x; j < groups; j += NT) {
    uint64_t base = j;
    for (int i = 0; i < k; i++) base = insert0(base, sorted[i]);
    cd x[16];
    uint64_t idx[16];
    for (int i = 0; i < dim; i++) {
      uint64_t v = base;
      for (int bit = 0; bit < k; bit++)
        if ((i >> (k - 1 - bit)) & 1) v |= uint64_t(1) << qs[bit];
      idx[i] = v;
      x[i] = ldc(st, v);
    }
    for (int r = 0; r < dim; r++) {
      cd out = {0.0, 0.0};
      for (int c = 0; c < dim; c++) out = cadd_rn(out, cmul_rn(mat_at(M, off, r * dim + c), x[c]));
      stc(st, idx[r], pruned(out));
    }
  }
}

// block sum of v in a fixed order (per-thread partial, then a tree); all
// threads get the result
template <int NT>
__device__ double t_block_sum(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int w = NT / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// collapseQubit (circuit.ts:55-72) on the shared-memory state
template <typename V, int NT>
__device__ int t_collapse(V* st, int n, int q, double rand, double* red) {
  if (q < 0 || q >= n) return 0;  // a qubit outside the state reads 0; the state is unchanged
  const uint64_t half = uint64_t(1) << (n - 1);
  double acc = 0.0;
  for (uint64_t j = threadIdx.x; j < half; j += NT)
    acc = __dadd_rn(acc, norm2_rn(ldc(st, insert0(j, q) | (uint64_t(1) << q))));
  const double p1 = t_block_sum<NT>(acc, red);
  const int outcome = rand < p1 ? 1 : 0;
  const double inv = 1 / sqrt(outcome == 1 ? p1 : 1 - p1);
  const uint64_t N = uint64_t(1) << n;
  for (uint64_t i = threadIdx.x; i < N; i += NT) {
    cd a = ldc(st, i);
    if ((int)((i >> q) & 1) == outcome) a = {__dmul_rn(a.re, inv), __dmul_rn(a.im, inv)};
    else a = {0.0, 0.0};
    stc(st, i, a);
  }
  return outcome;
}

template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_shots(const TOp* ops, int nops, const double* M, int64_t pauli0, int n,
                                              uint64_t init, const uint32_t* start, uint64_t shots, ket_noise nz,
                                              int ncbits, uint64_t* out_idx, uint8_t* out_bits) {
  typedef typename Vec2<R>::T V;
  extern __shared__ __align__(16) unsigned char smraw[];
  V* st = reinterpret_cast<V*>(smraw);
  const uint64_t N = uint64_t(1) << n;
  double* red = reinterpret_cast<double*>(smraw + sizeof(V) * N);
  uint8_t* bits = reinterpret_cast<uint8_t*>(red + NT);
  // sampling: per-thread chunk of C entries
  const uint64_t C = N >= (uint64_t)NT ? N / NT : 1;
  for (uint64_t shot = blockIdx.x; shot < shots; shot += gridDim.x) {
    uint32_t s = start[shot];
    for (uint64_t i = threadIdx.x; i < N; i += NT) {
      V v;
      v.x = (R)(i == init ? 1 : 0);
      v.y = (R)0;
      st[i] = v;
    }
    for (int b = threadIdx.x; b < ncbits; b += NT) bits[b] = 0;
    __syncthreads();
    for (int pc = 0; pc < nops; pc++) {
      const TOp o = ops[pc];
      switch (o.kind) {
        case KET_OP_SINGLE: t_apply2<V, NT>(st, n, o.q[0], -1, M, o.mat); break;
        case KET_OP_CONTROLLED: t_apply2<V, NT>(st, n, o.q[1], o.q[0], M, o.mat); break;
        case KET_OP_CNOT: t_permx<V, NT>(st, n, o.q[1], uint64_t(1) << o.q[0]); break;
        case KET_OP_TOFFOLI: t_permx<V, NT>(st, n, o.q[2], (uint64_t(1) << o.q[0]) | (uint64_t(1) << o.q[1])); break;
        case KET_OP_SWAP: t_swap<V, NT>(st, n, o.q[0], o.q[1], 0); break;
        case KET_OP_CSWAP: t_swap<V, NT>(st, n, o.q[1], o.q[2], uint64_t(1) << o.q[0]); break;
        case KET_OP_TWO: t_apply4<V, NT>(st, n, o.q[0], o.q[1], M, o.mat); break;
        case KET_OP_CSRSWAP: t_csrswap<V, NT>(st, n, o.q[0], o.q[1], o.q[2]); break;
        case KET_OP_UNITARY: t_applyk<V, NT>(st, n, o.q, o.k, M, o.mat); break;
        case T_NOISE1: {  // dep1 (circuit.ts:289-295)
          const double r = tdraw(s);
          if (r < nz.p1) {
            const double u = r / nz.p1;
            const int w = u < 1.0 / 3 ? 0 : u < 2.0 / 3 ? 1 : 2;
            t_apply2<V, NT>(st, n, o.q[0], -1, M, pauli0 + 4 * w);
          }
          break;
        }
        case T_NOISE2: {  // dep2 (circuit.ts:298-304), TWO_PAULI order
          const double r = tdraw(s);
          if (r < nz.p2) {
            int k = (int)floor(r / nz.p2 * 15);
            if (k > 14) k = 14;
            const int pa = (k + 1) >> 2, pb = (k + 1) & 3;  // k + 1 = 4 * pa + pb over {I, X, Y, Z}^2 \ {II}
            if (pa) { t_apply2<V, NT>(st, n, o.q[0], -1, M, pauli0 + 4 * (pa - 1)); __syncthreads(); }
            if (pb) t_apply2<V, NT>(st, n, o.q[1], -1, M, pauli0 + 4 * (pb - 1));
          }
          break;
        }
        case KET_OP_MEASURE: {
          const double r = tdraw(s);
          const int outcome = t_collapse<V, NT>(st, n, o.q[0], r, red);
          const int reported = (nz.pmeas != 0 && tdraw(s) < nz.pmeas) ? 1 - outcome : outcome;
          if (threadIdx.x == 0 && o.q[1] >= 0) bits[o.q[1]] = (uint8_t)reported;
          break;
        }
        case KET_OP_RESET: {
          const double r = tdraw(s);
          if (t_collapse<V, NT>(st, n, o.q[0], r, red) == 1) {
            __syncthreads();
            t_apply2<V, NT>(st, n, o.q[0], -1, M, pauli0);
          }
          break;
        }
        case KET_OP_IF: {
          int v = 0;
          for (int kk = 0; kk < o.q[1]; kk++)
            if (bits[o.q[0] + kk]) v |= 1 << kk;
          if (v != o.q[2]) pc += o.q[3];
          break;
        }
        default: break;  // barrier
      }
      __syncthreads();
    }
    // sampleSV (circuit.ts:75-83): the first index whose running sum of |a|^2
    // reaches the draw, else the last nonzero entry.  Chunk sums, then a walk
    // inside one chunk.
    const double r = tdraw(s);
    const uint64_t c0 = (uint64_t)threadIdx.x * C;
    double csum = 0.0;
    long long clast = -1;
    if (c0 < N)
      for (uint64_t i = c0; i < c0 + C; i++) {
        const double p = norm2_rn(ldc(st, i));
        if (p > 0) { csum = __dadd_rn(csum, p); clast = (long long)i; }
      }
    red[threadIdx.x] = csum;
    long long* lastk = reinterpret_cast<long long*>(bits + ((ncbits + 7) & ~7));
    lastk[threadIdx.x] = clast;
    __syncthreads();
    __shared__ long long pick;
    if (threadIdx.x == 0) {
      double cum = 0.0;
      long long last = -1, res = -1;
      for (int t = 0; t < NT && (uint64_t)t * C < N; t++) {
        if (lastk[t] >= 0) last = lastk[t];
        if (res < 0 && lastk[t] >= 0 && __dadd_rn(cum, red[t]) >= r) {
          double w = cum;
          for (uint64_t i = (uint64_t)t * C; i < (uint64_t)(t + 1) * C; i++) {
            const double p = norm2_rn(ldc(st, i));
            if (p > 0) {
              w = __dadd_rn(w, p);
              if (r <= w) { res = (long long)i; break; }
            }
          }
        }
        cum = __dadd_rn(cum, red[t]);
      }
      pick = res >= 0 ? res : (last >= 0 ? last : 0);
    }
    __syncthreads();
    uint64_t idx = (uint64_t)pick;
    if (nz.pmeas != 0)
      for (int q = 0; q < n; q++)
        if (tdraw(s) < nz.pmeas) idx ^= uint64_t(1) << q;
    if (threadIdx.x == 0) out_idx[shot] = idx;
    for (int b = threadIdx.x; b < ncbits; b += NT) out_bits[shot * (uint64_t)ncbits + b] = bits[b];
    __syncthreads();
  }
}

// xorshift32 as a linear map over GF(2)^32: col[k] = image of bit k
struct Jump {
  uint32_t col[32];
  uint32_t apply(uint32_t v) const {
    uint32_t o = 0;
    for (int k = 0; k < 32; k++)
      if ((v >> k) & 1) o ^= col[k];
    return o;
  }
};
Jump jump_power(uint64_t d) {
  Jump step, acc;
  for (int k = 0; k < 32; k++) {
    uint32_t s = 1u << k;
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    step.col[k] = s;
    acc.col[k] = 1u << k;
  }
  while (d) {
    if (d & 1) {
      Jump t;
      for (int k = 0; k < 32; k++) t.col[k] = step.apply(acc.col[k]);
      acc = t;
    }
    Jump sq;
    for (int k = 0; k < 32; k++) sq.col[k] = step.apply(step.col[k]);
    step = sq;
    d >>= 1;
  }
  return acc;
}

// Draws that ops[b, e) make per shot when that number does not depend on
// outcomes (no draw inside an if body), else -1.  Also lowers the ops to the
// device form.
int64_t lower_shots(const ket_op* ops, size_t b, size_t e, const ket_noise& nz, bool in_if, std::vector<TOp>& out) {
  int64_t draws = 0;
  for (size_t i = b; i < e; i++) {
    const ket_op& o = ops[i];
    TOp t;
    memset(&t, 0, sizeof(t));
    t.kind = o.kind;
    for (int j = 0; j < 4 && j < o.nq; j++) t.q[j] = o.q[j];
    t.mat = (int32_t)o.mat;
    t.k = o.nq;
    int64_t d = 0;
    bool noisy = false;
    switch (o.kind) {
      case KET_OP_SINGLE: noisy = nz.p1 != 0; break;
      case KET_OP_CNOT: case KET_OP_CONTROLLED: case KET_OP_SWAP: case KET_OP_TWO: noisy = nz.p2 != 0; break;
      case KET_OP_UNITARY: if (o.nq > 4) return -1; break;
      case KET_OP_MEASURE: d = 1 + (nz.pmeas != 0 ? 1 : 0); break;
      case KET_OP_RESET: d = 1; break;
      case KET_OP_IF: {
        out.push_back(t);
        const size_t at = out.size() - 1;
        const int64_t inner = lower_shots(ops, i + 1, i + 1 + o.q[3], nz, true, out);
        if (inner != 0) return -1;  // a body that draws makes the draw count depend on outcomes
        out[at].q[3] = (int32_t)(out.size() - at - 1);
        i += o.q[3];
        continue;
      }
      default: break;
    }
    out.push_back(t);
    if (noisy) {
      TOp z;
      memset(&z, 0, sizeof(z));
      z.kind = o.kind == KET_OP_SINGLE ? T_NOISE1 : T_NOISE2;
      z.q[0] = o.q[0];
      z.q[1] = o.q[1];
      out.push_back(z);
      d = 1;
    }
    if (in_if && d) return -1;
    draws += d;
  }
  return draws;
}

template <typename R, int NT>
cudaError_t launch_shots_t(const TOp* dops, int nops, const double* dmats, int64_t pauli0, int n, uint64_t init,
                           const uint32_t* dstart, uint64_t shots, const ket_noise& nz, int ncbits, uint64_t* dout,
                           uint8_t* dbits, cudaStream_t s) {
  const size_t smem = (sizeof(typename Vec2<R>::T) << n) + 8 * NT + ((ncbits + 7) & ~7) + 8 * NT;
  cudaError_t e = cudaFuncSetAttribute(k_shots<R, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_shots<R, NT>, NT, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const uint64_t grid = std::min<uint64_t>(shots, (uint64_t)per_sm * num_sms());
  k_shots<R, NT><<<(unsigned)grid, NT, smem, s>>>(dops, nops, dmats, pauli0, n, init, dstart, shots, nz, ncbits,
                                                  dout, dbits);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_shots(const TOp* dops, int nops, const double* dmats, int64_t pauli0, int n, uint64_t init,
                         const uint32_t* dstart, uint64_t shots, const ket_noise& nz, int ncbits, uint64_t* dout,
                         uint8_t* dbits, cudaStream_t s) {
  if (n <= 6) return launch_shots_t<R, 32>(dops, nops, dmats, pauli0, n, init, dstart, shots, nz, ncbits, dout, dbits, s);
  if (n <= 9) return launch_shots_t<R, 128>(dops, nops, dmats, pauli0, n, init, dstart, shots, nz, ncbits, dout, dbits, s);
  return launch_shots_t<R, 256>(dops, nops, dmats, pauli0, n, init, dstart, shots, nz, ncbits, dout, dbits, s);
}

// Largest state the batched kernel holds in shared memory.
int batched_max_qubits(int precision) { return precision == KET_C64 ? 13 : 12; }

int g_pershot_path = 0;  // ket_debug_pershot_path: 0 automatic, 1 host-driven only, 2 batched only

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// All shots in one launch: shot i starts from the stream state after i * D
// draws (D = draws per shot), found by the GF(2) jump of xorshift32.
int run_batched(ket_state* st, const std::vector<TOp>& tops, int64_t draws, const std::vector<double>& mats,
                int64_t pauli0, uint64_t init, const ket_noise& nz, size_t shots, uint32_t* prng, int ncbits,
                uint64_t* out_idx, uint8_t* out_bits) {
  ket_ctx* c = st->ctx;
  const Jump J = jump_power((uint64_t)draws);
  std::vector<uint32_t> start(shots);
  uint32_t s = *prng ? *prng : 1u;
  for (size_t i = 0; i < shots; i++) {
    start[i] = s;
    s = J.apply(s);
  }
  const size_t b_ops = align256(sizeof(TOp) * std::max<size_t>(1, tops.size()));
  const size_t b_mat = align256(8 * mats.size());
  const size_t b_start = align256(4 * shots), b_idx = align256(8 * shots), b_bits = align256(shots * ncbits + 1);
  void* scr;
  TRY(ctx_scratch(c, b_ops + b_mat + b_start + b_idx + b_bits, &scr));
  char* base = (char*)scr;
  TOp* dops = (TOp*)base;
  double* dmats = (double*)(base + b_ops);
  uint32_t* dstart = (uint32_t*)(base + b_ops + b_mat);
  uint64_t* didx = (uint64_t*)(base + b_ops + b_mat + b_start);
  uint8_t* dbits = (uint8_t*)(base + b_ops + b_mat + b_start + b_idx);
  cudaError_t e = cudaSuccess;
  if (!tops.empty()) e = cudaMemcpyAsync(dops, tops.data(), sizeof(TOp) * tops.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dmats, mats.data(), 8 * mats.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dstart, start.data(), 4 * shots, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(trajectory inputs)");
  c->h2d_bytes += sizeof(TOp) * tops.size() + 8 * mats.size() + 4 * shots;
  prof_begin(c);
  e = st->precision == KET_C64
          ? launch_shots<float>(dops, (int)tops.size(), dmats, pauli0, st->n, init, dstart, shots, nz, ncbits, didx,
                                dbits, c->stream)
          : launch_shots<double>(dops, (int)tops.size(), dmats, pauli0, st->n, init, dstart, shots, nz, ncbits, didx,
                                 dbits, c->stream);
  prof_end(c, PK_BATCH);
  if (e != cudaSuccess) return cuda_fail(e, "trajectory launch");
  e = cudaMemcpyAsync(out_idx, didx, 8 * shots, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && ncbits)
    e = cudaMemcpyAsync(out_bits, dbits, shots * (size_t)ncbits, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(trajectory outputs)");
  c->d2h_bytes += 8 * shots + shots * (size_t)ncbits;
  TRY(ctx_wait(c));
  *prng = s;
  return KET_OK;
}

// The op list's structure: every if-body lies inside its parent range;
// classical operands are in range.  Gates are collected for lower_ops.
int check_range(const ket_op* ops, size_t b, size_t e, int n, int ncbits, std::vector<ket_op>& gates) {
  for (size_t i = b; i < e; i++) {
    const ket_op& o = ops[i];
    switch (o.kind) {
      case KET_OP_MEASURE:
        if (o.nq != 2) return fail(KET_ERR_TYPE, "measure: nq must be 2 (qubit, classical bit)");
        if (o.q[1] < -1 || o.q[1] >= ncbits) return fail(KET_ERR_RANGE, "measure: classical bit out of range");
        break;
      case KET_OP_RESET:
        if (o.nq != 1) return fail(KET_ERR_TYPE, "reset: nq must be 1");
        if (o.q[0] < 0 || o.q[0] >= n)
          return fail(KET_ERR_RANGE, "qubit index " + std::to_string(o.q[0]) + " is out of range for a " +
                                         std::to_string(n) + "-qubit circuit");
        break;
      case KET_OP_IF: {
        if (o.nq != 4) return fail(KET_ERR_TYPE, "if: nq must be 4 (first bit, size, value, body length)");
        const int first = o.q[0], size = o.q[1], len = o.q[3];
        if (size < 0 || size > 31) return fail(KET_ERR_UNSUPPORTED, "if: registers of more than 31 bits");
        if (size > 0 && (first < 0 || first + size > ncbits)) return fail(KET_ERR_RANGE, "if: register out of range");
        if (len < 0 || i + 1 + (size_t)len > e) return fail(KET_ERR_TYPE, "if: body runs past its enclosing list");
        TRY(check_range(ops, i + 1, i + 1 + len, n, ncbits, gates));
        i += len;
        break;
      }
      default:
        gates.push_back(o);
        break;
    }
  }
  return KET_OK;
}

struct Runner {
  ket_state* st = nullptr;
  const ket_op* ops = nullptr;
  std::vector<double> mats;  // the caller's matrices, then X, Y, Z (gates.ts:15-17)
  size_t nmat = 0;
  int64_t pauli[4] = {0, 0, 0, 0};
  ket_noise nz{};
  uint32_t s = 1;
  std::vector<uint8_t> bits;
  std::vector<ket_op> seg;
  ket_exec_opts opts{};

  // makePrng's generator (circuit.ts:813-819)
  double draw() {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return (double)s / 4294967296.0;
  }
  int flush() {
    if (seg.empty()) return KET_OK;
    const int rc = ket_apply_ops(st, seg.data(), seg.size(), mats.data(), nmat, &opts);
    seg.clear();
    return rc;
  }
  void push_pauli(int which, int q) {
    ket_op o;
    memset(&o, 0, sizeof(o));
    o.kind = KET_OP_SINGLE;
    o.nq = 1;
    o.q[0] = q;
    o.mat = pauli[which];
    seg.push_back(o);
  }
  // dep1 / dep2 (circuit.ts:289-304): which Paulis a draw selects
  void dep1(int q) {
    const double r = draw();
    if (r >= nz.p1) return;
    const double u = r / nz.p1;
    push_pauli(u < 1.0 / 3 ? 1 : u < 2.0 / 3 ? 2 : 3, q);
  }
  void dep2(int a, int b) {
    static const int pairs[15][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 0}, {1, 1}, {1, 2}, {1, 3}, {2, 0},
                                     {2, 1}, {2, 2}, {2, 3}, {3, 0}, {3, 1}, {3, 2}, {3, 3}};
    const double r = draw();
    if (r >= nz.p2) return;
    int k = (int)std::floor(r / nz.p2 * 15);
    if (k > 14) k = 14;
    if (pairs[k][0]) push_pauli(pairs[k][0], a);
    if (pairs[k][1]) push_pauli(pairs[k][1], b);
  }
  // collapseQubit (circuit.ts:55-72); a qubit outside the state reads 0, as
  // the reference's mask then matches no index
  int collapse(int q, int& outcome) {
    TRY(flush());
    const double r = draw();
    double p1 = 0.0;
    const int n = st->n;
    const bool inside = q >= 0 && q < n;
    ket_ctx* c = st->ctx;
    if (inside) {
      const uint64_t half = uint64_t(1) << (n - 1);
      const uint64_t chunk = half > 4096 * 1024 ? (half + 4095) / 4096 : 1024;
      const int nb = (int)((half + chunk - 1) / chunk);
      void* scr;
      TRY(ctx_scratch(c, 8 * (size_t)nb + 64, &scr));
      double* part = (double*)scr;
      double* sum = part + nb;
      prof_begin(c);
      if (st->precision == KET_C64)
        k_prob_one<float><<<nb, KNT, 0, c->stream>>>((const float2*)st->amp, half, q, chunk, part);
      else
        k_prob_one<double><<<nb, KNT, 0, c->stream>>>((const double2*)st->amp, half, q, chunk, part);
      k_sum_in_order<<<1, 32, 0, c->stream>>>(part, nb, sum);
      prof_end(c, PK_READ);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "collapse reduction launch");
      c->d2h_bytes += 8;
      e = cudaMemcpyAsync(&p1, sum, 8, cudaMemcpyDeviceToHost, c->stream);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(P(q=1))");
      TRY(ctx_wait(c));
    }
    outcome = r < p1 ? 1 : 0;
    const double inv = 1 / std::sqrt(outcome == 1 ? p1 : 1 - p1);
    if (inside) {
      const uint64_t N = uint64_t(1) << n;
      const unsigned grid = (unsigned)std::min<uint64_t>((N + 255) / 256, 148 * 16);
      prof_begin(c);
      if (st->precision == KET_C64)
        k_collapse<float><<<grid, 256, 0, c->stream>>>((float2*)st->amp, N, q, outcome, inv);
      else
        k_collapse<double><<<grid, 256, 0, c->stream>>>((double2*)st->amp, N, q, outcome, inv);
      prof_end(c, PK_GATE);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "collapse launch");
    }
    return KET_OK;
  }
  // applyOps (circuit.ts:169-207) over ops[b, e)
  int run(size_t b, size_t e) {
    for (size_t i = b; i < e; i++) {
      const ket_op& o = ops[i];
      switch (o.kind) {
        case KET_OP_SINGLE:
          seg.push_back(o);
          if (nz.p1 != 0) dep1(o.q[0]);
          break;
        case KET_OP_CNOT: case KET_OP_CONTROLLED: case KET_OP_SWAP: case KET_OP_TWO:
          seg.push_back(o);
          if (nz.p2 != 0) dep2(o.q[0], o.q[1]);
          break;
        case KET_OP_BARRIER: break;
        case KET_OP_MEASURE: {
          int outcome;
          TRY(collapse(o.q[0], outcome));
          const int reported = (nz.pmeas != 0 && draw() < nz.pmeas) ? 1 - outcome : outcome;
          if (o.q[1] >= 0) bits[o.q[1]] = (uint8_t)reported;
          break;
        }
        case KET_OP_RESET: {
          int outcome;
          TRY(collapse(o.q[0], outcome));
          if (outcome == 1) push_pauli(1, o.q[0]);
          break;
        }
        case KET_OP_IF: {
          // cregValue (circuit.ts:164-166): the register as a little-endian integer
          int v = 0;
          for (int k = 0; k < o.q[1]; k++)
            if (bits[o.q[0] + k]) v |= 1 << k;
          if (v == o.q[2]) TRY(run(i + 1, i + 1 + o.q[3]));
          i += o.q[3];
          break;
        }
        default:  // toffoli, cswap, csrswap, unitary: no noise (circuit.ts:178-183)
          seg.push_back(o);
          break;
      }
    }
    return KET_OK;
  }
};

}  // namespace

extern "C" {

int ket_debug_pershot_path(int mode) {
  if (mode < 0 || mode > 2) return fail(KET_ERR_TYPE, "mode must be 0, 1 or 2");
  g_pershot_path = mode;
  return KET_OK;
}

int ket_run_shots(ket_state* st, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                  const ket_noise* noise, uint64_t init, size_t shots, uint32_t* prng_state, int ncbits,
                  uint64_t* out_idx, uint8_t* out_bits) {
  if (!st) return fail(KET_ERR_TYPE, "null state");
  if (nops && !ops) return fail(KET_ERR_TYPE, "null op list");
  if (!prng_state) return fail(KET_ERR_TYPE, "null prng state");
  if (ncbits < 0) return fail(KET_ERR_TYPE, "negative classical bit count");
  if (shots && !out_idx) return fail(KET_ERR_TYPE, "null output");
  if (shots && ncbits && !out_bits) return fail(KET_ERR_TYPE, "null classical-bit output");
  if (nmat && !mats) return fail(KET_ERR_TYPE, "null matrix buffer");
  if (init >> st->n) return fail(KET_ERR_RANGE, "initial index out of range");
  cudaSetDevice(st->ctx->device);
  // validate everything before touching the state
  std::vector<ket_op> gates;
  TRY(check_range(ops, 0, nops, st->n, ncbits, gates));
  {
    std::vector<Gate> lowered;
    std::string err;
    const int rc = lower_ops(st->n, gates.data(), gates.size(), mats, nmat, true, lowered, err);
    if (rc) return fail(rc, err);
  }
  const ket_noise nz0 = noise ? *noise : ket_noise{0.0, 0.0, 0.0};
  if (g_pershot_path != 1 && shots > 0 && st->n <= batched_max_qubits(st->precision) && ncbits <= 4096) {
    std::vector<TOp> tops;
    const int64_t op_draws = lower_shots(ops, 0, nops, nz0, false, tops);
    // per shot: the ops' draws, sampleSV's draw and the readout flips' draws
    const int64_t draws = op_draws < 0 ? -1 : op_draws + 1 + (nz0.pmeas != 0 ? st->n : 0);
    bool fits = draws > 0;
    for (const TOp& t : tops) fits = fits && t.mat >= -1;
    if (fits) {
      std::vector<double> tm(mats, mats + 2 * nmat);
      const int64_t pauli0 = (int64_t)nmat;
      static const double P[24] = {0, 0, 1, 0, 1, 0, 0, 0,    // X (gates.ts:15-17)
                                   0, 0, 0, -1, 0, 1, 0, 0,   // Y
                                   1, 0, 0, 0, 0, 0, -1, 0};  // Z
      tm.insert(tm.end(), P, P + 24);
      return run_batched(st, tops, draws, tm, pauli0, init, nz0, shots, prng_state, ncbits, out_idx, out_bits);
    }
  }
  if (g_pershot_path == 2) return fail(KET_ERR_UNSUPPORTED, "trajectories not batchable (state size or draws inside if)");
  Runner R;
  R.st = st;
  R.ops = ops;
  R.mats.assign(mats, mats + 2 * nmat);
  static const double P[3][8] = {{0, 0, 1, 0, 1, 0, 0, 0},     // X
                                 {0, 0, 0, -1, 0, 1, 0, 0},    // Y
                                 {1, 0, 0, 0, 0, 0, -1, 0}};   // Z
  for (int k = 0; k < 3; k++) {
    R.pauli[k + 1] = (int64_t)(R.mats.size() / 2);
    R.mats.insert(R.mats.end(), P[k], P[k] + 8);
  }
  R.nmat = R.mats.size() / 2;
  if (noise) R.nz = *noise;
  R.s = *prng_state ? *prng_state : 1u;
  R.bits.assign((size_t)ncbits, 0);
  ket_exec_opts_default(&R.opts);
  R.opts.prune = 1;
  for (size_t shot = 0; shot < shots; shot++) {
    TRY(ket_state_set_basis(st, init));
    std::fill(R.bits.begin(), R.bits.end(), 0);
    TRY(R.run(0, nops));
    TRY(R.flush());
    // sampleSV (circuit.ts:75-83) then the readout flips (:3466-3470)
    const double r = R.draw();
    uint64_t idx = 0;
    TRY(sample_indices(st, &r, 1, 0.0, &idx));
    if (R.nz.pmeas != 0)
      for (int q = 0; q < st->n; q++)
        if (R.draw() < R.nz.pmeas) idx ^= uint64_t(1) << q;
    out_idx[shot] = idx;
    if (ncbits) memcpy(out_bits + shot * (size_t)ncbits, R.bits.data(), (size_t)ncbits);
  }
  *prng_state = R.s;
  return KET_OK;
}

}  // extern "C"
