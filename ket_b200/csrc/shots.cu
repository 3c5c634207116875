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
//     One draw per shot does not pay for a whole sequential CDF, so above 12
//     qubits the draw walks chunk sums and then one chunk; that order of
//     additions differs from the sequential one only in rounding.
// The device state is the caller's ket_state, reset to |init> per shot.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "engine.h"

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
    TRY(sample_indices(st, &r, 1, 0.0, 12, &idx));
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
