// density.cpp -- runDM (density.ts:475-588) on the engine.
//
// The reference keeps rho as a sparse map keyed (row << n) | col and applies
// every op as U rho U^dagger, pruning each output entry once (dmSet).  Here
// rho is a dense 2n-qubit state with the same index: qubit n + q is qubit q of
// the row, qubit q is qubit q of the column.  U rho U^dagger is then one
// engine op on the row and column copies of U's qubits with the matrix
// U (x) conj(U), so the engine's per-op pruning is the reference's
// per-entry dmSet:
//   * single U on q    -> 4x4 on (n+q, q)
//   * two / controlled -> 16x16 on (n+a, n+b, a, b) (controlledGate, mps.ts:53-60)
//   * unitary on k <= 5 qubits -> 4^k x 4^k on the 2k copies
//   * cnot / swap / toffoli / cswap -> the permutation on the row copy and on
//     the column copy (applyPerm copies, no pruning)
//   * csrswap -> the reference's block rule (density.ts:532-575) as one 64x64
//     on (n+c, n+a, n+b, c, a, b): blocks with the row control set take
//     S rho S^dagger, the block with only the column control set takes
//     S^dagger rho S (its transpose-apply-transpose), the rest is unchanged;
//   * depolarize1 / depolarize2 (density.ts:193-264) -> their closed forms as
//     4x4 / 16x16 real maps on the row and column copies, after the gate they
//     follow (depolarize2 sums its 16 contributions at once where the
//     reference accumulates them one by one in its Map's order).
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

using namespace ket;

namespace {

typedef std::complex<double> zc;

struct Lowered {
  int n = 0;
  std::vector<ket_op> ops;
  std::vector<double> mats;

  void op(int kind, std::initializer_list<int> qs, const std::vector<zc>* m) {
    ket_op o;
    memset(&o, 0, sizeof(o));
    o.kind = kind;
    o.nq = (int)qs.size();
    int j = 0;
    for (int q : qs) o.q[j++] = q;
    o.mat = -1;
    if (m) {
      o.mat = (int64_t)(mats.size() / 2);
      for (const zc& z : *m) {
        mats.push_back(z.real());
        mats.push_back(z.imag());
      }
    }
    ops.push_back(o);
  }
  void op_q(int kind, const std::vector<int>& qs, const std::vector<zc>& m) {
    ket_op o;
    memset(&o, 0, sizeof(o));
    o.kind = kind;
    o.nq = (int)qs.size();
    for (size_t j = 0; j < qs.size(); j++) o.q[j] = qs[j];
    o.mat = (int64_t)(mats.size() / 2);
    for (const zc& z : m) {
      mats.push_back(z.real());
      mats.push_back(z.imag());
    }
    ops.push_back(o);
  }
};

// G (x) conj(G): index (i, j) -> (k, l) with coefficient G[i][k] conj(G[j][l]);
// rows of G act on the row copy (the more significant half of the local index)
std::vector<zc> kron_conj(const std::vector<zc>& g, int d) {
  std::vector<zc> m((size_t)d * d * d * d);
  for (int i = 0; i < d; i++)
    for (int j = 0; j < d; j++)
      for (int k = 0; k < d; k++)
        for (int l = 0; l < d; l++) m[(size_t)(i * d + j) * d * d + (k * d + l)] = g[i * d + k] * std::conj(g[j * d + l]);
  return m;
}

std::vector<zc> read_mat(const double* mats, int64_t off, size_t cnt) {
  std::vector<zc> g(cnt);
  for (size_t i = 0; i < cnt; i++) g[i] = zc(mats[2 * (off + i)], mats[2 * (off + i) + 1]);
  return g;
}

// depolarize1 (density.ts:193-222) on (row bit, column bit) of one qubit
std::vector<zc> dep1_map(double p) {
  const double sa = 1 - 2 * p / 3, sb = 2 * p / 3, cf = 1 - 4 * p / 3;
  std::vector<zc> m(16, 0.0);
  m[0 * 4 + 0] = sa; m[0 * 4 + 3] = sb;   // (0,0) <- sa rho00 + sb rho11
  m[3 * 4 + 3] = sa; m[3 * 4 + 0] = sb;   // (1,1) <- sa rho11 + sb rho00
  m[1 * 4 + 1] = cf; m[2 * 4 + 2] = cf;   // off-diagonal entries damp by 1 - 4p/3
  return m;
}

// depolarize2 (density.ts:239-264) on (row a, row b, column a, column b);
// PAULI15 (:226-231): {flip_a, flip_b, z_a, z_b}
std::vector<zc> dep2_map(double p) {
  static const int P15[15][4] = {{0, 1, 0, 0}, {0, 1, 0, 1}, {0, 0, 0, 1}, {1, 0, 0, 0}, {1, 1, 0, 0},
                                 {1, 1, 0, 1}, {1, 0, 0, 1}, {1, 0, 1, 0}, {1, 1, 1, 0}, {1, 1, 1, 1},
                                 {1, 0, 1, 1}, {0, 0, 1, 0}, {0, 1, 1, 0}, {0, 1, 1, 1}, {0, 0, 1, 1}};
  const double w1 = 1 - p, w2 = p / 15;
  std::vector<zc> m(256, 0.0);
  for (int in = 0; in < 16; in++) {
    const int ra = (in >> 3) & 1, rb = (in >> 2) & 1, ca = (in >> 1) & 1, cb = in & 1;
    m[in * 16 + in] += w1;
    for (const auto& P : P15) {
      const int out = ((ra ^ P[0]) << 3) | ((rb ^ P[1]) << 2) | ((ca ^ P[0]) << 1) | (cb ^ P[1]);
      const int parity = (P[2] * (ra ^ ca)) ^ (P[3] * (rb ^ cb));
      m[out * 16 + in] += parity ? -w2 : w2;
    }
  }
  return m;
}

// runDM's csrswap (density.ts:532-575) as a 64x64 on (row c, row a, row b,
// column c, column a, column b)
std::vector<zc> csrswap_map() {
  const double sq2 = 1 / std::sqrt(2.0);
  const zc S[16] = {1, 0, 0, 0, 0, sq2, zc(0, sq2), 0, 0, zc(0, sq2), sq2, 0, 0, 0, 0, 1};
  std::vector<zc> m(64 * 64, 0.0);
  for (int in = 0; in < 64; in++) {
    const int cr = (in >> 5) & 1, rab = (in >> 3) & 3, cc = (in >> 2) & 1, cab = in & 3;
    for (int orab = 0; orab < 4; orab++)
      for (int ocab = 0; ocab < 4; ocab++) {
        zc v;
        if (!cr && !cc) v = (orab == rab && ocab == cab) ? 1.0 : 0.0;
        else if (cr) v = S[orab * 4 + rab] * std::conj(S[ocab * 4 + cab]);  // S rho S^dagger
        else v = std::conj(S[orab * 4 + rab]) * S[ocab * 4 + cab];           // S^dagger rho S (S symmetric)
        const int out = (cr << 5) | (orab << 3) | (cc << 2) | ocab;
        m[(size_t)out * 64 + in] = v;
      }
  }
  return m;
}

#define TRY(x) do { int _rc = (x); if (_rc) return _rc; } while (0)

int check_dm(const ket_state* rho) {
  if (!rho) return fail(KET_ERR_TYPE, "null state");
  if (rho->n < 2 || rho->n % 2) return fail(KET_ERR_TYPE, "a density matrix is a state of 2n qubits, n >= 1");
  return KET_OK;
}

}  // namespace

extern "C" {

int ket_dm_run(ket_state* rho, const ket_op* ops, size_t nops, const double* mats, size_t nmat, double p1, double p2) {
  TRY(check_dm(rho));
  if (nops && !ops) return fail(KET_ERR_TYPE, "null op list");
  const int n = rho->n / 2;
  {
    std::vector<Gate> lowered;
    std::string err;
    const int rc = lower_ops(n, ops, nops, mats, nmat, true, lowered, err);
    if (rc) return fail(rc, err);
  }
  Lowered L;
  L.n = n;
  for (size_t i = 0; i < nops; i++) {
    const ket_op& o = ops[i];
    const int* q = o.q;
    bool noisy2 = false;
    switch (o.kind) {
      case KET_OP_SINGLE: {
        const std::vector<zc> m = kron_conj(read_mat(mats, o.mat, 4), 2);
        L.op(KET_OP_TWO, {n + q[0], q[0]}, &m);
        if (p1 > 0) {
          const std::vector<zc> d = dep1_map(p1);
          L.op(KET_OP_TWO, {n + q[0], q[0]}, &d);
        }
        break;
      }
      case KET_OP_CNOT:
        L.op(KET_OP_CNOT, {n + q[0], n + q[1]}, nullptr);
        L.op(KET_OP_CNOT, {q[0], q[1]}, nullptr);
        noisy2 = true;
        break;
      case KET_OP_SWAP:
        L.op(KET_OP_SWAP, {n + q[0], n + q[1]}, nullptr);
        L.op(KET_OP_SWAP, {q[0], q[1]}, nullptr);
        noisy2 = true;
        break;
      case KET_OP_TWO: case KET_OP_CONTROLLED: {
        std::vector<zc> g = read_mat(mats, o.mat, o.kind == KET_OP_TWO ? 16 : 4);
        if (o.kind == KET_OP_CONTROLLED)
          g = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, g[0], g[1], 0, 0, g[2], g[3]};
        L.op_q(KET_OP_UNITARY, {n + q[0], n + q[1], q[0], q[1]}, kron_conj(g, 4));
        noisy2 = true;
        break;
      }
      case KET_OP_TOFFOLI:
        L.op(KET_OP_TOFFOLI, {n + q[0], n + q[1], n + q[2]}, nullptr);
        L.op(KET_OP_TOFFOLI, {q[0], q[1], q[2]}, nullptr);
        break;
      case KET_OP_CSWAP:
        L.op(KET_OP_CSWAP, {n + q[0], n + q[1], n + q[2]}, nullptr);
        L.op(KET_OP_CSWAP, {q[0], q[1], q[2]}, nullptr);
        break;
      case KET_OP_CSRSWAP:
        L.op_q(KET_OP_UNITARY, {n + q[0], n + q[1], n + q[2], q[0], q[1], q[2]}, csrswap_map());
        break;
      case KET_OP_UNITARY: {
        if (o.nq > 5) return fail(KET_ERR_UNSUPPORTED, "dm(): unitary ops of more than 5 qubits");
        const int d = 1 << o.nq;
        std::vector<int> qs;
        for (int j = 0; j < o.nq; j++) qs.push_back(n + q[j]);
        for (int j = 0; j < o.nq; j++) qs.push_back(q[j]);
        L.op_q(KET_OP_UNITARY, qs, kron_conj(read_mat(mats, o.mat, (size_t)d * d), d));
        break;
      }
      default: break;  // barrier
    }
    if (noisy2 && p2 > 0) {
      const std::vector<zc> d = dep2_map(p2);
      L.op_q(KET_OP_UNITARY, {n + q[0], n + q[1], q[0], q[1]}, d);
    }
  }
  TRY(ket_state_set_basis(rho, 0));  // |0..0><0..0|
  ket_exec_opts o;
  ket_exec_opts_default(&o);
  o.prune = 1;
  return ket_apply_ops(rho, L.ops.data(), L.ops.size(), L.mats.data(), L.mats.size() / 2, &o);
}

int ket_dm_probs(const ket_state* rho, double* out) {
  TRY(check_dm(rho));
  if (!out) return fail(KET_ERR_TYPE, "null output");
  const int n = rho->n / 2;
  const uint64_t dim = uint64_t(1) << n;
  std::vector<uint64_t> idx(dim);
  for (uint64_t r = 0; r < dim; r++) idx[r] = (r << n) | r;
  std::vector<double> v(2 * dim);
  TRY(ket_amplitudes(rho, idx.data(), dim, v.data()));
  for (uint64_t r = 0; r < dim; r++) out[r] = v[2 * r];
  return KET_OK;
}

int ket_dm_bloch(const ket_state* rho, int q, double* out) {
  TRY(check_dm(rho));
  if (!out) return fail(KET_ERR_TYPE, "null output");
  const int n = rho->n / 2;
  if (q < 0 || q >= n)
    return fail(KET_ERR_RANGE, "qubit index " + std::to_string(q) + " is out of range for a " + std::to_string(n) +
                                   "-qubit circuit");
  const uint64_t dim = uint64_t(1) << n, qm = uint64_t(1) << q;
  std::vector<uint64_t> idx;
  idx.reserve(dim + dim / 2);
  for (uint64_t r = 0; r < dim; r++) idx.push_back((r << n) | r);
  for (uint64_t r = 0; r < dim; r++)
    if (!(r & qm)) idx.push_back((r << n) | (r | qm));
  std::vector<double> v(2 * idx.size());
  TRY(ket_amplitudes(rho, idx.data(), idx.size(), v.data()));
  double r00 = 0, r11 = 0, re = 0, im = 0;
  for (uint64_t r = 0; r < dim; r++) (r & qm ? r11 : r00) += v[2 * r];
  for (size_t k = dim; k < idx.size(); k++) {
    re += v[2 * k];
    im += v[2 * k + 1];
  }
  // DensityMatrix.blochAngles (density.ts:356-372)
  const double rz = r00 - r11, rx = 2 * re, ry = -2 * im;
  out[0] = std::acos(std::fmax(-1.0, std::fmin(1.0, rz)));
  out[1] = std::atan2(ry, rx);
  return KET_OK;
}

}  // extern "C"
