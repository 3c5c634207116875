// ket_oracle.cpp -- CPU restatement of the ket statevector path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the oracle that the GPU engine is
// checked against.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it; the product path (ket_b200/) never does.
//
// It restates, in plain C++ with IEEE FP64 and no FMA contraction
// (build with -ffp-contract=off), the algorithm of the reference TypeScript
// library dmvjs/ket:
//   src/complex.ts:10-24          complex add/mul/norm2/isNegligible
//   src/gates.ts:11-208           gate matrices
//   src/statevector.ts:16-280     sparse Map<bigint,Complex> kernels with
//                                 |a|^2 < 1e-14 pruning in accumulate()
//   src/circuit.ts:113-161        flattenOps / svFromBitstring / simulatePure
//   src/circuit.ts:813-819        makePrng (xorshift32)
//   src/circuit.ts:3406-3453      run() pure fast path (sort, CDF, lower bound)
//   src/circuit.ts:55-81, :169-207, :289-304, :3455-3481
//                                 the per-shot path: collapseQubit, sampleSV,
//                                 applyOps (measure / reset / if), dep1 / dep2
//   src/circuit.ts:1491-1518      amplitude / probability / marginals
//   src/circuit.ts:1462-1485      circuitMatrix
//   src/circuit.ts:4102-4129      blochAngles
//   src/density.ts:14-588         runDM: the density matrix with dmSet / dmAcc
//                                 pruning, depolarizing channels, purity,
//                                 entropy (Jacobi), blochAngles
//   src/circuit.ts:3700-3753      exactProbs / expectation
//   src/circuit.ts:1108-1146      #checkOp validation (RangeError / TypeError)
//   src/algorithms.ts:16-38       qft / iqft
//   src/algorithms.ts:231-276     maxCutHamiltonian / qaoa
//   src/algorithms.ts:301-336     vqe
//   src/algorithms.ts:366-399     realAmplitudes / efficientSU2
//   src/algorithms.ts:536-609     gradient (parameter shift) / minimize
//
// Three simulation modes:
//   ORC_SPARSE  the reference's own data structure: a hash map keyed by the
//               basis index, entries pruned exactly as accumulate() does.
//   ORC_DENSE   a dense FP64 vector with the same per-gate arithmetic and no
//               pruning (OpenMP over amplitude groups).
//   ORC_DENSE_PRUNE  dense, flushing every computed output with
//               |a|^2 < 1e-14 to zero -- the dense image of the sparse map.
//
// The workload generators at the end (seeded brickwork circuits, random
// 3-regular graphs, the transverse-field Ising chain and its ansatz) define
// the synthetic benchmark inputs; ket_b200/workloads.py draws the identical
// xorshift32 stream.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#include <map>
#include <unordered_map>
#include <unordered_set>
#include <algorithm>
#include <chrono>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- complex.ts
struct C { double re, im; };
static const C ZERO{0.0, 0.0};
static const C ONE{1.0, 0.0};
static inline C cx(double re, double im = 0.0) { return C{re, im}; }
static inline C add(C a, C b) { return C{a.re + b.re, a.im + b.im}; }
static inline C mul(C a, C b) { return C{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
static inline double norm2(C a) { return a.re * a.re + a.im * a.im; }
static inline bool negligible(C a) { return norm2(a) < 1e-14; }

// ---------------------------------------------------------------- gates.ts
typedef std::vector<C> Mat;  // row-major, 2x2 or 4x4 or 2^k x 2^k

static const double sq2 = 1.0 / std::sqrt(2.0);

static Mat m2(C a, C b, C c, C d) { return Mat{a, b, c, d}; }
static Mat gId() { return m2(ONE, ZERO, ZERO, ONE); }
static Mat gH() { return m2(cx(sq2), cx(sq2), cx(sq2), cx(-sq2)); }
static Mat gX() { return m2(ZERO, ONE, ONE, ZERO); }
static Mat gY() { return m2(ZERO, cx(0, -1), cx(0, 1), ZERO); }
static Mat gZ() { return m2(ONE, ZERO, ZERO, cx(-1)); }
static Mat gS() { return m2(ONE, ZERO, ZERO, cx(0, 1)); }
static Mat gSi() { return m2(ONE, ZERO, ZERO, cx(0, -1)); }
static Mat gT() { return m2(ONE, ZERO, ZERO, cx(sq2, sq2)); }
static Mat gTi() { return m2(ONE, ZERO, ZERO, cx(sq2, -sq2)); }
static Mat gV() { return m2(cx(.5, .5), cx(.5, -.5), cx(.5, -.5), cx(.5, .5)); }
static Mat gVi() { return m2(cx(.5, -.5), cx(.5, .5), cx(.5, .5), cx(.5, -.5)); }
static Mat gRx(double t) {
  double c = std::cos(t / 2), s = std::sin(t / 2);
  return m2(cx(c), cx(0, -s), cx(0, -s), cx(c));
}
static Mat gRy(double t) {
  double c = std::cos(t / 2), s = std::sin(t / 2);
  return m2(cx(c, 0), cx(-s), cx(s), cx(c));
}
static Mat gRz(double t) {
  double c = std::cos(t / 2), s = std::sin(t / 2);
  return m2(cx(c, -s), ZERO, ZERO, cx(c, s));
}
static Mat gU3(double th, double ph, double la) {
  double c = std::cos(th / 2), s = std::sin(th / 2);
  return m2(cx(c), cx(-s * std::cos(la), -s * std::sin(la)),
            cx(s * std::cos(ph), s * std::sin(ph)), cx(c * std::cos(ph + la), c * std::sin(ph + la)));
}
static Mat gU2(double ph, double la) { return gU3(M_PI / 2, ph, la); }
static Mat gU1(double la) { return m2(ONE, ZERO, ZERO, cx(std::cos(la), std::sin(la))); }
static Mat gGpi(double ph) {
  double c = std::cos(ph), s = std::sin(ph);
  return m2(ZERO, cx(c, -s), cx(c, s), ZERO);
}
static Mat gGpi2(double ph) {
  double c = std::cos(ph), s = std::sin(ph);
  return m2(cx(sq2), cx(-sq2 * s, -sq2 * c), cx(sq2 * s, -sq2 * c), cx(sq2));
}
static Mat m4(std::initializer_list<C> v) { return Mat(v); }
static Mat gXx(double t) {
  C co = cx(std::cos(t / 2)), ni = cx(0, -std::sin(t / 2));
  return m4({co, ZERO, ZERO, ni, ZERO, co, ni, ZERO, ZERO, ni, co, ZERO, ni, ZERO, ZERO, co});
}
static Mat gYy(double t) {
  C co = cx(std::cos(t / 2)), ni = cx(0, -std::sin(t / 2)), pi = cx(0, std::sin(t / 2));
  return m4({co, ZERO, ZERO, pi, ZERO, co, ni, ZERO, ZERO, ni, co, ZERO, pi, ZERO, ZERO, co});
}
static Mat gZz(double t) {
  double c = std::cos(t / 2), s = std::sin(t / 2);
  C m = cx(c, -s), p = cx(c, s);
  return m4({m, ZERO, ZERO, ZERO, ZERO, p, ZERO, ZERO, ZERO, ZERO, p, ZERO, ZERO, ZERO, ZERO, m});
}
static Mat gXy(double t) {
  C co = cx(std::cos(t / 2)), is = cx(0, std::sin(t / 2));
  return m4({ONE, ZERO, ZERO, ZERO, ZERO, co, is, ZERO, ZERO, is, co, ZERO, ZERO, ZERO, ZERO, ONE});
}
static Mat gMs(double p0, double p1) {
  double sp = std::sin(p0 + p1), cp = std::cos(p0 + p1);
  double sd = std::sin(p0 - p1), cd = std::cos(p0 - p1);
  return m4({cx(sq2), ZERO, ZERO, cx(-sp * sq2, -cp * sq2),
             ZERO, cx(sq2), cx(-sd * sq2, -cd * sq2), ZERO,
             ZERO, cx(sd * sq2, -cd * sq2), cx(sq2), ZERO,
             cx(sp * sq2, -cp * sq2), ZERO, ZERO, cx(sq2)});
}

// ---------------------------------------------------------------- Op IR (circuit.ts:20-47)
enum Kind { K_SINGLE, K_CNOT, K_SWAP, K_TWO, K_CONTROLLED, K_TOFFOLI, K_CSWAP, K_CSRSWAP, K_UNITARY, K_BARRIER,
            K_MEASURE, K_RESET, K_IF };

struct Op {
  Kind kind;
  std::vector<int> q;   // single:[q] cnot:[c,t] swap:[a,b] two:[a,b] controlled:[c,t]
                        // toffoli:[c1,c2,t] cswap/csrswap:[c,a,b] unitary: qs (qs[0]=MSB)
                        // measure / reset: [q]
  Mat m;
  int cbit = 0;                       // measure: classical bit (registers numbered consecutively)
  int reg0 = 0, regn = 0, value = 0;  // if: the register's first bit and size, the compared value
  std::vector<Op> body;               // if: the conditional ops
};

struct Circuit {
  int n;
  std::vector<Op> ops;
};

enum { ORC_OK = 0, ORC_RANGE = 1, ORC_TYPE = 2 };

static std::string g_err;

// #checkOp (circuit.ts:1113-1146)
static int check_op(const Circuit& c, const Op& op) {
  for (int q : op.q) {
    if (q < 0 || q >= c.n) {
      g_err = "qubit index " + std::to_string(q) + " is out of range for a " + std::to_string(c.n) + "-qubit circuit";
      return ORC_RANGE;
    }
  }
  if ((op.kind == K_CNOT || op.kind == K_CONTROLLED) && op.q[0] == op.q[1]) {
    g_err = "control and target qubits must differ (got " + std::to_string(op.q[0]) + ")";
    return ORC_TYPE;
  }
  if (op.kind == K_UNITARY) {
    if (op.q.empty()) { g_err = "unitary: qubits must be non-empty"; return ORC_TYPE; }
    size_t d = size_t(1) << op.q.size();
    if (op.m.size() != d * d) { g_err = "unitary: matrix shape"; return ORC_TYPE; }
  }
  return ORC_OK;
}

// Builder-method name -> op (circuit.ts:1152-1421, resolveParametric :1047-1073)
static int make_op(const std::string& name, const int* qs, int nq, const double* p, int np, Op& op) {
  auto need = [&](int k, int kp) -> bool {
    if (nq != k || np < kp) { g_err = "gate '" + name + "' arity"; return false; }
    return true;
  };
  op.q.assign(qs, qs + nq);
  op.m.clear();
  static const std::unordered_map<std::string, Mat (*)()> fixed1 = {
      {"id", gId}, {"h", gH}, {"x", gX}, {"y", gY}, {"z", gZ}, {"s", gS}, {"si", gSi}, {"sdg", gSi},
      {"t", gT}, {"ti", gTi}, {"tdg", gTi}, {"v", gV}, {"vi", gVi}, {"srn", gV}, {"srndg", gVi}};
  auto it = fixed1.find(name);
  if (it != fixed1.end()) { if (!need(1, 0)) return ORC_TYPE; op.kind = K_SINGLE; op.m = it->second(); return ORC_OK; }
  if (name == "rx") { if (!need(1, 1)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gRx(p[0]); return ORC_OK; }
  if (name == "ry") { if (!need(1, 1)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gRy(p[0]); return ORC_OK; }
  if (name == "rz" || name == "vz") { if (!need(1, 1)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gRz(p[0]); return ORC_OK; }
  if (name == "r2") { if (!need(1, 0)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gRz(M_PI / 2); return ORC_OK; }
  if (name == "r4") { if (!need(1, 0)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gRz(M_PI / 4); return ORC_OK; }
  if (name == "r8") { if (!need(1, 0)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gRz(M_PI / 8); return ORC_OK; }
  if (name == "u1" || name == "p") { if (!need(1, 1)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gU1(p[0]); return ORC_OK; }
  if (name == "u2") { if (!need(1, 2)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gU2(p[0], p[1]); return ORC_OK; }
  if (name == "u3") { if (!need(1, 3)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gU3(p[0], p[1], p[2]); return ORC_OK; }
  if (name == "gpi") { if (!need(1, 1)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gGpi(p[0]); return ORC_OK; }
  if (name == "gpi2") { if (!need(1, 1)) return ORC_TYPE; op.kind = K_SINGLE; op.m = gGpi2(p[0]); return ORC_OK; }
  if (name == "cnot" || name == "cx") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_CNOT; return ORC_OK; }
  if (name == "swap") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_SWAP; return ORC_OK; }
  if (name == "xx") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_TWO; op.m = gXx(p[0]); return ORC_OK; }
  if (name == "yy") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_TWO; op.m = gYy(p[0]); return ORC_OK; }
  if (name == "zz") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_TWO; op.m = gZz(p[0]); return ORC_OK; }
  if (name == "xy") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_TWO; op.m = gXy(p[0]); return ORC_OK; }
  if (name == "iswap") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_TWO; op.m = gXy(M_PI); return ORC_OK; }
  if (name == "srswap") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_TWO; op.m = gXy(M_PI / 2); return ORC_OK; }
  if (name == "ms") { if (!need(2, 2)) return ORC_TYPE; op.kind = K_TWO; op.m = gMs(p[0], p[1]); return ORC_OK; }
  static const std::unordered_map<std::string, Mat (*)()> fixedc = {
      {"cy", gY}, {"cz", gZ}, {"ch", gH}, {"cs", gS}, {"ct", gT}, {"csdg", gSi}, {"ctdg", gTi}, {"csrn", gV}};
  auto ic = fixedc.find(name);
  if (ic != fixedc.end()) { if (!need(2, 0)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = ic->second(); return ORC_OK; }
  if (name == "crx") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gRx(p[0]); return ORC_OK; }
  if (name == "cry") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gRy(p[0]); return ORC_OK; }
  if (name == "crz") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gRz(p[0]); return ORC_OK; }
  if (name == "cr2") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gRz(M_PI / 2); return ORC_OK; }
  if (name == "cr4") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gRz(M_PI / 4); return ORC_OK; }
  if (name == "cr8") { if (!need(2, 0)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gRz(M_PI / 8); return ORC_OK; }
  if (name == "cu1") { if (!need(2, 1)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gU1(p[0]); return ORC_OK; }
  if (name == "cu2") { if (!need(2, 2)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gU2(p[0], p[1]); return ORC_OK; }
  if (name == "cu3") { if (!need(2, 3)) return ORC_TYPE; op.kind = K_CONTROLLED; op.m = gU3(p[0], p[1], p[2]); return ORC_OK; }
  if (name == "ccx") { if (!need(3, 0)) return ORC_TYPE; op.kind = K_TOFFOLI; return ORC_OK; }
  if (name == "cswap") { if (!need(3, 0)) return ORC_TYPE; op.kind = K_CSWAP; return ORC_OK; }
  if (name == "csrswap") { if (!need(3, 0)) return ORC_TYPE; op.kind = K_CSRSWAP; return ORC_OK; }
  if (name == "barrier") { op.kind = K_BARRIER; return ORC_OK; }
  g_err = "unknown gate '" + name + "'";
  return ORC_TYPE;
}

static int circuit_add(Circuit& c, const std::string& name, std::vector<int> qs, std::vector<double> p) {
  Op op;
  int rc = make_op(name, qs.data(), (int)qs.size(), p.data(), (int)p.size(), op);
  if (rc) return rc;
  rc = check_op(c, op);
  if (rc) return rc;
  c.ops.push_back(std::move(op));
  return ORC_OK;
}

// ---------------------------------------------------------------- statevector.ts (sparse)
typedef std::unordered_map<uint64_t, C> SV;

struct PruneStats {
  uint64_t events = 0;     // accumulate() deletions of a nonzero value
  double max_abs = 0.0;    // largest |a| deleted
};

// accumulate (statevector.ts:19-27)
static inline void accumulate(SV& sv, uint64_t idx, C amp, PruneStats& ps) {
  auto it = sv.find(idx);
  C next = (it != sv.end()) ? add(it->second, amp) : amp;
  if (!negligible(next)) {
    if (it != sv.end()) it->second = next; else sv.emplace(idx, next);
  } else {
    if (it != sv.end()) sv.erase(it);
    double a = std::sqrt(norm2(next));
    if (a > 0) { ps.events++; if (a > ps.max_abs) ps.max_abs = a; }
  }
}
static inline C get(const SV& sv, uint64_t idx) {
  auto it = sv.find(idx);
  return it == sv.end() ? ZERO : it->second;
}

// applySingle (statevector.ts:47-65)
static SV applySingle(const SV& sv, int q, const Mat& g, PruneStats& ps) {
  SV next; next.reserve(sv.size() * 2);
  uint64_t mask = uint64_t(1) << q;
  std::unordered_set<uint64_t> seen; seen.reserve(sv.size());
  for (auto& kv : sv) {
    uint64_t base = kv.first & ~mask;
    if (!seen.insert(base).second) continue;
    C a0 = get(sv, base), a1 = get(sv, base | mask);
    accumulate(next, base, add(mul(g[0], a0), mul(g[1], a1)), ps);
    accumulate(next, base | mask, add(mul(g[2], a0), mul(g[3], a1)), ps);
  }
  return next;
}
// applyCNOT (:70-80)
static SV applyCNOT(const SV& sv, int c, int t) {
  SV next; next.reserve(sv.size());
  uint64_t cm = uint64_t(1) << c, tm = uint64_t(1) << t;
  for (auto& kv : sv) next[(kv.first & cm) ? kv.first ^ tm : kv.first] = kv.second;
  return next;
}
// applySWAP (:85-102)
static SV applySWAP(const SV& sv, int a, int b) {
  SV next; next.reserve(sv.size());
  uint64_t am = uint64_t(1) << a, bm = uint64_t(1) << b;
  for (auto& kv : sv) {
    bool ba = kv.first & am, bb = kv.first & bm;
    next[ba == bb ? kv.first : kv.first ^ am ^ bm] = kv.second;
  }
  return next;
}
// applyTwo (:110-132): local order [ctx, ctx|b, ctx|a, ctx|a|b], a = MSB
static SV applyTwo(const SV& sv, int a, int b, const Mat& g, PruneStats& ps) {
  SV next; next.reserve(sv.size() * 2);
  uint64_t ma = uint64_t(1) << a, mb = uint64_t(1) << b;
  std::unordered_set<uint64_t> seen; seen.reserve(sv.size());
  for (auto& kv : sv) {
    uint64_t ctx = kv.first & ~(ma | mb);
    if (!seen.insert(ctx).second) continue;
    uint64_t bases[4] = {ctx, ctx | mb, ctx | ma, ctx | ma | mb};
    C amps[4];
    for (int i = 0; i < 4; i++) amps[i] = get(sv, bases[i]);
    for (int r = 0; r < 4; r++) {
      C out = ZERO;
      for (int c = 0; c < 4; c++) out = add(out, mul(g[r * 4 + c], amps[c]));
      accumulate(next, bases[r], out, ps);
    }
  }
  return next;
}
// applyToffoli (:138-147)
static SV applyToffoli(const SV& sv, int c1, int c2, int t) {
  SV next; next.reserve(sv.size());
  uint64_t m1 = uint64_t(1) << c1, m2_ = uint64_t(1) << c2, tm = uint64_t(1) << t;
  for (auto& kv : sv) next[((kv.first & m1) && (kv.first & m2_)) ? kv.first ^ tm : kv.first] = kv.second;
  return next;
}
// applyCSwap (:153-168)
static SV applyCSwap(const SV& sv, int c, int a, int b) {
  SV next; next.reserve(sv.size());
  uint64_t cm = uint64_t(1) << c, am = uint64_t(1) << a, bm = uint64_t(1) << b;
  for (auto& kv : sv) {
    if (!(kv.first & cm)) { next[kv.first] = kv.second; continue; }
    bool ba = kv.first & am, bb = kv.first & bm;
    next[ba == bb ? kv.first : kv.first ^ am ^ bm] = kv.second;
  }
  return next;
}
// applyCsrSwap (:177-207)
static SV applyCsrSwap(const SV& sv, int c, int a, int b, PruneStats& ps) {
  SV next; next.reserve(sv.size() * 2);
  uint64_t cm = uint64_t(1) << c, am = uint64_t(1) << a, bm = uint64_t(1) << b;
  std::unordered_set<uint64_t> seen; seen.reserve(sv.size());
  for (auto& kv : sv) {
    uint64_t ctx = kv.first & ~(cm | am | bm);
    if (!seen.insert(ctx).second) continue;
    for (uint64_t cc : {uint64_t(0), cm}) {
      uint64_t bases[4] = {ctx | cc, ctx | cc | bm, ctx | cc | am, ctx | cc | am | bm};
      C amps[4];
      for (int i = 0; i < 4; i++) amps[i] = get(sv, bases[i]);
      if (cc == 0) {
        for (int r = 0; r < 4; r++) accumulate(next, bases[r], amps[r], ps);
      } else {
        accumulate(next, bases[0], amps[0], ps);
        accumulate(next, bases[3], amps[3], ps);
        C a01 = amps[1], a10 = amps[2];
        accumulate(next, bases[1], add(mul(cx(sq2, 0), a01), mul(cx(0, sq2), a10)), ps);
        accumulate(next, bases[2], add(mul(cx(0, sq2), a01), mul(cx(sq2, 0), a10)), ps);
      }
    }
  }
  return next;
}
// applyControlled (:212-234)
static SV applyControlled(const SV& sv, int c, int t, const Mat& g, PruneStats& ps) {
  SV next; next.reserve(sv.size() * 2);
  uint64_t cm = uint64_t(1) << c, tm = uint64_t(1) << t;
  std::unordered_set<uint64_t> seen; seen.reserve(sv.size());
  for (auto& kv : sv) {
    if (!(kv.first & cm)) { accumulate(next, kv.first, kv.second, ps); continue; }
    uint64_t base = kv.first & ~tm;
    if (!seen.insert(base).second) continue;
    C a0 = get(sv, base), a1 = get(sv, base | tm);
    accumulate(next, base, add(mul(g[0], a0), mul(g[1], a1)), ps);
    accumulate(next, base | tm, add(mul(g[2], a0), mul(g[3], a1)), ps);
  }
  return next;
}
// applyUnitary (:240-270)
static SV applyUnitary(const SV& sv, const std::vector<int>& qs, const Mat& m, PruneStats& ps) {
  int k = (int)qs.size();
  size_t dim = size_t(1) << k;
  std::vector<uint64_t> masks(k);
  uint64_t all = 0;
  for (int i = 0; i < k; i++) { masks[i] = uint64_t(1) << qs[i]; all |= masks[i]; }
  SV next; next.reserve(sv.size() * 2);
  std::unordered_set<uint64_t> seen; seen.reserve(sv.size());
  std::vector<uint64_t> bases(dim);
  std::vector<C> amps(dim);
  for (auto& kv : sv) {
    uint64_t ctx = kv.first & ~all;
    if (!seen.insert(ctx).second) continue;
    for (size_t i = 0; i < dim; i++) {
      uint64_t b = ctx;
      for (int bit = 0; bit < k; bit++) if ((i >> (k - 1 - bit)) & 1) b |= masks[bit];
      bases[i] = b;
      amps[i] = get(sv, b);
    }
    for (size_t r = 0; r < dim; r++) {
      C out = ZERO;
      for (size_t c = 0; c < dim; c++) out = add(out, mul(m[r * dim + c], amps[c]));
      accumulate(next, bases[r], out, ps);
    }
  }
  return next;
}

// ---------------------------------------------------------------- dense restatement
struct Dense {
  int n;
  std::vector<C> a;
  bool prune;
  PruneStats ps;
};

static inline C dprune(Dense& d, C v) {
  if (d.prune && negligible(v)) return ZERO;
  return v;
}

static void dense_apply(Dense& d, const Op& op) {
  const uint64_t N = uint64_t(1) << d.n;
  C* A = d.a.data();
  const bool pr = d.prune;
  auto P = [pr](C v) -> C { return (pr && negligible(v)) ? ZERO : v; };
  switch (op.kind) {
    case K_SINGLE: {
      uint64_t m = uint64_t(1) << op.q[0];
      const Mat& g = op.m;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)(N / 2); i++) {
        uint64_t lo = (uint64_t)i & (m - 1), hi = ((uint64_t)i & ~(m - 1)) << 1;
        uint64_t x0 = hi | lo, x1 = x0 | m;
        C a0 = A[x0], a1 = A[x1];
        A[x0] = P(add(mul(g[0], a0), mul(g[1], a1)));
        A[x1] = P(add(mul(g[2], a0), mul(g[3], a1)));
      }
      break;
    }
    case K_CONTROLLED: {
      uint64_t cm = uint64_t(1) << op.q[0], m = uint64_t(1) << op.q[1];
      const Mat& g = op.m;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)(N / 2); i++) {
        uint64_t lo = (uint64_t)i & (m - 1), hi = ((uint64_t)i & ~(m - 1)) << 1;
        uint64_t x0 = hi | lo, x1 = x0 | m;
        if (!(x0 & cm)) continue;
        C a0 = A[x0], a1 = A[x1];
        A[x0] = P(add(mul(g[0], a0), mul(g[1], a1)));
        A[x1] = P(add(mul(g[2], a0), mul(g[3], a1)));
      }
      break;
    }
    case K_CNOT: case K_TOFFOLI: {
      uint64_t cm = 0;
      for (size_t i = 0; i + 1 < op.q.size(); i++) cm |= uint64_t(1) << op.q[i];
      uint64_t m = uint64_t(1) << op.q.back();
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)(N / 2); i++) {
        uint64_t lo = (uint64_t)i & (m - 1), hi = ((uint64_t)i & ~(m - 1)) << 1;
        uint64_t x0 = hi | lo, x1 = x0 | m;
        if ((x0 & cm) != cm) continue;
        std::swap(A[x0], A[x1]);
      }
      break;
    }
    case K_SWAP: case K_CSWAP: {
      uint64_t cm = op.kind == K_CSWAP ? (uint64_t(1) << op.q[0]) : 0;
      int qa = op.q[op.q.size() - 2], qb = op.q.back();
      uint64_t am = uint64_t(1) << qa, bm = uint64_t(1) << qb;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)N; i++) {
        uint64_t x = (uint64_t)i;
        if ((x & cm) != cm) continue;
        if ((x & am) && !(x & bm)) std::swap(A[x], A[x ^ am ^ bm]);
      }
      break;
    }
    case K_TWO: case K_CSRSWAP: {
      Mat g = op.m;
      uint64_t cm = 0;
      int a = op.q[0], b = op.q[1];
      if (op.kind == K_CSRSWAP) {
        cm = uint64_t(1) << op.q[0]; a = op.q[1]; b = op.q[2];
        g = m4({ONE, ZERO, ZERO, ZERO, ZERO, cx(sq2, 0), cx(0, sq2), ZERO,
                ZERO, cx(0, sq2), cx(sq2, 0), ZERO, ZERO, ZERO, ZERO, ONE});
      }
      uint64_t ma = uint64_t(1) << a, mb = uint64_t(1) << b;
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)N; i++) {
        uint64_t x = (uint64_t)i;
        if (x & (ma | mb)) continue;
        if ((x & cm) != cm) continue;
        uint64_t bs[4] = {x, x | mb, x | ma, x | ma | mb};
        C am_[4];
        for (int j = 0; j < 4; j++) am_[j] = A[bs[j]];
        if (op.kind == K_CSRSWAP) {
          // statevector.ts:195-200: |c00>,|c11> pass through; the 01/10 block is computed
          A[bs[1]] = P(add(mul(cx(sq2, 0), am_[1]), mul(cx(0, sq2), am_[2])));
          A[bs[2]] = P(add(mul(cx(0, sq2), am_[1]), mul(cx(sq2, 0), am_[2])));
          continue;
        }
        for (int r = 0; r < 4; r++) {
          C out = ZERO;
          for (int c = 0; c < 4; c++) out = add(out, mul(g[r * 4 + c], am_[c]));
          A[bs[r]] = P(out);
        }
      }
      break;
    }
    case K_UNITARY: {
      int k = (int)op.q.size();
      size_t dim = size_t(1) << k;
      uint64_t all = 0;
      std::vector<uint64_t> masks(k);
      for (int i = 0; i < k; i++) { masks[i] = uint64_t(1) << op.q[i]; all |= masks[i]; }
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < (int64_t)N; i++) {
        uint64_t x = (uint64_t)i;
        if (x & all) continue;
        std::vector<uint64_t> bs(dim);
        std::vector<C> am_(dim);
        for (size_t j = 0; j < dim; j++) {
          uint64_t b = x;
          for (int bit = 0; bit < k; bit++) if ((j >> (k - 1 - bit)) & 1) b |= masks[bit];
          bs[j] = b; am_[j] = A[b];
        }
        for (size_t r = 0; r < dim; r++) {
          C out = ZERO;
          for (size_t c = 0; c < dim; c++) out = add(out, mul(op.m[r * dim + c], am_[c]));
          A[bs[r]] = P(out);
        }
      }
      break;
    }
    case K_BARRIER: case K_MEASURE: case K_RESET: case K_IF: break;
  }
}

// ---------------------------------------------------------------- simulatePure (circuit.ts:143-161)
struct State {
  int n;
  int mode;        // 0 sparse, 1 dense, 2 dense+prune
  SV sv;
  Dense d;
  PruneStats ps;
};

static State* simulate(const Circuit& c, uint64_t init, int mode) {
  State* s = new State();
  s->n = c.n;
  s->mode = mode;
  if (mode == 0) {
    s->sv.emplace(init, ONE);
    for (const Op& op : c.ops) {
      switch (op.kind) {
        case K_SINGLE: s->sv = applySingle(s->sv, op.q[0], op.m, s->ps); break;
        case K_CNOT: s->sv = applyCNOT(s->sv, op.q[0], op.q[1]); break;
        case K_CONTROLLED: s->sv = applyControlled(s->sv, op.q[0], op.q[1], op.m, s->ps); break;
        case K_SWAP: s->sv = applySWAP(s->sv, op.q[0], op.q[1]); break;
        case K_TOFFOLI: s->sv = applyToffoli(s->sv, op.q[0], op.q[1], op.q[2]); break;
        case K_CSWAP: s->sv = applyCSwap(s->sv, op.q[0], op.q[1], op.q[2]); break;
        case K_CSRSWAP: s->sv = applyCsrSwap(s->sv, op.q[0], op.q[1], op.q[2], s->ps); break;
        case K_TWO: s->sv = applyTwo(s->sv, op.q[0], op.q[1], op.m, s->ps); break;
        case K_UNITARY: s->sv = applyUnitary(s->sv, op.q, op.m, s->ps); break;
        case K_BARRIER: case K_MEASURE: case K_RESET: case K_IF: break;
      }
    }
  } else {
    s->d.n = c.n;
    s->d.prune = (mode == 2);
    s->d.a.assign(size_t(1) << c.n, ZERO);
    s->d.a[init] = ONE;
    for (const Op& op : c.ops) dense_apply(s->d, op);
  }
  return s;
}

static C state_get(const State* s, uint64_t idx) {
  if (s->mode == 0) return get(s->sv, idx);
  return s->d.a[idx];
}

// probabilities (statevector.ts:273-280), sorted ascending by index
static void probs_sorted(const State* s, std::vector<std::pair<uint64_t, double>>& out) {
  out.clear();
  if (s->mode == 0) {
    for (auto& kv : s->sv) {
      double p = kv.second.re * kv.second.re + kv.second.im * kv.second.im;
      if (p > 1e-14) out.emplace_back(kv.first, p);
    }
    std::sort(out.begin(), out.end());
  } else {
    uint64_t N = uint64_t(1) << s->n;
    for (uint64_t i = 0; i < N; i++) {
      const C& a = s->d.a[i];
      double p = a.re * a.re + a.im * a.im;
      if (p > 1e-14) out.emplace_back(i, p);
    }
  }
}

// makePrng (circuit.ts:813-819)
struct Prng {
  uint32_t s;
  explicit Prng(uint32_t seed) : s(seed ? seed : 1u) {}
  uint32_t next_u32() { s ^= s << 13; s ^= s >> 17; s ^= s << 5; return s; }
  double next() { return (double)next_u32() / 4294967296.0; }
};

// run() pure fast path (circuit.ts:3424-3453): returns the sampled index per shot
static void run_shots(const State* s, int shots, uint32_t seed, uint64_t* out) {
  std::vector<std::pair<uint64_t, double>> pr;
  probs_sorted(s, pr);
  std::vector<double> cum(pr.size());
  double acc = 0;
  for (size_t i = 0; i < pr.size(); i++) { acc += pr[i].second; cum[i] = acc; }
  if (!cum.empty()) cum.back() = 1.0;
  Prng rng(seed);
  for (int i = 0; i < shots; i++) {
    double r = rng.next();
    int64_t lo = 0, hi = (int64_t)cum.size() - 1;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (cum[mid] < r) lo = mid + 1; else hi = mid;
    }
    out[i] = cum.empty() ? 0 : pr[lo].first;
  }
}

// ---------------------------------------------------------------- the per-shot path
// Entries of a sparse state in ascending index order.
static std::vector<std::pair<uint64_t, C>> sorted_entries(const SV& sv) {
  std::vector<std::pair<uint64_t, C>> e(sv.begin(), sv.end());
  std::sort(e.begin(), e.end(), [](const std::pair<uint64_t, C>& a, const std::pair<uint64_t, C>& b) {
    return a.first < b.first;
  });
  return e;
}

// collapseQubit (circuit.ts:55-72).  P(q=1) is summed in ascending index
// order; the reference sums in its Map's insertion order, which differs from
// this only in rounding.
static int collapse(SV& sv, int q, double rand) {
  const uint64_t mask = (q >= 0 && q < 64) ? (uint64_t(1) << q) : 0;
  const auto e = sorted_entries(sv);
  double p1 = 0;
  for (const auto& kv : e)
    if (kv.first & mask) p1 += kv.second.re * kv.second.re + kv.second.im * kv.second.im;
  const int outcome = rand < p1 ? 1 : 0;
  const double inv = 1 / std::sqrt(outcome == 1 ? p1 : 1 - p1);
  SV next;
  next.reserve(e.size());
  for (const auto& kv : e)
    if (outcome == 1 ? (kv.first & mask) != 0 : (kv.first & mask) == 0)
      next.emplace(kv.first, C{kv.second.re * inv, kv.second.im * inv});
  sv = std::move(next);
  return outcome;
}

// sampleSV (circuit.ts:75-83)
static uint64_t sample_sv(const SV& sv, double rand) {
  const auto e = sorted_entries(sv);
  double cum = 0;
  for (const auto& kv : e) {
    cum += kv.second.re * kv.second.re + kv.second.im * kv.second.im;
    if (rand <= cum) return kv.first;
  }
  return e.empty() ? 0 : e.back().first;
}

struct Noise { double p1, p2, pm; };

// dep1 / dep2 (circuit.ts:289-304); TWO_PAULI order (:262-268), 0 = I
static void dep1(SV& sv, int q, double p, double rand, PruneStats& ps) {
  if (rand >= p) return;
  const double r = rand / p;
  if (r < 1.0 / 3) sv = applySingle(sv, q, gX(), ps);
  else if (r < 2.0 / 3) sv = applySingle(sv, q, gY(), ps);
  else sv = applySingle(sv, q, gZ(), ps);
}
static void dep2(SV& sv, int a, int b, double p, double rand, PruneStats& ps) {
  if (rand >= p) return;
  static const int pairs[15][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 0}, {1, 1}, {1, 2}, {1, 3}, {2, 0},
                                   {2, 1}, {2, 2}, {2, 3}, {3, 0}, {3, 1}, {3, 2}, {3, 3}};
  const int k = std::min((int)std::floor(rand / p * 15), 14);
  Mat (*const pauli[4])() = {nullptr, gX, gY, gZ};
  if (pairs[k][0]) sv = applySingle(sv, a, pauli[pairs[k][0]](), ps);
  if (pairs[k][1]) sv = applySingle(sv, b, pauli[pairs[k][1]](), ps);
}

// applyOps (circuit.ts:169-207)
static void apply_ops(const std::vector<Op>& ops, SV& sv, std::vector<uint8_t>& bits, Prng& rng, const Noise& nz,
                      PruneStats& ps) {
  for (const Op& op : ops) {
    switch (op.kind) {
      case K_SINGLE:
        sv = applySingle(sv, op.q[0], op.m, ps);
        if (nz.p1 != 0) dep1(sv, op.q[0], nz.p1, rng.next(), ps);
        break;
      case K_CNOT:
        sv = applyCNOT(sv, op.q[0], op.q[1]);
        if (nz.p2 != 0) dep2(sv, op.q[0], op.q[1], nz.p2, rng.next(), ps);
        break;
      case K_CONTROLLED:
        sv = applyControlled(sv, op.q[0], op.q[1], op.m, ps);
        if (nz.p2 != 0) dep2(sv, op.q[0], op.q[1], nz.p2, rng.next(), ps);
        break;
      case K_SWAP:
        sv = applySWAP(sv, op.q[0], op.q[1]);
        if (nz.p2 != 0) dep2(sv, op.q[0], op.q[1], nz.p2, rng.next(), ps);
        break;
      case K_TOFFOLI: sv = applyToffoli(sv, op.q[0], op.q[1], op.q[2]); break;
      case K_CSWAP: sv = applyCSwap(sv, op.q[0], op.q[1], op.q[2]); break;
      case K_CSRSWAP: sv = applyCsrSwap(sv, op.q[0], op.q[1], op.q[2], ps); break;
      case K_TWO:
        sv = applyTwo(sv, op.q[0], op.q[1], op.m, ps);
        if (nz.p2 != 0) dep2(sv, op.q[0], op.q[1], nz.p2, rng.next(), ps);
        break;
      case K_UNITARY: sv = applyUnitary(sv, op.q, op.m, ps); break;
      case K_MEASURE: {
        const int outcome = collapse(sv, op.q[0], rng.next());
        const int reported = (nz.pm != 0 && rng.next() < nz.pm) ? 1 - outcome : outcome;
        bits[op.cbit] = (uint8_t)reported;
        break;
      }
      case K_RESET:
        if (collapse(sv, op.q[0], rng.next()) == 1) sv = applySingle(sv, op.q[0], gX(), ps);
        break;
      case K_IF: {
        // cregValue (circuit.ts:164-166): the register as a little-endian integer
        int v = 0;
        for (int i = 0; i < op.regn; i++)
          if (bits[op.reg0 + i]) v |= 1 << i;
        if (v == op.value) apply_ops(op.body, sv, bits, rng, nz, ps);
        break;
      }
      case K_BARRIER: break;
    }
  }
}

// run() per-shot path (circuit.ts:3455-3481): one trajectory per shot from
// |init>; out_idx[s] = the sampled index after readout flips, out_bits[s *
// ncbits + b] = classical bit b at the end of shot s.  Returns the stream's
// state after the last draw.
static uint32_t run_pershot(const Circuit& c, uint64_t init, int shots, uint32_t seed, const Noise& nz, int ncbits,
                            uint64_t* out_idx, uint8_t* out_bits) {
  Prng rng(seed);
  PruneStats ps;
  std::vector<uint8_t> bits(ncbits);
  for (int i = 0; i < shots; i++) {
    std::fill(bits.begin(), bits.end(), 0);
    SV sv;
    sv.emplace(init, ONE);
    apply_ops(c.ops, sv, bits, rng, nz, ps);
    uint64_t idx = sample_sv(sv, rng.next());
    if (nz.pm != 0)
      for (int q = 0; q < c.n; q++)
        if (rng.next() < nz.pm) idx ^= uint64_t(1) << q;
    out_idx[i] = idx;
    for (int b = 0; b < ncbits; b++) out_bits[(size_t)i * ncbits + b] = bits[b];
  }
  return rng.s;
}

// circuitMatrix (circuit.ts:1462-1485): column col is simulatePure from
// |flip(col)> (sparse mode); rows and columns use q0 as the most significant bit
static void circuit_matrix(const Circuit& c, double* out) {
  const int n = c.n;
  const uint64_t dim = uint64_t(1) << n;
  auto flip = [n](uint64_t i) {
    uint64_t r = 0;
    for (int b = 0; b < n; b++)
      if (i & (uint64_t(1) << b)) r |= uint64_t(1) << (n - 1 - b);
    return r;
  };
  std::memset(out, 0, sizeof(double) * 2 * dim * dim);
  for (uint64_t col = 0; col < dim; col++) {
    State* s = simulate(c, flip(col), 0);
    for (auto& kv : s->sv) {
      const uint64_t at = flip(kv.first) * dim + col;
      out[2 * at] = kv.second.re;
      out[2 * at + 1] = kv.second.im;
    }
    delete s;
  }
}

// blochAngles (circuit.ts:4102-4129) over the entries in ascending index order;
// out = {rho00, rho11, Re rho01, Im rho01, theta, phi}
static void bloch(const State* s, int q, double* out) {
  const uint64_t mask = uint64_t(1) << q;
  std::vector<std::pair<uint64_t, C>> e;
  if (s->mode == 0) e = sorted_entries(s->sv);
  else
    for (uint64_t i = 0; i < s->d.a.size(); i++)
      if (s->d.a[i].re != 0 || s->d.a[i].im != 0) e.emplace_back(i, s->d.a[i]);
  double r00 = 0, r11 = 0, re = 0, im = 0;
  for (const auto& kv : e) {
    const C& a = kv.second;
    const double p = a.re * a.re + a.im * a.im;
    if (kv.first & mask) { r11 += p; continue; }
    r00 += p;
    const C a1 = state_get(s, kv.first | mask);
    if (a1.re != 0 || a1.im != 0) {
      re += a.re * a1.re + a.im * a1.im;
      im += a.im * a1.re - a.re * a1.im;
    }
  }
  const double rz = r00 - r11, rx = 2 * re, ry = -2 * im;
  out[0] = r00; out[1] = r11; out[2] = re; out[3] = im;
  out[4] = std::acos(std::max(-1.0, std::min(1.0, rz)));
  out[5] = std::atan2(ry, rx);
}

// ---------------------------------------------------------------- density.ts (runDM)
// The reference keeps rho sparse, key = (row << n) | col (density.ts:14-35);
// here an ordered map, so every iteration is in ascending key order (the
// reference's Map iterates in insertion order, which changes only the order of
// the sums in depolarize2 and so only their rounding).
typedef std::map<uint64_t, C> DMap;
static inline C conjc(C a) { return C{a.re, -a.im}; }
static inline C dm_get(const DMap& m, uint64_t k) {
  auto it = m.find(k);
  return it == m.end() ? ZERO : it->second;
}
static inline void dm_set(DMap& m, uint64_t k, C v) {  // dmSet (:23-27)
  if (!negligible(v)) m[k] = v;
  else m.erase(k);
}
static inline void dm_acc(DMap& m, uint64_t k, C v) {  // dmAcc (:29-35)
  auto it = m.find(k);
  C nx = it != m.end() ? add(it->second, v) : v;
  if (!negligible(nx)) m[k] = nx;
  else if (it != m.end()) m.erase(it);
}

// applySingle (:46-79)
static DMap dm_single(const DMap& dm, int n, int q, const Mat& g) {
  DMap next;
  const uint64_t dim_mask = (uint64_t(1) << n) - 1, qm = uint64_t(1) << q;
  const uint64_t krm = qm << n, kcm = qm;
  const C a = g[0], b = g[1], c = g[2], d = g[3];
  const C ca = conjc(a), cb = conjc(b), cc = conjc(c), cd = conjc(d);
  std::unordered_set<uint64_t> seen;
  for (const auto& kv : dm) {
    const uint64_t ctx = kv.first & ~krm & ~kcm;
    if (!seen.insert(ctx).second) continue;
    const uint64_t r0 = ctx >> n, c0 = ctx & dim_mask, r1 = r0 | qm, c1 = c0 | qm;
    const C p00 = dm_get(dm, (r0 << n) | c0), p01 = dm_get(dm, (r0 << n) | c1);
    const C p10 = dm_get(dm, (r1 << n) | c0), p11 = dm_get(dm, (r1 << n) | c1);
    const C t00 = add(mul(a, p00), mul(b, p10)), t01 = add(mul(a, p01), mul(b, p11));
    const C t10 = add(mul(c, p00), mul(d, p10)), t11 = add(mul(c, p01), mul(d, p11));
    dm_set(next, (r0 << n) | c0, add(mul(ca, t00), mul(cb, t01)));
    dm_set(next, (r0 << n) | c1, add(mul(cc, t00), mul(cd, t01)));
    dm_set(next, (r1 << n) | c0, add(mul(ca, t10), mul(cb, t11)));
    dm_set(next, (r1 << n) | c1, add(mul(cc, t10), mul(cd, t11)));
  }
  return next;
}

// applyUnitaryN (:133-180); applyTwo (:81-119) is its 2-qubit case with the
// same sums
static DMap dm_unitary(const DMap& dm, int n, const std::vector<int>& qs, const Mat& m) {
  DMap next;
  const uint64_t dim_mask = (uint64_t(1) << n) - 1;
  const int k = (int)qs.size();
  const size_t ld = size_t(1) << k;
  uint64_t all = 0;
  std::vector<uint64_t> masks(k);
  for (int i = 0; i < k; i++) { masks[i] = uint64_t(1) << qs[i]; all |= masks[i]; }
  auto bases = [&](uint64_t base) {
    std::vector<uint64_t> b(ld);
    for (size_t i = 0; i < ld; i++) {
      uint64_t v = base;
      for (int bit = 0; bit < k; bit++)
        if ((i >> (k - 1 - bit)) & 1) v |= masks[bit];
      b[i] = v;
    }
    return b;
  };
  std::unordered_set<uint64_t> seen;
  for (const auto& kv : dm) {
    const uint64_t ctx = kv.first & ~(all << n) & ~all;
    if (!seen.insert(ctx).second) continue;
    const std::vector<uint64_t> rb = bases(ctx >> n), cb = bases(ctx & dim_mask);
    std::vector<C> p(ld * ld), t(ld * ld);
    for (size_t ri = 0; ri < ld; ri++)
      for (size_t ci = 0; ci < ld; ci++) p[ri * ld + ci] = dm_get(dm, (rb[ri] << n) | cb[ci]);
    for (size_t ri = 0; ri < ld; ri++)
      for (size_t ci = 0; ci < ld; ci++) {
        C v = ZERO;
        for (size_t j = 0; j < ld; j++) v = add(v, mul(m[ri * ld + j], p[j * ld + ci]));
        t[ri * ld + ci] = v;
      }
    for (size_t ri = 0; ri < ld; ri++)
      for (size_t ci = 0; ci < ld; ci++) {
        C v = ZERO;
        for (size_t j = 0; j < ld; j++) v = add(v, mul(t[ri * ld + j], conjc(m[ci * ld + j])));
        dm_set(next, (rb[ri] << n) | cb[ci], v);
      }
  }
  return next;
}

// applyPerm (:122-130)
template <typename F>
static DMap dm_perm(const DMap& dm, int n, F f) {
  DMap next;
  const uint64_t dim_mask = (uint64_t(1) << n) - 1;
  for (const auto& kv : dm) next[(f(kv.first >> n) << n) | f(kv.first & dim_mask)] = kv.second;
  return next;
}

// depolarize1 (:193-222)
static DMap dm_dep1(const DMap& dm, int n, int q, double p) {
  if (p <= 0) return dm;
  DMap next;
  const uint64_t dim_mask = (uint64_t(1) << n) - 1, qm = uint64_t(1) << q;
  const double sa = 1 - 2 * p / 3, sb = 2 * p / 3, cf = 1 - 4 * p / 3;
  std::unordered_set<uint64_t> seen;
  for (const auto& kv : dm) {
    const uint64_t ctx = kv.first & ~(qm << n) & ~qm;
    if (!seen.insert(ctx).second) continue;
    const uint64_t r0 = ctx >> n, c0 = ctx & dim_mask, r1 = r0 | qm, c1 = c0 | qm;
    const C p00 = dm_get(dm, (r0 << n) | c0), p11 = dm_get(dm, (r1 << n) | c1);
    dm_set(next, (r0 << n) | c0, C{sa * p00.re + sb * p11.re, sa * p00.im + sb * p11.im});
    dm_set(next, (r1 << n) | c1, C{sa * p11.re + sb * p00.re, sa * p11.im + sb * p00.im});
    const C p01 = dm_get(dm, (r0 << n) | c1), p10 = dm_get(dm, (r1 << n) | c0);
    dm_set(next, (r0 << n) | c1, C{cf * p01.re, cf * p01.im});
    dm_set(next, (r1 << n) | c0, C{cf * p10.re, cf * p10.im});
  }
  return next;
}

// PAULI15 (:226-231): {flip_a, flip_b, z_a, z_b} of the 15 non-identity 2-qubit Paulis
static const int PAULI15[15][4] = {{0, 1, 0, 0}, {0, 1, 0, 1}, {0, 0, 0, 1}, {1, 0, 0, 0}, {1, 1, 0, 0},
                                   {1, 1, 0, 1}, {1, 0, 0, 1}, {1, 0, 1, 0}, {1, 1, 1, 0}, {1, 1, 1, 1},
                                   {1, 0, 1, 1}, {0, 0, 1, 0}, {0, 1, 1, 0}, {0, 1, 1, 1}, {0, 0, 1, 1}};

// depolarize2 (:239-264)
static DMap dm_dep2(const DMap& dm, int n, int a, int b, double p) {
  if (p <= 0) return dm;
  DMap next;
  const uint64_t dim_mask = (uint64_t(1) << n) - 1, ma = uint64_t(1) << a, mb = uint64_t(1) << b;
  const double w1 = 1 - p, w2 = p / 15;
  for (const auto& kv : dm) {
    const uint64_t r = kv.first >> n, c = kv.first & dim_mask;
    const C v = kv.second;
    dm_acc(next, (r << n) | c, C{w1 * v.re, w1 * v.im});
    const int bar = (int)((r >> a) & 1), bbr = (int)((r >> b) & 1), bac = (int)((c >> a) & 1), bbc = (int)((c >> b) & 1);
    for (const auto& P : PAULI15) {
      const uint64_t perm = (P[0] ? ma : 0) | (P[1] ? mb : 0);
      const int parity = (P[2] * (bar ^ bac)) ^ (P[3] * (bbr ^ bbc));
      const double s = parity ? -w2 : w2;
      dm_acc(next, ((r ^ perm) << n) | (c ^ perm), C{s * v.re, s * v.im});
    }
  }
  return next;
}

// runDM's csrswap (:532-575): blocks by the control bit of row and column
static DMap dm_csrswap(const DMap& dm, int n, int ctl, int a, int b) {
  const uint64_t cm = uint64_t(1) << ctl, dim_mask = (uint64_t(1) << n) - 1;
  const Mat S = {ONE, ZERO, ZERO, ZERO, ZERO, cx(sq2, 0), cx(0, sq2), ZERO,
                 ZERO, cx(0, sq2), cx(sq2, 0), ZERO, ZERO, ZERO, ZERO, ONE};
  DMap blk[4];
  for (const auto& kv : dm) {
    const uint64_t r = kv.first >> n, c = kv.first & dim_mask;
    blk[((r & cm) ? 2 : 0) | ((c & cm) ? 1 : 0)][kv.first] = kv.second;
  }
  const std::vector<int> ab = {a, b};
  DMap d11 = dm_unitary(blk[3], n, ab, S);
  DMap t01;
  for (const auto& kv : blk[1]) t01[((kv.first & dim_mask) << n) | (kv.first >> n)] = kv.second;
  DMap t01a = dm_unitary(t01, n, ab, S), d01;
  for (const auto& kv : t01a) d01[((kv.first & dim_mask) << n) | (kv.first >> n)] = kv.second;
  DMap d10 = dm_unitary(blk[2], n, ab, S);
  DMap out = blk[0];
  for (const DMap* m : {&d01, &d10, &d11})
    for (const auto& kv : *m) dm_acc(out, kv.first, kv.second);
  return out;
}

// controlledGate (mps.ts:53-60): diag(I, G), control = first (most significant) qubit
static Mat controlled_gate(const Mat& g) {
  return {ONE, ZERO, ZERO, ZERO, ZERO, ONE, ZERO, ZERO, ZERO, ZERO, g[0], g[1], ZERO, ZERO, g[2], g[3]};
}

// runDM (:475-588)
static DMap run_dm(const Circuit& c, double p1, double p2) {
  const int n = c.n;
  DMap dm;
  dm[0] = ONE;
  for (const Op& op : c.ops) {
    const std::vector<int>& q = op.q;
    switch (op.kind) {
      case K_SINGLE:
        dm = dm_single(dm, n, q[0], op.m);
        if (p1) dm = dm_dep1(dm, n, q[0], p1);
        break;
      case K_CNOT: {
        const uint64_t cm = uint64_t(1) << q[0], tm = uint64_t(1) << q[1];
        dm = dm_perm(dm, n, [=](uint64_t i) { return (i & cm) ? i ^ tm : i; });
        if (p2) dm = dm_dep2(dm, n, q[0], q[1], p2);
        break;
      }
      case K_SWAP: {
        const uint64_t am = uint64_t(1) << q[0], bm = uint64_t(1) << q[1];
        dm = dm_perm(dm, n, [=](uint64_t i) { return (((i & am) != 0) == ((i & bm) != 0)) ? i : i ^ am ^ bm; });
        if (p2) dm = dm_dep2(dm, n, q[0], q[1], p2);
        break;
      }
      case K_TWO:
        dm = dm_unitary(dm, n, {q[0], q[1]}, op.m);
        if (p2) dm = dm_dep2(dm, n, q[0], q[1], p2);
        break;
      case K_CONTROLLED:
        dm = dm_unitary(dm, n, {q[0], q[1]}, controlled_gate(op.m));
        if (p2) dm = dm_dep2(dm, n, q[0], q[1], p2);
        break;
      case K_TOFFOLI: {
        const uint64_t c1 = uint64_t(1) << q[0], c2 = uint64_t(1) << q[1], tm = uint64_t(1) << q[2];
        dm = dm_perm(dm, n, [=](uint64_t i) { return ((i & c1) && (i & c2)) ? i ^ tm : i; });
        break;
      }
      case K_CSWAP: {
        const uint64_t cm = uint64_t(1) << q[0], am = uint64_t(1) << q[1], bm = uint64_t(1) << q[2];
        dm = dm_perm(dm, n, [=](uint64_t i) {
          if (!(i & cm)) return i;
          return (((i & am) != 0) == ((i & bm) != 0)) ? i : i ^ am ^ bm;
        });
        break;
      }
      case K_CSRSWAP: dm = dm_csrswap(dm, n, q[0], q[1], q[2]); break;
      case K_UNITARY: dm = dm_unitary(dm, n, q, op.m); break;
      default: break;  // barrier (measure / reset / if are refused by the caller)
    }
  }
  return dm;
}

// DensityMatrix.entropy's Jacobi eigenvalue solver (:382-440), restated
static std::vector<double> jacobi_eigenvalues(std::vector<double> R, std::vector<double> I, int n) {
  for (int sweep = 0; sweep < 30 * n; sweep++) {
    double max_off = 0;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double o = R[p * n + q] * R[p * n + q] + I[p * n + q] * I[p * n + q];
        if (o > max_off) max_off = o;
      }
    if (max_off < 1e-28) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double ore = R[p * n + q], oim = I[p * n + q], off2 = ore * ore + oim * oim;
        if (off2 < 1e-28) continue;
        const double phi = std::atan2(oim, ore), mag = std::sqrt(off2);
        const double tau = (R[q * n + q] - R[p * n + p]) / 2;
        const double t = mag / (std::fabs(tau) + std::sqrt(tau * tau + mag * mag)) * (tau < 0 ? -1 : 1);
        const double cg = 1 / std::sqrt(1 + t * t), sg = t * cg;
        const double sre = sg * std::cos(phi), sim = sg * std::sin(phi);
        for (int k = 0; k < n; k++) {
          const double xr = R[p * n + k], xi = I[p * n + k], yr = R[q * n + k], yi = I[q * n + k];
          R[p * n + k] = cg * xr + sre * yr - sim * yi;
          I[p * n + k] = cg * xi + sre * yi + sim * yr;
          R[q * n + k] = -sre * xr + sim * xi + cg * yr;
          I[q * n + k] = -sre * xi - sim * xr + cg * yi;
        }
        for (int k = 0; k < n; k++) {
          const double xr = R[k * n + p], xi = I[k * n + p], yr = R[k * n + q], yi = I[k * n + q];
          R[k * n + p] = cg * xr + sre * yr + sim * yi;
          I[k * n + p] = cg * xi + sre * yi - sim * yr;
          R[k * n + q] = -sre * xr + sim * xi + cg * yr;
          I[k * n + q] = -sre * xi - sim * xr + cg * yi;
        }
      }
  }
  std::vector<double> ev(n);
  for (int i = 0; i < n; i++) ev[i] = R[i * n + i];
  return ev;
}

// ---------------------------------------------------------------- algorithms.ts
static Circuit qft(int n) {                       // algorithms.ts:16-26
  Circuit c{n, {}};
  for (int j = n - 1; j >= 0; j--) {
    circuit_add(c, "h", {j}, {});
    for (int k = j - 1; k >= 0; k--) circuit_add(c, "cu1", {k, j}, {M_PI / std::pow(2.0, j - k)});
  }
  for (int i = 0; i < n / 2; i++) circuit_add(c, "swap", {i, n - 1 - i}, {});
  return c;
}
static Circuit iqft(int n) {                      // algorithms.ts:31-38
  Circuit c{n, {}};
  for (int i = 0; i < n / 2; i++) circuit_add(c, "swap", {i, n - 1 - i}, {});
  for (int j = 0; j < n; j++) {
    for (int k = j - 1; k >= 0; k--) circuit_add(c, "cu1", {k, j}, {-M_PI / std::pow(2.0, j - k)});
    circuit_add(c, "h", {j}, {});
  }
  return c;
}

struct Term { double coeff; std::string ops; };   // PauliTerm, ops[0] acts on qubit n-1

// Circuit.expectation-style parity sum over exactProbs, with the PauliTerm
// convention of vqe (algorithms.ts:301-336).
static double vqe(const Circuit& ansatz, const std::vector<Term>& H, uint64_t init, int mode) {
  int n = ansatz.n;
  double energy = 0;
  for (const Term& t : H) {
    if ((int)t.ops.size() != n) { g_err = "ops length"; throw std::runtime_error(g_err); }
    if (std::fabs(t.coeff) < 1e-15) continue;
    std::string up = t.ops;
    for (char& ch : up) ch = (char)std::toupper(ch);
    if (up.find_first_of("XYZ") == std::string::npos) { energy += t.coeff; continue; }
    Circuit rot = ansatz;
    for (int q = 0; q < n; q++) {
      char p = up[n - 1 - q];
      if (p == 'X') circuit_add(rot, "h", {q}, {});
      else if (p == 'Y') circuit_add(rot, "rx", {q}, {M_PI / 2});
    }
    State* s = simulate(rot, init, mode);
    std::vector<std::pair<uint64_t, double>> pr;
    probs_sorted(s, pr);
    delete s;
    double exp = 0;
    for (auto& kv : pr) {
      int parity = 0;
      for (int q = 0; q < n; q++) {
        char p = up[n - 1 - q];
        if (p != 'I' && ((kv.first >> q) & 1)) parity ^= 1;
      }
      exp += (parity == 0 ? 1 : -1) * kv.second;
    }
    energy += t.coeff * exp;
  }
  return energy;
}

// Ansatz families (algorithms.ts:366-399 and the layered Ry/Rz + CNOT-ladder
// ansatz of the 24-qubit VQE workload)
enum { ANS_REAL_AMPLITUDES = 0, ANS_EFFICIENT_SU2 = 1, ANS_HEA_LADDER = 2 };

static int ansatz_params(int kind, int n, int reps) {
  if (kind == ANS_REAL_AMPLITUDES) return n * (reps + 1);
  if (kind == ANS_EFFICIENT_SU2) return 2 * n * (reps + 1);
  return 2 * n * reps;  // HEA_LADDER: reps layers of (ry,rz per qubit, cnot ladder)
}

static Circuit build_ansatz(int kind, int n, int reps, const double* p) {
  Circuit c{n, {}};
  int k = 0;
  if (kind == ANS_REAL_AMPLITUDES) {
    for (int r = 0; r < reps; r++) {
      for (int q = 0; q < n; q++) circuit_add(c, "ry", {q}, {p[k++]});
      for (int q = 0; q < n - 1; q++) circuit_add(c, "cnot", {q, q + 1}, {});
    }
    for (int q = 0; q < n; q++) circuit_add(c, "ry", {q}, {p[k++]});
  } else if (kind == ANS_EFFICIENT_SU2) {
    for (int r = 0; r < reps; r++) {
      for (int q = 0; q < n; q++) { circuit_add(c, "ry", {q}, {p[k++]}); circuit_add(c, "rz", {q}, {p[k++]}); }
      for (int q = 0; q < n - 1; q++) circuit_add(c, "cnot", {q, q + 1}, {});
    }
    for (int q = 0; q < n; q++) { circuit_add(c, "ry", {q}, {p[k++]}); circuit_add(c, "rz", {q}, {p[k++]}); }
  } else {
    for (int r = 0; r < reps; r++) {
      for (int q = 0; q < n; q++) { circuit_add(c, "ry", {q}, {p[k++]}); circuit_add(c, "rz", {q}, {p[k++]}); }
      for (int q = 0; q < n - 1; q++) circuit_add(c, "cnot", {q, q + 1}, {});
    }
  }
  return c;
}

// ---------------------------------------------------------------- workload generators
// Seeded brickwork layer stream: per layer, per qubit g = floor(rng*5) picks
// {H, T, Rx, Ry, Rz}; rotations then draw theta = rng*2pi; then CNOT(q,q+1)
// for q even on even layers, odd on odd layers.
static void brickwork(Circuit& c, int layers, Prng& rng) {
  int n = c.n;
  for (int l = 0; l < layers; l++) {
    for (int q = 0; q < n; q++) {
      int g = (int)std::floor(rng.next() * 5);
      if (g == 0) circuit_add(c, "h", {q}, {});
      else if (g == 1) circuit_add(c, "t", {q}, {});
      else {
        double th = rng.next() * 2 * M_PI;
        circuit_add(c, g == 2 ? "rx" : g == 3 ? "ry" : "rz", {q}, {th});
      }
    }
    for (int q = (l & 1); q + 1 < n; q += 2) circuit_add(c, "cnot", {q, q + 1}, {});
  }
}

// Random 3-regular graph by the pairing (configuration) model with rejection.
static std::vector<std::pair<int, int>> regular3(int n, Prng& rng) {
  for (;;) {
    std::vector<int> pts(3 * n);
    for (int i = 0; i < 3 * n; i++) pts[i] = i / 3;
    for (int i = 3 * n - 1; i >= 1; i--) {
      int j = (int)std::floor(rng.next() * (i + 1));
      std::swap(pts[i], pts[j]);
    }
    std::vector<std::pair<int, int>> e;
    bool ok = true;
    std::unordered_set<uint64_t> seen;
    for (int k = 0; k < 3 * n / 2 && ok; k++) {
      int u = pts[2 * k], v = pts[2 * k + 1];
      if (u == v) { ok = false; break; }
      if (u > v) std::swap(u, v);
      uint64_t key = (uint64_t)u * 4096 + v;
      if (!seen.insert(key).second) { ok = false; break; }
      e.emplace_back(u, v);
    }
    if (ok) return e;
  }
}

}  // namespace

// ============================================================================ C ABI
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_circuit_new(int n) { return new Circuit{n, {}}; }
void orc_circuit_free(void* c) { delete (Circuit*)c; }
void* orc_circuit_copy(void* c) { return new Circuit(*(Circuit*)c); }
int orc_circuit_nops(void* c) { return (int)((Circuit*)c)->ops.size(); }
int orc_circuit_qubits(void* c) { return ((Circuit*)c)->n; }

int orc_add(void* cp, const char* name, const int* qs, int nq, const double* params, int np) {
  Circuit& c = *(Circuit*)cp;
  Op op;
  int rc = make_op(name, qs, nq, params, np, op);
  if (rc) return rc;
  rc = check_op(c, op);
  if (rc) return rc;
  c.ops.push_back(std::move(op));
  return ORC_OK;
}

int orc_add_unitary(void* cp, const int* qs, int nq, const double* mat_re_im) {
  Circuit& c = *(Circuit*)cp;
  Op op;
  op.kind = K_UNITARY;
  op.q.assign(qs, qs + nq);
  size_t d = size_t(1) << nq;
  op.m.resize(d * d);
  for (size_t i = 0; i < d * d; i++) op.m[i] = C{mat_re_im[2 * i], mat_re_im[2 * i + 1]};
  int rc = check_op(c, op);
  if (rc) return rc;
  c.ops.push_back(std::move(op));
  return ORC_OK;
}

// Op i's kind, qubits and matrix (gate-matrix restatement check)
int orc_op_info(void* cp, int i, int* kind, int* qs, int* nq, double* mat, int mat_cap) {
  const Op& op = ((Circuit*)cp)->ops[i];
  *kind = op.kind;
  *nq = (int)op.q.size();
  for (size_t j = 0; j < op.q.size(); j++) qs[j] = op.q[j];
  int m = (int)op.m.size();
  for (int j = 0; j < m && j < mat_cap; j++) { mat[2 * j] = op.m[j].re; mat[2 * j + 1] = op.m[j].im; }
  return m;
}

// Classical ops (circuit.ts:1598-1642).  measure takes any q, as the
// reference's builder does not check it (an out-of-range qubit reads 0).
int orc_add_measure(void* cp, int q, int cbit) {
  Op op;
  op.kind = K_MEASURE;
  op.q = {q};
  op.cbit = cbit;
  ((Circuit*)cp)->ops.push_back(std::move(op));
  return ORC_OK;
}
int orc_add_reset(void* cp, int q) {
  Circuit& c = *(Circuit*)cp;
  if (q < 0 || q >= c.n) {
    g_err = "qubit index " + std::to_string(q) + " is out of range for a " + std::to_string(c.n) + "-qubit circuit";
    return ORC_RANGE;
  }
  Op op;
  op.kind = K_RESET;
  op.q = {q};
  c.ops.push_back(std::move(op));
  return ORC_OK;
}
// if: the ops of `body` (a circuit) run when bits [reg0, reg0 + regn) read as
// a little-endian integer equal value
int orc_add_if(void* cp, int reg0, int regn, int value, void* body) {
  Op op;
  op.kind = K_IF;
  op.reg0 = reg0;
  op.regn = regn;
  op.value = value;
  op.body = ((Circuit*)body)->ops;
  ((Circuit*)cp)->ops.push_back(std::move(op));
  return ORC_OK;
}
// run() per-shot path; returns the xorshift32 state after the last draw
uint32_t orc_run_pershot(void* cp, uint64_t init, int shots, uint32_t seed, double p1, double p2, double pm,
                         int ncbits, uint64_t* out_idx, uint8_t* out_bits) {
  return run_pershot(*(Circuit*)cp, init, shots, seed, Noise{p1, p2, pm}, ncbits, out_idx, out_bits);
}

// runDM and the DensityMatrix read-outs (density.ts:274-372, :475-588)
void* orc_dm_run(void* cp, double p1, double p2) { return new DMap(run_dm(*(Circuit*)cp, p1, p2)); }
void orc_dm_free(void* h) { delete (DMap*)h; }
uint64_t orc_dm_nnz(void* h) { return ((DMap*)h)->size(); }
// rho as a dense 2^n x 2^n row-major complex matrix
void orc_dm_dense(void* h, int n, double* out) {
  const uint64_t dim = uint64_t(1) << n;
  std::memset(out, 0, sizeof(double) * 2 * dim * dim);
  for (const auto& kv : *(DMap*)h) {
    out[2 * kv.first] = kv.second.re;
    out[2 * kv.first + 1] = kv.second.im;
  }
}
double orc_dm_purity(void* h) {  // purity (:314-318)
  double p = 0;
  for (const auto& kv : *(DMap*)h) p += kv.second.re * kv.second.re + kv.second.im * kv.second.im;
  return p;
}
double orc_dm_entropy(void* h, int n) {  // entropy (:328-346)
  const int dim = 1 << n;
  std::vector<double> re((size_t)dim * dim), im((size_t)dim * dim);
  for (const auto& kv : *(DMap*)h) {
    re[kv.first] = kv.second.re;
    im[kv.first] = kv.second.im;
  }
  double s = 0;
  for (double lam : jacobi_eigenvalues(re, im, dim))
    if (lam > 1e-14) s -= lam * std::log2(lam);
  return s;
}
void orc_dm_bloch(void* h, int n, int q, double* out) {  // blochAngles (:356-372)
  const uint64_t qm = uint64_t(1) << q, dim_mask = (uint64_t(1) << n) - 1;
  double r00 = 0, r11 = 0, re = 0, im = 0;
  for (const auto& kv : *(DMap*)h) {
    const uint64_t r = kv.first >> n, c = kv.first & dim_mask;
    if (r == c) {
      if (!(r & qm)) r00 += kv.second.re;
      else r11 += kv.second.re;
    } else if (!(r & qm) && c == (r | qm)) {
      re += kv.second.re;
      im += kv.second.im;
    }
  }
  const double rz = r00 - r11, rx = 2 * re, ry = -2 * im;
  out[0] = std::acos(std::max(-1.0, std::min(1.0, rz)));
  out[1] = std::atan2(ry, rx);
}

void orc_circuit_matrix(void* cp, double* out) { circuit_matrix(*(Circuit*)cp, out); }
void orc_bloch(void* sp, int q, double* out) { bloch((State*)sp, q, out); }

void* orc_simulate(void* cp, uint64_t init, int mode) { return simulate(*(Circuit*)cp, init, mode); }
void orc_state_free(void* s) { delete (State*)s; }

uint64_t orc_state_nnz(void* sp) {
  State* s = (State*)sp;
  if (s->mode == 0) return s->sv.size();
  uint64_t k = 0;
  for (auto& a : s->d.a) if (a.re != 0 || a.im != 0) k++;
  return k;
}

void orc_state_get(void* sp, uint64_t idx, double* re_im) {
  C a = state_get((State*)sp, idx);
  re_im[0] = a.re; re_im[1] = a.im;
}

void orc_state_dense(void* sp, double* out) {
  State* s = (State*)sp;
  uint64_t N = uint64_t(1) << s->n;
  if (s->mode == 0) {
    std::memset(out, 0, sizeof(double) * 2 * N);
    for (auto& kv : s->sv) { out[2 * kv.first] = kv.second.re; out[2 * kv.first + 1] = kv.second.im; }
  } else {
    std::memcpy(out, s->d.a.data(), sizeof(double) * 2 * N);
  }
}

void orc_state_prune_stats(void* sp, uint64_t* events, double* max_abs) {
  State* s = (State*)sp;
  *events = s->ps.events;
  *max_abs = s->ps.max_abs;
}

// exactProbs(): entries with p > 1e-14 sorted by index; returns the count
uint64_t orc_exact_probs(void* sp, uint64_t* idx, double* p, uint64_t cap) {
  std::vector<std::pair<uint64_t, double>> pr;
  probs_sorted((State*)sp, pr);
  for (uint64_t i = 0; i < pr.size() && i < cap; i++) { idx[i] = pr[i].first; p[i] = pr[i].second; }
  return pr.size();
}

void orc_run(void* sp, int shots, uint32_t seed, uint64_t* out_idx) { run_shots((State*)sp, shots, seed, out_idx); }

// marginals() (circuit.ts:1508-1518)
void orc_marginals(void* sp, double* out) {
  State* s = (State*)sp;
  for (int q = 0; q < s->n; q++) out[q] = 0;
  auto accum = [&](uint64_t idx, C a) {
    double p = a.re * a.re + a.im * a.im;
    for (int q = 0; q < s->n; q++) if ((idx >> q) & 1) out[q] += p;
  };
  if (s->mode == 0) for (auto& kv : s->sv) accum(kv.first, kv.second);
  else for (uint64_t i = 0; i < s->d.a.size(); i++) accum(i, s->d.a[i]);
}

// Circuit.expectation(pauli) (circuit.ts:3728-3753): pauli[q] acts on qubit q
double orc_expectation(void* cp, const char* pauli, uint64_t init, int mode) {
  Circuit rot = *(Circuit*)cp;
  int n = rot.n;
  std::string P(pauli);
  for (char& ch : P) ch = (char)std::toupper(ch);
  if (P.find_first_of("XYZ") == std::string::npos) return 1.0;
  for (int q = 0; q < n; q++) {
    if (P[q] == 'X') circuit_add(rot, "h", {q}, {});
    else if (P[q] == 'Y') circuit_add(rot, "rx", {q}, {M_PI / 2});
  }
  State* s = simulate(rot, init, mode);
  std::vector<std::pair<uint64_t, double>> pr;
  probs_sorted(s, pr);
  delete s;
  double e = 0;
  for (auto& kv : pr) {
    int parity = 0;
    for (int q = 0; q < n; q++) if (P[q] != 'I' && ((kv.first >> q) & 1)) parity ^= 1;
    e += (parity == 0 ? 1 : -1) * kv.second;
  }
  return e;
}

static std::vector<Term> terms_from(int nterms, const double* coeffs, const char* ops, int n) {
  std::vector<Term> H(nterms);
  for (int t = 0; t < nterms; t++) { H[t].coeff = coeffs[t]; H[t].ops.assign(ops + (size_t)t * n, n); }
  return H;
}

double orc_vqe(void* cp, int nterms, const double* coeffs, const char* ops, int mode) {
  Circuit& c = *(Circuit*)cp;
  try { return vqe(c, terms_from(nterms, coeffs, ops, c.n), 0, mode); } catch (...) { return NAN; }
}

int orc_ansatz_params(int kind, int n, int reps) { return ansatz_params(kind, n, reps); }
void* orc_ansatz(int kind, int n, int reps, const double* params) {
  return new Circuit(build_ansatz(kind, n, reps, params));
}

// gradient() by parameter shift (algorithms.ts:536-547)
void orc_gradient(int kind, int n, int reps, const double* params, int nterms, const double* coeffs,
                  const char* ops, int mode, double* grad) {
  int P = ansatz_params(kind, n, reps);
  std::vector<Term> H = terms_from(nterms, coeffs, ops, n);
  std::vector<double> pp(params, params + P);
  const double shift = M_PI / 2;
  for (int i = 0; i < P; i++) {
    std::vector<double> plus = pp, minus = pp;
    plus[i] = pp[i] + shift;
    minus[i] = pp[i] - shift;
    double ep = vqe(build_ansatz(kind, n, reps, plus.data()), H, 0, mode);
    double em = vqe(build_ansatz(kind, n, reps, minus.data()), H, 0, mode);
    grad[i] = 0.5 * (ep - em);
  }
}

// minimize() (algorithms.ts:591-609); returns steps, writes params/energy/converged
int orc_minimize(int kind, int n, int reps, double* params, int nterms, const double* coeffs, const char* ops,
                 double lr, int steps, double tol, int mode, double* energy, int* converged) {
  int P = ansatz_params(kind, n, reps);
  std::vector<Term> H = terms_from(nterms, coeffs, ops, n);
  std::vector<double> g(P);
  for (int step = 0; step < steps; step++) {
    orc_gradient(kind, n, reps, params, nterms, coeffs, ops, mode, g.data());
    double s = 0;
    for (double v : g) s += v * v;
    if (std::sqrt(s) < tol) {
      *energy = vqe(build_ansatz(kind, n, reps, params), H, 0, mode);
      *converged = 1;
      return step;
    }
    for (int i = 0; i < P; i++) params[i] = params[i] - lr * g[i];
  }
  *energy = vqe(build_ansatz(kind, n, reps, params), H, 0, mode);
  *converged = 0;
  return steps;
}

void* orc_qft(int n) { return new Circuit(qft(n)); }
void* orc_iqft(int n) { return new Circuit(iqft(n)); }

// qaoa() (algorithms.ts:260-276)
void* orc_qaoa(int n, const int* edges, int ne, const double* gamma, const double* beta, int p) {
  Circuit* c = new Circuit{n, {}};
  for (int q = 0; q < n; q++) circuit_add(*c, "h", {q}, {});
  for (int l = 0; l < p; l++) {
    for (int e = 0; e < ne; e++) {
      int u = edges[2 * e], v = edges[2 * e + 1];
      circuit_add(*c, "cnot", {u, v}, {});
      circuit_add(*c, "rz", {v}, {-gamma[l]});
      circuit_add(*c, "cnot", {u, v}, {});
    }
    for (int q = 0; q < n; q++) circuit_add(*c, "rx", {q}, {2 * beta[l]});
  }
  return c;
}

// maxCutHamiltonian() (algorithms.ts:231-241) into caller buffers; returns term count
int orc_maxcut_hamiltonian(int n, const int* edges, int ne, double* coeffs, char* ops) {
  if (ne == 0) return 0;
  coeffs[0] = ne / 2.0;
  for (int q = 0; q < n; q++) ops[q] = 'I';
  for (int e = 0; e < ne; e++) {
    char* o = ops + (size_t)(e + 1) * n;
    for (int q = 0; q < n; q++) o[q] = 'I';
    o[n - 1 - edges[2 * e]] = 'Z';
    o[n - 1 - edges[2 * e + 1]] = 'Z';
    coeffs[e + 1] = -0.5;
  }
  return ne + 1;
}

// Workload: seeded brickwork circuit (optionally followed by qft(n)); the
// generator's stream state after the circuit is returned in *state_out.
void* orc_brickwork(int n, int layers, uint32_t seed, int with_qft, uint32_t* state_out) {
  Prng rng(seed);
  Circuit* c = new Circuit{n, {}};
  brickwork(*c, layers, rng);
  if (with_qft) {
    Circuit q = qft(n);
    for (auto& op : q.ops) c->ops.push_back(op);
  }
  if (state_out) *state_out = rng.s;
  return c;
}

// Workload: one random 3-regular graph drawn from a xorshift32 stream state.
// Returns edge count; the advanced state in *state.
int orc_regular3(int n, uint32_t* state, int* edges) {
  Prng rng(*state);
  auto e = regular3(n, rng);
  for (size_t i = 0; i < e.size(); i++) { edges[2 * i] = e[i].first; edges[2 * i + 1] = e[i].second; }
  *state = rng.s;
  return (int)e.size();
}

// CPU-baseline timing: simulate ops [0, first) untimed, then time ops
// [first, first+count) in the given mode (sparse = the reference's algorithm).
// Returns the amplitude updates done in the timed range (sum over timed ops of
// the entries the op visits: the map size for the sparse path, 2^n dense).
uint64_t orc_time_ops(void* cp, uint64_t init, int mode, int first, int count, double* seconds) {
  const Circuit& c = *(Circuit*)cp;
  Circuit pre{c.n, {}}, timed{c.n, {}};
  for (int i = 0; i < (int)c.ops.size(); i++) {
    if (i < first) pre.ops.push_back(c.ops[i]);
    else if (i < first + count) timed.ops.push_back(c.ops[i]);
  }
  State* s = simulate(pre, init, mode);
  uint64_t updates = 0;
  auto t0 = std::chrono::steady_clock::now();
  if (mode == 0) {
    for (const Op& op : timed.ops) {
      updates += s->sv.size();
      switch (op.kind) {
        case K_SINGLE: s->sv = applySingle(s->sv, op.q[0], op.m, s->ps); break;
        case K_CNOT: s->sv = applyCNOT(s->sv, op.q[0], op.q[1]); break;
        case K_CONTROLLED: s->sv = applyControlled(s->sv, op.q[0], op.q[1], op.m, s->ps); break;
        case K_SWAP: s->sv = applySWAP(s->sv, op.q[0], op.q[1]); break;
        case K_TOFFOLI: s->sv = applyToffoli(s->sv, op.q[0], op.q[1], op.q[2]); break;
        case K_CSWAP: s->sv = applyCSwap(s->sv, op.q[0], op.q[1], op.q[2]); break;
        case K_CSRSWAP: s->sv = applyCsrSwap(s->sv, op.q[0], op.q[1], op.q[2], s->ps); break;
        case K_TWO: s->sv = applyTwo(s->sv, op.q[0], op.q[1], op.m, s->ps); break;
        case K_UNITARY: s->sv = applyUnitary(s->sv, op.q, op.m, s->ps); break;
        case K_BARRIER: case K_MEASURE: case K_RESET: case K_IF: break;
      }
    }
  } else {
    for (const Op& op : timed.ops) {
      updates += s->d.a.size();
      dense_apply(s->d, op);
    }
  }
  *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  delete s;
  return updates;
}

uint32_t orc_prng_next(uint32_t* state) { Prng r(*state); uint32_t v = r.next_u32(); *state = r.s; return v; }

}  // extern "C"
