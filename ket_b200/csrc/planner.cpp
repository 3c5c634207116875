// planner.cpp -- op validation, lowering and the greedy fusion planner.
//
// lower_ops() turns the reference's FlatOp list (circuit.ts:20-47, carried
// as ket_op) into internal gates: control qubits become a mask, diagonal and
// X-type matrices are recognised (they then need no amplitude pairing), and
// identity gates and barriers are dropped.  Validation mirrors #checkOp
// (circuit.ts:1113-1146): RangeError for an out-of-range qubit, TypeError for
// control == target or a malformed unitary.
//
// plan_passes() groups gates into tile passes.  A pass streams the state
// through tiles of 2^m amplitudes: the tile holds the L lowest qubits
// (contiguous in memory, so loads coalesce) plus m-L chosen high qubits.  A
// gate joins the pass when every qubit it mixes lies in the tile; control
// qubits and diagonal gates may sit anywhere, since their bit values are
// known from each amplitude's global index.  Gate order is preserved: a gate
// deferred to a later pass blocks every later gate that shares a qubit.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "engine.h"

namespace ket {

namespace {

inline bool is0(cd a) { return a.re == 0.0 && a.im == 0.0; }
inline bool is1(cd a) { return a.re == 1.0 && a.im == 0.0; }

int range_err(std::string& err, int q, int n) {
  err = "qubit index " + std::to_string(q) + " is out of range for a " + std::to_string(n) + "-qubit circuit";
  return KET_ERR_RANGE;
}

uint64_t bit(int q) { return uint64_t(1) << q; }

thread_local int g_anc = -1;  // ancilla of the plan being built (adjoint sweep)

// Qubits a gate touches (targets and controls).
uint64_t gate_qubits(const Gate& g) {
  uint64_t m = g.cmask;
  if (is_grad(g) && g_anc >= 0) m |= bit(g_anc);
  if (g.t0 >= 0) m |= bit(g.t0);
  if (g.t1 >= 0) m |= bit(g.t1);
  for (int q : g.tk) m |= bit(q);
  return m;
}

// Qubits whose amplitudes a gate mixes (must lie in the tile).
uint64_t gate_mix(const Gate& g) {
  if (is_grad(g)) {
    uint64_t m = bit(g_anc);
    if (g.type != G_GRADD) m |= bit(g.t0);
    if (g.type == G_GRADM2) m |= bit(g.t1);
    return m;
  }
  switch (g.type) {
    case G_DIAG1: case G_DIAG2: return 0;
    case G_MAT1: case G_X1: return bit(g.t0);
    case G_SWAP: case G_MAT2: return bit(g.t0) | bit(g.t1);
    case G_MATK: { uint64_t m = 0; for (int q : g.tk) m |= bit(q); return m; }
  }
  return 0;
}

// A 4x4 with every off-diagonal entry zero becomes a diagonal phase gate.
void lower_diag2(Gate& g) {
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++)
      if (r != c && !is0(g.m[r * 4 + c])) return;
  cd d[4] = {g.m[0], g.m[5], g.m[10], g.m[15]};
  g.type = G_DIAG2;
  for (int k = 0; k < 4; k++) g.m[k] = d[k];
}

bool fusable(const Gate& g) { return g.type != G_MATK || g.tk.size() <= 2; }

// Gates that can change amplitude magnitudes.  With the reference's per-gate
// pruning (accumulate(), statevector.ts:19-27) their relative order must be
// kept: pruning after G1 then G2 differs from pruning after G2 then G1.
// Diagonal phases and permutations preserve magnitudes, so they may move past
// mixing gates on other qubits without changing what gets pruned.
bool is_mixing(const Gate& g) { return g.type == G_MAT1 || g.type == G_MAT2 || g.type == G_MATK; }

}  // namespace

int lower_ops(int n, const ket_op* ops, size_t nops, const double* mats, size_t nmat, bool prune,
              std::vector<Gate>& out, std::string& err) {
  out.clear();
  out.reserve(nops);
  auto getm = [&](const ket_op& op, int k, cd* dst, std::vector<cd>* vdst) -> int {
    size_t cnt = size_t(1) << (2 * k);
    if (op.mat < 0 || (size_t)op.mat + cnt > nmat || mats == nullptr) {
      err = "matrix offset out of bounds for op";
      return KET_ERR_TYPE;
    }
    for (size_t i = 0; i < cnt; i++) {
      cd v{mats[2 * (op.mat + i)], mats[2 * (op.mat + i) + 1]};
      if (dst) dst[i] = v;
      if (vdst) vdst->push_back(v);
    }
    return KET_OK;
  };
  for (size_t i = 0; i < nops; i++) {
    const ket_op& op = ops[i];
    int need = -1;
    switch (op.kind) {
      case KET_OP_SINGLE: need = 1; break;
      case KET_OP_CNOT: case KET_OP_SWAP: case KET_OP_TWO: case KET_OP_CONTROLLED: need = 2; break;
      case KET_OP_TOFFOLI: case KET_OP_CSWAP: case KET_OP_CSRSWAP: need = 3; break;
      case KET_OP_UNITARY: case KET_OP_BARRIER: break;
      default: err = "unknown op kind " + std::to_string(op.kind); return KET_ERR_TYPE;
    }
    if (need >= 0 && op.nq != need) {
      err = "op " + std::to_string(i) + ": expected " + std::to_string(need) + " qubits";
      return KET_ERR_TYPE;
    }
    if (op.nq < 0 || op.nq > KET_MAX_OP_QUBITS) { err = "op qubit count out of bounds"; return KET_ERR_TYPE; }
    if (op.kind == KET_OP_UNITARY && op.nq == 0) { err = "unitary: qubits must be non-empty"; return KET_ERR_TYPE; }
    for (int j = 0; j < op.nq; j++)
      if (op.q[j] < 0 || op.q[j] >= n) return range_err(err, op.q[j], n);
    const int* q = op.q;
    Gate g;
    g.src_op = (int)i;
    switch (op.kind) {
      case KET_OP_BARRIER: continue;
      case KET_OP_CNOT:
        if (q[0] == q[1]) { err = "control and target qubits must differ (got " + std::to_string(q[0]) + ")"; return KET_ERR_TYPE; }
        g.type = G_X1; g.t0 = q[1]; g.cmask = bit(q[0]);
        break;
      case KET_OP_TOFFOLI:
        if (q[2] == q[0] || q[2] == q[1]) { err = "toffoli: target repeats a control qubit"; return KET_ERR_TYPE; }
        g.type = G_X1; g.t0 = q[2]; g.cmask = bit(q[0]) | bit(q[1]);
        break;
      case KET_OP_SWAP:
        if (q[0] == q[1]) continue;  // applySWAP with a == b is the identity
        g.type = G_SWAP; g.t0 = q[0]; g.t1 = q[1];
        break;
      case KET_OP_CSWAP:
        if (q[1] == q[2]) continue;
        if (q[0] == q[1] || q[0] == q[2]) { err = "cswap: control repeats a target qubit"; return KET_ERR_TYPE; }
        g.type = G_SWAP; g.t0 = q[1]; g.t1 = q[2]; g.cmask = bit(q[0]);
        break;
      case KET_OP_CSRSWAP: {
        if (q[1] == q[2] || q[0] == q[1] || q[0] == q[2]) { err = "csrswap: qubits must be distinct"; return KET_ERR_TYPE; }
        const double s = 1.0 / std::sqrt(2.0);
        g.type = G_MAT2; g.t0 = q[1]; g.t1 = q[2]; g.cmask = bit(q[0]); g.prune = prune;
        for (int k = 0; k < 16; k++) g.m[k] = cd{0, 0};
        g.m[0] = cd{1, 0}; g.m[5] = cd{s, 0}; g.m[6] = cd{0, s}; g.m[9] = cd{0, s}; g.m[10] = cd{s, 0}; g.m[15] = cd{1, 0};
        break;
      }
      case KET_OP_SINGLE: case KET_OP_CONTROLLED: {
        int t = op.kind == KET_OP_SINGLE ? q[0] : q[1];
        if (op.kind == KET_OP_CONTROLLED) {
          if (q[0] == q[1]) { err = "control and target qubits must differ (got " + std::to_string(q[0]) + ")"; return KET_ERR_TYPE; }
          g.cmask = bit(q[0]);
        }
        cd m[4];
        int rc = getm(op, 1, m, nullptr);
        if (rc) return rc;
        g.t0 = t;
        g.prune = prune;
        if (is0(m[1]) && is0(m[2])) {
          if (is1(m[0]) && is1(m[3])) continue;  // identity: outputs equal inputs bit for bit
          g.type = G_DIAG1; g.m[0] = m[0]; g.m[1] = m[3];
        } else if (is0(m[0]) && is0(m[3]) && is1(m[1]) && is1(m[2])) {
          g.type = G_X1; g.prune = false;  // 0*x0 + 1*x1 == x1 exactly: a permutation
        } else {
          g.type = G_MAT1;
          for (int k = 0; k < 4; k++) g.m[k] = m[k];
        }
        break;
      }
      case KET_OP_TWO: {
        if (q[0] == q[1]) { err = "two-qubit gate on a repeated qubit"; return KET_ERR_TYPE; }
        int rc = getm(op, 2, g.m, nullptr);
        if (rc) return rc;
        g.type = G_MAT2; g.t0 = q[0]; g.t1 = q[1]; g.prune = prune;
        lower_diag2(g);
        break;
      }
      case KET_OP_UNITARY: {
        int k = op.nq;
        for (int a = 0; a < k; a++)
          for (int b = a + 1; b < k; b++)
            if (q[a] == q[b]) { err = "unitary: repeated qubit"; return KET_ERR_TYPE; }
        g.prune = prune;
        if (k == 1) {
          cd m[4];
          int rc = getm(op, 1, m, nullptr);
          if (rc) return rc;
          g.t0 = q[0];
          if (is0(m[1]) && is0(m[2])) {
            if (is1(m[0]) && is1(m[3])) continue;
            g.type = G_DIAG1; g.m[0] = m[0]; g.m[1] = m[3];
          } else {
            g.type = G_MAT1;
            for (int j = 0; j < 4; j++) g.m[j] = m[j];
          }
        } else if (k == 2) {
          int rc = getm(op, 2, g.m, nullptr);
          if (rc) return rc;
          g.type = G_MAT2; g.t0 = q[0]; g.t1 = q[1];
          lower_diag2(g);
        } else {
          int rc = getm(op, k, nullptr, &g.mk);
          if (rc) return rc;
          g.type = G_MATK;
          g.tk.assign(q, q + k);
        }
        break;
      }
    }
    out.push_back(std::move(g));
  }
  return KET_OK;
}

namespace {

void mat_of(const Gate& g, cd m[4]) {
  if (g.type == G_MAT1) {
    for (int k = 0; k < 4; k++) m[k] = g.m[k];
  } else if (g.type == G_DIAG1) {
    m[0] = g.m[0]; m[1] = cd{0, 0}; m[2] = cd{0, 0}; m[3] = g.m[1];
  } else {  // G_X1
    m[0] = cd{0, 0}; m[1] = cd{1, 0}; m[2] = cd{1, 0}; m[3] = cd{0, 0};
  }
}

cd cmulh(cd a, cd b) { return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
cd caddh(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }

// Classify a 2x2 as identity (returns false), diagonal, X or general.
bool set_single(Gate& g, const cd m[4], bool prune) {
  if (is0(m[1]) && is0(m[2])) {
    if (is1(m[0]) && is1(m[3])) return false;
    g.type = G_DIAG1; g.m[0] = m[0]; g.m[1] = m[3]; g.prune = prune;
  } else if (is0(m[0]) && is0(m[3]) && is1(m[1]) && is1(m[2])) {
    g.type = G_X1; g.prune = false;
  } else {
    g.type = G_MAT1; g.prune = prune;
    for (int k = 0; k < 4; k++) g.m[k] = m[k];
  }
  return true;
}

}  // namespace

// Folding of uncontrolled single-qubit gates.  A gate G on qubit q merges with
// the previous uncontrolled single-qubit gate P on q into the one gate G*P when
// the gate that has to move to the other's position commutes with everything
// on q in between: a diagonal commutes with gates that use q only as a control
// and with other diagonals on q; an X or a general 2x2 needs q untouched.
// With the reference's pruning two magnitude-changing gates never merge (the
// reference prunes between them); a diagonal or an X preserves magnitudes, so
// merging it is exact.  The merged gate takes the position of the gate that
// can change magnitudes, so the order of those gates is unchanged.
void fold_single_qubit(std::vector<Gate>& gs, bool prune) {
  const size_t ng = gs.size();
  std::vector<int> cand(64, -1);
  std::vector<char> tmix(64, 0), tany(64, 0), dead(ng, 0);
  for (size_t i = 0; i < ng; i++) {
    Gate& g = gs[i];
    const bool single = (g.type == G_MAT1 || g.type == G_DIAG1 || g.type == G_X1) && g.cmask == 0;
    if (!single) {
      uint64_t tgt = 0, all = g.cmask;
      switch (g.type) {
        case G_MAT1: case G_X1: tgt = bit(g.t0); break;
        case G_SWAP: case G_MAT2: tgt = bit(g.t0) | bit(g.t1); break;
        case G_MATK: for (int q : g.tk) tgt |= bit(q); break;
        case G_DIAG1: all |= bit(g.t0); break;
        case G_DIAG2: all |= bit(g.t0) | bit(g.t1); break;
        default: break;
      }
      all |= tgt;
      for (int q = 0; q < 64; q++) {
        if ((all >> q) & 1) tany[q] = 1;
        if ((tgt >> q) & 1) tmix[q] = 1;
      }
      continue;
    }
    const int q = g.t0, p = cand[q];
    if (p >= 0) {
      Gate& P = gs[p];
      const bool pd = P.type == G_DIAG1, gd = g.type == G_DIAG1;
      const bool pm = P.type == G_MAT1, gm = g.type == G_MAT1;
      bool ok = (pd || gd) ? !tmix[q] : !tany[q];
      if (prune && pm && gm) ok = false;
      if (ok) {
        cd a[4], b[4], m[4];
        mat_of(g, a);
        mat_of(P, b);
        for (int r = 0; r < 2; r++)
          for (int c = 0; c < 2; c++) m[2 * r + c] = caddh(cmulh(a[2 * r], b[c]), cmulh(a[2 * r + 1], b[2 + c]));
        // the merged gate goes where the magnitude-changing gate was; between
        // two magnitude-preserving gates, where the moving diagonal allows
        const size_t pos = pm ? (size_t)p : (gm ? i : (pd ? i : (size_t)p));
        const size_t other = pos == i ? (size_t)p : i;
        Gate merged = gs[pos];
        const bool keep = set_single(merged, m, prune);
        dead[other] = 1;
        if (!keep) {
          dead[pos] = 1;
          cand[q] = -1;
        } else {
          gs[pos] = merged;
          cand[q] = (int)pos;
          if (pos == i) { tmix[q] = 0; tany[q] = 0; }
        }
        continue;
      }
    }
    cand[q] = (int)i;
    tmix[q] = 0;
    tany[q] = 0;
  }
  size_t w = 0;
  for (size_t i = 0; i < ng; i++)
    if (!dead[i]) {
      if (w != i) gs[w] = std::move(gs[i]);
      w++;
    }
  gs.resize(w);
}

int tile_qubits(int precision, int fusion) {
  int mx = 12;
  if (fusion > 0) return std::max(6, std::min(fusion, mx));
  return mx;
}

void plan_passes(int n, int precision, int fusion, bool keep_mix_order, Plan& plan) {
  plan.passes.clear();
  g_anc = plan.anc;
  const std::vector<Gate>& G = plan.gates;
  const int M = std::min(n, tile_qubits(precision, fusion));
  // L low qubits are contiguous in every tile: 2^L amplitudes per HBM chunk
  // (one TMA bulk copy each, >= 32 bytes so both precisions stay 16-byte sized).
  static int Lenv = getenv("KET_TILE_LOW") ? atoi(getenv("KET_TILE_LOW")) : 5;
  const int L = std::min(n, std::max(2, std::min(5, Lenv)));
  const uint64_t low = (L >= 64) ? ~uint64_t(0) : bit(L) - 1;
  std::vector<int> pending(G.size());
  for (size_t i = 0; i < G.size(); i++) pending[i] = (int)i;
  // what the sweeps ask of each gate, once
  struct Use {
    uint64_t qs;   // qubits it touches
    uint64_t mix;  // qubits it mixes
    bool mixing;   // keeps its order among mixing gates
    bool fus;      // can join a tile pass
  };
  std::vector<Use> use(G.size());
  for (size_t i = 0; i < G.size(); i++)
    use[i] = {gate_qubits(G[i]), gate_mix(G[i]), keep_mix_order && is_mixing(G[i]), fusable(G[i])};

  auto single_pass = [&](int gi) {
    Pass p;
    p.fused = false;
    p.gates.push_back(gi);
    plan.passes.push_back(std::move(p));
  };

  if (fusion == 0) {
    for (int gi : pending) single_pass(gi);
    return;
  }

  // Score of a pass over tile set S: the gates it would absorb (the sweep
  // below, counted).  With the reference's pruning, mixing gates must keep
  // their order, so how far a pass gets along them decides how many passes
  // follow: mixing gates absorbed count first, then all gates.
  // Every gate touches a qubit, so once the skipped gates block all of them
  // (B == everything) no later gate can join.
  const uint64_t allq = n >= 64 ? ~uint64_t(0) : bit(n) - 1;
  auto absorbed = [&](uint64_t S, std::vector<uint64_t>* cand) -> int {
    uint64_t B = 0;
    bool mixblocked = false;
    int taken = 0, tmix = 0;
    for (int gi : pending) {
      if ((B & allq) == allq) break;
      const Use& u = use[gi];
      const uint64_t qs = u.qs;
      const bool mixing = u.mixing;
      bool blocked = (qs & B) || (mixing && mixblocked) || !u.fus;
      uint64_t miss = u.mix & ~S;
      if (blocked || miss) {
        if (!blocked && miss && cand && cand->size() < 16) {
          bool dup = false;
          for (uint64_t c : *cand) dup |= (c == miss);
          if (!dup) cand->push_back(miss);
        }
        B |= qs;
        if (mixing) mixblocked = true;
        continue;
      }
      taken++;
      if (mixing) tmix++;
    }
    return tmix * 65536 + taken;
  };

  while (!pending.empty()) {
    // Grow the tile's qubit set one step at a time, each time adding the
    // missing targets of whichever frontier gate lets the pass absorb most.
    uint64_t S = (M >= n) ? (n >= 64 ? ~uint64_t(0) : bit(n) - 1) : low;
    if (plan.anc >= 0) S |= bit(plan.anc);
    while (__builtin_popcountll(S) < M) {
      std::vector<uint64_t> cand;
      absorbed(S, &cand);
      int best = -1;
      uint64_t bestS = S;
      for (uint64_t c : cand) {
        if (__builtin_popcountll(S | c) > M) continue;
        int v = absorbed(S | c, nullptr);
        if (v > best) { best = v; bestS = S | c; }
      }
      if (best < 0) break;
      S = bestS;
    }
    // Sweep: take every gate applicable in tile S, preserving order.
    Pass p;
    p.fused = true;
    p.m = M;
    p.L = L;
    uint64_t B = 0;
    bool mixblocked = false;
    std::vector<int> rest;
    for (int gi : pending) {
      const Use& u = use[gi];
      const uint64_t qs = u.qs;
      const bool mixing = u.mixing;
      if ((qs & B) || (mixing && mixblocked) || !u.fus || (u.mix & ~S)) {
        B |= qs;
        if (mixing) mixblocked = true;
        rest.push_back(gi);
        continue;
      }
      p.gates.push_back(gi);
    }
    if (p.gates.empty()) {
      // Front gate cannot be fused (wide unitary): run it alone.
      single_pass(pending[0]);
      pending.erase(pending.begin());
      continue;
    }
    for (int q = 0; q < n; q++)
      if (((S >> q) & 1) && !((low >> q) & 1)) p.hbits.push_back(q);
    // Pad the tile to M qubits with unused high qubits (keeps tile count fixed).
    for (int q = n - 1; (int)p.hbits.size() + L < M && q >= L; q--)
      if (!((S >> q) & 1)) { p.hbits.push_back(q); S |= bit(q); }
    std::sort(p.hbits.begin(), p.hbits.end());
    plan.passes.push_back(std::move(p));
    pending.swap(rest);
  }
}

}  // namespace ket
