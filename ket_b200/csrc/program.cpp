// program.cpp -- lowers one fused pass to the register-tiled program run by
// k_fused2: a sequence of gate ops, each addressed by the role (register bit,
// lane bit, anywhere-diagonal) its target plays in the current tile layout,
// with a layout exchange inserted whenever the next gate's target sits on a
// warp bit (or a two-qubit gate needs both targets in registers).
//
// Layout choice looks ahead: the tile bits needed soonest become register
// and lane bits, the ones needed latest become warp bits.  The first and last
// layouts keep lane bit l on tile bit l (l < 5) so the global load and store
// of each warp touch contiguous 128-byte lines.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "launch.h"

namespace ket {

namespace {

const int NB = KET_T2_BITS;

struct Lay {
  int pos[NB];   // role -> tile bit: 0..4 lanes, then NW warps, then NR registers
  int role[NB];  // tile bit -> role
};

thread_local int g_nreg = 4;  // register bits of the program being lowered (4 or 5)
inline int NRg() { return g_nreg; }
inline int NWg() { return 7 - g_nreg; }
inline int REG0() { return 5 + NWg(); }  // role of register bit 0

void fill_roles(Lay& l) {
  for (int r = 0; r < NB; r++) l.role[l.pos[r]] = r;
}

bool a0_compatible(const Lay& l) {
  for (int i = 0; i < 5; i++)
    if (l.pos[i] != i) return false;
  return true;
}

bool is_reg(const Lay& l, int tb) { return l.role[tb] >= REG0(); }
bool is_lane(const Lay& l, int tb) { return l.role[tb] < 5; }

// Tile-local bit of a global qubit, -1 when outside the tile.
int tpos(const Pass& p, int q) {
  if (q < 0) return -1;
  if (q < p.L) return q;
  for (size_t j = 0; j < p.hbits.size(); j++)
    if (p.hbits[j] == q) return p.L + (int)j;
  return -1;
}

thread_local int g_anc_tb = -1;  // tile bit of the adjoint ancilla in the pass being lowered
thread_local bool g_relabel = false;  // uncontrolled swaps of two tile bits become relabellings (FO_RELAY)

// An uncontrolled swap of two qubits of the tile: a relabelling of the layout.
bool relabel_gate(const Gate& g, const Pass& p) {
  return g_relabel && g.type == G_SWAP && g.cmask == 0 && tpos(p, g.t0) >= 0 && tpos(p, g.t1) >= 0;
}

bool fits(const Gate& g, const Pass& p, const Lay& l) {
  switch (g.type) {
    case G_GRADM: return is_reg(l, tpos(p, g.t0)) && is_reg(l, g_anc_tb);
    case G_GRADD: return is_reg(l, g_anc_tb);
    case G_GRADM2: return true;
    case G_DIAG1: case G_DIAG2: case G_SWAP: case G_MAT2: return true;  // SWAP/MAT2 work in any layout
    case G_MAT1: case G_X1: {
      int t = tpos(p, g.t0);
      return is_reg(l, t) || is_lane(l, t);
    }
    default: return false;
  }
}

// For each tile bit, the index of the first gate from `from` on whose
// target it is (kNever when none).
struct FirstUse {
  int next[NB];
};
const int kNever = 1 << 30;

// Fold gate i into the first uses of the gates after it.
void first_use_step(const Plan& plan, const Pass& p, size_t i, FirstUse& f) {
  const Gate& g = plan.gates[p.gates[i]];
  if (g.type == G_DIAG1 || g.type == G_DIAG2 || g.type == G_GRADD || g.type == G_GRADM2) return;
  if (relabel_gate(g, p)) return;  // needs no role
  const int ts[2] = {tpos(p, g.t0), g.type == G_SWAP || g.type == G_MAT2 ? tpos(p, g.t1) : -1};
  for (int t : ts)
    if (t >= 0) f.next[t] = (int)i;
}

// First uses for every start index 0..G, by one backward sweep.
std::vector<FirstUse> first_uses(const Plan& plan, const Pass& p) {
  const size_t G = p.gates.size();
  std::vector<FirstUse> f(G + 1);
  for (int b = 0; b < NB; b++) f[G].next[b] = kNever;
  for (size_t i = G; i-- > 0;) {
    f[i] = f[i + 1];
    first_use_step(plan, p, i, f[i]);
  }
  return f;
}

// Choose a layout for the gates from index `from` on, given their first uses.
Lay choose_with(const Plan& plan, const Pass& p, size_t from, bool a0, int precision, const FirstUse& fu) {
  const int* next = fu.next;
  struct Bits {  // a short list of tile bits
    int v[NB];
    int n = 0;
    void add(int b) { v[n++] = b; }
  };
  // the adjoint ancilla always sits in registers; a 2x2 probe's target too
  Bits must;
  if (g_anc_tb >= 0) must.add(g_anc_tb);
  if (from < p.gates.size()) {
    const Gate& g = plan.gates[p.gates[from]];
    if (g.type == G_GRADM) must.add(tpos(p, g.t0));
  }
  // tile bits by first use (soonest first, the lower bit first among
  // equals): a stable insertion sort
  int order[NB];
  for (int b = 0; b < NB; b++) {
    int j = b;
    for (; j > 0; j--) {
      const int y = order[j - 1];
      if (next[b] >= next[y]) break;
      order[j] = y;
    }
    order[j] = b;
  }
  Lay l;
  bool used[NB] = {};
  Bits regs, lanes, warps;
  auto take_reg = [&](int b) { regs.add(b); used[b] = true; };
  if (a0) {
    for (int b = 0; b < 5; b++) { lanes.add(b); used[b] = true; }
    for (int k = 0; k < must.n; k++) if (!used[must.v[k]] && regs.n < NRg()) take_reg(must.v[k]);
    for (int b : order) if (!used[b] && regs.n < NRg() && b >= 5) take_reg(b);
    for (int b : order) if (!used[b]) { warps.add(b); used[b] = true; }
  } else {
    for (int k = 0; k < must.n; k++) if (!used[must.v[k]] && regs.n < NRg()) take_reg(must.v[k]);
    for (int b : order) if (!used[b] && regs.n < NRg()) take_reg(b);
    for (int b : order) if (!used[b] && lanes.n < 5) { lanes.add(b); used[b] = true; }
    for (int b = 0; b < NB; b++) if (!used[b]) { warps.add(b); used[b] = true; }
    // Shared-memory bank spread: the swizzle folds tile bits mod 3 (c128) or
    // mod 4 (c64) into the low bits, so lanes 0..2 (0..3) should cover
    // distinct residues: the first lane of each residue in turn, then the rest
    // in their order.
    const int mod = precision == KET_C64 ? 4 : 3;
    Bits out;
    bool moved[NB] = {};
    for (int r = 0; r < mod; r++)
      for (int k = 0; k < lanes.n; k++)
        if (!moved[k] && lanes.v[k] % mod == r) { out.add(lanes.v[k]); moved[k] = true; break; }
    for (int k = 0; k < lanes.n; k++) if (!moved[k]) out.add(lanes.v[k]);
    lanes = out;
  }
  // the adjoint ancilla always occupies the top register bit (the kernel's
  // probes address it at compile time)
  const int top = NRg() - 1;
  if (g_anc_tb >= 0)
    for (int i = 0; i < top; i++)
      if (regs.v[i] == g_anc_tb) std::swap(regs.v[i], regs.v[top]);
  for (int i = 0; i < 5; i++) l.pos[i] = lanes.v[i];
  for (int i = 0; i < NWg(); i++) l.pos[5 + i] = warps.v[i];
  for (int i = 0; i < NRg(); i++) l.pos[REG0() + i] = regs.v[i];
  fill_roles(l);
  return l;
}

Lay choose(const Plan& plan, const Pass& p, size_t from, bool a0, int precision) {
  FirstUse f;
  for (int b = 0; b < NB; b++) f.next[b] = kNever;
  for (size_t i = p.gates.size(); i-- > from;) first_use_step(plan, p, i, f);
  return choose_with(plan, p, from, a0, precision, f);
}

// l with tile bits a and b exchanged: where the data stays after swapping them.
Lay relabeled(const Lay& l, int a, int b) {
  Lay r = l;
  for (int i = 0; i < NB; i++) {
    if (r.pos[i] == a) r.pos[i] = b;
    else if (r.pos[i] == b) r.pos[i] = a;
  }
  fill_roles(r);
  return r;
}

FOp make_exch(const Lay& l, int precision) {
  FOp o;
  memset(&o, 0, sizeof(o));
  o.type = FO_EXCH;
  uint16_t bx[NB];
  for (int i = 0; i < NB; i++) {
    o.pos[i] = (uint8_t)l.pos[i];
    bx[i] = (uint16_t)exch_offset(1u << l.pos[i], precision == KET_C64);
  }
  memcpy(o.m, bx, sizeof(bx));
  return o;
}

// Split a control mask over the current layout.
void controls(const Gate& g, const Pass& p, const Lay& l, FOp& o) {
  o.lmask = 0xffffffffu;
  for (int q = 0; q < 64; q++) {
    if (!((g.cmask >> q) & 1)) continue;
    int t = tpos(p, q);
    if (t < 0) { o.cctx |= uint64_t(1) << q; continue; }
    o.ctile |= 1u << t;
    int r = l.role[t];
    if (r >= REG0()) {
      o.creg |= (uint8_t)(1u << (r - REG0()));
    } else {
      o.cthr |= (uint8_t)(1u << r);  // lanes 0..4 -> tid bits 0..4, warps -> the tid bits above
      if (r < 5) {
        uint32_t lanes = 0;
        for (int ln = 0; ln < 32; ln++)
          if ((ln >> r) & 1) lanes |= 1u << ln;
        o.lmask &= lanes;
      }
    }
  }
}

FOp make_op(const Gate& g, const Pass& p, const Lay& l, bool prune) {
  FOp o;
  memset(&o, 0, sizeof(o));
  o.flags = (g.prune && prune) ? FOF_PRUNE : 0;
  o.d0 = o.d1 = -2;
  controls(g, p, l, o);
  int t0 = tpos(p, g.t0), t1 = tpos(p, g.t1);
  switch (g.type) {
    case G_MAT1: case G_X1: {
      bool reg = is_reg(l, t0);
      o.type = g.type == G_MAT1 ? (reg ? FO_MAT1R : FO_MAT1L) : (reg ? FO_X1R : FO_X1L);
      o.a = (uint8_t)(reg ? l.role[t0] - REG0() : l.role[t0]);
      o.b = (uint8_t)t0;  // tile bit (the shared-memory form of a multi-controlled X)
      bool real = true;
      for (int k = 0; k < 4; k++) {
        o.m[2 * k] = g.m[k].re;
        o.m[2 * k + 1] = g.m[k].im;
        real = real && g.m[k].im == 0.0;
      }
      bool rx = g.m[0].im == 0.0 && g.m[3].im == 0.0 && g.m[1].re == 0.0 && g.m[2].re == 0.0;
      if (g.type == G_MAT1 && real) o.flags |= FOF_REAL;
      else if (g.type == G_MAT1 && rx) o.flags |= FOF_RXFORM;
      break;
    }
    case G_SWAP:
      o.type = FO_SWAPS;
      o.a = (uint8_t)t0;
      o.b = (uint8_t)t1;
      break;
    case G_MAT2:
      o.type = FO_MAT2S;
      o.a = (uint8_t)t0;
      o.b = (uint8_t)t1;
      for (int k = 0; k < 16; k++) { o.m[2 * k] = g.m[k].re; o.m[2 * k + 1] = g.m[k].im; }
      break;
    case G_DIAG1: {
      // A phase keeps |a| (to the last bit), so the reference's pruning after
      // it can only fire on amplitudes it already pruned: no prune flag.
      o.flags &= ~FOF_PRUNE;
      for (int k = 0; k < 2; k++) { o.m[2 * k] = g.m[k].re; o.m[2 * k + 1] = g.m[k].im; }
      if (g.m[0].re == 1.0 && g.m[0].im == 0.0) o.flags |= FOF_D0ONE;
      if (t0 < 0) {
        o.type = FO_DIAGX;
        o.dg0 = uint64_t(1) << g.t0;
      } else if (is_reg(l, t0)) {
        o.type = FO_DIAGR;
        o.a = (uint8_t)(l.role[t0] - REG0());
      } else {
        o.type = FO_DIAGT;
        o.a = (uint8_t)l.role[t0];  // lanes 0..4 -> tid bits 0..4, warps -> the tid bits above
      }
      break;
    }
    case G_GRADM: {
      o.type = FO_GRADM;
      o.flags = 0;
      o.a = (uint8_t)(l.role[t0] - REG0());
      o.b = (uint8_t)(l.role[g_anc_tb] - REG0());
      o.slot = (int16_t)g.slot;
      for (int k = 0; k < 4; k++) { o.m[2 * k] = g.m[k].re; o.m[2 * k + 1] = g.m[k].im; }
      break;
    }
    case G_GRADD: {
      o.type = FO_GRADD;
      o.flags = 0;
      o.b = (uint8_t)(l.role[g_anc_tb] - REG0());
      o.slot = (int16_t)g.slot;
      if (t0 < 0) { o.flags |= FOF_TGT_CTX; o.dg0 = uint64_t(1) << g.t0; }
      else if (is_reg(l, t0)) o.a = (uint8_t)(l.role[t0] - REG0());
      else { o.flags |= FOF_TGT_THR; o.a = (uint8_t)l.role[t0]; }
      for (int k = 0; k < 2; k++) { o.m[2 * k] = g.m[k].re; o.m[2 * k + 1] = g.m[k].im; }
      break;
    }
    case G_GRADM2: {
      o.type = FO_GRADM2;
      o.flags = 0;
      o.a = (uint8_t)t0;
      o.b = (uint8_t)t1;
      o.anc = (int16_t)g_anc_tb;
      o.slot = (int16_t)g.slot;
      for (int k = 0; k < 16; k++) { o.m[2 * k] = g.m[k].re; o.m[2 * k + 1] = g.m[k].im; }
      break;
    }
    case G_DIAG2: {
      o.flags &= ~FOF_PRUNE;
      o.type = FO_DIAG;
      o.d0 = (int8_t)(t0 >= 0 ? t0 : -1);
      if (t0 < 0) o.dg0 = uint64_t(1) << g.t0;
      o.d1 = (int8_t)(t1 >= 0 ? t1 : -1);
      if (t1 < 0) o.dg1 = uint64_t(1) << g.t1;
      for (int k = 0; k < 4; k++) { o.m[2 * k] = g.m[k].re; o.m[2 * k + 1] = g.m[k].im; }
      break;
    }
    default: break;
  }
  return o;
}

}  // namespace

namespace {

int popc(uint64_t v) { return __builtin_popcountll(v); }

bool fan_member(const FOp& o) {
  return o.type == FO_DIAGR && (o.flags & FOF_D0ONE) && popc(o.creg) + popc(o.cthr) + popc(o.cctx) <= 1;
}

// Merge runs of phase gates on the same register bit into FO_CPHASE ops.
void merge_phase_fans(std::vector<FOp>& prog) {
  std::vector<FOp> out;
  out.reserve(prog.size());
  size_t i = 0;
  while (i < prog.size()) {
    size_t j = i;
    while (j < prog.size() && fan_member(prog[j]) && prog[j].a == prog[i].a) j++;
    // phases whose control is a register bit run as cheap compiled ops of
    // their own (4 of 16 slots each); a fan of only those costs more
    bool other = false;
    for (size_t k = i; k < j; k++) other = other || !prog[k].creg;
    if (!fan_member(prog[i]) || j - i < 2 || (!other && j - i < 6)) {
      out.push_back(prog[i]);
      i++;
      continue;
    }
    const int A = prog[i].a;
    const int nt = 1 << (NRg() - 1);  // slots with bit A set
    cd T[16], H[8];
    for (int k = 0; k < 16; k++) T[k] = cd{1, 0};
    for (int k = 0; k < 8; k++) H[k] = cd{1, 0};
    std::vector<std::pair<uint64_t, double>> terms;  // (mask, angle)
    auto mul = [](cd a, cd b) { return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; };
    for (size_t g = i; g < j; g++) {
      const FOp& o = prog[g];
      const cd ph{o.m[2], o.m[3]};
      if (o.cctx) {
        const double ang = std::atan2(ph.im, ph.re);
        bool found = false;
        for (auto& t : terms)
          if (t.first == o.cctx) { t.second += ang; found = true; }
        if (!found) terms.push_back({o.cctx, ang});
      } else if (o.cthr) {
        for (int sb = 0; sb < 8; sb++)
          if (o.cthr == (1u << sb)) H[sb] = mul(H[sb], ph);
      } else {
        for (int k = 0; k < nt; k++) {
          const int slot = ((k >> A) << (A + 1)) | (1 << A) | (k & ((1 << A) - 1));
          if ((slot & o.creg) == o.creg) T[k] = mul(T[k], ph);
        }
      }
    }
    FOp f;
    memset(&f, 0, sizeof(f));
    f.type = FO_CPHASE;
    f.a = (uint8_t)A;
    f.d0 = f.d1 = -2;
    for (int k = 0; k < nt; k++) { f.m[2 * k] = T[k].re; f.m[2 * k + 1] = T[k].im; }
    const size_t nrec = 1 + (terms.size() + KET_CPHASE_TERMS_PER_RECORD - 1) / KET_CPHASE_TERMS_PER_RECORD;
    f.lmask = (uint32_t)terms.size();
    f.ctile = (uint32_t)nrec;
    out.push_back(f);
    for (size_t r = 0; r < nrec; r++) {
      FOp c;
      memset(&c, 0, sizeof(c));
      c.opc = OC_NOP;
      c.type = FO_CONT;
      c.d0 = c.d1 = -2;
      double* d = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(&c) + 16);
      if (r == 0) {
        for (int k = 0; k < 8; k++) { d[2 * k] = H[k].re; d[2 * k + 1] = H[k].im; }
      } else {
        for (size_t t = 0; t < KET_CPHASE_TERMS_PER_RECORD; t++) {
          const size_t ti = (r - 1) * KET_CPHASE_TERMS_PER_RECORD + t;
          if (ti >= terms.size()) break;
          d[2 * t] = terms[ti].second;
          memcpy(&d[2 * t + 1], &terms[ti].first, 8);
        }
      }
      out.push_back(c);
    }
    i = j;
  }
  prog.swap(out);
}

// A phase gate diag(1, p) with |p| = 1 whose target and register-bit controls
// name at most one register bit (rb: that bit, or -1).
bool poly_member(const FOp& o, int& rb) {
  if (!(o.flags & FOF_D0ONE)) return false;
  if (o.type != FO_DIAGR && o.type != FO_DIAGT && o.type != FO_DIAGX) return false;
  const double r2 = o.m[2] * o.m[2] + o.m[3] * o.m[3];
  if (!(std::fabs(r2 - 1.0) <= 4e-16)) return false;
  const uint32_t regs = o.creg | (o.type == FO_DIAGR ? 1u << o.a : 0u);
  if (popc(regs) > 1) return false;
  rb = regs ? __builtin_ctz(regs) : -1;
  return true;
}

// Runs of at least this many phase gates become FO_PPOLY ops.
constexpr size_t kPolyMinRun = 6;

// One FO_PPOLY op and its records from prog[i, j), all poly members, whose
// (register bit, tm) groups number at most KET_PPOLY_MAX_GROUPS.
void emit_poly(const std::vector<FOp>& prog, size_t i, size_t j, std::vector<FOp>& out) {
  struct Grp {
    int rb;
    uint32_t tm;
    std::vector<PPolyTerm> terms;
  };
  std::vector<Grp> grps;
  uint8_t used = 0;
  for (size_t g = i; g < j; g++) {
    const FOp& o = prog[g];
    int rb;
    poly_member(o, rb);
    PPolyTerm t;
    t.re = o.m[2];
    t.im = o.m[3];
    t.cm = o.cctx | (o.type == FO_DIAGX ? o.dg0 : 0);
    t.unused = 0;
    const uint32_t tm = o.cthr | (o.type == FO_DIAGT ? 1u << o.a : 0u);
    Grp* G = nullptr;
    for (auto& x : grps)
      if (x.rb == rb && x.tm == tm) G = &x;
    if (!G) {
      grps.push_back({rb, tm, {}});
      G = &grps.back();
    }
    G->terms.push_back(t);
    if (rb >= 0) used |= (uint8_t)(1u << rb);
  }
  // groups of no register bit first, then bit 0, 1, ... (stable: first use)
  std::stable_sort(grps.begin(), grps.end(), [](const Grp& a, const Grp& b) { return a.rb < b.rb; });
  FOp f;
  memset(&f, 0, sizeof(f));
  f.type = FO_PPOLY;
  f.d0 = f.d1 = -2;
  f.b = used;
  f.lmask = (uint32_t)grps.size();
  uint32_t* cnt = reinterpret_cast<uint32_t*>(f.m);
  PPolyGroup* desc = reinterpret_cast<PPolyGroup*>(reinterpret_cast<unsigned char*>(f.m) + 32);
  std::vector<FOp> recs;
  for (size_t g = 0; g < grps.size(); g++) {
    cnt[grps[g].rb + 1]++;
    desc[g].tm = grps[g].tm;
    desc[g].n = (uint32_t)grps[g].terms.size();
    desc[g].rec = (uint32_t)recs.size() + 1;
    desc[g].unused = 0;
    for (size_t k = 0; k < grps[g].terms.size(); k++) {
      if (k % KET_PPOLY_TERMS_PER_RECORD == 0) {
        FOp c;
        memset(&c, 0, sizeof(c));
        c.opc = OC_NOP;
        c.type = FO_CONT;
        c.d0 = c.d1 = -2;
        recs.push_back(c);
      }
      PPolyTerm* d = reinterpret_cast<PPolyTerm*>(reinterpret_cast<unsigned char*>(&recs.back()) + 16);
      d[k % KET_PPOLY_TERMS_PER_RECORD] = grps[g].terms[k];
    }
  }
  f.ctile = (uint32_t)recs.size();
  out.push_back(f);
  out.insert(out.end(), recs.begin(), recs.end());
}

bool diagonal_op(const FOp& o) { return o.type == FO_DIAGR || o.type == FO_DIAGT || o.type == FO_DIAGX; }

// Merge the phase gates of each run of diagonal ops into FO_PPOLY ops placed
// first in the run, the run's other diagonal ops following in their order.
// All of them are diagonal, so only the order in which a thread multiplies
// their factors changes.
void merge_phase_polys(std::vector<FOp>& prog) {
  std::vector<FOp> out;
  out.reserve(prog.size());
  size_t i = 0;
  int rb;
  while (i < prog.size()) {
    if (!diagonal_op(prog[i])) {
      out.push_back(prog[i]);
      i++;
      continue;
    }
    size_t j = i;
    std::vector<size_t> mem, rest;
    while (j < prog.size() && diagonal_op(prog[j])) {
      (poly_member(prog[j], rb) ? mem : rest).push_back(j);
      j++;
    }
    if (mem.size() < kPolyMinRun) {
      for (size_t k = i; k < j; k++) out.push_back(prog[k]);
      i = j;
      continue;
    }
    std::vector<FOp> ms;
    for (size_t k : mem) ms.push_back(prog[k]);
    // split where a piece would need more groups than an op holds
    size_t s0 = 0;
    std::vector<std::pair<int, uint32_t>> keys;
    for (size_t k = 0; k <= ms.size(); k++) {
      if (k < ms.size()) {
        poly_member(ms[k], rb);
        const std::pair<int, uint32_t> key{rb, ms[k].cthr | (ms[k].type == FO_DIAGT ? 1u << ms[k].a : 0u)};
        if (std::find(keys.begin(), keys.end(), key) != keys.end()) continue;
        if (keys.size() < KET_PPOLY_MAX_GROUPS) {
          keys.push_back(key);
          continue;
        }
        keys.assign(1, key);
      }
      emit_poly(ms, s0, k, out);
      s0 = k;
    }
    for (size_t k : rest) out.push_back(prog[k]);
    i = j;
  }
  prog.swap(out);
}

// Deferred register swaps (FOF_SW, fused_abi.h), for the compiled kernels:
// an X on a register bit under thread or out-of-tile controls becomes a
// per-thread flag, and the ops after it read the flag where they can (a 2x2
// or general diagonal on that bit exchanges its matrix entries; exchanges,
// shared-memory ops and the store address the logical slots).  Where an op
// needs the register slots in logical order -- register controls on a
// swapped bit, a phase on one, merged phase ops, and a lane op whose partner
// lanes could disagree (a swap decided by a control on that lane bit) --
// FO_REAL carries the pending swaps out first.
void defer_swaps(std::vector<FOp>& prog) {
  const int nr = NRg();
  uint32_t pend = 0;               // register bits with pending swaps
  uint32_t src[KET_NR_MAX] = {};   // per register bit: thread-id bits of the controls that decided them (bit 8: outside the tile)
  std::vector<FOp> out;
  out.reserve(prog.size() + 8);
  auto clear = [&]() {
    pend = 0;
    for (int k = 0; k < nr; k++) src[k] = 0;
  };
  auto realize = [&](uint32_t m) {
    m &= pend;
    if (!m) return;
    FOp r;
    memset(&r, 0, sizeof(r));
    r.type = FO_REAL;
    r.creg = (uint8_t)m;
    r.d0 = r.d1 = -2;
    r.lmask = 0xffffffffu;
    out.push_back(r);
    pend &= ~m;
    for (int k = 0; k < nr; k++)
      if ((m >> k) & 1) src[k] = 0;
  };
  for (const FOp& in : prog) {
    FOp o = in;
    switch (o.type) {
      case FO_CONT:  // the records of the op before: kept right after it
      case FO_RELAY:  // no data moves
      case FO_SYNC:
        break;
      case FO_EXCH: case FO_SWAPS: case FO_MAT2S: case FO_DIAG:
        clear();  // written out through the logical slots
        break;
      case FO_X1R: {
        if (!o.creg) {
          if (o.cthr || o.cctx) {
            o.flags |= FOF_SW;
            pend |= 1u << o.a;
            src[o.a] |= o.cthr | (o.cctx ? 0x100u : 0u);
          }  // uncontrolled: a renaming, which commutes with the pending swaps
        } else if (!(o.creg & (o.creg - 1)) && !o.cthr && !o.cctx) {
          const int c = __builtin_ctz(o.creg);
          if ((pend >> c) & 1) {
            o.flags |= FOF_SW;
            pend |= 1u << o.a;
            src[o.a] |= src[c];
          }
        } else {
          clear();  // the shared-memory form (several controls)
        }
        break;
      }
      case FO_MAT1R:
        realize(o.creg);
        if ((pend >> o.a) & 1) o.flags |= FOF_SW;
        break;
      case FO_DIAGR:
        realize(o.creg);
        if ((pend >> o.a) & 1) {
          if (o.flags & FOF_D0ONE) realize(1u << o.a);
          else o.flags |= FOF_SW;
        }
        break;
      case FO_MAT1L: case FO_X1L: {
        uint32_t m = o.creg;
        for (int k = 0; k < nr; k++)
          if ((src[k] >> o.a) & 1) m |= 1u << k;
        realize(m);
        break;
      }
      case FO_DIAGT: case FO_DIAGX:
        realize(o.creg);
        break;
      default:  // merged phase ops and anything else
        realize(pend);
        break;
    }
    out.push_back(o);
  }
  prog.swap(out);  // the store takes what is still pending
}

// Deferred X gates on lane bits (FOF_SW on FO_X1L, compiled kernels): an X
// on lane bit a whose controls sit on thread bits or outside the tile moves
// amplitudes between lanes.  Instead each thread keeps its logical thread id
// (the lanes' amplitudes stay where they are; the X flips bit a of the
// logical id of the threads whose controls hold), every control and phase
// reads the logical id, and the next exchange, shared-memory op or store
// addresses the logical lanes.  A lane op needs its partners in place, so an
// X is deferred only when no lane op follows it before the layout is next
// written out.  The interpreter ignores the flag and moves the amplitudes.
void defer_lane_x(std::vector<FOp>& prog) {
  auto writes_layout = [](const FOp& o) {
    if (o.type == FO_EXCH || o.type == FO_SWAPS || o.type == FO_MAT2S || o.type == FO_DIAG) return true;
    return o.type == FO_X1R && o.creg && ((o.creg & (o.creg - 1)) || o.cthr || o.cctx);  // the shared-memory X
  };
  auto lane_op = [](const FOp& o) {
    return o.type == FO_MAT1L || (o.type == FO_X1L && o.creg) || o.type == FO_GRADM || o.type == FO_GRADD ||
           o.type == FO_GRADM2;
  };
  bool later_lane_op = false;  // scanning backwards: a lane op follows in the current segment
  for (size_t i = prog.size(); i-- > 0;) {
    FOp& o = prog[i];
    if (o.type == FO_CONT) continue;
    if (writes_layout(o)) {
      later_lane_op = false;
      continue;
    }
    if (o.type == FO_X1L && !o.creg && !later_lane_op) {
      o.flags |= FOF_SW;
      continue;
    }
    if (lane_op(o)) later_lane_op = true;
  }
}

}  // namespace

void assign_opcode(FOp& o) {
  const bool real = o.flags & FOF_REAL, rx = o.flags & FOF_RXFORM, d0one = o.flags & FOF_D0ONE;
  // a single control on a register bit (and none elsewhere) gets a compile-time variant
  int c1 = -1;
  if (o.creg && !(o.creg & (o.creg - 1)) && !o.cthr && !o.cctx)
    for (int k = 0; k < KET_NR_MAX; k++)
      if (o.creg == (1u << k)) c1 = k;
  switch (o.type) {
    case FO_EXCH: o.opc = OC_EXCH; break;
    case FO_MAT1R: o.opc = (uint8_t)(OC_MAT1R + 3 * o.a + (real ? 1 : rx ? 2 : 0)); break;
    case FO_MAT1L: o.opc = (uint8_t)(OC_MAT1L + (real ? 1 : rx ? 2 : 0)); break;
    case FO_X1R:
      if (!o.creg) o.opc = (uint8_t)(OC_X1R + o.a);
      else if (c1 >= 0) o.opc = (uint8_t)(OC_X1RC + 5 * o.a + c1);
      else o.opc = OC_X1S;  // several controls, some on register bits: rare
      break;
    case FO_X1L: o.opc = OC_X1L; break;
    case FO_DIAGR:
      if (d0one) o.opc = c1 >= 0 ? (uint8_t)(OC_DIAGR1C + 5 * o.a + c1) : (uint8_t)(OC_DIAGR1 + o.a);
      else o.opc = (uint8_t)(OC_DIAGR + o.a);
      break;
    case FO_DIAGT: o.opc = OC_DIAGT; break;
    case FO_DIAGX: o.opc = OC_DIAGX; break;
    case FO_DIAG: o.opc = OC_DIAG; break;
    case FO_SWAPS: o.opc = OC_SWAPS; break;
    case FO_MAT2S: o.opc = OC_MAT2S; break;
    case FO_GRADM: o.opc = (uint8_t)(OC_GRADM + o.a); break;
    case FO_GRADD: o.opc = OC_GRADD; break;
    case FO_GRADM2: o.opc = OC_GRADM2; break;
    case FO_CPHASE: o.opc = (uint8_t)(OC_CPHASE + o.a); break;
    case FO_PPOLY: o.opc = OC_PPOLY; break;
    case FO_REAL: o.opc = OC_REAL; break;
    case FO_RELAY: o.opc = OC_RELAY; break;
    case FO_SYNC: o.opc = OC_SYNC; break;
    case FO_CONT: o.opc = OC_NOP; break;
    default: o.opc = 0xff; break;
  }
}

namespace {

// Estimated cost, in milliseconds per op on a 2^30-amplitude complex128 state,
// of the program's ops by kind and placement.  Fitted to the event-timed
// passes of the 30-qubit brickwork step (compiled kernels, 4 register bits):
// a 2x2 on a register bit about 0.6 (general matrices more, real and Rx-like
// less), the same on a lane bit about 0.25 more (its shuffles), an X on a lane
// bit 0.4, an X on a register bit under a thread or out-of-tile control 0.22
// (conditional register moves; uncontrolled or register-controlled, a
// renaming), a diagonal 0.16, a layout exchange 0.45.
double exch_cost() {
  static const double c = [] {
    const char* e = getenv("KET_COST_EXCH");  // experiments only
    return e ? atof(e) : 0.45;
  }();
  return c;
}

double mat_form_cost(const Gate& g) {
  bool real = true;
  for (int k = 0; k < 4; k++) real = real && g.m[k].im == 0.0;
  const bool rx = g.m[0].im == 0.0 && g.m[3].im == 0.0 && g.m[1].re == 0.0 && g.m[2].re == 0.0;
  return real || rx ? 0.5 : 0.75;
}

double gate_cost(const Gate& g, const Pass& p, const Lay& l) {
  switch (g.type) {
    case G_MAT1: return mat_form_cost(g) + (is_lane(l, tpos(p, g.t0)) ? 0.25 : 0.0);
    case G_X1: {
      if (is_lane(l, tpos(p, g.t0))) return 0.4;
      int nreg = 0;
      bool other = false;
      for (int q = 0; q < 64; q++) {
        if (!((g.cmask >> q) & 1)) continue;
        const int t = tpos(p, q);
        if (t >= 0 && is_reg(l, t)) nreg++;
        else other = true;
      }
      if (nreg == 0) return other ? 0.22 : 0.0;
      if (nreg == 1 && !other) return 0.0;
      return 2 * exch_cost();  // several controls with one on a register bit: a shared-memory op
    }
    case G_DIAG1: return 0.16;
    default: return 2 * exch_cost();  // shared-memory ops: the same in every layout
  }
}

bool same_lay(const Lay& a, const Lay& b) { return memcmp(a.pos, b.pos, sizeof a.pos) == 0; }

// Layouts of a pass by dynamic programming over where to exchange.  Candidate
// layouts at gate i are the look-ahead layouts from i (one keeping the
// store's lanes, one not); the load layout is any lane-keeping candidate.
// The cheapest sequence of runs and exchanges under gate_cost, with the
// restore to a lane-keeping layout at the end, wins.  lay[i] is the layout
// gate i runs in.  False when no sequence fits (the caller falls back to the
// greedy rule).
bool plan_layouts(const Plan& plan, const Pass& p, int precision, std::vector<Lay>& lay) {
  const size_t G = p.gates.size();
  const std::vector<FirstUse> fu = first_uses(plan, p);
  std::vector<std::vector<Lay>> cand(G + 1);
  for (size_t i = 0; i <= G; i++) {
    for (int a0 = 1; a0 >= 0; a0--) {
      const Lay l = choose_with(plan, p, i, a0 != 0, precision, fu[i]);
      bool dup = false;
      for (const Lay& c : cand[i]) dup = dup || same_lay(c, l);
      if (!dup) cand[i].push_back(l);
    }
  }
  struct St {
    Lay l;
    double cost;
    int from;   // index of the state it came from (in the previous position's list), -1 at the start
    bool exch;  // entered by an exchange at this position
  };
  std::vector<std::vector<St>> at(G + 1);  // states in effect before gate i (after any exchange at i)
  std::vector<std::vector<St>> run(G + 1);  // states arriving at i by running gate i-1 (or the start)
  // a list keeps one state per layout, the cheapest (the first of equals)
  auto relax = [](std::vector<St>& v, const St& s) {
    for (St& o : v)
      if (same_lay(o.l, s.l)) {
        if (s.cost < o.cost) o = s;
        return;
      }
    v.push_back(s);
  };
  // starting layouts: every lane-keeping candidate
  for (size_t i = 0; i <= G; i++)
    for (const Lay& c : cand[i])
      if (a0_compatible(c)) relax(run[0], {c, 0.0, -1, false});
  // Every list holds distinct layouts: the start list and the exchange
  // targets by relax, the stays because the run list they copy does, and the
  // run list because running a gate keeps a layout and a relabelling maps
  // distinct layouts to distinct ones.
  for (size_t i = 0; i <= G; i++) {
    // stay
    at[i].reserve(run[i].size() + cand[i].size());
    for (size_t k = 0; k < run[i].size(); k++) {
      St s = run[i][k];
      s.from = (int)k;
      s.exch = false;
      at[i].push_back(s);
    }
    // or exchange to a candidate from the cheapest state of another layout
    // (the first of equals)
    for (const Lay& c : cand[i]) {
      if (i < G && !fits(plan.gates[p.gates[i]], p, c)) continue;
      if (i == G && !a0_compatible(c)) continue;
      int from = -1;
      double fc = 0;
      for (size_t k = 0; k < run[i].size(); k++) {
        if (same_lay(c, run[i][k].l)) continue;
        const double v = run[i][k].cost + exch_cost();
        if (from < 0 || v < fc) { from = (int)k; fc = v; }
      }
      if (from >= 0) relax(at[i], {c, fc, from, true});
    }
    if (i == G) break;
    const Gate& g = plan.gates[p.gates[i]];
    const bool rel = relabel_gate(g, p);
    run[i + 1].reserve(at[i].size());
    for (size_t k = 0; k < at[i].size(); k++) {
      const St& s = at[i][k];
      if (rel) {
        run[i + 1].push_back({relabeled(s.l, tpos(p, g.t0), tpos(p, g.t1)), s.cost, (int)k, false});
        continue;
      }
      if (!fits(g, p, s.l)) continue;
      run[i + 1].push_back({s.l, s.cost + gate_cost(g, p, s.l), (int)k, false});
    }
    if (run[i + 1].empty()) return false;
  }
  // the end: the store needs the lanes kept (a restore exchange otherwise)
  int best = -1;
  double bc = 0;
  for (size_t k = 0; k < at[G].size(); k++) {
    const St& s = at[G][k];
    if (!a0_compatible(s.l)) continue;
    if (best < 0 || s.cost < bc) { best = (int)k; bc = s.cost; }
  }
  if (best < 0) return false;
  // walk back: at[i][k] came from run[i][from]; run[i][k] came from at[i-1][from]
  lay.assign(G + 1, Lay());
  int k = best;
  for (size_t i = G + 1; i-- > 0;) {
    const St& s = at[i][k];
    lay[i] = s.l;
    const int r = s.from;  // index in run[i]
    if (i == 0) break;
    k = run[i][r].from;    // index in at[i-1]
  }
  return true;
}

// Switches for experiments, read once per process: the greedy layout rule
// instead of the cost-model planner (everywhere, or for adjoint passes),
// swaps as data moves instead of relabellings, and no deferred register
// swaps or lane X gates.
struct Switches {
  bool greedy = getenv("KET_GREEDY_LAYOUT") != nullptr;
  bool adjoint_greedy = getenv("KET_ADJOINT_GREEDY") != nullptr;
  bool no_relabel = getenv("KET_NO_RELABEL") != nullptr;
  bool no_defer = getenv("KET_NO_DEFER") != nullptr;
  bool no_lane_defer = getenv("KET_NO_LANE_DEFER") != nullptr;
};

const Switches& switches() {
  static const Switches s;
  return s;
}

}  // namespace

void plan_program(const Plan& plan, const Pass& p, int precision, bool prune, int nreg, std::vector<FOp>& prog,
                  uint8_t load_pos[KET_T2_BITS], uint8_t store_pos[KET_T2_BITS]) {
  prog.clear();
  g_nreg = nreg;
  g_anc_tb = plan.anc >= 0 ? tpos(p, plan.anc) : -1;
  std::vector<Lay> lay;
  // adjoint passes too (their probes fit only where the ancilla and a 2x2
  // probe's target sit in registers, which the candidates respect); their
  // swaps stay data moves
  const Switches& sw = switches();
  const bool dp = !sw.greedy && (g_anc_tb < 0 || !sw.adjoint_greedy);
  g_relabel = dp && g_anc_tb < 0 && !sw.no_relabel;
  if (dp && plan_layouts(plan, p, precision, lay)) {
    // lay[i]: the layout gate i runs in; lay[G]: the store layout
    Lay cur = lay[0];
    for (int i = 0; i < NB; i++) load_pos[i] = (uint8_t)cur.pos[i];
    for (size_t i = 0; i < p.gates.size(); i++) {
      if (!same_lay(lay[i], cur)) {
        cur = lay[i];
        prog.push_back(make_exch(cur, precision));
      }
      const Gate& g = plan.gates[p.gates[i]];
      if (relabel_gate(g, p)) {
        cur = relabeled(cur, tpos(p, g.t0), tpos(p, g.t1));
        FOp r = make_exch(cur, precision);
        r.type = FO_RELAY;
        prog.push_back(r);
        continue;
      }
      prog.push_back(make_op(g, p, cur, prune));
    }
    if (!same_lay(lay[p.gates.size()], cur)) {
      cur = lay[p.gates.size()];
      prog.push_back(make_exch(cur, precision));
    }
    for (int i = 0; i < NB; i++) store_pos[i] = (uint8_t)cur.pos[i];
    // Relabellings can make a thread store amplitudes that another thread
    // loaded.  An exchange puts a barrier between every load and every store;
    // without one, a barrier of its own does.
    bool barrier = false, moved = false;
    for (const FOp& o : prog) barrier = barrier || o.type == FO_EXCH;
    for (int r = 0; r < 5 + NWg(); r++) moved = moved || load_pos[r] != store_pos[r];
    if (moved && !barrier) {
      FOp b;
      memset(&b, 0, sizeof(b));
      b.type = FO_SYNC;
      b.d0 = b.d1 = -2;
      b.lmask = 0xffffffffu;
      prog.push_back(b);
    }
    if (g_anc_tb < 0) {  // the probe passes run no merged phase ops
      merge_phase_polys(prog);
      merge_phase_fans(prog);
    }
    if (!sw.no_defer) defer_swaps(prog);
    if (!sw.no_lane_defer) defer_lane_x(prog);
    for (FOp& o : prog) assign_opcode(o);
    g_relabel = false;
    return;
  }
  g_relabel = false;
  Lay cur = choose(plan, p, 0, true, precision);
  for (int i = 0; i < NB; i++) load_pos[i] = (uint8_t)cur.pos[i];
  for (size_t i = 0; i < p.gates.size(); i++) {
    const Gate& g = plan.gates[p.gates[i]];
    if (!fits(g, p, cur)) {
      // A layout with the store's lanes that holds every remaining gate saves
      // the exchange back to it at the end of the pass.
      Lay a0 = choose(plan, p, i, true, precision);
      bool all = true;
      for (size_t j = i; j < p.gates.size() && all; j++) all = fits(plan.gates[p.gates[j]], p, a0);
      cur = all ? a0 : choose(plan, p, i, false, precision);
      prog.push_back(make_exch(cur, precision));
    }
    prog.push_back(make_op(g, p, cur, prune));
  }
  if (!a0_compatible(cur)) {
    Lay last = choose(plan, p, p.gates.size(), true, precision);
    cur = last;
    prog.push_back(make_exch(cur, precision));
  }
  for (int i = 0; i < NB; i++) store_pos[i] = (uint8_t)cur.pos[i];
  if (g_anc_tb < 0) {
    merge_phase_polys(prog);
    merge_phase_fans(prog);
  }
  for (FOp& o : prog) assign_opcode(o);
}

}  // namespace ket
