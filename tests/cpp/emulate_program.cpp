// emulate_program.cpp -- TEST INFRASTRUCTURE: executes the fused-pass programs
// that the engine's planner emits (ket_b200/csrc/planner.cpp, program.cpp) on
// host arrays, following the semantics of the k_fused2 kernel op by op
// (layouts, exchanges, register / lane / diagonal / shared-memory
// ops, controls).  The tests compare it with direct gate-by-gate application,
// so planner and program-generator bugs show up without a GPU.
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "launch.h"

namespace ket {
int num_sms() { return 148; }
}

using namespace ket;
typedef std::complex<double> cx;

namespace {

// Thread/slot shape of the layouts being emulated: NR register bits, NW warp bits.
int NR = KET_FUSED_NREG, NW = 7 - KET_FUSED_NREG, NTH = 32 << (7 - KET_FUSED_NREG), NS = 1 << KET_FUSED_NREG;

struct Lay {
  std::vector<uint32_t> tbase;  // per thread
  uint32_t rp[KET_NR_MAX];
};

Lay make_lay(const uint8_t* pos) {
  Lay L;
  L.tbase.assign(NTH, 0);
  for (int t = 0; t < NTH; t++) {
    int lane = t & 31, warp = t >> 5;
    uint32_t v = 0;
    for (int l = 0; l < 5; l++) v |= (uint32_t)((lane >> l) & 1) << pos[l];
    for (int w = 0; w < NW; w++) v |= (uint32_t)((warp >> w) & 1) << pos[5 + w];
    L.tbase[t] = v;
  }
  for (int k = 0; k < NR; k++) L.rp[k] = 1u << pos[5 + NW + k];
  return L;
}

uint32_t rofs(const Lay& L, int j) {
  uint32_t o = 0;
  for (int k = 0; k < NR; k++)
    if ((j >> k) & 1) o |= L.rp[k];
  return o;
}

void prune(cx& a) {
  double n2 = a.real() * a.real() + a.imag() * a.imag();
  if (n2 < 1e-14) a = 0.0;
}

uint32_t slotmask(uint32_t creg) {
  uint32_t v = 0;
  for (int j = 0; j < NS; j++)
    if (((uint32_t)j & creg) == creg) v |= 1u << j;
  return v;
}

const double* record_data(const std::vector<FOp>& prog, size_t k) {
  return reinterpret_cast<const double*>(reinterpret_cast<const unsigned char*>(&prog[k]) + 16);
}

// Ops of each FOpType in the programs emulated since the last reset.
int64_t g_type_count[32];
// 1: emulate the compiled kernels' deferred register swaps (FOF_SW, FO_REAL:
// physical slot j of thread t holds logical slot j ^ sw[t]); 0: the
// interpreter's, which carries every swap out at once and ignores both.
int g_deferred = 1;
int64_t g_sw_count = 0;  // ops with FOF_SW in the programs emulated since the last reset
int g_lane_error = 0;    // a lane op met lanes moved by deferred lane X gates
int64_t g_lane_defer_count = 0;  // deferred lane X gates in the programs emulated since the last reset

void run_pass(const Plan& plan, const Pass& p, int n, bool prunef, cx* amp) {
  std::vector<FOp> prog;
  uint8_t lp[KET_T2_BITS], sp[KET_T2_BITS];
  plan_program(plan, p, KET_C128, prunef, NR, prog, lp, sp);
  for (const FOp& o : prog) {
    g_type_count[o.type & 31]++;
    if (o.type != FO_CONT && (o.flags & FOF_SW)) g_sw_count++;
    if (o.type == FO_X1L && (o.flags & FOF_SW)) g_lane_defer_count++;
  }
  const int L = p.L;
  auto gq = [&](int tb) { return tb < L ? tb : p.hbits[tb - L]; };
  uint64_t S = (uint64_t(1) << L) - 1;
  for (int q : p.hbits) S |= uint64_t(1) << q;
  std::vector<int> ctxbits;
  for (int q = 0; q < n; q++)
    if (!((S >> q) & 1)) ctxbits.push_back(q);
  const uint64_t ntiles = uint64_t(1) << (n - KET_T2_BITS);
  std::vector<cx> x(NTH * NS), sm(4096);
  auto gaddr = [&](uint64_t ctx, uint32_t tidx) {
    uint64_t g = ctx;
    for (int b = 0; b < KET_T2_BITS; b++)
      if ((tidx >> b) & 1) g |= uint64_t(1) << gq(b);
    return g;
  };
  for (uint64_t tile = 0; tile < ntiles; tile++) {
    uint64_t ctx = 0;
    for (size_t j = 0; j < ctxbits.size(); j++)
      if ((tile >> j) & 1) ctx |= uint64_t(1) << ctxbits[j];
    Lay Lc = make_lay(lp);
    for (int t = 0; t < NTH; t++)
      for (int j = 0; j < NS; j++) x[t * NS + j] = amp[gaddr(ctx, Lc.tbase[t] | rofs(Lc, j))];
    std::vector<uint32_t> sw(NTH, 0);
    // logical thread ids: deferred lane X gates (FOF_SW on FO_X1L) move the
    // lane bits of a thread's logical id, not its amplitudes
    std::vector<int> lt(NTH);
    for (int t = 0; t < NTH; t++) lt[t] = t;
    // move every thread's amplitudes to its logical thread (as the kernel's
    // logical-lane addressing of exchanges and stores does)
    auto lanes_home = [&]() {
      std::vector<cx> v = x;
      for (int t = 0; t < NTH; t++) {
        for (int j = 0; j < NS; j++) x[lt[t] * NS + j] = v[t * NS + j];
      }
      std::vector<uint32_t> s2(NTH);
      for (int t = 0; t < NTH; t++) s2[lt[t]] = sw[t];
      sw = s2;
      for (int t = 0; t < NTH; t++) lt[t] = t;
    };
    // carry out the pending swaps of register bits m (physical slot order = logical)
    auto realize = [&](uint32_t m) {
      for (int t = 0; t < NTH; t++) {
        const uint32_t s = sw[t] & m;
        if (!s) continue;
        std::vector<cx> v(x.begin() + t * NS, x.begin() + (t + 1) * NS);
        for (int j = 0; j < NS; j++) x[t * NS + (j ^ s)] = v[j];
        sw[t] &= ~m;
      }
    };
    for (size_t oi = 0; oi < prog.size(); oi++) {
      const FOp& op = prog[oi];
      if (op.type == FO_REAL) {
        realize(op.creg);
        continue;
      }
      if (op.type == FO_RELAY) {  // the data stays; the layout names its bits anew
        Lc = make_lay(op.pos);
        continue;
      }
      if (op.type == FO_SYNC) continue;  // a barrier: nothing to emulate
      // the kernel's exchanges and shared-memory ops write the logical slots
      const bool smem_x1 = op.type == FO_X1R && op.creg && ((op.creg & (op.creg - 1)) || op.cthr || op.cctx);
      if (op.type == FO_EXCH || op.type == FO_SWAPS || op.type == FO_MAT2S || op.type == FO_DIAG || smem_x1) {
        realize(0xffffffffu);
        lanes_home();
      }
      // a lane op needs the partner lanes in place: the program generator
      // defers no lane X before one
      if (op.type == FO_MAT1L || (op.type == FO_X1L && !(g_deferred && (op.flags & FOF_SW)))) {
        for (int t = 0; t < NTH; t++)
          if (lt[t] != t) g_lane_error = 1;
      }
      if (op.type == FO_CPHASE) {
        // phase fan on register bit a: T[k] * prod H[thread bits] * exp(i sum ctx angles)
        const double* H = record_data(prog, oi + 1);
        double th = 0.0;
        for (uint32_t t = 0; t < op.lmask; t++) {
          const size_t rec = t / KET_CPHASE_TERMS_PER_RECORD, w = t % KET_CPHASE_TERMS_PER_RECORD;
          const double* rd = record_data(prog, oi + 2 + rec);
          uint64_t mk;
          memcpy(&mk, &rd[2 * w + 1], 8);
          if (ctx & mk) th += rd[2 * w];
        }
        const cx E = std::polar(1.0, th);
        for (int t = 0; t < NTH; t++) {
          cx F = E;
          for (int sb = 0; sb < 8; sb++)
            if ((lt[t] >> sb) & 1) F *= cx(H[2 * sb], H[2 * sb + 1]);
          for (int j = 0; j < NS; j++) {
            if (!((j >> op.a) & 1)) continue;
            const int k = ((j >> (op.a + 1)) << op.a) | (j & ((1 << op.a) - 1));
            x[t * NS + j] *= cx(op.m[2 * k], op.m[2 * k + 1]) * F;
          }
        }
        oi += op.ctile;
        continue;
      }
      if (op.type == FO_PPOLY) {
        // group products over the matching terms, then per thread and register bit
        const uint32_t* cnt = reinterpret_cast<const uint32_t*>(op.m);
        const PPolyGroup* desc =
            reinterpret_cast<const PPolyGroup*>(reinterpret_cast<const unsigned char*>(op.m) + 32);
        std::vector<cx> K(op.lmask, cx(1.0, 0.0));
        for (uint32_t g = 0; g < op.lmask; g++)
          for (uint32_t k = 0; k < desc[g].n; k++) {
            const size_t rec = desc[g].rec + k / KET_PPOLY_TERMS_PER_RECORD;
            const PPolyTerm& tm =
                reinterpret_cast<const PPolyTerm*>(record_data(prog, oi + rec))[k % KET_PPOLY_TERMS_PER_RECORD];
            if ((ctx & tm.cm) == tm.cm) K[g] *= cx(tm.re, tm.im);
          }
        for (int t = 0; t < NTH; t++) {
          uint32_t g = 0;
          for (int seg = 0; seg <= KET_NR_MAX; seg++) {
            if (!cnt[seg]) continue;
            cx f(1.0, 0.0);
            for (uint32_t k = 0; k < cnt[seg]; k++, g++)
              if (((uint32_t)lt[t] & desc[g].tm) == desc[g].tm) f *= K[g];
            for (int j = 0; j < NS; j++)
              if (seg == 0 || ((j >> (seg - 1)) & 1)) x[t * NS + j] *= f;
          }
        }
        oi += op.ctile;
        continue;
      }
      if (op.type == FO_EXCH) {
        for (int t = 0; t < NTH; t++)
          for (int j = 0; j < NS; j++) sm[Lc.tbase[t] | rofs(Lc, j)] = x[t * NS + j];
        Lc = make_lay(op.pos);
        for (int t = 0; t < NTH; t++)
          for (int j = 0; j < NS; j++) x[t * NS + j] = sm[Lc.tbase[t] | rofs(Lc, j)];
        continue;
      }
      if ((ctx & op.cctx) != op.cctx) continue;
      const bool pr = op.flags & FOF_PRUNE;
      const bool dfr = g_deferred && (op.flags & FOF_SW);
      if (dfr && op.type == FO_X1R && !op.creg) {
        for (int t = 0; t < NTH; t++)
          if ((uint32_t)(lt[t] & op.cthr) == op.cthr) sw[t] ^= 1u << op.a;
        continue;
      }
      if (dfr && op.type == FO_X1L) {  // a deferred lane X: the logical ids move
        for (int t = 0; t < NTH; t++)
          if ((uint32_t)(lt[t] & op.cthr) == op.cthr) lt[t] ^= 1 << op.a;
        continue;
      }
      std::vector<cx> nx = x;
      for (int t = 0; t < NTH; t++) {
        const uint32_t sm_ = ((uint32_t)(lt[t] & op.cthr) == op.cthr) ? slotmask(op.creg) : 0;
        cx* xt = &x[t * NS];
        cx* nt = &nx[t * NS];
        const int lane = t & 31;
        // a 2x2 or diagonal on a register bit whose slot pairs this thread has exchanged
        const bool xs = dfr && (op.type == FO_MAT1R || op.type == FO_DIAGR) && ((sw[t] >> op.a) & 1);
        const cx m0(op.m[xs ? 6 : 0], op.m[xs ? 7 : 1]), m1(op.m[xs ? 4 : 2], op.m[xs ? 5 : 3]),
            m2(op.m[xs ? 2 : 4], op.m[xs ? 3 : 5]), m3(op.m[xs ? 0 : 6], op.m[xs ? 1 : 7]);
        // the diagonal's two entries
        const cx d0(op.m[xs ? 2 : 0], op.m[xs ? 3 : 1]), d1(op.m[xs ? 0 : 2], op.m[xs ? 1 : 3]);
        switch (op.type) {
          case FO_MAT1R: case FO_X1R:
            for (int j = 0; j < NS; j++) {
              if ((j >> op.a) & 1) continue;
              int j1 = j | (1 << op.a);
              if (!((sm_ >> j) & 1)) continue;
              if (op.type == FO_X1R) { nt[j] = xt[j1]; nt[j1] = xt[j]; continue; }
              nt[j] = m0 * xt[j] + m1 * xt[j1];
              nt[j1] = m2 * xt[j] + m3 * xt[j1];
            }
            break;
          case FO_MAT1L: case FO_X1L: {
            int bitv = (lane >> op.a) & 1;
            const cx* pt = &x[(t ^ (1 << op.a)) * NS];
            for (int j = 0; j < NS; j++) {
              if (!((sm_ >> j) & 1)) continue;
              if (op.type == FO_X1L) { nt[j] = pt[j]; continue; }
              nt[j] = bitv ? (m2 * pt[j] + m3 * xt[j]) : (m0 * xt[j] + m1 * pt[j]);
            }
            break;
          }
          case FO_DIAGR:
            for (int j = 0; j < NS; j++)
              if ((sm_ >> j) & 1) nt[j] = ((j >> op.a) & 1 ? d1 : d0) * xt[j];
            break;
          case FO_DIAGT: case FO_DIAGX: {
            bool one = op.type == FO_DIAGT ? ((lt[t] >> op.a) & 1) : ((ctx & op.dg0) != 0);
            for (int j = 0; j < NS; j++)
              if ((sm_ >> j) & 1) nt[j] = (one ? d1 : d0) * xt[j];
            break;
          }
          case FO_DIAG: {
            // d0, d1: tile bits, -1 = outside the tile; controls as a tile-bit mask
            for (int j = 0; j < NS; j++) {
              uint32_t idx = Lc.tbase[t] | rofs(Lc, j);
              if ((idx & op.ctile) != op.ctile) continue;
              int k0 = op.d0 >= 0 ? (int)((idx >> op.d0) & 1) : (int)((ctx & op.dg0) != 0);
              int k1 = op.d1 >= 0 ? (int)((idx >> op.d1) & 1) : (int)((ctx & op.dg1) != 0);
              int kk = 2 * k0 + k1;
              nt[j] = cx(op.m[2 * kk], op.m[2 * kk + 1]) * xt[j];
            }
            break;
          }
          default: break;
        }
      }
      if (op.type == FO_SWAPS || op.type == FO_MAT2S) {
        for (int t = 0; t < NTH; t++)
          for (int j = 0; j < NS; j++) sm[Lc.tbase[t] | rofs(Lc, j)] = x[t * NS + j];
        const int ta = op.a, tb = op.b, lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
        for (uint32_t g = 0; g < 1024; g++) {
          uint32_t lo_m = (1u << lo) - 1;
          uint32_t b0 = ((g & ~lo_m) << 1) | (g & lo_m);
          uint32_t hi_m = (1u << hi) - 1;
          b0 = ((b0 & ~hi_m) << 1) | (b0 & hi_m);
          if ((b0 & op.ctile) != op.ctile) continue;
          uint32_t idx[4] = {b0, b0 | (1u << tb), b0 | (1u << ta), b0 | (1u << ta) | (1u << tb)};
          if (op.type == FO_SWAPS) { std::swap(sm[idx[1]], sm[idx[2]]); continue; }
          cx v[4] = {sm[idx[0]], sm[idx[1]], sm[idx[2]], sm[idx[3]]};
          for (int r = 0; r < 4; r++) {
            cx y = 0;
            for (int c = 0; c < 4; c++) y += cx(op.m[8 * r + 2 * c], op.m[8 * r + 2 * c + 1]) * v[c];
            if (pr) prune(y);
            sm[idx[r]] = y;
          }
        }
        for (int t = 0; t < NTH; t++)
          for (int j = 0; j < NS; j++) nx[t * NS + j] = sm[Lc.tbase[t] | rofs(Lc, j)];
        x = nx;
        continue;
      }
      if (pr)
        for (auto& v : nx) prune(v);
      x = nx;
      if (dfr && op.type == FO_X1R && op.creg) {
        // X1RC on a deferred control bit C: flipping every pair along a adds the other half
        const int c = __builtin_ctz(op.creg);
        for (int t = 0; t < NTH; t++)
          if ((uint32_t)(lt[t] & op.cthr) == op.cthr) sw[t] ^= ((sw[t] >> c) & 1u) << op.a;
      }
    }
    realize(0xffffffffu);  // the store writes the logical slots and lanes
    lanes_home();
    Lay Ls = make_lay(sp);
    for (int t = 0; t < NTH; t++)
      for (int j = 0; j < NS; j++) amp[gaddr(ctx, Ls.tbase[t] | rofs(Ls, j))] = x[t * NS + j];
  }
}

}  // namespace

extern "C" {

// Apply ops to the n-qubit state re_im (interleaved) through the planner's
// fused programs, emulated.  Returns 0, or the lowering status; passes[0] =
// emulated register-tiled passes, passes[1] = other passes (not emulated: -1).
int emu_apply_nreg(int n, const ket_op* ops, size_t nops, const double* mats, size_t nmat, int prune, int fusion,
                   double* re_im, int64_t* passes, int nreg) {
  NR = nreg;
  NW = 7 - nreg;
  NTH = 32 << NW;
  NS = 1 << NR;
  Plan plan;
  std::string err;
  int rc = lower_ops(n, ops, nops, mats, nmat, prune != 0, plan.gates, err);
  if (rc) return rc;
  if (fusion != 0) fold_single_qubit(plan.gates, prune != 0);
  plan_passes(n, KET_C128, fusion, prune != 0, plan);
  cx* amp = reinterpret_cast<cx*>(re_im);
  passes[0] = passes[1] = 0;
  memset(g_type_count, 0, sizeof g_type_count);
  g_sw_count = 0;
  g_lane_error = 0;
  g_lane_defer_count = 0;
  for (const Pass& p : plan.passes) {
    if (!(p.fused && p.m == KET_T2_BITS && n >= KET_T2_BITS)) { passes[1]++; return -1; }
    run_pass(plan, p, n, prune != 0, amp);
    passes[0]++;
  }
  return g_lane_error ? -2 : 0;
}

// Ops of FOpType `type` in the programs of the last emu_apply call.
int64_t emu_type_count(int type) { return g_type_count[type & 31]; }

// 1 (the default): deferred register swaps as the compiled kernels run them; 0: as the interpreter.
void emu_set_deferred(int on) { g_deferred = on; }
int64_t emu_sw_count() { return g_sw_count; }
int64_t emu_lane_defer_count() { return g_lane_defer_count; }

int emu_apply(int n, const ket_op* ops, size_t nops, const double* mats, size_t nmat, int prune, int fusion,
              double* re_im, int64_t* passes) {
  return emu_apply_nreg(n, ops, nops, mats, nmat, prune, fusion, re_im, passes, KET_FUSED_NREG);
}

// Plan an op list as a run on an n-qubit state would (automatic fusion) and
// digest, with 64-bit FNV-1a, every register-tiled pass's load and store
// layouts and program bytes in order; nothing is emulated, so n may be 30.
// out[0] = the digest, out[1] = tiled passes, out[2] = program ops.
int emu_plan_digest(int n, int precision, const ket_op* ops, size_t nops, const double* mats, size_t nmat, int prune,
                    int nreg, uint64_t* out) {
  Plan plan;
  std::string err;
  int rc = lower_ops(n, ops, nops, mats, nmat, prune != 0, plan.gates, err);
  if (rc) return rc;
  fold_single_qubit(plan.gates, prune != 0);
  plan_passes(n, precision, -1, prune != 0, plan);
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&h](const void* d, size_t b) {
    const unsigned char* c = static_cast<const unsigned char*>(d);
    for (size_t i = 0; i < b; i++) { h ^= c[i]; h *= 0x100000001b3ull; }
  };
  out[1] = out[2] = 0;
  for (const Pass& p : plan.passes) {
    if (!(p.fused && p.m == KET_T2_BITS && n >= KET_T2_BITS)) continue;
    std::vector<FOp> prog;
    uint8_t lp[KET_T2_BITS], sp[KET_T2_BITS];
    plan_program(plan, p, precision, prune != 0, nreg, prog, lp, sp);
    mix(lp, sizeof lp);
    mix(sp, sizeof sp);
    if (!prog.empty()) mix(prog.data(), prog.size() * sizeof(FOp));
    out[1]++;
    out[2] += prog.size();
  }
  out[0] = h;
  return 0;
}

// The same digest for an adjoint-style reverse plan on n + 1 qubits: the
// lowered gates in reverse order, the ancilla on qubit n, and after every
// one-qubit matrix gate a 2x2 probe (G_GRADM) on its target, after every
// one-qubit diagonal a diagonal probe (G_GRADD); probe passes keep their
// order, pruning is off, as in the adjoint sweep.
int emu_adjoint_plan_digest(int n, const ket_op* ops, size_t nops, const double* mats, size_t nmat, int nreg,
                            uint64_t* out) {
  Plan fwd;
  std::string err;
  int rc = lower_ops(n, ops, nops, mats, nmat, false, fwd.gates, err);
  if (rc) return rc;
  Plan plan;
  plan.anc = n;
  int slot = 0;
  for (size_t k = fwd.gates.size(); k-- > 0;) {
    const Gate& g = fwd.gates[k];
    plan.gates.push_back(g);
    if (g.type != G_MAT1 && g.type != G_DIAG1) continue;
    Gate pr;
    pr.type = g.type == G_MAT1 ? G_GRADM : G_GRADD;
    pr.t0 = g.t0;
    pr.cmask = g.cmask;
    pr.slot = slot++;
    for (int q = 0; q < 4; q++) pr.m[q] = g.m[q];
    plan.gates.push_back(pr);
  }
  plan_passes(n + 1, KET_C128, -1, false, plan);
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&h](const void* d, size_t b) {
    const unsigned char* c = static_cast<const unsigned char*>(d);
    for (size_t i = 0; i < b; i++) { h ^= c[i]; h *= 0x100000001b3ull; }
  };
  out[1] = out[2] = 0;
  for (const Pass& p : plan.passes) {
    if (!(p.fused && p.m == KET_T2_BITS)) continue;
    std::vector<FOp> prog;
    uint8_t lp[KET_T2_BITS], sp[KET_T2_BITS];
    plan_program(plan, p, KET_C128, false, nreg, prog, lp, sp);
    mix(lp, sizeof lp);
    mix(sp, sizeof sp);
    if (!prog.empty()) mix(prog.data(), prog.size() * sizeof(FOp));
    out[1]++;
    out[2] += prog.size();
  }
  out[0] = h;
  return 0;
}
}
