// batch_vqe.cu -- vqe() energies of many parameterised circuits of uneven
// width in one persistent launch (ket_batch_vqe).
//
// The reference evaluates each energy on its own: vqe() (algorithms.ts:301-336)
// re-simulates the circuit per Pauli term, and a parameter sweep calls it once
// per parameter vector.  Here a batch names circuit templates (an op list whose
// parametric ops are bound to parameters, the same bindings as the adjoint
// gradient) and instances (a template and a parameter vector).  A persistent
// grid pulls instances from a queue, largest first; one CTA runs one instance
// with its whole state in shared memory (up to 13 qubits, 128 KB):
//   * |0...0>, then every op in order, with the reference's per-gate pruning
//     (accumulate(), statevector.ts:19-27) after each matrix op; parametric
//     matrices are formed on the device from the instance's parameters with
//     the formulas of gates.ts (Rx, Ry, Rz, U1, Gpi, Gpi2, their controlled
//     forms, Xx, Yy, Zz, Xy);
//   * E = ident + sum_t Re <psi| c_t P_t |psi> over the template's Pauli terms,
//     summed in a fixed order, so results repeat bit for bit.
// The launch (queue reset, kernel) is captured in a CUDA graph that is kept
// and replayed while the batch's shape and buffers stay the same; parameters
// are uploaded to the same addresses before each replay.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "launch.h"

namespace ket {
namespace {

constexpr int kVqeMaxQubits = 13;
constexpr int kVqeThreads = 256;

enum : uint8_t { BK_M1 = 0, BK_M2 = 1, BK_X = 2, BK_SWAP = 3 };

// One op of a template.  kind BK_M1: 2x2 on q0 with controls cmask (single,
// controlled, csrswap is BK_M2); BK_M2: 4x4 on q0 (MSB), q1 with controls;
// BK_X: X on q0 with controls (cnot, toffoli); BK_SWAP: swap q0, q1 with
// controls (swap, cswap).  fam >= 0: the matrix is G_fam(scale * theta[param]
// + shift); otherwise it is mats[moff ..].
struct BOp {
  uint8_t kind, q0, q1, prune;
  int16_t fam;
  int16_t pad;
  int32_t param;
  int32_t cmask;
  int64_t moff;
  double scale, shift;
};
static_assert(sizeof(BOp) == 40, "BOp layout");

struct BTmpl {
  int n, nops, nterms, pad;
  int64_t op_first, term_first;
  double ident;
};

struct BTerm {
  uint64_t flip, zm;
  double cre, cim;  // coeff * i^ny
};

struct BArgs {
  const BTmpl* tmpl;
  const BOp* ops;
  const double2* mats;
  const BTerm* terms;
  const int* inst_tmpl;
  const int* order;  // instances in launch order
  const double* theta;
  double* energy;
  unsigned int* next;
  int ninst, nparams;
};

// G_fam(a) into m (row-major, 2x2 or 4x4), the formulas of gates.ts.
__device__ void param_matrix(int fam, double a, double2* m) {
  double s, c;
  sincos(0.5 * a, &s, &c);
  const double sq2 = 0.70710678118654752440;
  switch (fam) {
    case KET_PG_RX: case KET_PG_CRX:
      m[0] = make_double2(c, 0); m[1] = make_double2(0, -s); m[2] = make_double2(0, -s); m[3] = make_double2(c, 0);
      return;
    case KET_PG_RY: case KET_PG_CRY:
      m[0] = make_double2(c, 0); m[1] = make_double2(-s, 0); m[2] = make_double2(s, 0); m[3] = make_double2(c, 0);
      return;
    case KET_PG_RZ: case KET_PG_CRZ:
      m[0] = make_double2(c, -s); m[1] = make_double2(0, 0); m[2] = make_double2(0, 0); m[3] = make_double2(c, s);
      return;
    case KET_PG_U1: case KET_PG_CU1: {
      double si, co;
      sincos(a, &si, &co);
      m[0] = make_double2(1, 0); m[1] = make_double2(0, 0); m[2] = make_double2(0, 0); m[3] = make_double2(co, si);
      return;
    }
    case KET_PG_GPI: {
      double si, co;
      sincos(a, &si, &co);
      m[0] = make_double2(0, 0); m[1] = make_double2(co, -si); m[2] = make_double2(co, si); m[3] = make_double2(0, 0);
      return;
    }
    case KET_PG_GPI2: {
      double si, co;
      sincos(a, &si, &co);
      m[0] = make_double2(sq2, 0); m[1] = make_double2(-sq2 * si, -sq2 * co);
      m[2] = make_double2(sq2 * si, -sq2 * co); m[3] = make_double2(sq2, 0);
      return;
    }
    default:
      break;
  }
  for (int k = 0; k < 16; k++) m[k] = make_double2(0, 0);
  if (fam == KET_PG_XX || fam == KET_PG_YY) {
    const double2 ni = make_double2(0, -s);
    const double2 corner = fam == KET_PG_XX ? ni : make_double2(0, s);
    m[0] = m[5] = m[10] = m[15] = make_double2(c, 0);
    m[3] = m[12] = corner;
    m[6] = m[9] = ni;
  } else if (fam == KET_PG_ZZ) {
    m[0] = m[15] = make_double2(c, -s);
    m[5] = m[10] = make_double2(c, s);
  } else {  // XY
    m[0] = m[15] = make_double2(1, 0);
    m[5] = m[10] = make_double2(c, 0);
    m[6] = m[9] = make_double2(0, s);
  }
}

__device__ __forceinline__ double2 cmac(double2 acc, double2 m, double2 x) {
  return make_double2(fma(m.x, x.x, fma(-m.y, x.y, acc.x)), fma(m.x, x.y, fma(m.y, x.x, acc.y)));
}

// accumulate()'s flush: |a|^2 < 1e-14 becomes an exact zero.
__device__ __forceinline__ double2 prune2(double2 v) {
  return norm2_ref(v.x, v.y) < 1e-14 ? make_double2(0.0, 0.0) : v;
}

// Shared-memory position of amplitude i: the three low index bits XORed with
// bits 3-5, so that pairs and quads on low qubits spread over the banks.
__device__ __forceinline__ uint32_t swz3(uint32_t i) { return i ^ ((i >> 3) & 7u); }

// The matrix of op k into m: formed from the instance's parameter, or copied.
__device__ __forceinline__ void op_matrix(const BArgs& a, const BOp& op, const double* th, double2* m) {
  if (op.fam >= 0) {
    param_matrix(op.fam, op.scale * th[op.param] + op.shift, m);
  } else {
    const int ne = op.kind == BK_M1 ? 4 : 16;
    for (int e = 0; e < ne; e++) m[e] = a.mats[op.moff + e];
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_batch_vqe(BArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* s = reinterpret_cast<double2*>(smraw);
  __shared__ double2 gm[2][16];  // the current op's matrix and the next one's
  __shared__ double red[32];
  __shared__ int item_sh;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) item_sh = (int)atomicAdd(a.next, 1u);
    __syncthreads();
    const int it = item_sh;
    __syncthreads();
    if (it >= a.ninst) break;
    const int inst = a.order[it];
    const BTmpl T = a.tmpl[a.inst_tmpl[inst]];
    const int n = T.n;
    const uint32_t N = 1u << n;
    const double* th = a.theta + (size_t)inst * a.nparams;
    for (uint32_t i = tid; i < N; i += NT) s[swz3(i)] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
    if (tid == 0 && T.nops > 0) {
      const BOp op0 = a.ops[T.op_first];
      if (op0.kind == BK_M1 || op0.kind == BK_M2) op_matrix(a, op0, th, gm[0]);
    }
    for (int k = 0; k < T.nops; k++) {
      const BOp op = a.ops[T.op_first + k];
      // one barrier per op: op k-1 is done with s and with gm[(k+1)&1], and
      // gm[k&1] (written during op k-1) is ready
      __syncthreads();
      if (tid == 0 && k + 1 < T.nops) {  // the next op's matrix, while this op runs
        const BOp nx = a.ops[T.op_first + k + 1];
        if (nx.kind == BK_M1 || nx.kind == BK_M2) op_matrix(a, nx, th, gm[(k + 1) & 1]);
      }
      const double2* M = gm[k & 1];
      const uint32_t cm = (uint32_t)op.cmask;
      const bool pr = op.prune != 0;
      if (op.kind == BK_M1 || op.kind == BK_X) {
        const int t = op.q0;
        for (uint32_t p = tid; p < N / 2; p += NT) {
          const uint32_t i0 = insert0_32(p, t), i1 = i0 | (1u << t);
          if ((i0 & cm) != cm) continue;
          const uint32_t a0 = swz3(i0), a1 = swz3(i1);
          const double2 x0 = s[a0], x1 = s[a1];
          if (op.kind == BK_X) {
            s[a0] = x1;
            s[a1] = x0;
          } else {
            double2 y0 = cmac(cmac(make_double2(0, 0), M[0], x0), M[1], x1);
            double2 y1 = cmac(cmac(make_double2(0, 0), M[2], x0), M[3], x1);
            if (pr) { y0 = prune2(y0); y1 = prune2(y1); }
            s[a0] = y0;
            s[a1] = y1;
          }
        }
      } else {
        const int qa = op.q0, qb = op.q1;
        const int lo = qa < qb ? qa : qb, hi = qa < qb ? qb : qa;
        for (uint32_t g = tid; g < N / 4; g += NT) {
          const uint32_t b0 = insert0_32(insert0_32(g, lo), hi);
          if ((b0 & cm) != cm) continue;
          const uint32_t i1 = b0 | (1u << qb), i2 = b0 | (1u << qa), i3 = i1 | i2;
          if (op.kind == BK_SWAP) {
            const double2 t1 = s[swz3(i1)];
            s[swz3(i1)] = s[swz3(i2)];
            s[swz3(i2)] = t1;
          } else {
            const uint32_t idx[4] = {swz3(b0), swz3(i1), swz3(i2), swz3(i3)};
            const double2 x[4] = {s[idx[0]], s[idx[1]], s[idx[2]], s[idx[3]]};
#pragma unroll
            for (int r = 0; r < 4; r++) {
              double2 y = make_double2(0, 0);
#pragma unroll
              for (int c = 0; c < 4; c++) y = cmac(y, M[4 * r + c], x[c]);
              s[idx[r]] = pr ? prune2(y) : y;
            }
          }
        }
      }
    }
    __syncthreads();
    double e = 0.0;
    for (int t = 0; t < T.nterms; t++) {
      const BTerm tm = a.terms[T.term_first + t];
      for (uint32_t y = tid; y < N; y += NT) {
        const uint32_t x = y ^ (uint32_t)tm.flip;
        const double2 v = s[swz3(x)], p = s[swz3(y)];
        const double sg = (__popc(x & (uint32_t)tm.zm) & 1) ? -1.0 : 1.0;
        const double lr = sg * (tm.cre * v.x - tm.cim * v.y), li = sg * (tm.cre * v.y + tm.cim * v.x);
        e += p.x * lr + p.y * li;
      }
    }
    e = block_sum<NT>(e, red);
    if (tid == 0) a.energy[inst] = e + T.ident;
  }
}

// Device image of the batch: offsets into the workspace.
struct Layout {
  size_t tmpl, ops, mats, terms, inst, order, theta, energy, next, total;
};

}  // namespace
}  // namespace ket

using namespace ket;

extern "C" int ket_batch_vqe(ket_ctx* c, int ntmpl, const ket_batch_template* tp, const ket_op* ops,
                             const double* mats, size_t nmat, const ket_param_binding* binds, const double* coeffs,
                             const char* pauli, int ninst, const int* inst_tmpl, const double* theta, int nparams,
                             int use_graph, double* energy) {
  if (!c || ntmpl < 0 || ninst < 0 || nparams < 0) return fail(KET_ERR_TYPE, "null context or negative count");
  if (ninst == 0) return KET_OK;
  if (!tp || !ops || !inst_tmpl || !energy || (nparams > 0 && !theta)) return fail(KET_ERR_TYPE, "null argument");
  cudaSetDevice(c->device);
  // ---- templates: validate and encode
  std::vector<BTmpl> bt(ntmpl);
  std::vector<BOp> bops;
  std::vector<BTerm> bterms;
  int maxn = 1;
  for (int j = 0; j < ntmpl; j++) {
    const ket_batch_template& T = tp[j];
    const int n = T.nqubits;
    if (n < 1 || n > kVqeMaxQubits)
      return fail(KET_ERR_UNSUPPORTED, "batch templates take 1.." + std::to_string(kVqeMaxQubits) +
                                           " qubits (one instance's state lives in shared memory)");
    if (T.nops < 0 || T.nbinds < 0 || T.nterms < 0 || T.op_first < 0 || T.bind_first < 0 || T.term_first < 0 ||
        T.pauli_first < 0)
      return fail(KET_ERR_TYPE, "template " + std::to_string(j) + ": negative count or offset");
    if (T.nterms > 0 && (!coeffs || !pauli)) return fail(KET_ERR_TYPE, "null Hamiltonian");
    if (T.nbinds > 0 && !binds) return fail(KET_ERR_TYPE, "null bindings");
    const ket_op* to = ops + T.op_first;
    {  // RangeError / TypeError as the reference's builder (circuit.ts:1113-1146)
      std::vector<Gate> chk;
      std::string err;
      const int rc = lower_ops(n, to, (size_t)T.nops, mats, nmat, true, chk, err);
      if (rc) return fail(rc, "template " + std::to_string(j) + ": " + err);
    }
    std::vector<int> bind_of(T.nops, -1);
    for (int b = 0; b < T.nbinds; b++) {
      const ket_param_binding& pb = binds[T.bind_first + b];
      if (pb.op < 0 || pb.op >= T.nops) return fail(KET_ERR_RANGE, "binding op index out of range");
      if (pb.param < 0 || pb.param >= nparams) return fail(KET_ERR_RANGE, "binding parameter index out of range");
      if (pb.gate < KET_PG_RX || pb.gate > KET_PG_XY) return fail(KET_ERR_TYPE, "unknown parametric gate");
      const int want = (pb.gate >= KET_PG_CRX && pb.gate <= KET_PG_CU1) ? KET_OP_CONTROLLED
                       : pb.gate >= KET_PG_XX                           ? KET_OP_TWO
                                                                        : KET_OP_SINGLE;
      if (to[pb.op].kind != want) return fail(KET_ERR_TYPE, "binding gate does not match the op kind");
      if (bind_of[pb.op] >= 0) return fail(KET_ERR_TYPE, "an op has two bindings");
      bind_of[pb.op] = b;
    }
    BTmpl& B = bt[j];
    B.n = n;
    B.op_first = (int64_t)bops.size();
    for (int k = 0; k < T.nops; k++) {
      const ket_op& op = to[k];
      BOp o;
      memset(&o, 0, sizeof(o));
      o.fam = -1;
      o.param = -1;
      o.prune = 1;
      const int* q = op.q;
      switch (op.kind) {
        case KET_OP_BARRIER: continue;
        case KET_OP_SINGLE: o.kind = BK_M1; o.q0 = (uint8_t)q[0]; o.moff = op.mat; break;
        case KET_OP_CONTROLLED: o.kind = BK_M1; o.q0 = (uint8_t)q[1]; o.cmask = 1 << q[0]; o.moff = op.mat; break;
        case KET_OP_TWO: o.kind = BK_M2; o.q0 = (uint8_t)q[0]; o.q1 = (uint8_t)q[1]; o.moff = op.mat; break;
        case KET_OP_CNOT: o.kind = BK_X; o.q0 = (uint8_t)q[1]; o.cmask = 1 << q[0]; break;
        case KET_OP_TOFFOLI: o.kind = BK_X; o.q0 = (uint8_t)q[2]; o.cmask = (1 << q[0]) | (1 << q[1]); break;
        case KET_OP_SWAP: o.kind = BK_SWAP; o.q0 = (uint8_t)q[0]; o.q1 = (uint8_t)q[1]; break;
        case KET_OP_CSWAP: o.kind = BK_SWAP; o.q0 = (uint8_t)q[1]; o.q1 = (uint8_t)q[2]; o.cmask = 1 << q[0]; break;
        case KET_OP_CSRSWAP:  // sqrt(iSWAP) on (q1, q2) when q0 is set (applyCsrSwap, statevector.ts:177-207)
          o.kind = BK_M2; o.q0 = (uint8_t)q[1]; o.q1 = (uint8_t)q[2]; o.cmask = 1 << q[0]; o.moff = -1; break;
        case KET_OP_UNITARY:
          if (op.nq == 1) { o.kind = BK_M1; o.q0 = (uint8_t)q[0]; o.moff = op.mat; break; }
          if (op.nq == 2) { o.kind = BK_M2; o.q0 = (uint8_t)q[0]; o.q1 = (uint8_t)q[1]; o.moff = op.mat; break; }
          return fail(KET_ERR_UNSUPPORTED, "batch templates take unitaries of 1 or 2 qubits");
        default:
          return fail(KET_ERR_UNSUPPORTED, "batch templates take pure gate ops only (no measure, reset or if)");
      }
      const int b = bind_of[k];
      if (b >= 0) {
        const ket_param_binding& pb = binds[T.bind_first + b];
        o.fam = (int16_t)pb.gate;
        o.param = pb.param;
        o.scale = pb.scale;
        o.shift = pb.shift;
      } else if (o.kind == BK_M1 || o.kind == BK_M2) {
        const int64_t need = o.kind == BK_M1 ? 4 : 16;
        if (o.moff != -1 && (o.moff < 0 || (size_t)(o.moff + need) > nmat))
          return fail(KET_ERR_TYPE, "op matrix offset out of bounds");
      }
      bops.push_back(o);
    }
    B.nops = (int)((int64_t)bops.size() - B.op_first);
    // Hamiltonian (PauliTerm convention: ops[0] acts on qubit n-1; |coeff| < 1e-15 skipped,
    // identity terms add their coeff, algorithms.ts:283-336)
    B.term_first = (int64_t)bterms.size();
    B.ident = 0.0;
    for (int t = 0; t < T.nterms; t++) {
      const double cf = coeffs[T.term_first + t];
      const char* ps = pauli + T.pauli_first + (int64_t)t * n;
      for (int q = 0; q < n; q++)
        if (ps[q] == 0) return fail(KET_ERR_TYPE, "ops length must equal ansatz.qubits (" + std::to_string(n) + ")");
      if (std::fabs(cf) < 1e-15) continue;
      uint64_t flip = 0, zm = 0;
      int ny = 0;
      bool any = false;
      for (int q = 0; q < n; q++) {
        const char ch = (char)toupper((unsigned char)ps[n - 1 - q]);
        if (ch == 'I') continue;
        any = true;
        if (ch == 'X' || ch == 'Y') flip |= uint64_t(1) << q;
        if (ch != 'X') zm |= uint64_t(1) << q;
        if (ch == 'Y') ny++;
      }
      if (!any) { B.ident += cf; continue; }
      static const double pr[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};  // i^ny
      bterms.push_back(BTerm{flip, zm, cf * pr[ny & 3][0], cf * pr[ny & 3][1]});
    }
    B.nterms = (int)((int64_t)bterms.size() - B.term_first);
    maxn = std::max(maxn, n);
  }
  // the csrswap block, appended to the matrices
  std::vector<double> dm(mats ? mats : nullptr, mats ? mats + 2 * nmat : nullptr);
  const int64_t csr_off = (int64_t)(dm.size() / 2);
  {
    const double h = 1.0 / std::sqrt(2.0);
    double blk[32] = {0};
    blk[0] = 1; blk[2 * 5] = h; blk[2 * 6 + 1] = h; blk[2 * 9 + 1] = h; blk[2 * 10] = h; blk[2 * 15] = 1;
    dm.insert(dm.end(), blk, blk + 32);
  }
  for (BOp& o : bops)
    if ((o.kind == BK_M1 || o.kind == BK_M2) && o.fam < 0 && o.moff == -1) o.moff = csr_off;
  // ---- instances, largest first
  std::vector<int> order(ninst);
  for (int i = 0; i < ninst; i++) {
    if (inst_tmpl[i] < 0 || inst_tmpl[i] >= ntmpl) return fail(KET_ERR_RANGE, "instance template index out of range");
    order[i] = i;
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const BTmpl &X = bt[inst_tmpl[x]], &Y = bt[inst_tmpl[y]];
    return ((int64_t)X.nops << X.n) > ((int64_t)Y.nops << Y.n);
  });
  // ---- workspace
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  Layout L;
  L.tmpl = 0;
  L.ops = L.tmpl + al(sizeof(BTmpl) * std::max(ntmpl, 1));
  L.mats = L.ops + al(sizeof(BOp) * std::max<size_t>(bops.size(), 1));
  L.terms = L.mats + al(8 * dm.size());
  L.inst = L.terms + al(sizeof(BTerm) * std::max<size_t>(bterms.size(), 1));
  L.order = L.inst + al(4 * (size_t)ninst);
  L.theta = L.order + al(4 * (size_t)ninst);
  L.energy = L.theta + al(8 * std::max<size_t>((size_t)ninst * nparams, 1));
  L.next = L.energy + al(8 * (size_t)ninst);
  L.total = L.next + 256;
  if (c->vqe_work_bytes < L.total) {
    int rc = ctx_wait(c);
    if (rc) return rc;
    if (c->vqe_graph_exec) { cudaGraphExecDestroy(c->vqe_graph_exec); c->vqe_graph_exec = nullptr; }
    c->vqe_graph_key = 0;
    if (c->vqe_work) cudaFree(c->vqe_work);
    c->vqe_work = nullptr;
    c->vqe_work_bytes = 0;
    rc = dev_alloc(&c->vqe_work, L.total);
    if (rc) return rc;
    c->vqe_work_bytes = L.total;
  }
  char* base = (char*)c->vqe_work;
  std::vector<unsigned char> img(L.theta, 0);  // everything before the parameters, one copy
  memcpy(img.data() + L.tmpl, bt.data(), sizeof(BTmpl) * ntmpl);
  if (!bops.empty()) memcpy(img.data() + L.ops, bops.data(), sizeof(BOp) * bops.size());
  memcpy(img.data() + L.mats, dm.data(), 8 * dm.size());
  if (!bterms.empty()) memcpy(img.data() + L.terms, bterms.data(), sizeof(BTerm) * bterms.size());
  memcpy(img.data() + L.inst, inst_tmpl, 4 * (size_t)ninst);
  memcpy(img.data() + L.order, order.data(), 4 * (size_t)ninst);
  cudaError_t e = cudaMemcpyAsync(base, img.data(), img.size(), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess && nparams > 0)
    e = cudaMemcpyAsync(base + L.theta, theta, 8 * (size_t)ninst * nparams, cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(batch)");
  c->h2d_bytes += img.size() + 8 * (size_t)ninst * nparams;
  BArgs a;
  a.tmpl = (const BTmpl*)(base + L.tmpl);
  a.ops = (const BOp*)(base + L.ops);
  a.mats = (const double2*)(base + L.mats);
  a.terms = (const BTerm*)(base + L.terms);
  a.inst_tmpl = (const int*)(base + L.inst);
  a.order = (const int*)(base + L.order);
  a.theta = (const double*)(base + L.theta);
  a.energy = (double*)(base + L.energy);
  a.next = (unsigned int*)(base + L.next);
  a.ninst = ninst;
  a.nparams = nparams;
  // ---- launch: a resident grid sized for the widest template's shared memory
  const size_t smem = size_t(16) << maxn;
  static std::atomic<uint64_t> attr_set{0};
  const uint64_t bit = uint64_t(1) << (c->device & 63);
  if (!(attr_set.load() & bit)) {
    e = cudaFuncSetAttribute(k_batch_vqe<kVqeThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             16 << kVqeMaxQubits);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(k_batch_vqe)");
    attr_set.fetch_or(bit);
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_vqe<kVqeThreads>, kVqeThreads, smem);
  const int grid = std::max(1, std::min(num_sms() * std::max(1, per_sm), ninst));
  auto record = [&]() -> cudaError_t {
    cudaMemsetAsync(a.next, 0, 4, c->stream);
    k_batch_vqe<kVqeThreads><<<grid, kVqeThreads, smem, c->stream>>>(a);
    return cudaGetLastError();
  };
  prof_begin(c);
  if (!use_graph) {
    e = record();
  } else {
    uint64_t key = 1469598103934665603ull;
    auto mix = [&](const void* p, size_t nb) {
      for (size_t i = 0; i < nb; i++) key = (key ^ ((const unsigned char*)p)[i]) * 1099511628211ull;
    };
    mix(&a, sizeof(a));
    mix(&smem, sizeof(smem));
    mix(&grid, sizeof(grid));
    if (c->vqe_graph_exec && c->vqe_graph_key == key) {
      e = cudaGraphLaunch(c->vqe_graph_exec, c->stream);
    } else {
      cudaGraph_t graph;
      e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t er = record();
        e = cudaStreamEndCapture(c->stream, &graph);
        if (er != cudaSuccess) e = er;
      }
      if (e == cudaSuccess) {
        if (c->vqe_graph_exec) { cudaGraphExecDestroy(c->vqe_graph_exec); c->vqe_graph_exec = nullptr; }
        c->vqe_graph_key = 0;
        e = cudaGraphInstantiate(&c->vqe_graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e == cudaSuccess) {
          c->vqe_graph_key = key;
          e = cudaGraphLaunch(c->vqe_graph_exec, c->stream);
        }
      }
    }
  }
  prof_end(c, PK_BATCH);
  if (e != cudaSuccess) return cuda_fail(e, "batch vqe launch");
  e = cudaMemcpyAsync(energy, a.energy, 8 * (size_t)ninst, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(energy)");
  c->d2h_bytes += 8 * (size_t)ninst;
  return ctx_wait(c);
}
