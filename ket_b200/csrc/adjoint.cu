// adjoint.cu -- adjoint (reverse-sweep) gradients of <psi(theta)|H|psi(theta)>
// and the parameter-shift reference, behind ket_adjoint_gradient and
// ket_shift_gradient.
//
// The reference differentiates by parameter shift (algorithms.ts:536-547):
// 2P energy evaluations, each a full re-simulation.  Here one forward pass
// builds psi = U|init>, lambda = H psi, and one reverse sweep walks the gates
// backwards, un-applying each to psi and lambda and reading every parameter's
// derivative as 2 Re <lambda| G^dagger dG |psi> on the way.
//
// psi and lambda live in one buffer of 2^(n+1) amplitudes whose top qubit n
// selects psi (0) or lambda (1); un-applying a gate to that (n+1)-qubit state
// un-applies it to both, so the reverse sweep reuses the fused tile passes.
// The probes G^dagger dG are read-only ops inside those passes (FO_GRAD*),
// accumulated per CTA in a fixed order and reduced deterministically.
//
// Checkpoints: the forward state is stored every C ops (C ~ sqrt(#ops) by
// default) and restored at the matching point of the reverse sweep, which
// bounds the drift of un-applying gates in floating point.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <complex>
#include <cstring>
#include <map>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "launch.h"
#include "read.h"
#include "jit.h"

namespace ket {

typedef std::complex<double> zc;

namespace {

// ---------------------------------------------------------------- parametric gates (gates.ts)
// G(a) and dG/da for the one-parameter families, restating gates.ts:25-153
// (Rx, Ry, Rz, U1, Gpi, Gpi2, Xx, Yy, Zz, Xy) and their entry-wise derivatives.
int gate_dim(int pg) { return pg >= KET_PG_XX ? 4 : 2; }

void gate_and_deriv(int pg, double a, zc* G, zc* dG) {
  const zc I(0, 1);
  const double sq2 = 1.0 / std::sqrt(2.0);
  double c = std::cos(a / 2), s = std::sin(a / 2);
  switch (pg) {
    case KET_PG_RX: case KET_PG_CRX:
      G[0] = c; G[1] = -I * s; G[2] = -I * s; G[3] = c;
      dG[0] = -s / 2; dG[1] = -I * (c / 2); dG[2] = -I * (c / 2); dG[3] = -s / 2;
      break;
    case KET_PG_RY: case KET_PG_CRY:
      G[0] = c; G[1] = -s; G[2] = s; G[3] = c;
      dG[0] = -s / 2; dG[1] = -c / 2; dG[2] = c / 2; dG[3] = -s / 2;
      break;
    case KET_PG_RZ: case KET_PG_CRZ:
      G[0] = zc(c, -s); G[1] = 0; G[2] = 0; G[3] = zc(c, s);
      dG[0] = zc(-s / 2, -c / 2); dG[1] = 0; dG[2] = 0; dG[3] = zc(-s / 2, c / 2);
      break;
    case KET_PG_U1: case KET_PG_CU1:
      G[0] = 1; G[1] = 0; G[2] = 0; G[3] = zc(std::cos(a), std::sin(a));
      dG[0] = 0; dG[1] = 0; dG[2] = 0; dG[3] = zc(-std::sin(a), std::cos(a));
      break;
    case KET_PG_GPI: {
      double co = std::cos(a), si = std::sin(a);
      G[0] = 0; G[1] = zc(co, -si); G[2] = zc(co, si); G[3] = 0;
      dG[0] = 0; dG[1] = zc(-si, -co); dG[2] = zc(-si, co); dG[3] = 0;
      break;
    }
    case KET_PG_GPI2: {
      double co = std::cos(a), si = std::sin(a);
      G[0] = sq2; G[1] = zc(-sq2 * si, -sq2 * co); G[2] = zc(sq2 * si, -sq2 * co); G[3] = sq2;
      dG[0] = 0; dG[1] = zc(-sq2 * co, sq2 * si); dG[2] = zc(sq2 * co, sq2 * si); dG[3] = 0;
      break;
    }
    default: {  // two-qubit families, 4x4 row-major (first qubit = MSB)
      for (int k = 0; k < 16; k++) { G[k] = 0; dG[k] = 0; }
      const zc co = c, dco = -s / 2;
      if (pg == KET_PG_XX || pg == KET_PG_YY) {
        const zc ni = -I * s, dni = -I * (c / 2);
        const zc corner = pg == KET_PG_XX ? ni : -ni, dcorner = pg == KET_PG_XX ? dni : -dni;
        G[0] = G[5] = G[10] = G[15] = co; dG[0] = dG[5] = dG[10] = dG[15] = dco;
        G[3] = G[12] = corner; dG[3] = dG[12] = dcorner;
        G[6] = G[9] = ni; dG[6] = dG[9] = dni;
      } else if (pg == KET_PG_ZZ) {
        G[0] = G[15] = zc(c, -s); G[5] = G[10] = zc(c, s);
        dG[0] = dG[15] = zc(-s / 2, -c / 2); dG[5] = dG[10] = zc(-s / 2, c / 2);
      } else {  // XY
        G[0] = G[15] = 1;
        G[5] = G[10] = co; dG[5] = dG[10] = dco;
        G[6] = G[9] = I * s; dG[6] = dG[9] = I * (c / 2);
      }
      break;
    }
  }
}

bool pg_controlled(int pg) { return pg >= KET_PG_CRX && pg <= KET_PG_CU1; }

int expected_kind(int pg) {
  if (pg_controlled(pg)) return KET_OP_CONTROLLED;
  if (pg >= KET_PG_XX) return KET_OP_TWO;
  return KET_OP_SINGLE;
}

// ---------------------------------------------------------------- H psi
struct Term {
  uint64_t flip, zm;
  int ny;
  double coeff;
};

int parse_terms(int n, int nterms, const double* coeffs, const char* ops, std::vector<Term>& out, double& ident) {
  ident = 0;
  out.clear();
  for (int t = 0; t < nterms; t++) {
    const char* o = ops + (size_t)t * n;
    for (int j = 0; j < n; j++)
      if (o[j] == 0) return fail(KET_ERR_TYPE, "ops length must equal ansatz.qubits (" + std::to_string(n) + ")");
    if (std::fabs(coeffs[t]) < 1e-15) continue;
    Term tm{0, 0, 0, coeffs[t]};
    bool any = false;
    for (int q = 0; q < n; q++) {
      char ch = (char)toupper((unsigned char)o[n - 1 - q]);
      if (ch == 'X' || ch == 'Y' || ch == 'Z') any = true;
      if (ch == 'I') continue;
      uint64_t b = uint64_t(1) << q;
      if (ch == 'X' || ch == 'Y') tm.flip |= b;
      if (ch != 'X') tm.zm |= b;
      if (ch == 'Y') tm.ny++;
    }
    if (!any) { ident += coeffs[t]; continue; }
    out.push_back(tm);
  }
  return KET_OK;
}

struct DevTerm {
  uint64_t flip, zm;
  double cre, cim;  // coeff * i^ny
};

// lambda_y = sum_t coeff_t i^ny_t (-1)^popc((y^f_t) & zm_t) psi_{y^f_t}  (+ ident * psi_y),
// and per-block partials of Re <psi|lambda>.
__global__ void k_hpsi(const double2* psi, double2* lam, uint64_t N, const DevTerm* terms, int nt, double ident,
                       double* partial) {
  __shared__ double red[32];
  double e = 0.0;
  for (uint64_t y = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; y < N; y += (uint64_t)gridDim.x * blockDim.x) {
    double2 p = psi[y];
    double lr = ident * p.x, li = ident * p.y;
    for (int t = 0; t < nt; t++) {
      const DevTerm tm = terms[t];
      const uint64_t x = y ^ tm.flip;
      const double2 v = psi[x];
      const double sg = (__popcll(x & tm.zm) & 1) ? -1.0 : 1.0;
      lr = fma(sg, tm.cre * v.x - tm.cim * v.y, lr);
      li = fma(sg, tm.cre * v.y + tm.cim * v.x, li);
    }
    lam[y] = make_double2(lr, li);
    e += p.x * lr + p.y * li;
  }
  double t = block_sum<256>(e, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

__global__ void k_sum_fixed(const double* partial, int n, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double a = 0.0;
  for (int i = 0; i < n; i++) a += partial[i];
  *out = a;
}

// ---------------------------------------------------------------- helpers
void daggerize(const ket_op& op, const double* mats, std::vector<double>& out_mats, ket_op& out) {
  out = op;
  if (op.kind == KET_OP_SINGLE || op.kind == KET_OP_CONTROLLED || op.kind == KET_OP_TWO || op.kind == KET_OP_UNITARY) {
    int k = op.kind == KET_OP_UNITARY ? op.nq : (op.kind == KET_OP_TWO ? 2 : 1);
    int d = 1 << k;
    out.mat = (int64_t)(out_mats.size() / 2);
    for (int r = 0; r < d; r++)
      for (int c = 0; c < d; c++) {
        const double* e = mats + 2 * (op.mat + (int64_t)c * d + r);  // (G^dagger)[r][c] = conj(G[c][r])
        out_mats.push_back(e[0]);
        out_mats.push_back(-e[1]);
      }
  }
  // CNOT / SWAP / Toffoli / CSWAP are their own inverses; csrswap's block is
  // built by the lowering (its inverse is handled as a dagger of the 4x4).
}

}  // namespace

// Reverse-sweep runner: like run_plan, with gradient probes reduced per pass
// into slot_out (device, indexed by the probes' global slot).
// Nothing waits: the probe partials (gpart) and the op images are reused by
// later passes in stream order, and the caller reads the status word once at
// the end.
static int run_plan_grad(ket_state* s, Plan& plan, double* slot_out, double* gpart, size_t gpart_cap,
                         int specialize) {
  ket_ctx* c = s->ctx;
  const size_t np = plan.passes.size();
  ket_exec_opts o;
  ket_exec_opts_default(&o);
  o.prune = 0;
  o.specialize = specialize;
  auto probes_of = [&](size_t i, int& slot_lo) {
    int nprobe = 0;
    slot_lo = 1 << 30;
    for (int gi : plan.passes[i].gates)
      if (is_grad(plan.gates[gi])) { nprobe++; slot_lo = std::min(slot_lo, plan.gates[gi].slot); }
    return nprobe;
  };
  for (size_t i = 0; i < np;) {
    const Pass& p = plan.passes[i];
    int slot_lo;
    const int nprobe = probes_of(i, slot_lo);
    if (nprobe == 0) {
      // a run of passes without probes: the ordinary runner, in one call
      size_t j = i + 1;
      int lo2;
      while (j < np && probes_of(j, lo2) == 0) j++;
      int rc = run_plan(s, plan, o, false, i, j);
      if (rc) return rc;
      i = j;
      continue;
    }
    i++;
    if (!(p.fused && p.m == KET_T2_BITS && s->n >= KET_T2_BITS))
      return fail(KET_ERR_UNSUPPORTED, "adjoint probe outside a register-tiled pass");
    std::vector<FOp> prog;
    Pass2Args a;
    memset(&a, 0, sizeof(a));
    plan_program(plan, p, s->precision, false, 4, prog, a.load_pos, a.store_pos);
    // the probes of this pass write slots 0..nprobe-1 (they are consecutive)
    for (FOp& f : prog)
      if (f.type == FO_GRADM || f.type == FO_GRADD || f.type == FO_GRADM2) f.slot = (int16_t)(f.slot - slot_lo);
    a.nreg = 4;  // probes: 256 threads, ancilla on register bit 3
    void* dev;
    size_t fb = sizeof(FOp) * prog.size();
    int rc = ctx_scratch(c, fb + 256, &dev);
    if (rc) return rc;
    c->h2d_bytes += fb;
    rc = ctx_upload(c, dev, prog.data(), fb);
    if (rc) return rc;
    a.amp = s->amp;
    a.ops = reinterpret_cast<const FOp*>(dev);
    a.nops = (int)prog.size();
    a.n = s->n;
    a.L = p.L;
    a.nh = (int)p.hbits.size();
    for (int j = 0; j < a.nh; j++) a.hbits[j] = p.hbits[j];
    uint64_t S = (uint64_t(1) << p.L) - 1;
    for (int q : p.hbits) S |= uint64_t(1) << q;
    for (int q = 0; q < s->n; q++)
      if (!((S >> q) & 1)) a.ctxbits[a.nctx++] = q;
    a.pairbit = -1;  // the probes sum per CTA: one tile per thread
    a.thr = 1e-14;
    a.qthr = 1e-7;
    a.status = c->d_status;
    a.gpart = gpart;
    a.nslots = nprobe;
    // the probe pass on a kernel compiled for its program where one is ready
    // (or, with specialize = 1, after compiling it), else on the interpreter
    JitFn jf;
    if (specialize >= 0 && nprobe <= KET_JIT_MAX_PROBES) {
      std::vector<JitPass> jp{JitPass{prog.data(), (int)prog.size(), s->n, 4, a.load_pos, false}};
      std::vector<JitFn> fns;
      std::string err;
      rc = jit_prepare(jp, s->precision, specialize, c->stream, fns, err);
      if (rc) return fail(rc, err);
      jf = fns[0];
    }
    const int nctas = jf.fn ? (int)jit_grid(s->n) : std::min<int>(fused2_grid(4), 1 << (s->n - KET_T2_BITS));
    if ((size_t)nctas * nprobe * 8 > gpart_cap) return fail(KET_ERR_UNSUPPORTED, "too many gradient probes in a pass");
    prof_begin(c);
    cudaError_t e = jf.fn ? jit_launch(jf, a, s->precision, c->stream) : launch_fused2(a, s->precision, c->stream);
    prof_end(c, PK_ADJOINT);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint pass launch");
    e = launch_grad_reduce(gpart, nctas, nprobe, slot_out + slot_lo, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint reduce launch");
    c->launches += 1;
  }
  return KET_OK;
}

}  // namespace ket

using namespace ket;

namespace {

struct Bound {
  std::vector<double> mats;     // forward matrices with parameters bound
  std::vector<zc> D;            // per binding: G^dagger dG (times the angle scale), 2x2 or 4x4
};

int bind_params(const ket_op* ops, size_t nops, const double* mats, size_t nmat, const ket_param_binding* binds,
                size_t nbinds, const double* theta, int nparams, Bound& b) {
  b.mats.assign(mats, mats + 2 * nmat);
  b.D.assign(nbinds * 16, zc(0));
  for (size_t i = 0; i < nbinds; i++) {
    const ket_param_binding& pb = binds[i];
    if (pb.op < 0 || (size_t)pb.op >= nops) return fail(KET_ERR_RANGE, "binding op index out of range");
    if (pb.param < 0 || pb.param >= nparams) return fail(KET_ERR_RANGE, "binding parameter index out of range");
    if (pb.gate < KET_PG_RX || pb.gate > KET_PG_XY) return fail(KET_ERR_TYPE, "unknown parametric gate");
    const ket_op& op = ops[pb.op];
    if (op.kind != expected_kind(pb.gate)) return fail(KET_ERR_TYPE, "binding gate does not match the op kind");
    const int d = gate_dim(pb.gate);
    if (op.mat < 0 || (size_t)op.mat + d * d > nmat) return fail(KET_ERR_TYPE, "binding matrix offset out of bounds");
    const double angle = pb.scale * theta[pb.param] + pb.shift;
    zc G[16], dG[16];
    gate_and_deriv(pb.gate, angle, G, dG);
    for (int k = 0; k < d * d; k++) {
      b.mats[2 * (op.mat + k)] = G[k].real();
      b.mats[2 * (op.mat + k) + 1] = G[k].imag();
    }
    // D = G^dagger dG * scale
    for (int r = 0; r < d; r++)
      for (int c = 0; c < d; c++) {
        zc acc = 0;
        for (int k = 0; k < d; k++) acc += std::conj(G[k * d + r]) * dG[k * d + c];
        b.D[i * 16 + r * d + c] = acc * pb.scale;
      }
  }
  return KET_OK;
}

// Lower a single op into gates (0 or 1), with pruning off.
int lower_one(int n, const ket_op& op, const double* mats, size_t nmat, std::vector<Gate>& out) {
  std::string err;
  int rc = lower_ops(n, &op, 1, mats, nmat, false, out, err);
  if (rc) return fail(rc, err);
  return KET_OK;
}

// A checkpoint of psi: device memory while the budget allows, pinned host
// memory beyond it.
struct Ckpt {
  void* p = nullptr;
  bool host = false;
};

struct AdjWork {
  ket_state full;   // 2^(n+1): psi | lambda
  ket_state psi;    // view of the first half
  std::vector<Ckpt> ckpt;
  double* slot_out = nullptr;  // [batch][nbinds] probe sums
  double* gpart = nullptr;
  size_t gpart_cap = 0;
  DevTerm* terms = nullptr;
  double* epart = nullptr;     // Hpsi partials, then [batch] energies
};

// Device bytes the adjoint may spend on checkpoints (ket_debug_adjoint_budget);
// negative = whatever free memory allows, keeping 2 GiB spare.
int64_t g_ckpt_device_budget = -1;

}  // namespace

extern "C" {

int ket_adjoint_gradient(ket_ctx* ctx, int n, uint64_t init, const ket_op* ops, size_t nops, const double* mats,
                         size_t nmat, const ket_param_binding* binds, size_t nbinds, const double* params,
                         int nparams, int batch, int nterms, const double* coeffs, const char* pauli_ops,
                         int checkpoint_every, double* energy, double* grad) {
  if (!ctx || (nops && !ops) || (nbinds && !binds) || (batch > 0 && nparams > 0 && !params) || !energy ||
      (nparams > 0 && batch > 0 && !grad))
    return fail(KET_ERR_TYPE, "null argument");
  if (n < KET_T2_BITS || n + 1 > KET_MAX_QUBITS)
    return fail(KET_ERR_UNSUPPORTED, "adjoint gradients need 12 <= qubits < 40");
  if (batch < 0 || nparams < 0) return fail(KET_ERR_TYPE, "negative batch or parameter count");
  if ((init >> n) != 0) return fail(KET_ERR_RANGE, "initial basis index out of range");
  cudaSetDevice(ctx->device);
  std::vector<Term> terms;
  double ident = 0;
  int rc = parse_terms(n, nterms, coeffs, pauli_ops, terms, ident);
  if (rc) return rc;
  // validate the op list once (RangeError / TypeError as the reference)
  {
    Plan chk;
    std::string err;
    rc = lower_ops(n, ops, nops, mats, nmat, false, chk.gates, err);
    if (rc) return fail(rc, err);
  }
  // op -> binding
  std::vector<int> bind_of(nops, -1);
  for (size_t i = 0; i < nbinds; i++) {
    if (binds[i].op < 0 || (size_t)binds[i].op >= nops) return fail(KET_ERR_RANGE, "binding op index out of range");
    if (bind_of[binds[i].op] >= 0) return fail(KET_ERR_TYPE, "an op has two bindings");
    bind_of[binds[i].op] = (int)i;
  }
  // checkpoint spacing
  // The reverse sweep recomputes psi by un-applying each gate (exact inverses
  // in FP64), so checkpoints only bound the rounding drift, about 1e-16 per
  // gate; a few suffice.  Automatic spacing: 8 sqrt(#ops) ops, i.e. about
  // sqrt(#ops)/8 segments (3 for the 568-gate, 8-layer ansatz: one every
  // three layers).  Each segment costs at least one pass over the state, so
  // fewer, longer segments also mean fuller passes.
  int C = checkpoint_every;
  if (C == 0) C = std::max(1, 8 * (int)std::ceil(std::sqrt((double)std::max<size_t>(nops, 1))));
  if (C < 0) C = (int)nops + 1;
  const int nseg = std::max(1, (int)((nops + C - 1) / C));
  const size_t half = size_t(16) << n;

  AdjWork w;
  void* buf = nullptr;
  rc = dev_alloc(&buf, 2 * half);
  if (rc) return rc;
  w.full.ctx = ctx; w.full.n = n + 1; w.full.precision = KET_C128; w.full.amp = buf; w.full.bytes = 2 * half;
  w.psi.ctx = ctx; w.psi.n = n; w.psi.precision = KET_C128; w.psi.amp = buf; w.psi.bytes = half;
  auto cleanup = [&]() {
    ctx_wait(ctx);
    for (const Ckpt& k : w.ckpt) {
      if (k.host) cudaFreeHost(k.p);
      else cudaFree(k.p);
    }
    if (w.slot_out) cudaFree(w.slot_out);
    if (w.gpart) cudaFree(w.gpart);
    if (w.terms) cudaFree(w.terms);
    if (w.epart) cudaFree(w.epart);
    cudaFree(buf);
  };
  // Checkpoints for segments 1..nseg-1: in device memory while it holds
  // them (2 GiB spare, or the debug budget), then in pinned host memory, so a
  // state too large to keep more than one device copy still restores psi at
  // every segment boundary.
  {
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    const size_t spare = size_t(2) << 30;
    size_t dev_room = freeb > spare ? freeb - spare : 0;
    if (g_ckpt_device_budget >= 0) dev_room = std::min(dev_room, (size_t)g_ckpt_device_budget);
    for (int sgi = 1; sgi < nseg; sgi++) {
      Ckpt k;
      if (dev_room >= half) {
        if (dev_alloc(&k.p, half) == KET_OK) {
          dev_room -= half;
          w.ckpt.push_back(k);
          continue;
        }
        g_err.clear();
        dev_room = 0;
      }
      if (cudaHostAlloc(&k.p, half, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        break;  // no room anywhere: later segments are un-applied without a restore
      }
      k.host = true;
      w.ckpt.push_back(k);
    }
  }
  const int nck = (int)w.ckpt.size();  // checkpoints for segments 1..nck
  auto save = [&](int sg) {            // psi at the start of segment sg
    const Ckpt& k = w.ckpt[sg - 1];
    return cudaMemcpyAsync(k.p, buf, half, k.host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream);
  };
  auto restore = [&](int sg) {
    const Ckpt& k = w.ckpt[sg - 1];
    return cudaMemcpyAsync(buf, k.p, half, k.host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream);
  };
  std::vector<DevTerm> dterms;
  for (const Term& t : terms) {
    zc ph = std::pow(zc(0, 1), t.ny & 3) * t.coeff;
    dterms.push_back(DevTerm{t.flip, t.zm, ph.real(), ph.imag()});
  }
  const int hblocks = 1024;
  const size_t nslot = std::max<size_t>(nbinds, 1);
  rc = dev_alloc((void**)&w.slot_out, sizeof(double) * nslot * std::max(batch, 1));
  if (!rc) {
    w.gpart_cap = (size_t)2 * num_sms() * 8 * KET_JIT_MAX_PROBES;  // CTAs x warps x probes of one pass
    rc = dev_alloc((void**)&w.gpart, sizeof(double) * w.gpart_cap);
  }
  if (!rc) rc = dev_alloc((void**)&w.terms, sizeof(DevTerm) * std::max<size_t>(dterms.size(), 1));
  if (!rc) rc = dev_alloc((void**)&w.epart, sizeof(double) * (hblocks + 8 + std::max(batch, 1)));
  if (rc) { cleanup(); return rc; }
  if (!dterms.empty())
    cudaMemcpyAsync(w.terms, dterms.data(), sizeof(DevTerm) * dterms.size(), cudaMemcpyHostToDevice, ctx->stream);
  if (batch > 0) cudaMemsetAsync(w.slot_out, 0, sizeof(double) * nslot * batch, ctx->stream);
  // Batches run their passes on kernels compiled for each pass's program
  // (compiled once, on the first vector, and reused by the rest); a single
  // vector uses compiled kernels that are ready and the interpreter otherwise.
  const int specialize = batch >= 8 ? 1 : 0;
  ket_exec_opts fo;
  ket_exec_opts_default(&fo);
  fo.prune = 0;
  fo.specialize = specialize;
  double* d_energy = w.epart + hblocks + 8;
  std::vector<int> slot_bind;  // slot -> binding index (the same for every vector)

  // Every vector's passes are queued without a host wait: the host plans
  // vector b+1 while the GPU runs vector b, and the energies and probe sums
  // stay on the device until the end.
  // KET_ADJ_TIMING=1: host seconds spent queueing the batch and waiting for it, to stderr
  static const bool timing = getenv("KET_ADJ_TIMING") != nullptr;
  const auto t_start = std::chrono::steady_clock::now();
  // host seconds per section (with KET_ADJ_TIMING): binding, forward planning,
  // forward launches, energy, reverse gates, reverse planning, probe passes
  double sec[7] = {0, 0, 0, 0, 0, 0, 0};
  auto t_last = t_start;
  auto tick = [&](int k) {
    if (!timing) return;
    const auto now = std::chrono::steady_clock::now();
    sec[k] += std::chrono::duration<double>(now - t_last).count();
    t_last = now;
  };
  for (int b = 0; b < batch; b++) {
    const double* theta = params + (size_t)b * nparams;
    Bound bd;
    tick(6);
    rc = bind_params(ops, nops, mats, nmat, binds, nbinds, theta, nparams, bd);
    if (rc) { cleanup(); return rc; }
    tick(0);
    // ---- forward, segment by segment, saving checkpoints
    cudaMemsetAsync(buf, 0, 2 * half, ctx->stream);
    static const double one[2] = {1.0, 0.0};
    rc = ctx_upload(ctx, (char*)buf + 16 * init, one, 16);
    if (rc) { cleanup(); return rc; }
    for (int sg = 0; sg < nseg; sg++) {
      size_t lo = (size_t)sg * C, hi = std::min(nops, lo + C);
      if (sg >= 1 && sg <= nck && save(sg) != cudaSuccess) { cleanup(); return cuda_fail(cudaGetLastError(), "checkpoint save"); }
      Plan fp;
      std::string err;
      rc = lower_ops(n, ops + lo, hi - lo, bd.mats.data(), nmat, false, fp.gates, err);
      if (rc) { cleanup(); return fail(rc, err); }
      if (fp.gates.empty()) continue;
      plan_passes(n, KET_C128, -1, false, fp);
      tick(1);
      rc = run_plan(&w.psi, fp, fo, false);
      if (rc) { cleanup(); return rc; }
      tick(2);
    }
    // ---- lambda = H psi, energy
    prof_begin(ctx);
    k_hpsi<<<hblocks, 256, 0, ctx->stream>>>((const double2*)buf, (double2*)((char*)buf + half), uint64_t(1) << n,
                                             w.terms, (int)dterms.size(), ident, w.epart);
    k_sum_fixed<<<1, 32, 0, ctx->stream>>>(w.epart, hblocks, d_energy + b);
    prof_end(ctx, PK_ADJOINT);
    ctx->launches += 1;
    tick(3);
    // ---- reverse sweep
    double* slots_b = w.slot_out + (size_t)b * nslot;
    std::vector<int> sb;
    for (int sg = nseg - 1; sg >= 0; sg--) {
      size_t lo = (size_t)sg * C, hi = std::min(nops, lo + C);
      // restore psi at the end of this segment
      if (sg + 1 <= nck && sg + 1 < nseg && restore(sg + 1) != cudaSuccess) {
        cleanup();
        return cuda_fail(cudaGetLastError(), "checkpoint restore");
      }
      Plan bp;
      bp.anc = n;
      std::vector<double> dmats;
      for (size_t k = hi; k-- > lo;) {
        ket_op dop;
        daggerize(ops[k], bd.mats.data(), dmats, dop);
        std::vector<Gate> gs;
        if (ops[k].kind == KET_OP_CSRSWAP) {
          // lower, then dagger the 4x4 block the lowering built
          rc = lower_one(n, ops[k], bd.mats.data(), nmat, gs);
          if (rc) { cleanup(); return rc; }
          for (Gate& g : gs) {
            cd m[16];
            for (int r = 0; r < 4; r++)
              for (int c = 0; c < 4; c++) m[r * 4 + c] = cd{g.m[c * 4 + r].re, -g.m[c * 4 + r].im};
            for (int q = 0; q < 16; q++) g.m[q] = m[q];
          }
        } else if (dop.kind != KET_OP_BARRIER) {
          rc = lower_one(n, dop, dmats.data(), dmats.size() / 2, gs);
          if (rc) { cleanup(); return rc; }
        }
        for (Gate& g : gs) { g.src_op = (int)k; bp.gates.push_back(g); }
        int bi = bind_of[k];
        if (bi >= 0) {
          const ket_param_binding& pb = binds[bi];
          const ket_op& op = ops[k];
          Gate pr;
          pr.src_op = (int)k;
          pr.slot = (int)sb.size();
          sb.push_back(bi);
          const zc* D = &bd.D[(size_t)bi * 16];
          const int d = gate_dim(pb.gate);
          bool diag = true;
          for (int r = 0; r < d; r++)
            for (int c = 0; c < d; c++)
              if (r != c && D[r * d + c] != zc(0)) diag = false;
          if (d == 2) {
            pr.t0 = op.kind == KET_OP_CONTROLLED ? op.q[1] : op.q[0];
            if (op.kind == KET_OP_CONTROLLED) pr.cmask = uint64_t(1) << op.q[0];
            if (diag) {
              pr.type = G_GRADD;
              pr.m[0] = cd{D[0].real(), D[0].imag()};
              pr.m[1] = cd{D[3].real(), D[3].imag()};
            } else {
              pr.type = G_GRADM;
              for (int q = 0; q < 4; q++) pr.m[q] = cd{D[q].real(), D[q].imag()};
            }
          } else {
            pr.type = G_GRADM2;
            pr.t0 = op.q[0];
            pr.t1 = op.q[1];
            for (int q = 0; q < 16; q++) pr.m[q] = cd{D[q].real(), D[q].imag()};
          }
          bp.gates.push_back(pr);
        }
      }
      if (bp.gates.empty()) continue;
      tick(4);
      plan_passes(n + 1, KET_C128, -1, false, bp);
      tick(5);
      // probes must stay in order within each pass: slots are consecutive per pass by construction
      rc = run_plan_grad(&w.full, bp, slots_b, w.gpart, w.gpart_cap, specialize);
      if (rc) { cleanup(); return rc; }
      tick(6);
    }
    if (b == 0) slot_bind = sb;
  }
  std::vector<double> slot_val(nslot * std::max(batch, 1)), e_all(std::max(batch, 1));
  if (batch > 0) {
    cudaMemcpyAsync(e_all.data(), d_energy, 8 * (size_t)batch, cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(slot_val.data(), w.slot_out, 8 * nslot * batch, cudaMemcpyDeviceToHost, ctx->stream);
    ctx->d2h_bytes += 8 * (size_t)batch * (nslot + 1);
  }
  const auto t_queued = std::chrono::steady_clock::now();
  rc = ctx_wait(ctx);
  if (!rc) rc = check_status(ctx);
  if (timing) {
    const auto t_done = std::chrono::steady_clock::now();
    fprintf(stderr, "ket_adjoint_gradient: %d vectors, %d segments: queued in %.3f s, then waited %.3f s\n", batch,
            nseg, std::chrono::duration<double>(t_queued - t_start).count(),
            std::chrono::duration<double>(t_done - t_queued).count());
    fprintf(stderr, "  host s: bind %.3f, forward plan %.3f, forward launch %.3f, energy %.3f, reverse gates %.3f,"
            " reverse plan %.3f, probe passes %.3f\n", sec[0], sec[1], sec[2], sec[3], sec[4], sec[5], sec[6]);
  }
  if (rc) { cleanup(); return rc; }
  for (int b = 0; b < batch; b++) {
    energy[b] = e_all[b];
    double* g = grad + (size_t)b * nparams;
    for (int p = 0; p < nparams; p++) g[p] = 0.0;
    // dE/dtheta = sum over bound ops of 2 Re<lambda|G^dagger dG|psi>; slots were
    // numbered in reverse op order, so add them back in forward order
    const double* sv = slot_val.data() + (size_t)b * nslot;
    for (size_t sl = slot_bind.size(); sl-- > 0;) g[binds[slot_bind[sl]].param] += 2.0 * sv[sl];
  }
  cleanup();
  return KET_OK;
}

int ket_debug_adjoint_budget(int64_t device_bytes) {
  g_ckpt_device_budget = device_bytes;
  return KET_OK;
}

// Parameter-shift gradient on the same engine (algorithms.ts:536-547): for each
// parameter, E(theta + pi/2 e_k) and E(theta - pi/2 e_k) by full forward
// simulations, grad_k = (E+ - E-)/2.  Reference semantics of the energy (the
// reference re-simulates per Pauli term; one simulation and the Pauli sum
// give the same value).
int ket_shift_gradient(ket_ctx* ctx, int n, uint64_t init, const ket_op* ops, size_t nops, const double* mats,
                       size_t nmat, const ket_param_binding* binds, size_t nbinds, const double* params, int nparams,
                       int batch, int nterms, const double* coeffs, const char* pauli_ops, int prune, double* energy,
                       double* grad) {
  if (!ctx || (nops && !ops) || (nbinds && !binds) || !energy || (nparams > 0 && (!params || !grad)))
    return fail(KET_ERR_TYPE, "null argument");
  if (n < 1 || n > KET_MAX_QUBITS) return fail(KET_ERR_RANGE, "qubit count out of range");
  cudaSetDevice(ctx->device);
  ket_state* st = nullptr;
  int rc = ket_state_alloc(ctx, n, KET_C128, &st);
  if (rc) return rc;
  ket_exec_opts o;
  ket_exec_opts_default(&o);
  o.prune = prune ? 1 : 0;
  std::vector<double> th(nparams);
  auto energy_at = [&](const double* t, double* e) -> int {
    Bound bd;
    int r = bind_params(ops, nops, mats, nmat, binds, nbinds, t, nparams, bd);
    if (r) return r;
    r = ket_state_set_basis(st, init);
    if (r) return r;
    r = ket_apply_ops(st, ops, nops, bd.mats.data(), nmat, &o);
    if (r) return r;
    return ket_expect_pauli_sum(st, nterms, coeffs, pauli_ops, e);
  };
  const double shift = M_PI / 2;
  for (int b = 0; b < batch && !rc; b++) {
    const double* theta = params + (size_t)b * nparams;
    rc = energy_at(theta, &energy[b]);
    for (int k = 0; k < nparams && !rc; k++) {
      double ep = 0, em = 0;
      std::copy(theta, theta + nparams, th.begin());
      th[k] = theta[k] + shift;
      rc = energy_at(th.data(), &ep);
      if (rc) break;
      th[k] = theta[k] - shift;
      rc = energy_at(th.data(), &em);
      grad[(size_t)b * nparams + k] = 0.5 * (ep - em);
    }
  }
  ket_state_free(st);
  return rc;
}

}  // extern "C"
