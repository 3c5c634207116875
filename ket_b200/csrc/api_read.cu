// api_read.cu -- read-out entry points of the C ABI (include/ket_sv.h).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "ctx.h"
#include "read.h"

using namespace ket;

namespace {

int check_state(const ket_state* s) {
  if (!s) return fail(KET_ERR_TYPE, "null state");
  cudaSetDevice(s->ctx->device);
  return KET_OK;
}

int h2d(ket_ctx* c, void* dst, const void* src, size_t bytes) {
  if (!bytes) return KET_OK;
  c->h2d_bytes += bytes;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
  return e == cudaSuccess ? KET_OK : cuda_fail(e, "cudaMemcpyAsync(H2D)");
}
int d2h(ket_ctx* c, void* dst, const void* src, size_t bytes) {
  if (!bytes) return KET_OK;
  c->d2h_bytes += bytes;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
  return e == cudaSuccess ? KET_OK : cuda_fail(e, "cudaMemcpyAsync(D2H)");
}
int launched(cudaError_t e) { return e == cudaSuccess ? KET_OK : cuda_fail(e, "kernel launch"); }

// Launch a read-out kernel bracketed for accounting/profiling.
#define LAUNCH_READ(c, expr) (prof_begin(c), prof_end_ret((c), (expr)))
// The same for a launcher that issues two kernels (block partials, then their
// fixed-order sum): the launch counter counts both.
#define LAUNCH_READ2(c, expr) ((c)->launches++, LAUNCH_READ(c, expr))
int prof_end_ret(ket_ctx* c, cudaError_t e) {
  prof_end(c, PK_READ);
  return launched(e);
}

#define TRY(x) do { int _rc = (x); if (_rc) return _rc; } while (0)

char* align_up(char* p, size_t a) { return (char*)(((uintptr_t)p + a - 1) & ~(uintptr_t)(a - 1)); }

}  // namespace

extern "C" {

int ket_amplitudes(const ket_state* s, const uint64_t* idx, size_t k, double* out) {
  TRY(check_state(s));
  if (k && (!idx || !out)) return fail(KET_ERR_TYPE, "null argument");
  const uint64_t N = uint64_t(1) << s->n;
  for (size_t i = 0; i < k; i++)
    if (idx[i] >= N) return fail(KET_ERR_RANGE, "amplitude index out of range");
  if (!k) return KET_OK;
  void* scr;
  TRY(ctx_scratch(s->ctx, 8 * k + 16 * k + 512, &scr));
  uint64_t* di = (uint64_t*)scr;
  double* dout = (double*)align_up((char*)(di + k), 256);
  TRY(h2d(s->ctx, di, idx, 8 * k));
  TRY(LAUNCH_READ(s->ctx, launch_gather(s->amp, s->precision, di, k, dout, s->ctx->stream)));
  TRY(d2h(s->ctx, out, dout, 16 * k));
  return ctx_wait(s->ctx);
}

int ket_norm2(const ket_state* s, double* out) {
  TRY(check_state(s));
  if (!out) return fail(KET_ERR_TYPE, "null argument");
  void* scr;
  TRY(ctx_scratch(s->ctx, norm2_scratch(s->n) + 64, &scr));
  double* res = (double*)scr;
  TRY(LAUNCH_READ2(s->ctx, launch_norm2(s->amp, s->n, s->precision, res + 8, res, s->ctx->stream)));
  TRY(d2h(s->ctx, out, res, 8));
  return ctx_wait(s->ctx);
}

int ket_state_compare(const ket_state* a, const ket_state* b, double* overlap_re_im, double* max_abs_diff) {
  TRY(check_state(a));
  TRY(check_state(b));
  if (!overlap_re_im && !max_abs_diff) return fail(KET_ERR_TYPE, "null argument");
  if (a->n != b->n) return fail(KET_ERR_TYPE, "states of different sizes");
  if (a->ctx != b->ctx) return fail(KET_ERR_TYPE, "states of different contexts");
  void* scr;
  TRY(ctx_scratch(a->ctx, compare_scratch(a->n) + 64, &scr));
  double* res = (double*)scr;
  TRY(LAUNCH_READ2(a->ctx, launch_compare(a->amp, a->precision, b->amp, b->precision, a->n, res + 8, res,
                                         a->ctx->stream)));
  double h[3];
  TRY(d2h(a->ctx, h, res, 24));
  TRY(ctx_wait(a->ctx));
  if (overlap_re_im) { overlap_re_im[0] = h[0]; overlap_re_im[1] = h[1]; }
  if (max_abs_diff) *max_abs_diff = h[2];
  return KET_OK;
}

int ket_probs_dense(const ket_state* s, double thr, double* out) {
  TRY(check_state(s));
  if (!out) return fail(KET_ERR_TYPE, "null argument");
  const uint64_t N = uint64_t(1) << s->n;
  const uint64_t chunk = std::min<uint64_t>(N, uint64_t(1) << 24);
  void* scr;
  TRY(ctx_scratch(s->ctx, 8 * chunk, &scr));
  for (uint64_t off = 0; off < N; off += chunk) {
    TRY(LAUNCH_READ(s->ctx, launch_probs_dense(s->amp, s->precision, off, chunk, thr, (double*)scr, s->ctx->stream)));
    TRY(d2h(s->ctx, out + off, scr, 8 * chunk));
    TRY(ctx_wait(s->ctx));
  }
  return KET_OK;
}

int ket_probs_sparse(const ket_state* s, double thr, uint64_t* idx, double* p, uint64_t cap, uint64_t* count) {
  TRY(check_state(s));
  if (!count || (cap && (!idx || !p))) return fail(KET_ERR_TYPE, "null argument");
  const uint64_t N = uint64_t(1) << s->n;
  const uint64_t chunk = kept_chunk(s->n), nb = (N + chunk - 1) / chunk;
  void* scr;
  TRY(ctx_scratch(s->ctx, 16 * nb + 512, &scr));
  uint64_t* dcounts = (uint64_t*)scr;
  TRY(LAUNCH_READ(s->ctx, launch_count_kept(s->amp, s->n, s->precision, thr, dcounts, s->ctx->stream)));
  std::vector<uint64_t> counts(nb), offs(nb);
  TRY(d2h(s->ctx, counts.data(), dcounts, 8 * nb));
  TRY(ctx_wait(s->ctx));
  uint64_t total = 0;
  for (uint64_t b = 0; b < nb; b++) { offs[b] = total; total += counts[b]; }
  *count = total;
  uint64_t ncopy = std::min(total, cap);
  if (ncopy == 0) return KET_OK;
  TRY(ctx_scratch(s->ctx, 8 * nb + 16 * ncopy + 1024, &scr));
  uint64_t* doffs = (uint64_t*)scr;
  uint64_t* didx = (uint64_t*)align_up((char*)(doffs + nb), 256);
  double* dp = (double*)align_up((char*)(didx + ncopy), 256);
  TRY(h2d(s->ctx, doffs, offs.data(), 8 * nb));
  TRY(LAUNCH_READ(s->ctx, launch_compact_kept(s->amp, s->n, s->precision, thr, doffs, ncopy, didx, dp, s->ctx->stream)));
  TRY(d2h(s->ctx, idx, didx, 8 * ncopy));
  TRY(d2h(s->ctx, p, dp, 8 * ncopy));
  return ctx_wait(s->ctx);
}

int ket_marginals(const ket_state* s, double* out) {
  TRY(check_state(s));
  if (!out) return fail(KET_ERR_TYPE, "null argument");
  const uint64_t N = uint64_t(1) << s->n;
  const uint64_t nb = (N + marg_chunk(s->n) - 1) / marg_chunk(s->n);
  void* scr;
  TRY(ctx_scratch(s->ctx, 8 * (nb * s->n + s->n) + 512, &scr));
  double* res = (double*)scr;
  double* partial = (double*)align_up((char*)(res + s->n), 256);
  TRY(LAUNCH_READ2(s->ctx, launch_marginals(s->amp, s->n, s->precision, partial, res, s->ctx->stream)));
  TRY(d2h(s->ctx, out, res, 8 * s->n));
  return ctx_wait(s->ctx);
}

int ket_marginal_dist(const ket_state* s, const int* qubits, int m, double* out) {
  TRY(check_state(s));
  if (!out || (m && !qubits)) return fail(KET_ERR_TYPE, "null argument");
  if (m < 1 || m > KET_MAX_MARGINAL_QUBITS) return fail(KET_ERR_TYPE, "marginal_dist supports 1..12 qubits");
  MarginalSpec spec;
  memset(&spec, 0, sizeof(spec));
  spec.m = m;
  for (int k = 0; k < m; k++) {
    if (qubits[k] < 0 || qubits[k] >= s->n) return fail(KET_ERR_RANGE, "qubit index out of range");
    if ((spec.mask >> qubits[k]) & 1) return fail(KET_ERR_TYPE, "repeated qubit in marginal_dist");
    spec.q[k] = qubits[k];
    spec.mask |= uint64_t(1) << qubits[k];
  }
  int c = mdist_chunk_bits(s->n, m);
  uint64_t nb = uint64_t(1) << (s->n - c);
  uint64_t width = uint64_t(1) << m;
  void* scr;
  TRY(ctx_scratch(s->ctx, 8 * (nb * width + width) + 512, &scr));
  double* res = (double*)scr;
  double* partial = (double*)align_up((char*)(res + width), 256);
  TRY(LAUNCH_READ2(s->ctx, launch_marginal_dist(s->amp, s->n, s->precision, spec, partial, res, s->ctx->stream)));
  TRY(d2h(s->ctx, out, res, 8 * width));
  return ctx_wait(s->ctx);
}

int ket_sample(const ket_state* s, const double* r, size_t shots, double thr, uint64_t* out) {
  return ket::sample_indices(s, r, shots, thr, out);
}

}  // extern "C"

namespace ket {

int sample_indices(const ket_state* s, const double* r, size_t shots, double thr, uint64_t* out) {
  TRY(check_state(s));
  if (shots && (!r || !out)) return fail(KET_ERR_TYPE, "null argument");
  if (!shots) return KET_OK;
  for (size_t i = 0; i < shots; i++)
    if (!(r[i] >= 0.0 && r[i] <= 1.0)) return fail(KET_ERR_RANGE, "a draw outside [0, 1]");
  size_t need = sample_scratch(s->n) + 16 * shots + 1024;
  void* scr;
  TRY(ctx_scratch(s->ctx, need, &scr));
  double* dr = (double*)scr;
  uint64_t* dout = (uint64_t*)align_up((char*)(dr + shots), 256);
  void* work = align_up((char*)(dout + shots), 256);
  TRY(h2d(s->ctx, dr, r, 8 * shots));
  s->ctx->launches += sample_launches() - 1;  // LAUNCH_READ counts one
  TRY(LAUNCH_READ(s->ctx, launch_sample(s->amp, s->n, s->precision, thr, dr, shots, work, dout, s->ctx->stream)));
  TRY(d2h(s->ctx, out, dout, 8 * shots));
  return ctx_wait(s->ctx);
}

}  // namespace ket

namespace {

struct Term {
  double coeff;
  uint64_t flip, zm;
  int ny;
};

// Sum over groups of Pauli terms that share (flip mask, i^nY phase).
int pauli_terms_expect(const ket_state* s, const std::vector<Term>& terms, double* out) {
  std::map<std::pair<uint64_t, int>, std::vector<const Term*>> groups;
  for (const Term& t : terms) groups[{t.flip, t.ny & 3}].push_back(&t);
  std::vector<PauliGroup> gl;
  for (auto& kv : groups) {
    const auto& v = kv.second;
    for (size_t o = 0; o < v.size(); o += KET_PAULI_GROUP_TERMS) {
      PauliGroup g;
      memset(&g, 0, sizeof(g));
      g.flip = kv.first.first;
      g.ny = kv.first.second;
      g.nterms = (int)std::min<size_t>(KET_PAULI_GROUP_TERMS, v.size() - o);
      for (int j = 0; j < g.nterms; j++) { g.zm[j] = v[o + j]->zm; g.coeff[j] = v[o + j]->coeff; }
      gl.push_back(g);
    }
  }
  if (gl.empty()) { *out = 0.0; return KET_OK; }
  void* scr;
  TRY(ctx_scratch(s->ctx, pauli_scratch(s->n) + 8 * gl.size() + 512, &scr));
  double* res = (double*)scr;
  double* partial = (double*)align_up((char*)(res + gl.size()), 256);
  for (size_t i = 0; i < gl.size(); i++)
    TRY(LAUNCH_READ2(s->ctx, launch_pauli_group(s->amp, s->n, s->precision, gl[i], partial, res + i, s->ctx->stream)));
  std::vector<double> h(gl.size());
  TRY(d2h(s->ctx, h.data(), res, 8 * gl.size()));
  TRY(ctx_wait(s->ctx));
  double e = 0.0;
  for (double v : h) e += v;
  *out = e;
  return KET_OK;
}

}  // namespace

extern "C" {

int ket_expect_pauli(const ket_state* s, const char* pauli, double* out) {
  TRY(check_state(s));
  if (!pauli || !out) return fail(KET_ERR_TYPE, "null argument");
  if ((int)strlen(pauli) != s->n)
    return fail(KET_ERR_TYPE, "pauli length must equal qubits (" + std::to_string(s->n) + ")");
  Term t{1.0, 0, 0, 0};
  bool any = false;
  for (int q = 0; q < s->n; q++) {
    char ch = (char)toupper((unsigned char)pauli[q]);
    if (ch != 'I' && ch != 'X' && ch != 'Y' && ch != 'Z') return fail(KET_ERR_TYPE, "pauli must contain only I, X, Y, Z");
    if (ch == 'I') continue;
    any = true;
    uint64_t b = uint64_t(1) << q;
    if (ch == 'X' || ch == 'Y') t.flip |= b;
    if (ch == 'Y' || ch == 'Z') t.zm |= b;
    if (ch == 'Y') t.ny++;
  }
  if (!any) { *out = 1.0; return KET_OK; }  // circuit.ts:3735
  return pauli_terms_expect(s, std::vector<Term>{t}, out);
}

int ket_expect_pauli_sum(const ket_state* s, int nterms, const double* coeffs, const char* ops, double* out) {
  TRY(check_state(s));
  if (!out || (nterms && (!coeffs || !ops))) return fail(KET_ERR_TYPE, "null argument");
  const int n = s->n;
  double ident = 0.0;
  std::vector<Term> terms;
  for (int t = 0; t < nterms; t++) {
    const char* o = ops + (size_t)t * n;
    for (int j = 0; j < n; j++)
      if (o[j] == 0) return fail(KET_ERR_TYPE, "ops length must equal ansatz.qubits (" + std::to_string(n) + ")");
    if (std::fabs(coeffs[t]) < 1e-15) continue;      // algorithms.ts:308
    Term tm{coeffs[t], 0, 0, 0};
    bool any = false;
    for (int q = 0; q < n; q++) {
      char ch = (char)toupper((unsigned char)o[n - 1 - q]);  // ops[n-1-q] acts on qubit q
      if (ch == 'X' || ch == 'Y' || ch == 'Z') any = true;
      if (ch == 'I') continue;
      uint64_t b = uint64_t(1) << q;
      // X -> h, Y -> rx(pi/2), anything else counts in the parity like Z (algorithms.ts:313-327)
      if (ch == 'X' || ch == 'Y') tm.flip |= b;
      if (ch != 'X') tm.zm |= b;
      if (ch == 'Y') tm.ny++;
    }
    if (!any) { ident += coeffs[t]; continue; }      // algorithms.ts:310
    terms.push_back(tm);
  }
  double e = 0.0;
  TRY(pauli_terms_expect(s, terms, &e));
  *out = ident + e;
  return KET_OK;
}

}  // extern "C"
