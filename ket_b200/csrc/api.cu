// api.cu -- the C ABI of the statevector engine (include/ket_sv.h).
//
// Control flow per call: validate on the host (mirroring the reference's
// synchronous throws), launch on the context's stream, then wait with a
// deadline by polling an event (never an unbounded synchronize), and report
// CUDA failures as status codes with a thread-local message.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "launch.h"
#include "jit.h"
#include "read.h"

namespace ket {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  return KET_ERR_CUDA;
}

// Allocation fault injection (host side): the N-th device allocation from now
// fails with KET_ERR_OOM.  Set by ket_debug_fail_alloc() or KET_FAIL_ALLOC_AFTER.
static long long g_fail_after = -2;

static bool alloc_should_fail() {
  if (g_fail_after == -2) {
    const char* e = getenv("KET_FAIL_ALLOC_AFTER");
    g_fail_after = e ? atoll(e) : -1;
  }
  if (g_fail_after < 0) return false;
  if (g_fail_after == 0) { g_fail_after = -1; return true; }
  g_fail_after--;
  return false;
}

int dev_alloc(void** p, size_t bytes) {
  *p = nullptr;
  if (alloc_should_fail()) return fail(KET_ERR_OOM, "device allocation failed (injected)");
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(KET_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
  }
  return KET_OK;
}

int ctx_scratch(ket_ctx* ctx, size_t bytes, void** out) {
  bytes = std::max<size_t>(bytes, 256);
  if (ctx->scratch_bytes < bytes) {
    int rc = ctx_wait(ctx);
    if (rc) return rc;
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    size_t want = std::max(bytes, size_t(1) << 20);
    rc = dev_alloc(&ctx->scratch, want);
    if (rc) return rc;
    ctx->scratch_bytes = want;
  }
  *out = ctx->scratch;
  return KET_OK;
}

double wait_deadline_s() {
  const char* e = getenv("KET_WAIT_TIMEOUT_S");
  return e ? atof(e) : 1800.0;
}

int ctx_upload(ket_ctx* c, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return KET_OK;
  constexpr size_t kSlots = 16;
  if (c->stage_ring.empty()) c->stage_ring.resize(kSlots);
  ket_ctx::StageSlot& sl = c->stage_ring[c->stage_next];
  c->stage_next = (c->stage_next + 1) % kSlots;
  cudaError_t e;
  if (sl.used && (e = cudaEventSynchronize(sl.ev)) != cudaSuccess) return cuda_fail(e, "staging slot");
  if (sl.cap < bytes) {
    if (sl.p) cudaFreeHost(sl.p);
    sl.p = nullptr;
    sl.cap = 0;
    const size_t cap = std::max<size_t>(bytes, 64 << 10);
    if (cudaHostAlloc(&sl.p, cap, cudaHostAllocDefault) != cudaSuccess) {
      // no pinned memory to be had: copy from the caller's buffer (the copy
      // may then wait for the stream, as any copy from pageable memory does)
      cudaGetLastError();
      sl.p = nullptr;
      sl.used = false;
      if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
        return cuda_fail(e, "cudaMemcpyAsync(upload)");
      return KET_OK;
    }
    sl.cap = cap;
  }
  if (!sl.ev && (e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming)) != cudaSuccess)
    return cuda_fail(e, "cudaEventCreate");
  memcpy(sl.p, src, bytes);
  if ((e = cudaMemcpyAsync(dst, sl.p, bytes, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess)
    return cuda_fail(e, "cudaMemcpyAsync(upload)");
  if ((e = cudaEventRecord(sl.ev, c->stream)) != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  sl.used = true;
  return KET_OK;
}

int ctx_wait(ket_ctx* ctx) {
  cudaError_t e = cudaEventRecord(ctx->done, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  auto t0 = std::chrono::steady_clock::now();
  const double limit = wait_deadline_s();
  int spins = 0;
  for (;;) {
    e = cudaEventQuery(ctx->done);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return cuda_fail(e, "device execution");
    if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > limit) return fail(KET_ERR_TIMEOUT, "device work did not finish within the wait deadline");
  }
  return KET_OK;
}

static size_t amp_bytes(int precision) { return precision == KET_C64 ? 8 : 16; }

void prof_begin(ket_ctx* c) {
  if (!c->prof) return;
  if (c->prof_next + 2 > c->ev_pool.size()) {
    for (int i = 0; i < 64; i++) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) { c->prof = false; return; }
      c->ev_pool.push_back(e);
    }
  }
  cudaEventRecord(c->ev_pool[c->prof_next], c->stream);
}

void prof_end(ket_ctx* c, int kind) {
  c->launches++;
  if (!c->prof || c->prof_next + 2 > c->ev_pool.size()) return;
  cudaEventRecord(c->ev_pool[c->prof_next + 1], c->stream);
  c->prof_kind.push_back(kind);
  c->prof_next += 2;
}

}  // namespace ket

using namespace ket;

extern "C" {

const char* ket_last_error(void) { return g_err.c_str(); }
int ket_abi_version(void) { return KET_SV_ABI_VERSION; }

void ket_exec_opts_default(ket_exec_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->fusion = -1;
  o->prune = 1;
}

int ket_debug_fail_alloc(int after) {
  g_fail_after = after;
  return KET_OK;
}

int ket_ctx_create(int device, ket_ctx** out) {
  if (!out) return fail(KET_ERR_TYPE, "null output pointer");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(KET_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  }
  if (device < 0 || device >= count) return fail(KET_ERR_RANGE, "device index out of range");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  ket_ctx* c = new ket_ctx();
  c->device = device;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cuda_fail(e, "cudaStreamCreate"); }
  e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming);
  if (e != cudaSuccess) { cudaStreamDestroy(c->stream); delete c; return cuda_fail(e, "cudaEventCreate"); }
  void* st = nullptr;
  int rc = dev_alloc(&st, 256);
  if (rc) { cudaEventDestroy(c->done); cudaStreamDestroy(c->stream); delete c; return rc; }
  c->d_status = (int*)st;
  cudaMemsetAsync(c->d_status, 0, 256, c->stream);
  *out = c;
  return KET_OK;
}

int ket_ctx_destroy(ket_ctx* c) {
  if (!c) return KET_OK;
  cudaSetDevice(c->device);
  ctx_wait(c);
  if (c->scratch) cudaFree(c->scratch);
  if (c->scratch2) cudaFree(c->scratch2);
  if (c->d_status) cudaFree(c->d_status);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->vqe_graph_exec) cudaGraphExecDestroy(c->vqe_graph_exec);
  if (c->vqe_work) cudaFree(c->vqe_work);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  for (auto& sl : c->stage_ring) {
    if (sl.p) cudaFreeHost(sl.p);
    if (sl.ev) cudaEventDestroy(sl.ev);
  }
  cudaEventDestroy(c->done);
  cudaStreamDestroy(c->stream);
  delete c;
  return KET_OK;
}

int ket_ctx_scratch_bytes(const ket_ctx* c, uint64_t* out) {
  if (!c || !out) return fail(KET_ERR_TYPE, "null argument");
  *out = c->scratch_bytes + c->scratch2_bytes;
  return KET_OK;
}

int ket_ctx_profile(ket_ctx* c, int enable) {
  if (!c) return fail(KET_ERR_TYPE, "null context");
  c->prof = enable != 0;
  c->prof_kind.clear();
  c->prof_next = 0;
  return KET_OK;
}

int ket_ctx_profile_read(ket_ctx* c, int* kinds, float* ms, size_t cap, size_t* count) {
  if (!c || !count) return fail(KET_ERR_TYPE, "null argument");
  int rc = ctx_wait(c);
  if (rc) return rc;
  size_t n = c->prof_kind.size();
  *count = n;
  for (size_t i = 0; i < n && i < cap; i++) {
    if (kinds) kinds[i] = c->prof_kind[i];
    float t = 0.f;
    cudaEventElapsedTime(&t, c->ev_pool[2 * i], c->ev_pool[2 * i + 1]);
    if (ms) ms[i] = t;
  }
  c->prof_kind.clear();
  c->prof_next = 0;
  return KET_OK;
}

int ket_ctx_io_bytes(const ket_ctx* c, uint64_t* h2d, uint64_t* d2h) {
  if (!c) return fail(KET_ERR_TYPE, "null context");
  if (h2d) *h2d = c->h2d_bytes;
  if (d2h) *d2h = c->d2h_bytes;
  return KET_OK;
}

int ket_ctx_stream(const ket_ctx* c, void** out) {
  if (!c || !out) return fail(KET_ERR_TYPE, "null argument");
  *out = (void*)c->stream;
  return KET_OK;
}

int ket_ctx_launch_count(const ket_ctx* c, uint64_t* out) {
  if (!c || !out) return fail(KET_ERR_TYPE, "null argument");
  *out = c->launches;
  return KET_OK;
}

int ket_state_alloc(ket_ctx* c, int n, int precision, ket_state** out) {
  if (!c || !out) return fail(KET_ERR_TYPE, "null argument");
  *out = nullptr;
  if (n < 1 || n > KET_MAX_QUBITS) return fail(KET_ERR_RANGE, "qubit count out of range: " + std::to_string(n));
  if (precision != KET_C128 && precision != KET_C64) return fail(KET_ERR_TYPE, "precision must be KET_C128 or KET_C64");
  cudaSetDevice(c->device);
  size_t bytes = amp_bytes(precision) << n;
  void* p = nullptr;
  int rc = dev_alloc(&p, bytes);
  if (rc) return rc;
  ket_state* s = new ket_state();
  s->ctx = c;
  s->n = n;
  s->precision = precision;
  s->amp = p;
  s->bytes = bytes;
  rc = ket_state_set_basis(s, 0);
  if (rc) { cudaFree(p); delete s; return rc; }
  *out = s;
  return KET_OK;
}

int ket_state_free(ket_state* s) {
  if (!s) return KET_OK;
  cudaSetDevice(s->ctx->device);
  ctx_wait(s->ctx);
  cudaFree(s->amp);
  delete s;
  return KET_OK;
}

int ket_state_qubits(const ket_state* s, int* n, int* precision) {
  if (!s) return fail(KET_ERR_TYPE, "null state");
  if (n) *n = s->n;
  if (precision) *precision = s->precision;
  return KET_OK;
}

int ket_state_set_basis(ket_state* s, uint64_t idx) {
  if (!s) return fail(KET_ERR_TYPE, "null state");
  if (s->n < 64 && (idx >> s->n) != 0) return fail(KET_ERR_RANGE, "basis index out of range");
  cudaSetDevice(s->ctx->device);
  cudaError_t e = cudaMemsetAsync(s->amp, 0, s->bytes, s->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  s->ctx->h2d_bytes += s->precision == KET_C64 ? 8 : 16;
  if (s->precision == KET_C64) {
    float one[2] = {1.0f, 0.0f};
    e = cudaMemcpyAsync((char*)s->amp + 8 * idx, one, 8, cudaMemcpyHostToDevice, s->ctx->stream);
  } else {
    double one[2] = {1.0, 0.0};
    e = cudaMemcpyAsync((char*)s->amp + 16 * idx, one, 16, cudaMemcpyHostToDevice, s->ctx->stream);
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
  return ctx_wait(s->ctx);
}

int ket_state_set_amplitudes(ket_state* s, uint64_t off, uint64_t cnt, const double* re_im) {
  if (!s || (!re_im && cnt)) return fail(KET_ERR_TYPE, "null argument");
  uint64_t N = uint64_t(1) << s->n;
  if (off > N || cnt > N - off) return fail(KET_ERR_RANGE, "amplitude range out of bounds");
  if (cnt == 0) return KET_OK;
  cudaSetDevice(s->ctx->device);
  if (s->precision == KET_C128) {
    cudaError_t e = cudaMemcpyAsync((char*)s->amp + 16 * off, re_im, 16 * cnt, cudaMemcpyHostToDevice, s->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
    return ctx_wait(s->ctx);
  }
  std::vector<float> tmp(2 * cnt);
  for (uint64_t i = 0; i < 2 * cnt; i++) tmp[i] = (float)re_im[i];
  cudaError_t e = cudaMemcpyAsync((char*)s->amp + 8 * off, tmp.data(), 8 * cnt, cudaMemcpyHostToDevice, s->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
  return ctx_wait(s->ctx);
}

int ket_state_get_amplitudes(const ket_state* s, uint64_t off, uint64_t cnt, double* re_im) {
  if (!s || (!re_im && cnt)) return fail(KET_ERR_TYPE, "null argument");
  uint64_t N = uint64_t(1) << s->n;
  if (off > N || cnt > N - off) return fail(KET_ERR_RANGE, "amplitude range out of bounds");
  if (cnt == 0) return KET_OK;
  cudaSetDevice(s->ctx->device);
  if (s->precision == KET_C128) {
    cudaError_t e = cudaMemcpyAsync(re_im, (char*)s->amp + 16 * off, 16 * cnt, cudaMemcpyDeviceToHost, s->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
    return ctx_wait(s->ctx);
  }
  std::vector<float> tmp(2 * cnt);
  cudaError_t e = cudaMemcpyAsync(tmp.data(), (char*)s->amp + 8 * off, 8 * cnt, cudaMemcpyDeviceToHost, s->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
  int rc = ctx_wait(s->ctx);
  if (rc) return rc;
  for (uint64_t i = 0; i < 2 * cnt; i++) re_im[i] = tmp[i];
  return KET_OK;
}

int ket_state_copy(ket_state* dst, const ket_state* src) {
  if (!dst || !src) return fail(KET_ERR_TYPE, "null state");
  if (dst->n != src->n || dst->precision != src->precision) return fail(KET_ERR_TYPE, "state shape mismatch");
  cudaSetDevice(dst->ctx->device);
  cudaError_t e = cudaMemcpyAsync(dst->amp, src->amp, src->bytes, cudaMemcpyDeviceToDevice, dst->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync");
  return ctx_wait(dst->ctx);
}

int ket_plan_stats(int n, int precision, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                   const ket_exec_opts* opts, int64_t passes[3]) {
  ket_exec_opts o;
  if (opts) o = *opts; else ket_exec_opts_default(&o);
  if (n < 1 || n > KET_MAX_QUBITS) return fail(KET_ERR_RANGE, "qubit count out of range");
  Plan plan;
  std::string err;
  int rc = lower_ops(n, ops, nops, mats, nmat, o.prune != 0, plan.gates, err);
  if (rc) return fail(rc, err);
  if (o.fusion != 0) fold_single_qubit(plan.gates, o.prune != 0);
  plan_passes(n, precision, o.fusion, o.prune != 0, plan);
  passes[0] = passes[1] = passes[2] = 0;
  for (auto& p : plan.passes) {
    if (p.fused) passes[0]++; else passes[1]++;
    passes[2] += (int64_t)p.gates.size();
  }
  return KET_OK;
}

int ket_plan_program_stats(int n, int precision, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                           const ket_exec_opts* opts, int64_t counts[16]) {
  ket_exec_opts o;
  if (opts) o = *opts; else ket_exec_opts_default(&o);
  if (n < 1 || n > KET_MAX_QUBITS) return fail(KET_ERR_RANGE, "qubit count out of range");
  Plan plan;
  std::string err;
  int rc = lower_ops(n, ops, nops, mats, nmat, o.prune != 0, plan.gates, err);
  if (rc) return fail(rc, err);
  if (o.fusion != 0) fold_single_qubit(plan.gates, o.prune != 0);
  plan_passes(n, precision, o.fusion, o.prune != 0, plan);
  for (int i = 0; i < 16; i++) counts[i] = 0;
  for (auto& p : plan.passes) {
    if (!(p.fused && p.m == KET_T2_BITS && n >= KET_T2_BITS)) { counts[15]++; continue; }
    std::vector<FOp> prog;
    uint8_t lp[KET_T2_BITS], sp[KET_T2_BITS];
    plan_program(plan, p, precision, o.prune != 0, tiled_nreg(n, o.reg_bits), prog, lp, sp);
    for (const FOp& f : prog) {
      if (f.type == FO_PPOLY) counts[FO_CPHASE]++;  // merged phase ops share one count
      else if (f.type <= FO_CPHASE) counts[f.type]++;  // probes (12-14) never occur here
      if (f.type == FO_MAT1R || f.type == FO_MAT1L) counts[(f.flags & (FOF_REAL | FOF_RXFORM)) ? 13 : 12]++;
    }
    counts[14]++;
  }
  return KET_OK;
}

int ket_debug_stage_drop(int64_t tile) {
  jit_debug_stage_drop(tile);
  return KET_OK;
}

int ket_jit_wait(void) {
  const int rc = jit_wait_all();
  return rc ? fail(rc, "a run-time compile of a pass kernel failed") : KET_OK;
}

int ket_jit_shutdown(void) {
  jit_shutdown();
  return KET_OK;
}

int ket_jit_stats(int64_t out[4], double* compile_seconds) {
  if (!out) return fail(KET_ERR_TYPE, "null argument");
  jit_stats(out, compile_seconds);
  return KET_OK;
}

int ket_jit_compile(int n, int precision, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                    const ket_exec_opts* opts, int64_t* kernels, char* log, size_t logcap) {
  ket_exec_opts o;
  if (opts) o = *opts; else ket_exec_opts_default(&o);
  if (n < 1 || n > KET_MAX_QUBITS) return fail(KET_ERR_RANGE, "qubit count out of range");
  if (o.reg_bits != 0 && o.reg_bits != 4 && o.reg_bits != 5) return fail(KET_ERR_RANGE, "reg_bits must be 0, 4 or 5");
  if (kernels) *kernels = 0;
  if (log && logcap) log[0] = 0;
  Plan plan;
  std::string err;
  int rc = lower_ops(n, ops, nops, mats, nmat, o.prune != 0, plan.gates, err);
  if (rc) return fail(rc, err);
  if (o.fusion != 0) fold_single_qubit(plan.gates, o.prune != 0);
  plan_passes(n, precision, o.fusion, o.prune != 0, plan);
  std::vector<std::vector<FOp>> progs;
  std::vector<std::vector<uint8_t>> lps;
  for (auto& p : plan.passes) {
    if (!(p.fused && p.m == KET_T2_BITS && n >= KET_T2_BITS)) continue;
    progs.emplace_back();
    lps.emplace_back(KET_T2_BITS);
    uint8_t sp[KET_T2_BITS];
    plan_program(plan, p, precision, o.prune != 0, tiled_nreg(n, o.reg_bits), progs.back(), lps.back().data(), sp);
  }
  std::vector<JitPass> jp;
  for (size_t i = 0; i < progs.size(); i++)
    jp.push_back(JitPass{progs[i].data(), (int)progs[i].size(), n, tiled_nreg(n, o.reg_bits), lps[i].data(),
                         use_staged(n, o.stage)});
  std::string clog;
  rc = jit_compile(jp, precision, kernels, clog);
  if (log && logcap) {
    strncpy(log, clog.c_str(), logcap - 1);
    log[logcap - 1] = 0;
  }
  return rc ? fail(rc, "run-time compile of a pass kernel failed") : KET_OK;
}

int ket_apply_ops(ket_state* s, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                  const ket_exec_opts* opts) {
  if (!s) return fail(KET_ERR_TYPE, "null state");
  if (nops && !ops) return fail(KET_ERR_TYPE, "null op list");
  ket_exec_opts o;
  if (opts) o = *opts; else ket_exec_opts_default(&o);
  if (o.reg_bits != 0 && o.reg_bits != 4 && o.reg_bits != 5) return fail(KET_ERR_RANGE, "reg_bits must be 0, 4 or 5");
  Plan plan;
  std::string err;
  int rc = lower_ops(s->n, ops, nops, mats, nmat, o.prune != 0, plan.gates, err);
  if (rc) return fail(rc, err);
  if (o.fusion != 0) fold_single_qubit(plan.gates, o.prune != 0);
  if (plan.gates.empty()) return KET_OK;
  plan_passes(s->n, s->precision, o.fusion, o.prune != 0, plan);
  return run_plan(s, plan, o);
}

}  // extern "C"

namespace ket {

int run_plan(ket_state* s, const Plan& plan, const ket_exec_opts& o, bool wait, size_t first, size_t last) {
  ket_ctx* c = s->ctx;
  cudaSetDevice(c->device);
  const bool prune = o.prune != 0;
  // Device image: v2 programs (FOp), v1 programs (DevOp), then MATK descriptors.
  // passes [first, last) of the plan
  last = std::min(last, plan.passes.size());
  first = std::min(first, last);
  const size_t np = last - first;
  std::vector<FOp> fops;
  std::vector<DevOp> devops;
  std::vector<size_t> off(np, 0), matk_off(np, 0);
  std::vector<Pass2Args> p2(np);
  std::vector<bool> use2(np, false);
  size_t matk_bytes = 0;
  // Register-tiled passes: compiled kernels (jit.cpp) use programs with
  // tiled_nreg(n) register bits; a pass whose kernel is not ready runs on the
  // interpreter with KET_FUSED_NREG.
  const int jit_nr = tiled_nreg(s->n, o.reg_bits);
  std::vector<std::vector<FOp>> progs(np);
  std::vector<JitFn> jf(np);
  auto lower_pass = [&](size_t i, int nreg) {
    Pass2Args& a = p2[i];
    memset(&a, 0, sizeof(a));
    a.nreg = nreg;
    plan_program(plan, plan.passes[first + i], s->precision, prune, nreg, progs[i], a.load_pos, a.store_pos);
  };
  for (size_t i = 0; i < np; i++) {
    const Pass& p = plan.passes[first + i];
    if (p.fused && p.m == KET_T2_BITS && s->n >= KET_T2_BITS) {
      use2[i] = true;
      lower_pass(i, o.specialize < 0 ? KET_FUSED_NREG : jit_nr);
    }
  }
  if (o.specialize >= 0) {
    std::vector<JitPass> jp(np);
    for (size_t i = 0; i < np; i++)
      if (use2[i])
        jp[i] = JitPass{progs[i].data(), (int)progs[i].size(), s->n, jit_nr, p2[i].load_pos,
                        use_staged(s->n, o.stage) && plan.passes[first + i].L == 5};
    std::string err;
    int rc = jit_prepare(jp, s->precision, o.specialize, c->stream, jf, err);
    if (rc) return fail(rc, err);
    for (size_t i = 0; i < np; i++)
      if (use2[i] && !jf[i].fn && jit_nr != KET_FUSED_NREG) lower_pass(i, KET_FUSED_NREG);
  }
  for (size_t i = 0; i < np; i++) {
    const Pass& p = plan.passes[first + i];
    if (use2[i]) {
      const std::vector<FOp>& prog = progs[i];
      Pass2Args& a = p2[i];
      off[i] = fops.size();
      fops.insert(fops.end(), prog.begin(), prog.end());
      a.amp = s->amp;
      a.nops = (int)prog.size();
      a.n = s->n;
      a.L = p.L;
      a.nh = (int)p.hbits.size();
      for (int j = 0; j < a.nh; j++) a.hbits[j] = p.hbits[j];
      uint64_t S = (uint64_t(1) << p.L) - 1;
      for (int q : p.hbits) S |= uint64_t(1) << q;
      a.nctx = 0;
      for (int q = 0; q < s->n; q++)
        if (!((S >> q) & 1)) a.ctxbits[a.nctx++] = q;
      a.pairbit = choose_pairbit(prog, a);
      a.thr = 1e-14;
      a.qthr = 1e-7;
      a.status = c->d_status;
    } else if (p.fused) {
      off[i] = devops.size();
      for (int gi : p.gates) devops.push_back(encode_devop(plan.gates[gi], p, prune));
    } else {
      const Gate& g = plan.gates[p.gates[0]];
      if (g.type == G_MATK) {
        matk_off[i] = matk_bytes;
        matk_bytes += 64 + 16 * g.mk.size();
        matk_bytes = (matk_bytes + 255) & ~size_t(255);
      }
    }
  }
  const size_t f_bytes = ((sizeof(FOp) * fops.size()) + 255) & ~size_t(255);
  const size_t d_bytes = ((sizeof(DevOp) * devops.size()) + 255) & ~size_t(255);
  const size_t total = f_bytes + d_bytes + matk_bytes;
  void* dev = nullptr;
  if (total) {
    int rc = ctx_scratch(c, total, &dev);
    if (rc) return rc;
    std::vector<unsigned char> host(total, 0);
    if (!fops.empty()) memcpy(host.data(), fops.data(), sizeof(FOp) * fops.size());
    if (!devops.empty()) memcpy(host.data() + f_bytes, devops.data(), sizeof(DevOp) * devops.size());
    for (size_t i = 0; i < np; i++) {
      const Pass& p = plan.passes[first + i];
      if (p.fused) continue;
      const Gate& g = plan.gates[p.gates[0]];
      if (g.type != G_MATK) continue;
      unsigned char* dst = host.data() + f_bytes + d_bytes + matk_off[i];
      int* q = reinterpret_cast<int*>(dst);
      for (size_t j = 0; j < g.tk.size(); j++) q[j] = g.tk[j];
      memcpy(dst + 64, g.mk.data(), 16 * g.mk.size());
    }
    c->h2d_bytes += total;
    int urc = ctx_upload(c, dev, host.data(), total);
    if (urc) return urc;
  }
  const FOp* dfops = reinterpret_cast<const FOp*>(dev);
  const DevOp* dops = reinterpret_cast<const DevOp*>((const char*)dev + f_bytes);
  for (size_t i = 0; i < np; i++) {
    const Pass& p = plan.passes[first + i];
    cudaError_t e;
    int kind = use2[i] ? PK_FUSED2 : (p.fused ? PK_FUSED1 : PK_GATE);
    prof_begin(c);
    if (use2[i]) {
      p2[i].ops = dfops + off[i];
      e = jf[i].fn ? jit_launch(jf[i], p2[i], s->precision, c->stream) : launch_fused2(p2[i], s->precision, c->stream);
    } else if (p.fused) {
      PassArgs a;
      memset(&a, 0, sizeof(a));
      a.amp = s->amp;
      a.ops = dops + off[i];
      a.nops = (int)p.gates.size();
      a.n = s->n;
      a.m = p.m;
      a.L = p.L;
      a.nh = (int)p.hbits.size();
      for (int j = 0; j < a.nh; j++) a.hbits[j] = p.hbits[j];
      uint64_t S = (p.L >= 64) ? ~uint64_t(0) : ((uint64_t(1) << p.L) - 1);
      for (int q : p.hbits) S |= uint64_t(1) << q;
      a.nctx = 0;
      for (int q = 0; q < s->n; q++)
        if (!((S >> q) & 1)) a.ctxbits[a.nctx++] = q;
      a.thr = 1e-14;
      a.qthr = 1e-7;
      e = launch_fused(a, s->precision, c->stream);
    } else {
      const Gate& g = plan.gates[p.gates[0]];
      const void* mk =
          g.type == G_MATK ? (const void*)((const char*)dev + f_bytes + d_bytes + matk_off[i]) : nullptr;
      e = launch_gate(g, s->precision, s->amp, s->n, mk, c->stream);
    }
    prof_end(c, kind);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  }
  if (!wait) return KET_OK;
  int rc = ctx_wait(c);
  if (rc) return rc;
  return check_status(c);
}

// Read and clear the device status word (set by kernels whose bounded waits ran out).
int check_status(ket_ctx* c) {
  int st = 0;
  cudaError_t e = cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "status read");
  if (st != 0) {
    cudaMemset(c->d_status, 0, sizeof(int));
    return fail(st, "a device-side bounded wait ran out (status " + std::to_string(st) + ")");
  }
  return KET_OK;
}

}  // namespace ket
