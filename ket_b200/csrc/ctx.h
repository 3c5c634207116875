// ctx.h -- context and state handles behind the opaque C ABI types.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "ket_sv.h"
#include "engine.h"

struct ket_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  void* scratch = nullptr;       // op images, reduction partials, sampling CDFs
  size_t scratch_bytes = 0;
  void* scratch2 = nullptr;      // second pool (adjoint states, batch workspace)
  size_t scratch2_bytes = 0;
  cudaGraphExec_t graph_exec = nullptr;  // last captured batch launch (ket_batch_qaoa)
  uint64_t graph_key = 0;
  void* vqe_work = nullptr;              // ket_batch_vqe: its device workspace
  size_t vqe_work_bytes = 0;
  cudaGraphExec_t vqe_graph_exec = nullptr;  // ket_batch_vqe: last captured launch
  uint64_t vqe_graph_key = 0;
  // launch accounting and optional per-launch CUDA-event timing
  int* d_status = nullptr;        // device status word written by kernels (bounded waits)
  uint64_t launches = 0;
  uint64_t h2d_bytes = 0, d2h_bytes = 0;  // host<->device copies made by the context
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> prof_kind;     // kind of each timed launch
  size_t prof_next = 0;           // next free event pair
  int batch_threads = 256;        // ket_batch_qaoa: threads per CTA (set by ket_batch_config)
  int batch_tile = 12;            // ket_batch_qaoa: tile width in qubits
  // Pinned staging for uploads of op programs (ctx_upload): a copy from
  // pageable memory may wait for the stream, which would keep the host from
  // planning ahead of the GPU.  A slot is reused once its copy has run.
  struct StageSlot {
    void* p = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    bool used = false;
  };
  std::vector<StageSlot> stage_ring;
  size_t stage_next = 0;
};

struct ket_state {
  ket_ctx* ctx = nullptr;
  int n = 0;
  int precision = KET_C128;
  void* amp = nullptr;
  size_t bytes = 0;
};

namespace ket {

extern thread_local std::string g_err;
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);
int dev_alloc(void** p, size_t bytes);
int ctx_scratch(ket_ctx* ctx, size_t bytes, void** out);
int ctx_wait(ket_ctx* ctx);
// Copy bytes from host memory to device memory dst, in stream order, through
// the context's pinned staging ring: the call returns without waiting for
// the stream (unless every slot's copy is still queued).
int ctx_upload(ket_ctx* ctx, void* dst, const void* src, size_t bytes);
// Run a plan's passes on the state's stream.  wait = false returns once the
// launches are queued (the caller waits and reads the status word later);
// every buffer the passes read is stream-ordered, so queued plans may follow
// one another.  first, last: run only passes [first, last) of the plan.
int run_plan(ket_state* s, const Plan& plan, const ket_exec_opts& o, bool wait = true, size_t first = 0,
             size_t last = SIZE_MAX);
int check_status(ket_ctx* c);
// ket_sample with the sequential CDF up to seq_qubits qubits (see read.h).
int sample_indices(const ket_state* s, const double* r, size_t shots, double thr, uint64_t* out);

// Launch kinds reported by ket_ctx_profile_read.
enum { PK_FUSED2 = 0, PK_FUSED1 = 1, PK_GATE = 2, PK_READ = 3, PK_ADJOINT = 4, PK_BATCH = 5 };
// Bracket one kernel launch on ctx->stream (counts it; times it when profiling).
void prof_begin(ket_ctx* c);
void prof_end(ket_ctx* c, int kind);

}  // namespace ket
