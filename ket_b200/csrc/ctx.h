// ctx.h -- context and state handles behind the opaque C ABI types.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "../../include/ket_sv.h"
#include "engine.h"

struct ket_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  void* scratch = nullptr;       // op images, reduction partials, sampling CDFs
  size_t scratch_bytes = 0;
  void* scratch2 = nullptr;      // second pool (adjoint states, batch workspace)
  size_t scratch2_bytes = 0;
  cudaGraphExec_t graph_exec = nullptr;  // last captured batch launch
  uint64_t graph_key = 0;
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
int run_plan(ket_state* s, const Plan& plan, const ket_exec_opts& o);

}  // namespace ket
