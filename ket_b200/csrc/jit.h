// jit.h -- register-tiled pass kernels compiled at run time (jit.cpp).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fused_abi.h"

namespace ket {

// Under the automatic policy, states below this many qubits always use the
// interpreter (a pass takes under a millisecond there, so compiling pays off
// only after thousands of runs).
#define KET_JIT_AUTO_QUBITS 26

struct JitPass {
  const FOp* prog = nullptr;  // host copy of the pass's program; null = not a register-tiled pass
  int nops = 0;
  int nqubits = 0;
};
struct JitFn {
  void* fn = nullptr;  // CUfunction, null = run the interpreter
};

// For each pass, the compiled kernel to launch (null where none is ready).
// mode: ket_exec_opts.specialize (0 automatic, 1 always, -1 never).
int jit_prepare(const std::vector<JitPass>& passes, int precision, int mode, int device, std::vector<JitFn>& out,
                std::string& err);
cudaError_t jit_launch(const JitFn& f, const Pass2Args& a, int precision, cudaStream_t s);
// Wait until no compile is queued or running.
int jit_wait_all();
// out: kernels known, compiled, failed, launches; *compile_s: compile seconds summed over threads.
void jit_stats(int64_t out[4], double* compile_s);
// Compile (on the pool, waiting) the kernels of all listed passes that are not
// compiled yet; no GPU needed.  *distinct: kernels the passes need.
int jit_compile(const std::vector<JitPass>& passes, int precision, int64_t* distinct, std::string& log);

}  // namespace ket
