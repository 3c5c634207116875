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
// Distinct program shapes a process compiles at most (their modules stay
// loaded for the life of the process).
#define KET_JIT_MAX_KERNELS 4096

struct JitPass {
  const FOp* prog = nullptr;  // host copy of the pass's program; null = not a register-tiled pass
  int nops = 0;
  int nqubits = 0;
  int nreg = KET_FUSED_NREG;  // register bits of the program's layouts (4 or 5)
  const uint8_t* load_pos = nullptr;  // the program's load layout (role -> tile bit)
  bool staged = false;        // tiles staged in shared memory by TMA copies (jit_ops.cuh)
};

// Register bits of the programs of compiled pass kernels for an n-qubit
// state.  Below KET_JIT_AUTO_QUBITS: 5, the interpreter's (128 threads of 32
// amplitudes), so a compiled kernel gives the interpreter's result bit for
// bit.  From there on: 4 (256 threads of 16 amplitudes, two CTAs and 16 warps
// per SM), the faster shape for compiled kernels and much the slower one for
// the interpreter, which keeps 5; KET_JIT_NREG=5 in the environment keeps 5
// throughout.  Register and lane forms of a gate round alike, but merged
// phase fans group their factors by role, so there the two paths agree to
// rounding rather than bit for bit.  reg_bits (ket_exec_opts.reg_bits) 4 or 5
// forces that count at any size; 0 leaves the choice above.
int tiled_nreg(int nqubits, int reg_bits = 0);
// Probes a compiled adjoint pass holds at most (its shared-memory sums).
#define KET_JIT_MAX_PROBES 512

struct JitFn {
  bool staged = false;              // the staged form (one CTA per SM, two tile groups, TMA copies)
  bool grad = false;                // an adjoint probe pass
  void* fn = nullptr;               // CUfunction, null = run the interpreter
  unsigned long long cops = 0;      // device address of the kernel's constant op array
  size_t cops_bytes = 0;
};

// For each pass, the compiled kernel to launch on this stream (null where none
// is ready).  Each stream gets its own instance of a kernel's module, since a
// launch first fills the module's constant op array.
// mode: ket_exec_opts.specialize (0 automatic, 1 always, -1 never).
int jit_prepare(const std::vector<JitPass>& passes, int precision, int mode, cudaStream_t stream,
                std::vector<JitFn>& out, std::string& err);
cudaError_t jit_launch(const JitFn& f, const Pass2Args& a, int precision, cudaStream_t s);
// Dynamic shared memory of a pass kernel (without probe sums).
int pass_smem(int precision, bool staged);
// CTAs of a register-load pass kernel on an n-qubit state (two per SM at most).
unsigned jit_grid(int n);
// Whether a pass of n qubits with these options runs the staged form
// (ket_exec_opts.stage: 1 always, -1 never, 0 automatic).
bool use_staged(int n, int stage);
// Test hook of the staged form's bounded waits (ket_debug_stage_drop).
void jit_debug_stage_drop(int64_t tile);
// Wait until no compile is queued or running.
int jit_wait_all();
// Drop queued compiles and wait for running ones.  A host calls this before it
// exits: a compile still running when the process tears down NVRTC's statics
// would crash the exit.
void jit_shutdown();
// out: kernels known, compiled, failed, launches; *compile_s: compile seconds summed over threads.
void jit_stats(int64_t out[4], double* compile_s);
// Compile (on the pool, waiting) the kernels of all listed passes that are not
// compiled yet; no GPU needed.  *distinct: kernels the passes need.
int jit_compile(const std::vector<JitPass>& passes, int precision, int64_t* distinct, std::string& log);

}  // namespace ket
