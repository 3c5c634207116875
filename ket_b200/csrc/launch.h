// launch.h -- kernel launchers shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "engine.h"
#include "fused_abi.h"

namespace ket {

// Device form of one gate inside a fused tile pass.
struct DevOp {
  int32_t type;    // GType
  int32_t b0, b1;  // tile-local bit of t0 / t1, -1 when the qubit is outside the tile
  int32_t flags;   // bit 0: prune outputs
  uint32_t ctile;  // control bits inside the tile (tile-local positions)
  uint32_t pad;
  uint64_t cctx;   // control bits outside the tile (global positions)
  uint64_t g0, g1; // DIAG: global mask of t0 / t1 when outside the tile
  double m[32];    // interleaved complex matrix (MAT1: 4, DIAG1: 2, DIAG2: 4, MAT2: 16 entries)
};

struct PassArgs {
  void* amp;
  const DevOp* ops;
  int nops;
  int n, m, L, nh, nctx;
  int hbits[KET_MAX_TILE_HBITS];
  int ctxbits[KET_MAX_CTX_BITS];
  double thr, qthr;  // pruning threshold and its square root
};

// ---------------------------------------------------------------- register-tiled pass
// The op records (FOp) and arguments (Pass2Args) are in fused_abi.h.

// Fill in op.opc from op.type, op.a, op.flags and op.creg.
void assign_opcode(FOp& op);

// Sum the adjoint partials of one pass: out[s] = sum over CTAs and warps (fixed order).
cudaError_t launch_grad_reduce(const double* gpart, int nctas, int nslots, double* out, cudaStream_t s);
// Persistent grid of the register-tiled pass for a register-bit count.
int fused2_grid(int nreg);
// Fill a.lgb, a.sgb and a.lbx (per-role byte offsets in the state and in the
// exchange buffer) from the layouts and tile bits.
void fill_pass2_offsets(Pass2Args& a, int precision);
// A qubit outside the tile (index into a.ctxbits) that no op of the program
// reads as a control or a diagonal target, or -1.
int choose_pairbit(const std::vector<FOp>& prog, const Pass2Args& a);

// Lower one fused pass to a register-tiled program (segments + exchanges).
void plan_program(const Plan& plan, const Pass& p, int precision, bool prune, int nreg, std::vector<FOp>& prog,
                  uint8_t load_pos[KET_T2_BITS], uint8_t store_pos[KET_T2_BITS]);
cudaError_t launch_fused2(const Pass2Args& a, int precision, cudaStream_t s);

struct Ctx;

// Encode a gate for a fused pass.
DevOp encode_devop(const Gate& g, const Pass& p, bool prune);
// Single-gate pass over the whole state.
cudaError_t launch_gate(const Gate& g, int precision, void* amp, int n, const void* dev_matk, cudaStream_t s);
// Fused tile pass.
cudaError_t launch_fused(const PassArgs& a, int precision, cudaStream_t s);

int num_sms();

}  // namespace ket
