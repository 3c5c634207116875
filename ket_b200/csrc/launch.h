// launch.h -- kernel launchers shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "engine.h"

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

#define KET_MAX_TILE_HBITS 16
#define KET_MAX_CTX_BITS 48

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
// The tile's 12 bits are split into roles: 5 lane bits, 3 warp bits, 4 register
// bits (each thread holds 16 amplitudes).  A layout lists, for lane bits 0..4,
// warp bits 0..2 and register bits 0..3, which tile bit plays that role.
#define KET_T2_BITS 12
enum FOpType : uint8_t {
  FO_EXCH = 0,    // re-layout the tile through shared memory
  FO_MAT1R = 1,   // 2x2 on register bit a
  FO_MAT1L = 2,   // 2x2 on lane bit a (warp shuffles)
  FO_X1R = 3,     // X on register bit a
  FO_X1L = 4,     // X on lane bit a
  FO_SWAPS = 5,   // swap tile bits a, b (controls allowed) through shared memory
  FO_MAT2S = 6,   // 4x4 on tile bits a (MSB), b through shared memory
  FO_RELABEL = 11,// no data movement: the layout's role -> tile-bit map changes (uncontrolled SWAP)
  FO_DIAG = 7,    // diag phase on tile bits d0 (and d1), anywhere (general form)
  FO_DIAGR = 8,   // diag(m0, m1) on register bit a
  FO_DIAGT = 9,   // diag(m0, m1) on thread-id bit a (lane 0-4 / warp 5-7): one phase per thread
  FO_DIAGX = 10,  // diag(m0, m1) on a qubit outside the tile (mask dg0): one phase per tile
  FO_GRADM = 12,  // adjoint probe, D 2x2 on register bit a, ancilla register bit b, slot d1
  FO_GRADD = 13,  // adjoint probe, D = diag(m0, m1) on target a (register / thread / outside, see flags)
  FO_GRADM2 = 14  // adjoint probe, D 4x4 on tile bits a (MSB), b through shared memory; ancilla tile bit d0
};

// flags
#define FOF_PRUNE 1u    // flush computed amplitudes with |a|^2 < 1e-14
#define FOF_REAL 2u     // MAT1: every matrix entry is real
#define FOF_D0ONE 4u    // DIAG*: m0 == 1 exactly (only bit-1 amplitudes change)
#define FOF_RXFORM 8u   // MAT1: m00, m11 real and m01, m10 imaginary (Rx-like)
#define FOF_TGT_THR 32u // FO_GRADD: target is a thread-id bit (a)
#define FOF_TGT_CTX 64u // FO_GRADD: target is outside the tile (mask dg0)

struct FOp {
  uint8_t type, a, b, flags;
  uint8_t pos[KET_T2_BITS];   // FO_EXCH: new layout
  uint32_t creg;              // controls on register bits (bit k = register bit k)
  uint32_t cthr;              // controls on thread-id bits (lane bits 0-4, warp bits 5-7)
  uint32_t ctile;             // FO_DIAG: controls inside the tile (tile-bit mask)
  int16_t d0, d1;             // FO_DIAG: tile bit of t0 / t1, -1 = outside the tile, -2 = none
  uint64_t cctx;              // controls on global bits outside the tile
  uint64_t dg0, dg1;          // FO_DIAG*: global mask of t0 / t1 when outside the tile
  uint64_t pad;               // header = 64 bytes
  double m[32];
};

struct Pass2Args {
  void* amp;
  const FOp* ops;
  int nops;
  int n, L, nh, nctx;
  uint8_t load_pos[KET_T2_BITS];   // layout used for the global load
  uint8_t store_pos[KET_T2_BITS];  // layout in force at the global store
  int hbits[KET_MAX_TILE_HBITS];   // global qubit of tile bits L..11
  int ctxbits[KET_MAX_CTX_BITS];
  double thr, qthr;
  int* status;                     // device status word: set to KET_ERR_TIMEOUT if a bounded wait ran out
  double* gpart;                   // adjoint: per-CTA gradient partials [cta][slot][warp]
  int nslots;                      // adjoint: gradient probes in this pass
};

// Sum the adjoint partials of one pass: out[s] = sum over CTAs and warps (fixed order).
cudaError_t launch_grad_reduce(const double* gpart, int nctas, int nslots, double* out, cudaStream_t s);
int fused2_grid();

// Lower one fused pass to a register-tiled program (segments + exchanges).
void plan_program(const Plan& plan, const Pass& p, int precision, bool prune, std::vector<FOp>& prog,
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
