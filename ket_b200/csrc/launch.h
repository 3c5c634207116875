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

struct Ctx;

// Encode a gate for a fused pass.
DevOp encode_devop(const Gate& g, const Pass& p, bool prune);
// Single-gate pass over the whole state.
cudaError_t launch_gate(const Gate& g, int precision, void* amp, int n, const void* dev_matk, cudaStream_t s);
// Fused tile pass.
cudaError_t launch_fused(const PassArgs& a, int precision, cudaStream_t s);

int num_sms();

}  // namespace ket
