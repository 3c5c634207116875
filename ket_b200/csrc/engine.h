// engine.h -- host-side structures of the statevector engine.
#pragma once

#include <stdint.h>
#include <string>
#include <vector>

#include "ket_sv.h"

namespace ket {

struct cd {
  double re, im;
};

// Internal gate after lowering a ket_op (controls folded into a mask).
enum GType : int32_t {
  G_MAT1 = 0,   // 2x2 on t0, controls cmask
  G_DIAG1 = 1,  // diag(d0, d1) on t0, controls cmask
  G_X1 = 2,     // X on t0 (CNOT / Toffoli), controls cmask
  G_SWAP = 3,   // swap t0, t1, controls cmask
  G_MAT2 = 4,   // 4x4 on (t0 = MSB, t1), controls cmask
  G_MATK = 5,   // dense 2^k x 2^k on tk (tk[0] = MSB)
  G_DIAG2 = 6,  // diag(m0..m3) on (t0 = MSB, t1), controls cmask
  // Adjoint-sweep probes (read-only): on a state whose top qubit `anc` splits
  // it into psi (anc = 0) and lambda (anc = 1), accumulate Re<lambda|D|psi>
  // into gradient slot `slot`.
  G_GRADM = 7,  // D 2x2 on t0, controls cmask
  G_GRADD = 8,  // D = diag(m0, m1) on t0, controls cmask
  G_GRADM2 = 9  // D 4x4 on (t0 = MSB, t1), controls cmask
};

struct Gate {
  GType type;
  int t0 = -1, t1 = -1;
  uint64_t cmask = 0;
  bool prune = false;         // computed outputs are flushed when |a|^2 < 1e-14
  cd m[16] = {};              // MAT1: m[0..3]; DIAG1: m[0], m[1]; DIAG2: m[0..3]; MAT2: m[0..15]
  std::vector<int> tk;        // MATK targets
  std::vector<cd> mk;         // MATK matrix
  int src_op = -1;            // index of the ket_op it came from
  int slot = -1;              // G_GRAD*: gradient slot
};

// Tile pass: the tile holds qubits {0..L-1} U hbits; gates are applied in order.
struct Pass {
  bool fused = false;
  int m = 0;                  // tile qubits
  int L = 0;                  // low contiguous qubits in the tile
  std::vector<int> hbits;     // global positions of tile bits L..m-1
  std::vector<int> gates;     // indices into the gate list
};

struct Plan {
  std::vector<Gate> gates;
  std::vector<Pass> passes;
  int anc = -1;               // adjoint sweep: qubit that selects psi / lambda, kept in every tile
};

inline bool is_grad(const Gate& g) { return g.type == G_GRADM || g.type == G_GRADD || g.type == G_GRADM2; }

// Lower and validate an op list (mirrors #checkOp, circuit.ts:1113-1146).
int lower_ops(int n, const ket_op* ops, size_t nops, const double* mats, size_t nmat, bool prune,
              std::vector<Gate>& out, std::string& err);
// Merge uncontrolled single-qubit gates on the same qubit where that is exact
// (with pruning: only when one of the two preserves magnitudes).
void fold_single_qubit(std::vector<Gate>& gates, bool prune);
// Greedy fusion planner.
void plan_passes(int n, int precision, int fusion, bool keep_mix_order, Plan& plan);

// Tile width used for fused passes at a given precision.
int tile_qubits(int precision, int fusion);

}  // namespace ket
