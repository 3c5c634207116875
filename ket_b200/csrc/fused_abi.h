// fused_abi.h -- the register-tiled pass's op records and launch arguments.
//
// Shared by the host (planner, launchers) and by device code, including the
// pass kernels compiled at run time (jit.cpp), so it holds only plain types:
// no host headers when compiled by the runtime compiler.
#pragma once

#ifdef __CUDACC_RTC__
typedef unsigned char uint8_t;
typedef signed char int8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <stdint.h>
#include <cuda_runtime.h>
#endif

#define KET_MAX_TILE_HBITS 16
#define KET_MAX_CTX_BITS 48

namespace ket {

// ---------------------------------------------------------------- register-tiled pass
// The tile's 12 bits are split into roles: 5 lane bits, NW warp bits and NR
// register bits (NW + NR = 7; each thread holds 2^NR amplitudes).  Role r < 5
// is lane bit r, 5 <= r < 5 + NW is warp bit r - 5 (thread-id bit r), and r >=
// 5 + NW is register bit r - 5 - NW.  A layout lists which tile bit plays
// each role.  Ordinary passes use NR = 5 (128 threads per CTA, two CTAs per
// SM); adjoint passes use NR = 4 (256 threads).
#define KET_T2_BITS 12
#define KET_NR_MAX 5
// Register bits of ordinary (non-adjoint) passes.
#define KET_FUSED_NREG 5
enum FOpType : uint8_t {
  FO_EXCH = 0,    // re-layout the tile through shared memory
  FO_MAT1R = 1,   // 2x2 on register bit a
  FO_MAT1L = 2,   // 2x2 on lane bit a (warp shuffles)
  FO_X1R = 3,     // X on register bit a
  FO_X1L = 4,     // X on lane bit a
  FO_SWAPS = 5,   // swap tile bits a, b (controls on tile bits: ctile) through shared memory
  FO_MAT2S = 6,   // 4x4 on tile bits a (MSB), b through shared memory
  FO_DIAG = 7,    // 4-entry diagonal on tile bits d0 (MSB), d1 (-1 = outside the tile), through shared memory
  FO_DIAGR = 8,   // diag(m0, m1) on register bit a
  FO_DIAGT = 9,   // diag(m0, m1) on thread-id bit a (lane 0-4 / warp 5-7): one phase per thread
  FO_DIAGX = 10,  // diag(m0, m1) on a qubit outside the tile (mask dg0): one phase per tile
  FO_CPHASE = 11, // fan of phases on register bit a (see below), followed by continuation records
  FO_GRADM = 12,  // adjoint probe, D 2x2 on register bit a (ancilla on register bit 3)
  FO_GRADD = 13,  // adjoint probe, D = diag(m0, m1) on target a (register / thread / outside, see flags)
  FO_GRADM2 = 14, // adjoint probe, D 4x4 on tile bits a (MSB), b through shared memory; ancilla tile bit anc
  FO_CONT = 15,   // continuation record of the op before it (data only, never dispatched)
  FO_PPOLY = 16,  // phases of a run of controlled-phase gates (see below), followed by continuation records
  FO_REAL = 17,   // compiled kernels: carry out the deferred register swaps of the register bits in creg (see FOF_SW)
  FO_RELAY = 18,  // an uncontrolled swap of two tile bits as a relabelling: the layout pos (as FO_EXCH's) takes
                  // effect with no data moved
  FO_SYNC = 19    // a barrier of the tile's threads: every load of the tile is done before any store (a program
                  // whose relabellings move amplitudes between threads but that holds no exchange)
};

// flags
#define FOF_PRUNE 1u    // flush computed amplitudes with |a|^2 < 1e-14
#define FOF_REAL 2u     // MAT1: every matrix entry is real
#define FOF_D0ONE 4u    // DIAG*: m0 == 1 exactly (only bit-1 amplitudes change)
#define FOF_RXFORM 8u   // MAT1: m00, m11 real and m01, m10 imaginary (Rx-like)
// FOF_SW: deferred register swaps (compiled kernels only; the interpreter and
// the emulator carry every swap out at once and ignore it).  An X on register
// bit a under thread or out-of-tile controls only records, per thread, that
// the slot pairs along a are exchanged (sw ^= 1 << a) instead of moving them;
// physical slot j then holds logical slot j ^ sw.  FOF_SW on such an X marks
// it deferred; on an X controlled by one register bit C it adds that the
// thread's sw bit C moves to a as well; on a 2x2 or a diagonal on register
// bit a it makes the op exchange its matrix rows and columns (its d0 and d1)
// where the thread's sw bit a is set.  Exchanges, shared-memory ops and the
// store address the logical slots, which clears sw; FO_REAL carries out the
// pending swaps where an op needs the logical order in registers.
#define FOF_SW 16u
#define FOF_TGT_THR 32u // FO_GRADD: target is a thread-id bit (a)
#define FOF_TGT_CTX 64u // FO_GRADD: target is outside the tile (mask dg0)

// Kernel op codes: one flat dispatch per op (the type, the target's register
// bit, the matrix form and a register control are folded in by the host).
enum FOpCode : uint8_t {
  OC_EXCH = 0,
  OC_MAT1R = 1,       // + 3 * A + form (form 0 general, 1 real, 2 Rx-like): 1..15
  OC_MAT1L = 16,      // + form: 16..18
  OC_X1R = 19,        // + A: 19..23 (no register control)
  OC_X1RC = 24,       // + 5 * A + C: 24..48, X on register bit A controlled by register bit C only
  OC_X1L = 49,
  OC_DIAGR = 50,      // + A: 50..54 (general diag)
  OC_DIAGR1 = 55,     // + A: 55..59 (m0 == 1)
  OC_DIAGR1C = 60,    // + 5 * A + C: 60..84 (m0 == 1, controlled by register bit C only)
  OC_DIAGT = 85,
  OC_DIAGX = 86,
  OC_DIAG = 87,
  OC_SWAPS = 88,
  OC_MAT2S = 89,
  OC_GRADM = 90,      // + A: 90..93
  OC_GRADD = 94,
  OC_GRADM2 = 95,
  OC_X1S = 96,        // X on tile bit b with controls ctile, through shared memory (multi-controlled X)
  OC_CPHASE = 97,     // + A: 97..101, phase fan on register bit A
  OC_PPOLY = 102,     // phases of a run of controlled-phase gates
  OC_REAL = 103,      // FO_REAL: carry out the deferred swaps of the register bits in creg (compiled kernels)
  OC_RELAY = 104,     // FO_RELAY: the new layout's exchange offsets, no data moved
  OC_SYNC = 105,      // FO_SYNC: the tile's threads meet
  OC_NOP = 0xFF       // continuation record: dispatched as an op that does nothing
};

// FO_CPHASE: a run of phase gates diag(1, e^{i phi}) on one target (register
// bit A), each with at most one control, merged into one op.  Every amplitude
// whose bit A is 1 is multiplied by
//   T[k] * prod_{thread-id bits s set} H[s] * exp(i * sum_{terms: ctx & mask} angle)
// where k is the slot index with bit A removed.  m holds T[0 .. 2^(NR-1)-1]
// (constant and register-bit controls).  Continuation records (FO_CONT) follow
// the op; each has a 16-byte header that makes it a no-op (OC_NOP, no
// controls).  Record 0 holds H[0..7] (lanes, then warps) after its header;
// records 1.. hold the out-of-tile controls as (angle, global qubit mask)
// double2 pairs, 19 per record.  The op's `lmask` field holds the number of
// pairs and `ctile` the number of records.
//
// FO_PPOLY: a run of phase gates diag(1, p), |p| = 1, on any targets and with
// any controls, where each gate's target and register-bit controls name at
// most one register bit, merged into one op.  Term t multiplies the amplitude
// in slot j of thread tid of the tile at ctx by p_t when (ctx & cm_t) ==
// cm_t, (tid & tm_t) == tm_t and slot j has the term's register bit (if it
// names one).  Terms are grouped by (register bit, tm); lane g of each warp
// multiplies the phases of group g's terms that match the tile, in term
// order, and every thread multiplies the group products whose tm it matches
// into one factor per register bit (and one for groups without), which its
// slots then take.  The op's m holds, as uint32, the number of groups of
// each register bit (none first, then bit 0, 1, ...) and, from byte 32, one
// descriptor {tm, number of terms, record, unused} per group (at most
// KET_PPOLY_MAX_GROUPS); `lmask` is the number of groups, `b` the register
// bits that some group names and `ctile` the number of records.  A group's
// terms {double re, im; uint64 cm; uint64 unused} (32 bytes) fill records
// from its own (`record` counts from the op: 1 is the first after it), 9 per
// record after the record's 16-byte no-op header.
enum : int {
  KET_CPHASE_TERMS_PER_RECORD = 19,
  KET_PPOLY_TERMS_PER_RECORD = 9,
  KET_PPOLY_MAX_GROUPS = 14
};
struct PPolyTerm {
  double re, im;
  uint64_t cm, unused;
};
struct PPolyGroup {
  uint32_t tm, n, rec, unused;
};

struct FOp {
  // bytes 0..15: everything the kernel needs to decide whether and how an op runs
  uint8_t opc;                // FOpCode
  uint8_t a;                  // target: register bit / lane bit / thread-id bit / tile bit (by type)
  uint8_t flags;
  uint8_t creg;               // controls on register bits (bit k = register bit k)
  uint8_t cthr;               // controls on thread-id bits (lane bits 0-4, then the warp bits)
  int8_t d0, d1;              // FO_DIAG: tile bits of t0 (MSB) and t1, -1 = outside the tile
  uint8_t type;               // FOpType (host-side classification, used by the planner's tests)
  uint64_t cctx;              // controls on global bits outside the tile
  // bytes 16..31
  uint32_t lmask;             // lanes whose lane-bit controls hold (shuffle member mask)
  uint32_t ctile;             // shared-memory ops: controls as a tile-bit mask
  int16_t slot, anc;          // adjoint probes: gradient slot; FO_GRADM2: ancilla tile bit
  uint8_t b;                  // shared-memory ops: second tile bit
  uint8_t pad0[3];
  // bytes 32..63
  uint64_t dg0, dg1;          // DIAGX / DIAG / GRADD: global mask of the target(s) outside the tile
  uint8_t pos[KET_T2_BITS];   // FO_EXCH: new layout (role -> tile bit)
  uint32_t pad1;
  // FO_EXCH: m holds, as 12 uint16, the swizzled byte offset of each role's tile
  // bit in the exchange buffer (see exch_offset); other ops: the matrix
  double m[32];
};
static_assert(sizeof(FOp) == 64 + 256, "FOp layout");
static_assert(16 + KET_PPOLY_TERMS_PER_RECORD * sizeof(PPolyTerm) <= sizeof(FOp), "FO_PPOLY record");
static_assert(32 + KET_PPOLY_MAX_GROUPS * sizeof(PPolyGroup) <= sizeof(FOp::m), "FO_PPOLY groups");

// Byte offset of tile index i in the XOR-swizzled exchange buffer.  The map is
// linear over GF(2), so the offset of a sum of disjoint bits is the XOR of
// their offsets.
__host__ __device__ inline uint32_t exch_offset(uint32_t i, bool c64) {
  return c64 ? ((i ^ (((i >> 4) ^ (i >> 8)) & 15u)) << 3) : ((i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u)) << 4);
}

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
  int nreg;                        // register bits of the layouts (4 or 5)
  int pairbit;                     // index into ctxbits of the qubit that tells apart the two tiles a
                                   // thread holds, -1 = one tile per thread (see choose_pairbit)
  // filled by launch_fused2 from the fields above:
  uint64_t lgb[KET_T2_BITS];       // byte offset in the state of each role's tile bit, load layout
  uint64_t sgb[KET_T2_BITS];       // same, store layout
  uint32_t lbx[KET_T2_BITS];       // exchange-buffer offset of each role's tile bit, load layout
  int64_t drop_tile;               // staged form, test hook: this tile's copies are skipped (-1 = none)
};

}  // namespace ket
