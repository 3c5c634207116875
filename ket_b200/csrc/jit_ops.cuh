// jit_ops.cuh -- the body of a register-tiled pass compiled for one program.
//
// k_fused2 interprets a program: every thread fetches each op's header,
// dispatches on its op code and runs the matching code for the op's target
// register bit, register controls and matrix form.  A pass kernel compiled
// for one program (jit.cpp writes one `step<...>` call per op and compiles the
// source at run time) has all of that as template arguments instead:
//   * no op fetch or dispatch, and the code of consecutive ops can overlap;
//   * the ops' matrices and masks are constant-bank operands (COp);
//   * register controls are compile-time slot masks;
//   * X and CNOT on register bits are renamings of the tile's registers, so
//     they cost no instruction.
// Everything else -- matrices, exchange layouts, shuffle member masks,
// out-of-tile controls and phase-fan terms -- is still read from the op
// records at run time, so one compiled kernel serves every program of the
// same shape (a parameterised circuit at any angles, the same circuit on any
// state).  The arithmetic of every op is the interpreter's (fused_ops.cuh),
// so results equal k_fused2's bit for bit.
#pragma once

#include "fused_ops.cuh"

namespace ket {
namespace jit {

template <int NS>
__host__ __device__ constexpr uint32_t slotmask(int creg) {
  uint32_t v = 0;
  for (int j = 0; j < NS; j++)
    if ((j & creg) == creg) v |= 1u << j;
  return v;
}

// A swap the compiler resolves by renaming: the tile lives in registers
// indexed only by constants, so straight-line code needs no moves.
template <typename R>
__device__ __forceinline__ void swp(cpx<R>& a, cpx<R>& b) {
  const cpx<R> t = a;
  a = b;
  b = t;
}

// The part of an op record a compiled kernel reads on every tile: the FOp's
// 64-byte header and its first 8 matrix entries.  The host copies it for each
// launch into the module's constant array, so these reads are constant-bank
// operands rather than loads; the rest (phase-fan tables, 4x4 matrices) is read
// from the global copy of the program.
struct COp {
  uint8_t opc, a, flags, creg, cthr;
  int8_t d0, d1;
  uint8_t type;
  uint64_t cctx;
  uint32_t lmask, ctile;
  int16_t slot, anc;
  uint8_t b, pad0[3];
  uint64_t dg0, dg1;
  uint8_t pos[KET_T2_BITS];
  uint32_t pad1;
  double m[8];
};
static_assert(sizeof(COp) == 128, "COp layout");
#ifndef __CUDACC_RTC__  // checked where the host side includes this header
static_assert(__builtin_offsetof(COp, m) == __builtin_offsetof(FOp, m), "COp mirrors FOp");
static_assert(__builtin_offsetof(COp, dg0) == __builtin_offsetof(FOp, dg0), "COp mirrors FOp");
#endif

// FO_EXCH's new layout: its 12 uint16 exchange-buffer offsets are in m[0..2].
template <int NR>
__device__ __forceinline__ SLay<NR> exch_slay_c(const COp& c, int lane, int warp) {
  uint32_t bx[12];
#pragma unroll
  for (int r = 0; r < 12; r++)
    bx[r] = (uint32_t)((unsigned long long)__double_as_longlong(c.m[r >> 2]) >> (16 * (r & 3))) & 0xffffu;
  return make_slay<NR>(bx, lane, warp);
}

// ---------------------------------------------------------------- mbarriers
#define KET_STAGE_WAIT_NS 2000000000ull
// Status words the staged loop writes: KET_ERR_TIMEOUT and KET_ERR_CUDA of
// ket_sv.h (the run-time compiler sees only these headers; jit.cpp checks that
// the values agree).
constexpr int kStageTimeout = 5, kStageMisaligned = 4;

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the phase of `parity` to complete; false once KET_STAGE_WAIT_NS has
// passed without it.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try(bar, parity))
    if (global_ns() - t0 > KET_STAGE_WAIT_NS) return false;
  return true;
}
// Per-tile context of the ops.
struct Tile {
  uint32_t smb;   // exchange buffer (shared-memory address)
  int tid, lane, warp;
  int ltid;       // logical thread id: tid with the lane bits moved by deferred lane X gates (FOF_SW on FO_X1L)
  uint64_t ctx0;  // global index bits of the tile outside its 12 bits
  double* sgrad;  // adjoint probe passes: the CTA's partial sums [slot][warp] in shared memory
  uint32_t sw;    // deferred register swaps (FOF_SW): physical slot j holds logical slot j ^ sw
  uint32_t bar;   // staged form: the named barrier of the tile's thread group
  uint32_t xbar;  // register form: mbarrier on which the warps announce their reads of the exchange buffer
  uint32_t xcnt;  // register form: exchange-buffer uses so far (every warp takes the same ones)
  int* status;    // the call's status word (a bounded wait that ran out)
};

// The barrier among the threads that hold a tile.  In the staged form
// (KET_STAGED_THREADS defined: a CTA of two tile groups of that many threads)
// only the tile's group takes part, on its named barrier; otherwise the whole
// CTA.
__device__ __forceinline__ void tile_sync(const Tile& t) {
#ifdef KET_STAGED_THREADS
  asm volatile("bar.sync %0, %1;" ::"r"(t.bar), "n"(KET_STAGED_THREADS) : "memory");
#else
  (void)t;
  __syncthreads();
#endif
}

// Reuse of the exchange buffer.  An exchange writes the tile into the buffer,
// meets the other warps, and reads its new slots back; the next use of the
// buffer must not write before every warp has done those reads.  In the
// register form each warp announces its reads on an mbarrier right after
// them, and the next use waits for that phase -- normally long complete --
// instead of holding a barrier of the whole CTA.  The staged form keeps its
// group barrier.
__device__ __forceinline__ void xbuf_acquire(Tile& t) {
#ifdef KET_STAGED_THREADS
  tile_sync(t);
#else
  if (t.xcnt && !mbar_wait(t.xbar, (t.xcnt - 1) & 1)) atomicExch(t.status, kStageTimeout);
#endif
}
__device__ __forceinline__ void xbuf_release(Tile& t) {
#ifndef KET_STAGED_THREADS
  __syncwarp();
  if (t.lane == 0) mbar_arrive(t.xbar);
  t.xcnt++;
#else
  (void)t;
#endif
}

// The layout sl as seen from the logical slots and lanes: slot j's amplitude,
// held in physical slot j ^ sw of this thread, goes to the exchange-buffer
// address of logical slot j of the logical thread ltid.
template <int NR>
__device__ __forceinline__ SLay<NR> logical_slay(const SLay<NR>& sl, const Tile& t) {
  SLay<NR> w = sl;
#pragma unroll
  for (int k = 0; k < NR; k++)
    if ((t.sw >> k) & 1) w.b ^= sl.s[k];
  const uint32_t dl = (uint32_t)(t.tid ^ t.ltid) & 31u;  // lane bits moved by deferred lane X gates
#pragma unroll
  for (int r = 0; r < 5; r++)
    if ((dl >> r) & 1) w.b ^= sl.l[r];
  return w;
}

// Carry out the deferred swaps of register bits M (a compile-time mask).
template <typename R, int NR, int M>
__device__ __forceinline__ void realize_swaps(cpx<R> (&x)[1 << NR], Tile& t) {
#pragma unroll
  for (int k = 0; k < NR; k++) {
    if (!((M >> k) & 1)) continue;
    const bool s = (t.sw >> k) & 1;
#pragma unroll
    for (int j = 0; j < (1 << NR); j++) {
      if (j & (1 << k)) continue;
      const cpx<R> a = x[j], b = x[j | (1 << k)];
      x[j] = sel<R>(s, b, a);
      x[j | (1 << k)] = sel<R>(s, a, b);
    }
  }
  t.sw &= ~(uint32_t)M;
}

// Rare ops on the shared-memory copy of the tile, as in k_fused2.
template <typename R, int NR, int OPC, int FL>
__device__ __forceinline__ void smem_op(cpx<R> (&x)[1 << NR], const SLay<NR>& sl, const FOp* op, Tile& t) {
  constexpr int NT = 32 << (7 - NR);
  constexpr double thr = 1e-14, qthr = 1e-7;
  const uint4 h = __ldg(reinterpret_cast<const uint4*>(op));
  const uint4 h2 = __ldg(reinterpret_cast<const uint4*>(op) + 1);
  const uint32_t ct = h2.y;
  const int oa = (h.x >> 8) & 0xff, ob = (int)(h2.w & 0xffu);
  const double* M = op->m;
  const uint32_t smb = t.smb;
  xbuf_acquire(t);
  write_tile<R, NR>(smb, logical_slay<NR>(sl, t), x);
  // the tile comes back in logical order below; a probe (read-only, it keeps
  // the registers) never has swaps or lane moves pending: the program
  // generator carries them out or defers none before a probe
  t.sw = 0;
  t.ltid = t.tid;
  tile_sync(t);
  if constexpr (OPC == OC_GRADM2) {
    // Re<lambda| D |psi> with D 4x4 on tile bits a (MSB), b; the ancilla tile
    // bit selects psi (0) / lambda (1).  Read-only: the registers keep the tile.
    const int slot = (int16_t)(h2.z & 0xffff), anc = (int16_t)(h2.z >> 16);
    int b3[3] = {oa, ob, anc};
    for (int u = 1; u < 3; u++)
      for (int v = u; v > 0 && b3[v - 1] > b3[v]; v--) {
        const int w = b3[v];
        b3[v] = b3[v - 1];
        b3[v - 1] = w;
      }
    double acc = 0.0;
    for (uint32_t g = t.tid; g < (1u << (KET_T2_BITS - 3)); g += NT) {
      const uint32_t b0 = insert0_32(insert0_32(insert0_32(g, b3[0]), b3[1]), b3[2]);
      if ((b0 & ct) != ct) continue;
      const uint32_t idx[4] = {b0, b0 | (1u << ob), b0 | (1u << oa), b0 | (1u << oa) | (1u << ob)};
      cpx<R> v[4];
      for (int c = 0; c < 4; c++) lds(smb + swz<R>(idx[c]), v[c]);
      for (int r = 0; r < 4; r++) {
        cpx<R> s0 = mac2<R>((R)__ldg(M + 8 * r), (R)__ldg(M + 8 * r + 1), v[0], (R)__ldg(M + 8 * r + 2),
                            (R)__ldg(M + 8 * r + 3), v[1]);
        cpx<R> s1 = mac2<R>((R)__ldg(M + 8 * r + 4), (R)__ldg(M + 8 * r + 5), v[2], (R)__ldg(M + 8 * r + 6),
                            (R)__ldg(M + 8 * r + 7), v[3]);
        cpx<R> lam;
        lds(smb + swz<R>(idx[r] | (1u << anc)), lam);
        acc += (double)lam.re * (s0.re + s1.re) + (double)lam.im * (s0.im + s1.im);
      }
    }
    grad_accum(t.sgrad, slot, t.warp, t.lane, acc);
    xbuf_release(t);
    return;
  } else if constexpr (OPC == OC_X1S) {
    for (uint32_t g = t.tid; g < (1u << (KET_T2_BITS - 1)); g += NT) {
      const uint32_t i0 = insert0_32(g, ob);
      if ((i0 & ct) != ct) continue;
      cpx<R> t0, t1;
      lds(smb + swz<R>(i0), t0);
      lds(smb + swz<R>(i0 | (1u << ob)), t1);
      sts(smb + swz<R>(i0), t1);
      sts(smb + swz<R>(i0 | (1u << ob)), t0);
    }
  } else if constexpr (OPC == OC_DIAG) {
    const int b0t = (int8_t)(h.y >> 8), b1t = (int8_t)(h.y >> 16);
    const uint64_t dg0 = __ldg(reinterpret_cast<const unsigned long long*>(op) + 4);
    const uint64_t dg1 = __ldg(reinterpret_cast<const unsigned long long*>(op) + 5);
    const int u0 = (int)((t.ctx0 & dg0) != 0), u1 = (int)((t.ctx0 & dg1) != 0);
    for (uint32_t i = t.tid; i < (1u << KET_T2_BITS); i += NT) {
      if ((i & ct) != ct) continue;
      const int k0 = b0t >= 0 ? (int)((i >> b0t) & 1) : u0;
      const int k1 = b1t >= 0 ? (int)((i >> b1t) & 1) : u1;
      const int kk = 2 * k0 + k1;
      cpx<R> v;
      lds(smb + swz<R>(i), v);
      v = cmul<R>((R)__ldg(M + 2 * kk), (R)__ldg(M + 2 * kk + 1), v);
      sts(smb + swz<R>(i), v);
    }
  } else {
    const int ta = oa, tb = ob;
    const int lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
    for (uint32_t g = t.tid; g < (1u << (KET_T2_BITS - 2)); g += NT) {
      const uint32_t b0 = insert0_32(insert0_32(g, lo), hi);
      if ((b0 & ct) != ct) continue;
      const uint32_t i1 = b0 | (1u << tb), i2 = b0 | (1u << ta), i3 = b0 | (1u << ta) | (1u << tb);
      if constexpr (OPC == OC_SWAPS) {
        cpx<R> t1, t2;
        lds(smb + swz<R>(i1), t1);
        lds(smb + swz<R>(i2), t2);
        sts(smb + swz<R>(i1), t2);
        sts(smb + swz<R>(i2), t1);
      } else {
        const uint32_t idx[4] = {b0, i1, i2, i3};
        cpx<R> v[4];
        for (int c = 0; c < 4; c++) lds(smb + swz<R>(idx[c]), v[c]);
        for (int r = 0; r < 4; r++) {
          cpx<R> s0 = mac2<R>((R)__ldg(M + 8 * r), (R)__ldg(M + 8 * r + 1), v[0], (R)__ldg(M + 8 * r + 2),
                              (R)__ldg(M + 8 * r + 3), v[1]);
          cpx<R> s1 = mac2<R>((R)__ldg(M + 8 * r + 4), (R)__ldg(M + 8 * r + 5), v[2], (R)__ldg(M + 8 * r + 6),
                              (R)__ldg(M + 8 * r + 7), v[3]);
          cpx<R> y;
          y.re = s0.re + s1.re;
          y.im = s0.im + s1.im;
          if (FL & FOF_PRUNE) prune_amp(y, thr, qthr);
          sts(smb + swz<R>(idx[r]), y);
        }
      }
    }
  }
  tile_sync(t);
  read_tile<R, NR>(smb, sl, x);
  xbuf_release(t);
}

// One op of the program.  OPC: op code; FL: flags; CREG: register controls;
// CTHR: thread-id controls; CCTX: whether the op has controls outside the
// tile; LA: the lane or thread-id bit of lane ops and thread diagonals.
// c: the op's constant copy; g: the op in the global copy of the program.
template <typename R, int NR, int OPC, int FL, int CREG, uint32_t CTHR, bool CCTX, int LA>
__device__ __forceinline__ void step(cpx<R> (&x)[1 << NR], SLay<NR>& sl, const COp& c, const FOp* g,
                                     Tile& t) {
  constexpr int NS = 1 << NR;
  constexpr double thr = 1e-14, qthr = 1e-7;
  if constexpr (OPC == OC_EXCH) {
    xbuf_acquire(t);
    write_tile<R, NR>(t.smb, logical_slay<NR>(sl, t), x);
    t.sw = 0;
    t.ltid = t.tid;
    tile_sync(t);
    sl = exch_slay_c<NR>(c, t.lane, t.warp);
    read_tile<R, NR>(t.smb, sl, x);
    xbuf_release(t);
    return;
  }
  if constexpr (OPC == OC_REAL) {
    realize_swaps<R, NR, CREG>(x, t);
    return;
  }
  if constexpr (OPC == OC_RELAY) {  // a relabelling swap: the data stays, the layout changes
    sl = exch_slay_c<NR>(c, t.lane, t.warp);
    return;
  }
  if constexpr (OPC == OC_SYNC) {  // every load of the tile done before any store
    tile_sync(t);
    return;
  }
  if constexpr (CCTX) {
    if ((t.ctx0 & c.cctx) != c.cctx) return;  // uniform over the CTA
  }
  if constexpr (OPC == OC_SWAPS || OPC == OC_MAT2S || OPC == OC_DIAG || OPC == OC_X1S || OPC == OC_GRADM2) {
    smem_op<R, NR, OPC, FL>(x, sl, g, t);
    return;
  }
  if constexpr ((OPC >= OC_GRADM && OPC < OC_GRADM + 4) || OPC == OC_GRADD) {
    // adjoint probe <lambda|D|psi> over this thread's amplitudes (register bit
    // 3 selects psi / lambda); every lane takes part in the warp sum, so
    // threads whose thread-bit controls fail add zero
    bool thr_ok = true;
    if constexpr (CTHR != 0) thr_ok = ((uint32_t)t.ltid & CTHR) == CTHR;
    const uint32_t smask = thr_ok ? (slotmask<NS>(CREG) & full_mask<NS>()) : 0u;
    double acc;
    if constexpr (OPC == OC_GRADD) {
      const R d0r = (R)c.m[0], d0i = (R)c.m[1], d1r = (R)c.m[2], d1i = (R)c.m[3];
      if (c.flags & (FOF_TGT_THR | FOF_TGT_CTX)) {
        const bool one = (c.flags & FOF_TGT_CTX) ? (t.ctx0 & c.dg0) != 0 : (bool)((t.ltid >> c.a) & 1);
        acc = grad_d<R, -1>(x, one ? d1r : d0r, one ? d1i : d0i, one ? d1r : d0r, one ? d1i : d0i, smask);
      } else if (c.a == 0) {
        acc = grad_d<R, 0>(x, d0r, d0i, d1r, d1i, smask);
      } else if (c.a == 1) {
        acc = grad_d<R, 1>(x, d0r, d0i, d1r, d1i, smask);
      } else {
        acc = grad_d<R, 2>(x, d0r, d0i, d1r, d1i, smask);
      }
    } else {
      const R d[8] = {(R)c.m[0], (R)c.m[1], (R)c.m[2], (R)c.m[3], (R)c.m[4], (R)c.m[5], (R)c.m[6], (R)c.m[7]};
      acc = grad_m<R, OPC - OC_GRADM>(x, d, smask);
    }
    grad_accum(t.sgrad, c.slot, t.warp, t.lane, acc);
    return;
  }
  if constexpr (CTHR != 0) {
    if (((uint32_t)t.ltid & CTHR) != CTHR) return;
  }
  constexpr uint32_t SM = slotmask<NS>(CREG);
  if constexpr (OPC >= OC_MAT1R && OPC < OC_MAT1R + 15) {
    constexpr int A = (OPC - OC_MAT1R) / 3, F = (OPC - OC_MAT1R) % 3;
    if constexpr ((FL & FOF_SW) != 0) {
      // slot pairs along A exchanged in this thread: rows and columns of the matrix too
      const bool s = (t.sw >> A) & 1;
      const R m[8] = {(R)(s ? c.m[6] : c.m[0]), (R)(s ? c.m[7] : c.m[1]), (R)(s ? c.m[4] : c.m[2]),
                      (R)(s ? c.m[5] : c.m[3]), (R)(s ? c.m[2] : c.m[4]), (R)(s ? c.m[3] : c.m[5]),
                      (R)(s ? c.m[0] : c.m[6]), (R)(s ? c.m[1] : c.m[7])};
      mat1_reg<R, A, F, NS>(x, m, SM);
    } else {
      const R m[8] = {(R)c.m[0], (R)c.m[1], (R)c.m[2], (R)c.m[3], (R)c.m[4], (R)c.m[5], (R)c.m[6], (R)c.m[7]};
      mat1_reg<R, A, F, NS>(x, m, SM);
    }
  } else if constexpr (OPC >= OC_MAT1L && OPC < OC_MAT1L + 3) {
    const uint32_t members = c.lmask;
    const bool bitv = (t.lane >> LA) & 1;
    // own output = c0 * own + c1 * partner
    const R c0r = (R)(bitv ? c.m[6] : c.m[0]), c0i = (R)(bitv ? c.m[7] : c.m[1]);
    const R c1r = (R)(bitv ? c.m[4] : c.m[2]), c1i = (R)(bitv ? c.m[5] : c.m[3]);
#pragma unroll
    for (int j = 0; j < NS; j++) {
      if (!((SM >> j) & 1)) continue;
      const cpx<R> p = shfl_xor_c<R>(x[j], 1 << LA, members);
      cpx<R> y;
      if constexpr (OPC == OC_MAT1L + 1) {
        y.re = fma(c0r, x[j].re, c1r * p.re);
        y.im = fma(c0r, x[j].im, c1r * p.im);
      } else if constexpr (OPC == OC_MAT1L + 2) {
        y.re = fma(c0r, x[j].re, -c1i * p.im);
        y.im = fma(c0r, x[j].im, c1i * p.re);
      } else {
        y = mac2<R>(c0r, c0i, x[j], c1r, c1i, p);
      }
      x[j] = y;
    }
  } else if constexpr (OPC >= OC_X1R && OPC < OC_X1R + 5) {
    constexpr int A = OPC - OC_X1R;
    if constexpr ((FL & FOF_SW) != 0) {
      t.sw ^= 1u << A;  // deferred: this thread passed the op's controls
      return;
    }
#pragma unroll
    for (int j = 0; j < NS; j++)
      if (!(j & (1 << A)) && ((SM >> j) & 1)) swp<R>(x[j], x[j | (1 << A)]);
  } else if constexpr (OPC >= OC_X1RC && OPC < OC_X1RC + 25) {
    constexpr int A = (OPC - OC_X1RC) / 5, C = (OPC - OC_X1RC) % 5;
#pragma unroll
    for (int j = 0; j < NS; j++)
      if (!(j & (1 << A)) && (j & (1 << C))) swp<R>(x[j], x[j | (1 << A)]);
    // a deferred swap on the control bit: the pairs whose logical control
    // bit is 1 are the other half, which flipping every pair along A adds
    if constexpr ((FL & FOF_SW) != 0) t.sw ^= ((t.sw >> C) & 1u) << A;
  } else if constexpr (OPC == OC_X1L) {
    if constexpr ((FL & FOF_SW) != 0) {
      t.ltid ^= 1 << LA;  // deferred: this thread passed the op's controls; its amplitudes stay
      return;
    }
    const uint32_t members = c.lmask;
#pragma unroll
    for (int j = 0; j < NS; j++)
      if ((SM >> j) & 1) x[j] = shfl_xor_c<R>(x[j], 1 << LA, members);
  } else if constexpr ((OPC >= OC_DIAGR && OPC < OC_DIAGR + 5) || (OPC >= OC_DIAGR1 && OPC < OC_DIAGR1 + 5)) {
    constexpr bool ONE = OPC >= OC_DIAGR1;
    constexpr int A = OPC - (ONE ? OC_DIAGR1 : OC_DIAGR);
    if constexpr ((FL & FOF_SW) != 0 && !ONE) {
      const bool s = (t.sw >> A) & 1;
      diag_reg<R, A, ONE, NS>(x, (R)(s ? c.m[2] : c.m[0]), (R)(s ? c.m[3] : c.m[1]), (R)(s ? c.m[0] : c.m[2]),
                              (R)(s ? c.m[1] : c.m[3]), SM);
    } else {
      diag_reg<R, A, ONE, NS>(x, (R)c.m[0], (R)c.m[1], (R)c.m[2], (R)c.m[3], SM);
    }
  } else if constexpr (OPC >= OC_DIAGR1C && OPC < OC_DIAGR1C + 25) {
    constexpr int A = (OPC - OC_DIAGR1C) / 5, C = (OPC - OC_DIAGR1C) % 5;
    diag1c_reg<R, A, C, NS>(x, (R)c.m[2], (R)c.m[3]);
  } else if constexpr (OPC >= OC_CPHASE && OPC < OC_CPHASE + 5) {
    constexpr int A = OPC - OC_CPHASE;
    const uint4 h2 = __ldg(reinterpret_cast<const uint4*>(g) + 1);
    phase_fan<R, A, 1, NS>(reinterpret_cast<cpx<R>(&)[1][NS]>(x), g, h2.x, t.ctx0, 0, t.tid, t.ltid);
  } else if constexpr (OPC == OC_PPOLY) {
    phase_poly<R, 1, NS>(reinterpret_cast<cpx<R>(&)[1][NS]>(x), g, t.ctx0, 0, t.tid, t.ltid);
  } else if constexpr (OPC == OC_DIAGT || OPC == OC_DIAGX) {
    bool one;
    if constexpr (OPC == OC_DIAGT) one = (t.ltid >> LA) & 1;
    else one = (t.ctx0 & c.dg0) != 0;
    if ((FL & FOF_D0ONE) && !one) return;
    phase_all<R, NS>(x, (R)(one ? c.m[2] : c.m[0]), (R)(one ? c.m[3] : c.m[1]), SM);
  } else {
    // handled above (the exchange and the shared-memory ops return early)
    static_assert(OPC == OC_NOP || OPC == OC_EXCH || OPC == OC_SWAPS || OPC == OC_MAT2S || OPC == OC_DIAG ||
                      OPC == OC_X1S || OPC == OC_REAL || OPC == OC_RELAY || OPC == OC_SYNC || (OPC >= OC_GRADM && OPC <= OC_GRADM2),
                  "op code without a compiled form");
    return;
  }
  if constexpr ((FL & FOF_PRUNE) != 0) prune_slots<R, NS>(x, thr, qthr);
}

// ---------------------------------------------------------------- store
// The store base of the thread's logical lane: gs (the physical lane's and
// warp's offsets) corrected for the lane bits deferred lane X gates moved.
__device__ __forceinline__ uint64_t logical_base(uint64_t gs, const uint64_t* sgb, const Tile& t) {
  const uint32_t dl = (uint32_t)(t.tid ^ t.ltid) & 31u;
#pragma unroll
  for (int r = 0; r < 5; r++)
    if ((dl >> r) & 1) gs += ((t.ltid >> r) & 1) ? sgb[r] : (uint64_t)0 - sgb[r];
  return gs;
}
// Store the tile: physical slot j holds logical slot j ^ t.sw, which goes to
// the address of the logical slot.  With a register bit k swapped, bit k of
// the address offset is taken where the physical slot's bit k is clear: the
// base gains that bit's offset and the slot's own term turns negative
// (unsigned arithmetic, exact modulo 2^64).
template <typename R, int NR>
__device__ __forceinline__ void store_tile(char* p, const uint64_t* rb, uint32_t sw, const cpx<R> (&x)[1 << NR]) {
  typedef typename Vec2<R>::T V;
  uint64_t sk[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) {
    const bool s = (sw >> k) & 1;
    if (s) p += rb[k];
    sk[k] = s ? (uint64_t)0 - rb[k] : rb[k];
  }
#pragma unroll
  for (int j = 0; j < (1 << NR); j++) {
    uint64_t o = 0;
#pragma unroll
    for (int k = 0; k < NR; k++)
      if (j & (1 << k)) o += sk[k];
    st_amp<R>(reinterpret_cast<V*>(p + o), x[j]);
  }
}

// The tile loop around a program: load each tile in the load layout, run the
// ops, store it in the store layout -- the same addressing as k_fused2.
// GRAD: an adjoint probe pass; its probes add into per-(slot, warp) partial
// sums in shared memory after the exchange buffer, written to a.gpart per CTA
// at the end (k_grad_reduce adds them in a fixed order).
template <typename R, int NR, bool GRAD = false, typename Body>
__device__ __forceinline__ void run_tiles(const Pass2Args& a, Body body) {
  constexpr int NW = 7 - NR, NS = 1 << NR, NT = 32 << NW;
  typedef typename Vec2<R>::T V;
  extern __shared__ __align__(128) unsigned char smraw[];
  Tile t;
  t.smb = (uint32_t)__cvta_generic_to_shared(smraw);
  t.tid = threadIdx.x;
  t.lane = t.tid & 31;
  t.warp = t.tid >> 5;
  t.sgrad = reinterpret_cast<double*>(smraw + ((size_t)sizeof(V) << KET_T2_BITS));
  __shared__ __align__(8) unsigned long long xbar_word;
  t.xbar = (uint32_t)__cvta_generic_to_shared(&xbar_word);
  t.xcnt = 0;
  t.status = a.status;
  if (t.tid == 0) {
    mbar_init(t.xbar, NT / 32);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if constexpr (GRAD)
    for (int i = t.tid; i < a.nslots * 8; i += NT) t.sgrad[i] = 0.0;
  __syncthreads();
  char* const amp = reinterpret_cast<char*>(a.amp);
  const uint64_t ntiles = uint64_t(1) << (a.n - KET_T2_BITS);
  uint64_t gl = 0, gs = 0;
#pragma unroll
  for (int r = 0; r < 5; r++)
    if ((t.lane >> r) & 1) {
      gl += a.lgb[r];
      gs += a.sgb[r];
    }
#pragma unroll
  for (int r = 0; r < NW; r++)
    if ((t.warp >> r) & 1) {
      gl += a.lgb[5 + r];
      gs += a.sgb[5 + r];
    }
  cpx<R> x[NS];
  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    t.ctx0 = ctx_of(a, tile);
    {
      const char* p = amp + t.ctx0 * sizeof(V) + gl;
#pragma unroll
      for (int j = 0; j < NS; j++) {
        uint64_t o = 0;
#pragma unroll
        for (int k = 0; k < NR; k++)
          if (j & (1 << k)) o += a.lgb[5 + NW + k];
        x[j] = ld_amp<R>(reinterpret_cast<const V*>(p + o));
      }
    }
    SLay<NR> sl = make_slay<NR>(a.lbx, t.lane, t.warp);
    t.sw = 0;
    t.ltid = t.tid;
    body(x, sl, t);
    store_tile<R, NR>(amp + t.ctx0 * sizeof(V) + logical_base(gs, a.sgb, t), a.sgb + 5 + NW, t.sw, x);
  }
  if constexpr (GRAD) {
    __syncthreads();
    for (int i = t.tid; i < a.nslots * 8; i += NT) a.gpart[(size_t)blockIdx.x * a.nslots * 8 + i] = t.sgrad[i];
  }
}

// ---------------------------------------------------------------- staged tile loop
// The same pass with every tile staged in shared memory by the tensor-memory
// accelerator.  One CTA per SM runs two tile groups of NT threads (16 warps
// at 4 register bits, as the register-load form's two CTAs) over NSTAGE
// stages: the CTA's k-th tile lands in stage k % NSTAGE and group k % 2 runs
// it, so while both groups compute, the next tile is already on its way.  A
// tile lands in its natural order -- byte offset = tile index x amplitude
// size, tile bits 0-4 the 5 contiguous low qubits, bits 5-11 the pass's high
// qubits -- as 128 boxes of a 2-D tensor map over the state, {the 2^5
// amplitudes of a row (as 2 x 32 reals), rows}: box j is the row at the
// tile's context plus the high qubits set in j.
//
// Per tile k in stage s: the group waits until the copy of tile k has been
// issued (a per-stage count in shared memory: the mbarrier's phase parity
// alone cannot tell tile k from tile k - NSTAGE when the group runs ahead of
// the other one) and for `full[s]`, reads the tile into
// registers in the load layout, runs the ops -- exchanges and shared-memory
// ops use the stage itself as their buffer, on the group's own named barrier
// -- then every thread fences its shared-memory writes against the async
// proxy, the group meets at its barrier, and the group's first warp arms
// `full[s]` with the byte count of tile k + NSTAGE and issues its boxes (4 per
// lane) before the group stores its registers straight to the state.  The
// stage's next user is the other group, which waits for `full[s]` again.
// Every wait is bounded in time: past KET_STAGE_WAIT_NS the status word gets
// KET_ERR_TIMEOUT, the group (all together, by a barrier vote) stops, and
// before the CTA exits thread 0 waits for the last copy issued into every
// stage.
struct __align__(64) TMap {
  unsigned long long w[16];
};

// Wait until *p >= want (a count another warp of the CTA raises); false once
// KET_STAGE_WAIT_NS has passed without it.
__device__ __forceinline__ bool wait_count(const uint32_t* p, uint32_t want) {
  const volatile uint32_t* v = p;
  if (*v >= want) return true;
  const uint64_t t0 = global_ns();
  while (*v < want)
    if (global_ns() - t0 > KET_STAGE_WAIT_NS) return false;
  return true;
}
__device__ __forceinline__ void tma_load2(uint32_t dst, const TMap* m, int row, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"((unsigned long long)m), "r"(0), "r"(row), "r"(bar)
      : "memory");
}
// AND of v over the NT threads of the group on named barrier `bar`.
template <int NT>
__device__ __forceinline__ bool all_group_threads(bool v, uint32_t bar) {
  uint32_t r;
  asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred p, %2, %3, q;\n selp.u32 %0, 1, 0, p;\n}"
               : "=r"(r)
               : "r"((uint32_t)v), "r"(bar), "n"(NT)
               : "memory");
  return r != 0;
}

template <typename R, int NR, int NSTAGE, typename Body>
__device__ __forceinline__ void run_tiles_staged(const Pass2Args& a, const TMap* tm, Body body) {
  constexpr int NW = 7 - NR, NS = 1 << NR, NT = 32 << NW;  // NT: threads of one tile group
  constexpr int NG = 2;                                      // tile groups per CTA
  static_assert(NSTAGE > NG, "a stage in flight beside each group's");
  typedef typename Vec2<R>::T V;
  constexpr uint32_t TB = (uint32_t)sizeof(V) << KET_T2_BITS;  // bytes per tile
  constexpr int nbox = 1 << (KET_T2_BITS - 5);                 // one box per row of 2^5 amplitudes
  constexpr uint32_t boxb = TB / (uint32_t)nbox;
  extern __shared__ __align__(1024) unsigned char smraw[];
  const uint32_t sm0 = (uint32_t)__cvta_generic_to_shared(smraw);
  const uint32_t full0 = sm0 + NSTAGE * TB;
  uint32_t* const issued = reinterpret_cast<uint32_t*>(smraw + NSTAGE * TB + 8 * NSTAGE);  // fills per stage
  const int tid = threadIdx.x;
  if (sm0 & 1023u) {  // the copies need aligned stages: refuse rather than misalign
    if (tid == 0) atomicExch(a.status, kStageMisaligned);
    return;
  }
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; s++) {
      mbar_init(full0 + 8 * s, 1);
      *(volatile uint32_t*)(issued + s) = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  const uint64_t ntiles = uint64_t(1) << (a.n - KET_T2_BITS);
  const uint32_t nk = ntiles > blockIdx.x ? (uint32_t)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0u;
  const int grp = tid / NT;
  Tile t;
  t.tid = tid - grp * NT;
  t.lane = t.tid & 31;
  t.warp = t.tid >> 5;
  t.bar = 1 + grp;
  // the CTA's k-th tile into stage k % NSTAGE, by one whole warp (4 boxes a lane)
  auto fill = [&](uint32_t k) {
    const uint32_t s = k % NSTAGE;
    const uint64_t tile = blockIdx.x + (uint64_t)k * gridDim.x;
    if ((int64_t)tile == a.drop_tile) return;  // test hook: the group's wait for it runs out
    const uint64_t ctx0 = ctx_of(a, tile);
    if (t.lane == 0) {
      *(volatile uint32_t*)(issued + s) = k / NSTAGE + 1;
      mbar_expect_tx(full0 + 8 * s, TB);
    }
    __syncwarp();
    for (int j = t.lane; j < nbox; j += 32) {
      uint64_t idx = ctx0;
#pragma unroll
      for (int e = 0; e < KET_T2_BITS - 5; e++)
        if ((j >> e) & 1) idx |= uint64_t(1) << a.hbits[e];
      tma_load2(sm0 + s * TB + (uint32_t)j * boxb, tm, (int)(idx >> 5), full0 + 8 * s);
    }
  };
  if (grp == 0 && t.warp == 0)
    for (uint32_t k = 0; k < nk && k < (uint32_t)NSTAGE; k++) fill(k);
  char* const amp = reinterpret_cast<char*>(a.amp);
  uint64_t gs = 0;
#pragma unroll
  for (int r = 0; r < 5; r++)
    if ((t.lane >> r) & 1) gs += a.sgb[r];
#pragma unroll
  for (int r = 0; r < NW; r++)
    if ((t.warp >> r) & 1) gs += a.sgb[5 + r];
  // the staged tile in the load layout: role r's tile bit at byte sizeof(V) << bit
  uint32_t nbx[KET_T2_BITS];
#pragma unroll
  for (int r = 0; r < KET_T2_BITS; r++) nbx[r] = (uint32_t)sizeof(V) << a.load_pos[r];
  const SLay<NR> nat = make_slay<NR>(nbx, t.lane, t.warp);
  cpx<R> x[NS];
  for (uint32_t k = grp; k < nk; k += NG) {
    const uint32_t s = k % NSTAGE;
    const bool landed = wait_count(issued + s, k / NSTAGE + 1) && mbar_wait(full0 + 8 * s, (k / NSTAGE) & 1);
    if (!all_group_threads<NT>(landed, t.bar)) {
      if (t.tid == 0) atomicExch(a.status, kStageTimeout);
      break;
    }
    const uint64_t tile = blockIdx.x + (uint64_t)k * gridDim.x;
    t.ctx0 = ctx_of(a, tile);
    t.smb = sm0 + s * TB;
    read_tile<R, NR>(t.smb, nat, x);
    SLay<NR> sl = make_slay<NR>(a.lbx, t.lane, t.warp);
    t.sw = 0;
    t.ltid = t.tid;
    body(x, sl, t);
    // the stage is free once every thread of the group is past its last
    // shared-memory access; its next copy comes from the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tile_sync(t);
    if (t.warp == 0 && k + NSTAGE < nk) fill(k + NSTAGE);
    store_tile<R, NR>(amp + t.ctx0 * sizeof(V) + logical_base(gs, a.sgb, t), a.sgb + 5 + NW, t.sw, x);
  }
  // no copy may still be landing when the CTA exits
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < NSTAGE; s++)
      if (issued[s] && !mbar_wait(full0 + 8 * s, (issued[s] - 1) & 1)) atomicExch(a.status, kStageTimeout);
}

}  // namespace jit
}  // namespace ket
