// kernels_fused.cu -- the register-tiled fused gate pass.
//
// A CTA owns a tile of 2^12 amplitudes at a time: the L lowest qubits
// (contiguous in HBM) plus 12-L high qubits chosen by the planner.  The tile's
// 12 bits are split into 5 lane bits, NW warp bits and NR register bits
// (NW + NR = 7): ordinary passes use NR = 5 (128 threads holding 32 amplitudes
// each, two CTAs per SM, so one CTA's tile loads overlap the other's
// arithmetic), adjoint passes NR = 4 (256 threads, 16 amplitudes).  A gate whose
// target is a register bit is applied inside each thread, a gate on a lane
// bit uses warp shuffles, and a gate on a warp bit first re-lays the tile out
// through shared memory (FO_EXCH).  Diagonal gates need no pairing and apply
// on any qubit, in or out of the tile.  The global load and store use a
// layout whose lane bits are the tile's low bits, so every warp touches whole
// 128-byte lines.  A pass costs one read and one write of the state however
// many gates it holds.
//
// The kernel is issue-bound, so the per-op overhead is kept small:
//   * an op's first 16 bytes hold everything needed to skip or dispatch it,
//     and the next op's header is fetched while the current one runs;
//   * the exchange buffer is XOR-swizzled with a map that is linear over
//     GF(2), so the 16 slot addresses of a thread are its base address XOR
//     combinations of four per-layout constants (15 XORs per layout);
//   * global addresses are a per-thread base plus sums of four per-layout
//     byte offsets computed on the host;
//   * threads whose thread-bit controls fail skip an op outright (shuffles
//     use the mask of lanes that take part);
//   * the per-gate pruning of the reference (|a|^2 < 1e-14 -> 0) is screened
//     with FP32 min/max over the high words of all 16 amplitudes; the exact
//     FP64 test runs only when some amplitude is below 1e-7 in magnitude.
#include <algorithm>

#include "common.cuh"
#include "fused_ops.cuh"
#include "launch.h"

namespace ket {

namespace {

__constant__ uint32_t c_slotmask[32];  // slots j < 32 with (j & creg) == creg

// ---------------------------------------------------------------- the pass
template <typename R, bool GRAD, int TT, int NR>
__global__ void __launch_bounds__(32 << (7 - NR), NR == 5 ? 2 : 1) k_fused2(Pass2Args a) {
  constexpr int NW = 7 - NR, NT = 32 << NW, NS = 1 << NR;  // warp bits, threads, slots per thread
  typedef typename Vec2<R>::T V;
  extern __shared__ __align__(128) unsigned char smraw[];
  // shared memory: one exchange buffer per tile a thread holds | gradient partials
  constexpr uint32_t TB = (uint32_t)sizeof(cpx<R>) << KET_T2_BITS;
  const uint32_t smb = (uint32_t)__cvta_generic_to_shared(smraw);
  double* sgrad = reinterpret_cast<double*>(smraw + TB * TT);  // [slot][warp]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (GRAD) {
    for (int i = threadIdx.x; i < a.nslots * 8; i += NT) sgrad[i] = 0.0;
    __syncthreads();
  }
  constexpr double thr = 1e-14, qthr = 1e-7;  // accumulate()'s threshold (statevector.ts:24) and its root
  char* const amp = reinterpret_cast<char*>(a.amp);
  // Each thread holds TT tiles that differ only in tile-index bit a.pairbit, a
  // qubit outside the tile that no op of the pass reads: every op then acts
  // on all TT tiles the same way.
  const uint64_t ngroups = (uint64_t(1) << (a.n - KET_T2_BITS)) / TT;
  const uint64_t pairq = TT > 1 ? uint64_t(1) << a.ctxbits[a.pairbit] : 0;
  cpx<R> x[TT][NS];

  for (uint64_t grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const uint64_t tile0 = TT > 1 ? insert0(grp, a.pairbit) : grp;
    const uint64_t ctx0 = ctx_of(a, tile0);
    {
      uint64_t gl = 0;
#pragma unroll
      for (int r = 0; r < 5; r++)
        if ((lane >> r) & 1) gl += a.lgb[r];
#pragma unroll
      for (int r = 0; r < NW; r++)
        if ((warp >> r) & 1) gl += a.lgb[5 + r];
#pragma unroll
      for (int t = 0; t < TT; t++) {
        const char* p = amp + (ctx0 | (t ? pairq : 0)) * sizeof(V) + gl;
#pragma unroll
        for (int j = 0; j < NS; j++) {
          uint64_t o = 0;
#pragma unroll
          for (int k = 0; k < NR; k++)
            if (j & (1 << k)) o += a.lgb[5 + NW + k];
          x[t][j] = ld_amp<R>(reinterpret_cast<const V*>(p + o));
        }
      }
    }
    SLay<NR> sl = make_slay<NR>(a.lbx, lane, warp);
    uint4 hn = a.nops > 0 ? __ldg(reinterpret_cast<const uint4*>(a.ops)) : make_uint4(0u, 0u, 0u, 0u);
    for (int k = 0; k < a.nops; k++) {
      const FOp* op = a.ops + k;
      const uint4 h = hn;
      if (k + 1 < a.nops) hn = __ldg(reinterpret_cast<const uint4*>(op + 1));
      // the matrix is loaded before decoding, so its latency overlaps the dispatch
      const double2* mp = reinterpret_cast<const double2*>(op->m);
      const double2 q0 = __ldg(mp), q1 = __ldg(mp + 1), q2 = __ldg(mp + 2), q3 = __ldg(mp + 3);
      const int opc = h.x & 0xff, oa = (h.x >> 8) & 0xff;
      const uint32_t fl = (h.x >> 16) & 0xffu, creg = h.x >> 24, cthr = h.y & 0xffu;
      if (opc == OC_EXCH) {
        __syncthreads();
#pragma unroll
        for (int t = 0; t < TT; t++) write_tile<R, NR>(smb + t * TB, sl, x[t]);
        __syncthreads();
        sl = exch_slay<NR>(op, lane, warp);
#pragma unroll
        for (int t = 0; t < TT; t++) read_tile<R, NR>(smb + t * TB, sl, x[t]);
        continue;
      }
      if (opc == OC_RELAY) {  // a relabelling swap: the data stays, the layout changes
        sl = exch_slay<NR>(op, lane, warp);
        continue;
      }
      if (opc == OC_SYNC) {  // every load of the tile done before any store
        __syncthreads();
        continue;
      }
      const uint64_t cctx = ((uint64_t)h.w << 32) | h.z;
      if ((ctx0 & cctx) != cctx) continue;  // uniform over the CTA (and the same for all TT tiles)
      const double* M = op->m;
      if (opc == OC_SWAPS || opc == OC_MAT2S || opc == OC_GRADM2 || opc == OC_DIAG || opc == OC_X1S) {
        // Rare ops (controlled swaps, dense 4x4s, two-qubit diagonals,
        // multi-controlled X, two-qubit probes) run on the shared-memory copy of
        // the tiles, in the current layout, with small code.
        if (opc == OC_GRADM2 && !GRAD) continue;
        const uint4 h2 = __ldg(reinterpret_cast<const uint4*>(op) + 1);
        const uint32_t ct = h2.y;
        const int ob = (int)(h2.w & 0xffu);
        __syncthreads();
#pragma unroll
        for (int t = 0; t < TT; t++) write_tile<R, NR>(smb + t * TB, sl, x[t]);
        __syncthreads();
        const int ta = oa, tb = ob;
        if (GRAD && opc == OC_GRADM2) {
          const int slot = (int16_t)(h2.z & 0xffff), anc = (int16_t)(h2.z >> 16);
          int b3[3] = {ta, tb, anc};
          for (int u = 1; u < 3; u++)
            for (int v = u; v > 0 && b3[v - 1] > b3[v]; v--) { int w = b3[v]; b3[v] = b3[v - 1]; b3[v - 1] = w; }
          double acc = 0.0;
          for (uint32_t g = tid; g < (1u << (KET_T2_BITS - 3)); g += NT) {
            uint32_t b0 = insert0_32(insert0_32(insert0_32(g, b3[0]), b3[1]), b3[2]);
            if ((b0 & ct) != ct) continue;
            const uint32_t idx[4] = {b0, b0 | (1u << tb), b0 | (1u << ta), b0 | (1u << ta) | (1u << tb)};
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
          grad_accum(sgrad, slot, warp, lane, acc);
          continue;  // read-only: registers still hold the tile
        }
        if (opc == OC_X1S) {
          for (uint32_t g = tid; g < (uint32_t)TT << (KET_T2_BITS - 1); g += NT) {
            const uint32_t base = smb + (g >> (KET_T2_BITS - 1)) * TB;
            const uint32_t i0 = insert0_32(g & ((1u << (KET_T2_BITS - 1)) - 1), ob);
            if ((i0 & ct) != ct) continue;
            cpx<R> t0, t1;
            lds(base + swz<R>(i0), t0);
            lds(base + swz<R>(i0 | (1u << ob)), t1);
            sts(base + swz<R>(i0), t1);
            sts(base + swz<R>(i0 | (1u << ob)), t0);
          }
          __syncthreads();
#pragma unroll
          for (int t = 0; t < TT; t++) read_tile<R, NR>(smb + t * TB, sl, x[t]);
          continue;
        }
        if (opc == OC_DIAG) {
          // d0, d1: tile bits of the two qubits, -1 = outside the tile
          const int b0t = (int8_t)(h.y >> 8), b1t = (int8_t)(h.y >> 16);
          const uint64_t dg0 = __ldg(reinterpret_cast<const unsigned long long*>(op) + 4);
          const uint64_t dg1 = __ldg(reinterpret_cast<const unsigned long long*>(op) + 5);
          const int u0 = (int)((ctx0 & dg0) != 0), u1 = (int)((ctx0 & dg1) != 0);
          for (uint32_t g = tid; g < (uint32_t)TT << KET_T2_BITS; g += NT) {
            const uint32_t base = smb + (g >> KET_T2_BITS) * TB, i = g & ((1u << KET_T2_BITS) - 1);
            if ((i & ct) != ct) continue;
            const int k0 = b0t >= 0 ? (int)((i >> b0t) & 1) : u0;
            const int k1 = b1t >= 0 ? (int)((i >> b1t) & 1) : u1;
            const int kk = 2 * k0 + k1;
            cpx<R> v;
            lds(base + swz<R>(i), v);
            v = cmul<R>((R)__ldg(M + 2 * kk), (R)__ldg(M + 2 * kk + 1), v);
            sts(base + swz<R>(i), v);
          }
          __syncthreads();
#pragma unroll
          for (int t = 0; t < TT; t++) read_tile<R, NR>(smb + t * TB, sl, x[t]);
          continue;
        }
        const int lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
        const bool pr = fl & FOF_PRUNE;
        for (uint32_t g = tid; g < (uint32_t)TT << (KET_T2_BITS - 2); g += NT) {
          const uint32_t base = smb + (g >> (KET_T2_BITS - 2)) * TB;
          uint32_t b0 = insert0_32(insert0_32(g & ((1u << (KET_T2_BITS - 2)) - 1), lo), hi);
          if ((b0 & ct) != ct) continue;
          const uint32_t i1 = b0 | (1u << tb), i2 = b0 | (1u << ta), i3 = b0 | (1u << ta) | (1u << tb);
          if (opc == OC_SWAPS) {
            cpx<R> t1, t2;
            lds(base + swz<R>(i1), t1);
            lds(base + swz<R>(i2), t2);
            sts(base + swz<R>(i1), t2);
            sts(base + swz<R>(i2), t1);
            continue;
          }
          const uint32_t idx[4] = {b0, i1, i2, i3};
          cpx<R> v[4];
          for (int c = 0; c < 4; c++) lds(base + swz<R>(idx[c]), v[c]);
          for (int r = 0; r < 4; r++) {
            cpx<R> s0 = mac2<R>((R)__ldg(M + 8 * r), (R)__ldg(M + 8 * r + 1), v[0], (R)__ldg(M + 8 * r + 2),
                                (R)__ldg(M + 8 * r + 3), v[1]);
            cpx<R> s1 = mac2<R>((R)__ldg(M + 8 * r + 4), (R)__ldg(M + 8 * r + 5), v[2], (R)__ldg(M + 8 * r + 6),
                                (R)__ldg(M + 8 * r + 7), v[3]);
            cpx<R> y;
            y.re = s0.re + s1.re;
            y.im = s0.im + s1.im;
            if (pr) prune_amp(y, thr, qthr);
            sts(base + swz<R>(idx[r]), y);
          }
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < TT; t++) read_tile<R, NR>(smb + t * TB, sl, x[t]);
        continue;  // pruning already done
      }
      const bool thr_ok = ((uint32_t)tid & cthr) == cthr;
      if (GRAD && opc >= OC_GRADM && opc <= OC_GRADD) {  // adjoint passes hold no phase fans (the host merges none there)
        // <lambda|D|psi> over this thread's amplitudes: register bit 3 of the
        // slot index selects psi (0) or lambda (1) -- the planner pins the
        // ancilla there.  Every lane takes part in the warp sum.  (TT == 1)
        const uint4 h2 = __ldg(reinterpret_cast<const uint4*>(op) + 1);
        const int slot = (int16_t)(h2.z & 0xffff);
        const uint32_t smask = thr_ok ? (c_slotmask[creg] & full_mask<NS>()) : 0u;
        double acc = 0.0;
        if (opc != OC_GRADD) {
          R d[8];
          load_m8<R>(op, d);
          switch (oa) {
            case 0: acc = grad_m<R, 0>(x[0], d, smask); break;
            case 1: acc = grad_m<R, 1>(x[0], d, smask); break;
            default: acc = grad_m<R, 2>(x[0], d, smask); break;
          }
        } else {
          const R d0r = (R)__ldg(M + 0), d0i = (R)__ldg(M + 1), d1r = (R)__ldg(M + 2), d1i = (R)__ldg(M + 3);
          if (fl & (FOF_TGT_THR | FOF_TGT_CTX)) {
            const bool one = (fl & FOF_TGT_CTX) ? (ctx0 & op->dg0) != 0 : (bool)((tid >> oa) & 1);
            acc = grad_d<R, -1>(x[0], one ? d1r : d0r, one ? d1i : d0i, one ? d1r : d0r, one ? d1i : d0i, smask);
          } else {
            switch (oa) {
              case 0: acc = grad_d<R, 0>(x[0], d0r, d0i, d1r, d1i, smask); break;
              case 1: acc = grad_d<R, 1>(x[0], d0r, d0i, d1r, d1i, smask); break;
              default: acc = grad_d<R, 2>(x[0], d0r, d0i, d1r, d1i, smask); break;
            }
          }
        }
        grad_accum(sgrad, slot, warp, lane, acc);
        continue;
      }
      // Thread-local ops and shuffles among the lanes that take part: a thread
      // whose thread-bit controls fail leaves its amplitudes alone.
      if (!thr_ok) continue;
      const uint32_t smask = creg ? (c_slotmask[creg] & full_mask<NS>()) : full_mask<NS>();
      switch (opc) {
#define KET_MAT1R(A, F)                                                                   \
  case OC_MAT1R + 3 * A + F:                                                              \
    if constexpr (A < NR) {                                                               \
      const R m[8] = {(R)q0.x, (R)q0.y, (R)q1.x, (R)q1.y, (R)q2.x, (R)q2.y, (R)q3.x, (R)q3.y}; \
      for (int t = 0; t < TT; t++) mat1_reg<R, A, F, NS>(x[t], m, smask);                 \
    }                                                                                     \
    break;
        KET_MAT1R(0, 0) KET_MAT1R(0, 1) KET_MAT1R(0, 2)
        KET_MAT1R(1, 0) KET_MAT1R(1, 1) KET_MAT1R(1, 2)
        KET_MAT1R(2, 0) KET_MAT1R(2, 1) KET_MAT1R(2, 2)
        KET_MAT1R(3, 0) KET_MAT1R(3, 1) KET_MAT1R(3, 2)
        KET_MAT1R(4, 0) KET_MAT1R(4, 1) KET_MAT1R(4, 2)
#undef KET_MAT1R
        case OC_MAT1L: case OC_MAT1L + 1: case OC_MAT1L + 2: {
          const uint32_t members = __ldg(reinterpret_cast<const uint32_t*>(op) + 4);
          const int bitv = (lane >> oa) & 1;
          // own output = c0 * own + c1 * partner
          const double2 e0 = bitv ? q3 : q0;
          const double2 e1 = bitv ? q2 : q1;
          const R c0r = (R)e0.x, c0i = (R)e0.y, c1r = (R)e1.x, c1i = (R)e1.y;
          const int msk = 1 << oa;
          if (opc == OC_MAT1L + 1) {
#pragma unroll
            for (int t = 0; t < TT; t++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
              cpx<R> p = shfl_xor_c<R>(x[t][j], msk, members);
              cpx<R> y;
              y.re = fma(c0r, x[t][j].re, c1r * p.re);
              y.im = fma(c0r, x[t][j].im, c1r * p.im);
              x[t][j] = smask == full_mask<NS>() ? y : sel<R>((smask >> j) & 1, y, x[t][j]);
            }
          } else if (opc == OC_MAT1L + 2) {
#pragma unroll
            for (int t = 0; t < TT; t++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
              cpx<R> p = shfl_xor_c<R>(x[t][j], msk, members);
              cpx<R> y;
              y.re = fma(c0r, x[t][j].re, -c1i * p.im);
              y.im = fma(c0r, x[t][j].im, c1i * p.re);
              x[t][j] = smask == full_mask<NS>() ? y : sel<R>((smask >> j) & 1, y, x[t][j]);
            }
          } else {
#pragma unroll
            for (int t = 0; t < TT; t++)
#pragma unroll
            for (int j = 0; j < NS; j++) {
              cpx<R> p = shfl_xor_c<R>(x[t][j], msk, members);
              cpx<R> y = mac2<R>(c0r, c0i, x[t][j], c1r, c1i, p);
              x[t][j] = smask == full_mask<NS>() ? y : sel<R>((smask >> j) & 1, y, x[t][j]);
            }
          }
          break;
        }
#define KET_X1R(A) \
  case OC_X1R + A: if constexpr (A < NR) { for (int t = 0; t < TT; t++) x1_reg<R, A, NS>(x[t]); } break;
        KET_X1R(0) KET_X1R(1) KET_X1R(2) KET_X1R(3) KET_X1R(4)
#undef KET_X1R
#define KET_X1RC(A, C) \
  case OC_X1RC + 5 * A + C: if constexpr (A < NR && C < NR) { for (int t = 0; t < TT; t++) x1c_reg<R, A, C, NS>(x[t]); } break;
        KET_X1RC(0, 1) KET_X1RC(0, 2) KET_X1RC(0, 3) KET_X1RC(0, 4)
        KET_X1RC(1, 0) KET_X1RC(1, 2) KET_X1RC(1, 3) KET_X1RC(1, 4)
        KET_X1RC(2, 0) KET_X1RC(2, 1) KET_X1RC(2, 3) KET_X1RC(2, 4)
        KET_X1RC(3, 0) KET_X1RC(3, 1) KET_X1RC(3, 2) KET_X1RC(3, 4)
        KET_X1RC(4, 0) KET_X1RC(4, 1) KET_X1RC(4, 2) KET_X1RC(4, 3)
#undef KET_X1RC
        case OC_X1L: {
          const uint32_t members = __ldg(reinterpret_cast<const uint32_t*>(op) + 4);
          const int msk = 1 << oa;
#pragma unroll
          for (int t = 0; t < TT; t++)
#pragma unroll
          for (int j = 0; j < NS; j++) {
            cpx<R> p = shfl_xor_c<R>(x[t][j], msk, members);
            x[t][j] = smask == full_mask<NS>() ? p : sel<R>((smask >> j) & 1, p, x[t][j]);
          }
          break;
        }
#define KET_DIAGR(A, ONE)                                                                   \
  case (ONE ? OC_DIAGR1 : OC_DIAGR) + A:                                                    \
    if constexpr (A < NR) {                                                                 \
      for (int t = 0; t < TT; t++) diag_reg<R, A, ONE, NS>(x[t], (R)q0.x, (R)q0.y, (R)q1.x, (R)q1.y, smask); \
    }                                                                                       \
    break;
        KET_DIAGR(0, false) KET_DIAGR(1, false) KET_DIAGR(2, false) KET_DIAGR(3, false) KET_DIAGR(4, false)
        KET_DIAGR(0, true) KET_DIAGR(1, true) KET_DIAGR(2, true) KET_DIAGR(3, true) KET_DIAGR(4, true)
#undef KET_DIAGR
#define KET_DIAGR1C(A, C)                                                                   \
  case OC_DIAGR1C + 5 * A + C:                                                              \
    if constexpr (A < NR && C < NR) {                                                       \
      for (int t = 0; t < TT; t++) diag1c_reg<R, A, C, NS>(x[t], (R)q1.x, (R)q1.y);         \
    }                                                                                       \
    break;
        KET_DIAGR1C(0, 1) KET_DIAGR1C(0, 2) KET_DIAGR1C(0, 3) KET_DIAGR1C(0, 4)
        KET_DIAGR1C(1, 0) KET_DIAGR1C(1, 2) KET_DIAGR1C(1, 3) KET_DIAGR1C(1, 4)
        KET_DIAGR1C(2, 0) KET_DIAGR1C(2, 1) KET_DIAGR1C(2, 3) KET_DIAGR1C(2, 4)
        KET_DIAGR1C(3, 0) KET_DIAGR1C(3, 1) KET_DIAGR1C(3, 2) KET_DIAGR1C(3, 4)
        KET_DIAGR1C(4, 0) KET_DIAGR1C(4, 1) KET_DIAGR1C(4, 2) KET_DIAGR1C(4, 3)
#undef KET_DIAGR1C
#define KET_CPHASE(A)                                                                         \
  case OC_CPHASE + A:                                                                         \
    if constexpr (A < NR) {                                                                   \
      const uint4 h2 = __ldg(reinterpret_cast<const uint4*>(op) + 1);                        \
      phase_fan<R, A, TT, NS>(x, op, h2.x, ctx0, pairq, tid, tid);                            \
    }                                                                                         \
    break; /* the continuation records that follow run as no-ops */
        KET_CPHASE(0) KET_CPHASE(1) KET_CPHASE(2) KET_CPHASE(3) KET_CPHASE(4)
#undef KET_CPHASE
        case OC_PPOLY:
          phase_poly<R, TT, NS>(x, op, ctx0, pairq, tid, tid);
          break;  // the continuation records that follow run as no-ops
        case OC_DIAGT: case OC_DIAGX: {
          bool one;
          if (opc == OC_DIAGT) one = (tid >> oa) & 1;
          else one = (ctx0 & __ldg(reinterpret_cast<const unsigned long long*>(op) + 4)) != 0;
          if ((fl & FOF_D0ONE) && !one) break;
          const double2 e = one ? q1 : q0;
          for (int t = 0; t < TT; t++) phase_all<R, NS>(x[t], (R)e.x, (R)e.y, smask);
          break;
        }
        default: break;
      }
      if (fl & FOF_PRUNE)  // mixing ops only (the planner clears the flag elsewhere)
#pragma unroll
        for (int t = 0; t < TT; t++) prune_slots<R, NS>(x[t], thr, qthr);
    }
    // the planner leaves the store layout in force here
    {
      uint64_t gs = 0;
#pragma unroll
      for (int r = 0; r < 5; r++)
        if ((lane >> r) & 1) gs += a.sgb[r];
#pragma unroll
      for (int r = 0; r < NW; r++)
        if ((warp >> r) & 1) gs += a.sgb[5 + r];
#pragma unroll
      for (int t = 0; t < TT; t++) {
        char* p = amp + (ctx0 | (t ? pairq : 0)) * sizeof(V) + gs;
#pragma unroll
        for (int j = 0; j < NS; j++) {
          uint64_t o = 0;
#pragma unroll
          for (int k = 0; k < NR; k++)
            if (j & (1 << k)) o += a.sgb[5 + NW + k];
          st_amp<R>(reinterpret_cast<V*>(p + o), x[t][j]);
        }
      }
    }
  }
  if (GRAD) {
    __syncthreads();
    for (int i = threadIdx.x; i < a.nslots * 8; i += NT) a.gpart[(size_t)blockIdx.x * a.nslots * 8 + i] = sgrad[i];
  }
}

// out[s] = sum over CTAs c and warps w of gpart[c][s][w], in a fixed order.
__global__ void k_grad_reduce(const double* gpart, int nctas, int nslots, double* out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  double acc = 0.0;
  for (int c = 0; c < nctas; c++)
    for (int w = 0; w < 8; w++) acc += gpart[((size_t)c * nslots + s) * 8 + w];
  out[s] = acc;
}

// Resident CTAs per SM for a register-bit count: 5 -> two CTAs of 128 threads
// (255 registers each), 4 -> one CTA of 256 threads.
constexpr int ctas_per_sm(int nreg) { return nreg == 5 ? 2 : 1; }

template <typename R, bool GRAD, int TT, int NR>
cudaError_t launch_tt(const Pass2Args& a, cudaStream_t s) {
  constexpr int NT = 32 << (7 - NR);
  static bool init = false;
  if (!init) {
    cudaFuncSetAttribute(k_fused2<R, GRAD, TT, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, 110 * 1024);
    init = true;
  }
  const size_t tb = sizeof(cpx<R>) << KET_T2_BITS;
  const size_t smem = TT * tb + (GRAD ? sizeof(double) * 8 * (size_t)a.nslots : 0);
  const uint64_t ngroups = (uint64_t(1) << (a.n - KET_T2_BITS)) / TT;
  const unsigned blocks = (unsigned)std::min<uint64_t>(ngroups, (uint64_t)fused2_grid(NR));
  k_fused2<R, GRAD, TT, NR><<<blocks, NT, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename R, bool GRAD>
cudaError_t launch_t(const Pass2Args& in, cudaStream_t s) {
  static bool init = false;
  if (!init) {
    uint32_t sm[32];
    for (int c = 0; c < 32; c++) {
      uint32_t v = 0;
      for (int j = 0; j < 32; j++)
        if ((j & c) == c) v |= 1u << j;
      sm[c] = v;
    }
    cudaMemcpyToSymbol(c_slotmask, sm, sizeof(sm));
    init = true;
  }
  Pass2Args a = in;
  fill_pass2_offsets(a, sizeof(R) == 4 ? KET_C64 : KET_C128);
  if constexpr (GRAD) {
    return launch_tt<R, true, 1, 4>(a, s);  // probes: 16 slots, ancilla on register bit 3
  } else {
    if (a.nreg == 5) return launch_tt<R, false, 1, 5>(a, s);
    return launch_tt<R, false, 1, 4>(a, s);
  }
}

}  // namespace

int fused2_grid(int nreg) { return num_sms() * ctas_per_sm(nreg); }

void fill_pass2_offsets(Pass2Args& a, int precision) {
  const bool c64 = precision == KET_C64;
  // per-role byte offsets in the state and in the exchange buffer
  auto gbit = [&](int tb) -> uint64_t {
    const int q = tb < a.L ? tb : a.hbits[tb - a.L];
    return (uint64_t(1) << q) * (c64 ? 8u : 16u);
  };
  for (int r = 0; r < KET_T2_BITS; r++) {
    a.lgb[r] = gbit(a.load_pos[r]);
    a.sgb[r] = gbit(a.store_pos[r]);
    a.lbx[r] = exch_offset(1u << a.load_pos[r], c64);
  }
}

int choose_pairbit(const std::vector<FOp>& prog, const Pass2Args& a) {
  uint64_t used = 0;  // (a phase fan's out-of-tile terms are evaluated per tile: not counted)
  for (const FOp& o : prog)
    if (o.type != FO_CONT) used |= o.cctx | o.dg0 | o.dg1;
  for (int j = 0; j < a.nctx; j++)
    if (!((used >> a.ctxbits[j]) & 1)) return j;
  return -1;
}

cudaError_t launch_fused2(const Pass2Args& a, int precision, cudaStream_t s) {
  if (a.nslots > 0) return precision == KET_C64 ? launch_t<float, true>(a, s) : launch_t<double, true>(a, s);
  return precision == KET_C64 ? launch_t<float, false>(a, s) : launch_t<double, false>(a, s);
}

cudaError_t launch_grad_reduce(const double* gpart, int nctas, int nslots, double* out, cudaStream_t s) {
  k_grad_reduce<<<(nslots + 127) / 128, 128, 0, s>>>(gpart, nctas, nslots, out);
  return cudaGetLastError();
}

}  // namespace ket
