// fused_ops.cuh -- device building blocks of the register-tiled pass: the
// exchange buffer's addressing, the pruning screen, and the gate arithmetic
// on register and lane bits.  Used by k_fused2 (kernels_fused.cu) and by the
// pass kernels compiled at run time for one program each (jit.cpp).
#pragma once

#include "fused_abi.h"
#include "common.cuh"

namespace ket {

// ---------------------------------------------------------------- shared memory
__device__ __forceinline__ void sts(uint32_t a, const cpx<double>& v) {
  asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.re), "d"(v.im) : "memory");
}
__device__ __forceinline__ void sts(uint32_t a, const cpx<float>& v) {
  asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.re), "f"(v.im) : "memory");
}
__device__ __forceinline__ void lds(uint32_t a, cpx<double>& v) {
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.re), "=d"(v.im) : "r"(a) : "memory");
}
__device__ __forceinline__ void lds(uint32_t a, cpx<float>& v) {
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.re), "=f"(v.im) : "r"(a) : "memory");
}

template <typename R>
__device__ __forceinline__ uint32_t swz(uint32_t i) {
  return exch_offset(i, sizeof(R) == 4);
}

// A thread's view of a layout in the exchange buffer: slot j lives at byte
// b ^ XOR over the set bits k of j of s[k].
template <int NR>
struct SLay {
  uint32_t b, s[NR];
  uint32_t l[5];  // the lane bits' offsets (deferred lane moves address the logical lanes with them)
};

template <int NR>
__device__ __forceinline__ uint32_t soff(const SLay<NR>& l, int j) {
  uint32_t o = l.b;
#pragma unroll
  for (int k = 0; k < NR; k++)
    if (j & (1 << k)) o ^= l.s[k];
  return o;
}

// bx[r] = exchange offset of role r's tile bit (roles: 5 lanes, 7-NR warps, NR registers).
template <int NR>
__device__ __forceinline__ SLay<NR> make_slay(const uint32_t* bx, int lane, int warp) {
  constexpr int NW = 7 - NR;
  SLay<NR> l;
  uint32_t b = 0;
#pragma unroll
  for (int r = 0; r < 5; r++)
    if ((lane >> r) & 1) b ^= bx[r];
#pragma unroll
  for (int r = 0; r < NW; r++)
    if ((warp >> r) & 1) b ^= bx[5 + r];
  l.b = b;
#pragma unroll
  for (int k = 0; k < NR; k++) l.s[k] = bx[5 + NW + k];
#pragma unroll
  for (int r = 0; r < 5; r++) l.l[r] = bx[r];
  return l;
}

// FO_EXCH keeps the new layout's 12 offsets as uint16 in its matrix area.
template <int NR>
__device__ __forceinline__ SLay<NR> exch_slay(const FOp* op, int lane, int warp) {
  const uint4 q0 = __ldg(reinterpret_cast<const uint4*>(op->m));
  const uint2 q1 = __ldg(reinterpret_cast<const uint2*>(op->m) + 2);
  const uint32_t w[6] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y};
  uint32_t bx[12];
#pragma unroll
  for (int r = 0; r < 12; r++) bx[r] = (w[r >> 1] >> (16 * (r & 1))) & 0xffffu;
  return make_slay<NR>(bx, lane, warp);
}

template <typename R, int NR>
__device__ __forceinline__ void write_tile(uint32_t smb, const SLay<NR>& l, const cpx<R>* x) {
#pragma unroll
  for (int j = 0; j < (1 << NR); j++) sts(smb + soff<NR>(l, j), x[j]);
}
template <typename R, int NR>
__device__ __forceinline__ void read_tile(uint32_t smb, const SLay<NR>& l, cpx<R>* x) {
#pragma unroll
  for (int j = 0; j < (1 << NR); j++) lds(smb + soff<NR>(l, j), x[j]);
}

// Mask of all NS slots.
template <int NS>
__device__ __forceinline__ constexpr uint32_t full_mask() {
  return NS == 32 ? 0xffffffffu : ((1u << NS) - 1u);
}

// ---------------------------------------------------------------- pruning screen
__device__ __forceinline__ float hiabs(double v) { return fabsf(__int_as_float(__double2hiint(v))); }
__device__ __forceinline__ float hiabs(float v) { return fabsf(v); }
// Screening thresholds: for doubles the high word read as a float preserves
// the order of |v|; 0x3E7AD7F3 lies just above the high word of 1e-7.
__device__ __forceinline__ float tiny_screen(double) { return __int_as_float(0x3E7AD7F3); }
__device__ __forceinline__ float tiny_screen(float) { return __int_as_float(0x33D6BF96); }  // just above 1e-7f

// Three-input minimum (sm_100, PTX of CUDA 12.9 on): min over N values in
// about N/2 instructions.  KET_NO_MIN3: an older runtime compiler.
__device__ __forceinline__ float fmin3(float a, float b, float c) {
#ifdef KET_NO_MIN3
  return fminf(fminf(a, b), c);
#else
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#endif
}
// t[0] = min(t[0..N)), one tree level of three-input minima at a time.
template <int N>
__device__ __forceinline__ void min_tree(float* t) {
  if constexpr (N > 1) {
    constexpr int M = (N + 2) / 3;
#pragma unroll
    for (int i = 0; i < M; i++) {
      const int a = 3 * i;  // a >= i: t[i] is written after its inputs are read
      if (a + 2 < N) t[i] = fmin3(t[a], t[a + 1], t[a + 2]);
      else if (a + 1 < N) t[i] = fminf(t[a], t[a + 1]);
      else t[i] = t[a];
    }
    min_tree<M>(t);
  }
}

template <typename R, int NS>
__device__ __forceinline__ void prune_slots(cpx<R>* x, double thr, double qthr) {
  // an amplitude can be pruned only if both components are below 1e-7
  float t[NS];
#pragma unroll
  for (int j = 0; j < NS; j++) t[j] = fmaxf(hiabs(x[j].re), hiabs(x[j].im));
  min_tree<NS>(t);
  if (t[0] < tiny_screen(R(0))) {
#pragma unroll
    for (int j = 0; j < NS; j++) prune_amp(x[j], thr, qthr);
  }
}

// ---------------------------------------------------------------- register and lane ops
template <typename R>
__device__ __forceinline__ cpx<R> shfl_xor_c(cpx<R> v, int mask, uint32_t members) {
  cpx<R> o;
  o.re = __shfl_xor_sync(members, v.re, mask);
  o.im = __shfl_xor_sync(members, v.im, mask);
  return o;
}

template <typename R>
__device__ __forceinline__ cpx<R> sel(bool p, cpx<R> a, cpx<R> b) {
  cpx<R> o;
  o.re = p ? a.re : b.re;
  o.im = p ? a.im : b.im;
  return o;
}

// Register swaps go through inline PTX with tied operands: every amplitude
// stays in its own loop-carried variable, so a permutation op does not force
// the register allocator to re-home the whole tile across the op loop.
__device__ __forceinline__ void swap_c(cpx<double>& a, cpx<double>& b) {
  asm("{\n .reg .f64 t;\n mov.f64 t, %0;\n mov.f64 %0, %2;\n mov.f64 %2, t;\n"
      " mov.f64 t, %1;\n mov.f64 %1, %3;\n mov.f64 %3, t;\n}"
      : "+d"(a.re), "+d"(a.im), "+d"(b.re), "+d"(b.im));
}
__device__ __forceinline__ void swap_c(cpx<float>& a, cpx<float>& b) {
  asm("{\n .reg .f32 t;\n mov.f32 t, %0;\n mov.f32 %0, %2;\n mov.f32 %2, t;\n"
      " mov.f32 t, %1;\n mov.f32 %1, %3;\n mov.f32 %3, t;\n}"
      : "+f"(a.re), "+f"(a.im), "+f"(b.re), "+f"(b.im));
}
// y0 = m00 x0 + m01 x1, y1 = m10 x0 + m11 x1, in place: the cross terms are
// formed first, so each output overwrites its own input with its last use and
// the loop-carried registers need no copies.  FORM 1: all entries real;
// FORM 2: m00, m11 real and m01, m10 imaginary (Rx-like); 0: general.
template <typename R, int FORM>
__device__ __forceinline__ void mat2x2(cpx<R>& x0, cpx<R>& x1, const R* m) {
  if (FORM == 2) {
    const R p1 = m[3] * x1.im, p2 = m[3] * x1.re, p3 = m[5] * x0.im, p4 = m[5] * x0.re;
    x0.re = fma(m[0], x0.re, -p1);
    x0.im = fma(m[0], x0.im, p2);
    x1.re = fma(m[6], x1.re, -p3);
    x1.im = fma(m[6], x1.im, p4);
  } else if (FORM == 1) {
    const R p1 = m[2] * x1.re, p2 = m[2] * x1.im, p3 = m[4] * x0.re, p4 = m[4] * x0.im;
    x0.re = fma(m[0], x0.re, p1);
    x0.im = fma(m[0], x0.im, p2);
    x1.re = fma(m[6], x1.re, p3);
    x1.im = fma(m[6], x1.im, p4);
  } else {
    // cross terms m01 x1 and m10 x0
    const R c0r = fma(m[2], x1.re, -m[3] * x1.im), c0i = fma(m[2], x1.im, m[3] * x1.re);
    const R c1r = fma(m[4], x0.re, -m[5] * x0.im), c1i = fma(m[4], x0.im, m[5] * x0.re);
    const R t0 = fma(-m[1], x0.im, c0r), u0 = fma(m[1], x0.re, c0i);
    const R t1 = fma(-m[7], x1.im, c1r), u1 = fma(m[7], x1.re, c1i);
    x0.re = fma(m[0], x0.re, t0);
    x0.im = fma(m[0], x0.im, u0);
    x1.re = fma(m[6], x1.re, t1);
    x1.im = fma(m[6], x1.im, u1);
  }
}

// x *= (mr + i mi), in place.
template <typename R>
__device__ __forceinline__ void cmul_in(cpx<R>& x, R mr, R mi) {
  const R p = mi * x.im, q = mi * x.re;
  x.re = fma(mr, x.re, -p);
  x.im = fma(mr, x.im, q);
}

template <typename R, int A, int FORM, int NS>
__device__ __forceinline__ void mat1_reg(cpx<R>* x, const R* m, uint32_t smask) {
  if (smask == full_mask<NS>()) {
#pragma unroll
    for (int j = 0; j < NS; j++) {
      if (j & (1 << A)) continue;
      mat2x2<R, FORM>(x[j], x[j | (1 << A)], m);
    }
  } else {
#pragma unroll
    for (int j = 0; j < NS; j++) {
      if (j & (1 << A)) continue;
      const int j1 = j | (1 << A);
      cpx<R> a0 = x[j], a1 = x[j1];
      mat2x2<R, FORM>(a0, a1, m);
      const bool p = (smask >> j) & 1;
      x[j] = sel<R>(p, a0, x[j]);
      x[j1] = sel<R>(p, a1, x[j1]);
    }
  }
}

// X on register bit A where register bit C is 1 (a CNOT inside the thread).
template <typename R, int A, int C, int NS>
__device__ __forceinline__ void x1c_reg(cpx<R>* x) {
#pragma unroll
  for (int j = 0; j < NS; j++)
    if (!(j & (1 << A)) && (j & (1 << C))) swap_c(x[j], x[j | (1 << A)]);
}

// diag(1, d1) on register bit A where register bit C is 1 (a controlled phase).
template <typename R, int A, int C, int NS>
__device__ __forceinline__ void diag1c_reg(cpx<R>* x, R d1r, R d1i) {
#pragma unroll
  for (int j = 0; j < NS; j++)
    if ((j & (1 << A)) && (j & (1 << C))) cmul_in<R>(x[j], d1r, d1i);
}

// X on register bit A (no register controls: other controls skip the thread).
template <typename R, int A, int NS>
__device__ __forceinline__ void x1_reg(cpx<R>* x) {
#pragma unroll
  for (int j = 0; j < NS; j++)
    if (!(j & (1 << A))) swap_c(x[j], x[j | (1 << A)]);
}

// diag(d0, d1) on register bit A; D0ONE: d0 == 1, so bit-0 slots are untouched.
template <typename R, int A, bool D0ONE, int NS>
__device__ __forceinline__ void diag_reg(cpx<R>* x, R d0r, R d0i, R d1r, R d1i, uint32_t smask) {
  if (smask == full_mask<NS>()) {
#pragma unroll
    for (int j = 0; j < NS; j++) {
      const bool one = (j >> A) & 1;
      if (D0ONE && !one) continue;
      cmul_in<R>(x[j], one ? d1r : d0r, one ? d1i : d0i);
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < NS; j++) {
    const bool one = (j >> A) & 1;
    if (D0ONE && !one) continue;
    cpx<R> y = cmul<R>(one ? d1r : d0r, one ? d1i : d0i, x[j]);
    x[j] = sel<R>((smask >> j) & 1, y, x[j]);
  }
}

template <typename R, int NS>
__device__ __forceinline__ void phase_all(cpx<R>* x, R dr, R di, uint32_t smask) {
  if (smask == full_mask<NS>()) {
#pragma unroll
    for (int j = 0; j < NS; j++) cmul_in<R>(x[j], dr, di);
    return;
  }
#pragma unroll
  for (int j = 0; j < NS; j++) {
    cpx<R> y = cmul<R>(dr, di, x[j]);
    x[j] = sel<R>((smask >> j) & 1, y, x[j]);
  }
}

template <typename R>
__device__ __forceinline__ void load_m8(const FOp* op, R* m) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(op->m) + q);
    m[2 * q] = (R)v.x;
    m[2 * q + 1] = (R)v.y;
  }
}

// ---------------------------------------------------------------- tiles
// Global index bits of a tile outside its 12 tile qubits.
__device__ __forceinline__ uint64_t ctx_of(const Pass2Args& a, uint64_t tile) {
  uint64_t cb = 0;
  for (int j = 0; j < a.nctx; j++)
    if ((tile >> j) & 1) cb |= uint64_t(1) << a.ctxbits[j];
  return cb;
}

// ---------------------------------------------------------------- adjoint probes
// Adjoint passes use 16 slots per thread: register bit 3 selects psi (0) / lambda (1).
// Re<lambda| D |psi> with D 2x2 on register bit A.
template <typename R, int A>
__device__ __forceinline__ double grad_m(const cpx<R>* x, const R* d, uint32_t smask) {
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    if ((j >> A) & 1) continue;
    if (!((smask >> j) & 1)) continue;
    const int j1 = j | (1 << A);
    cpx<R> u0 = mac2<R>(d[0], d[1], x[j], d[2], d[3], x[j1]);
    cpx<R> u1 = mac2<R>(d[4], d[5], x[j], d[6], d[7], x[j1]);
    acc += (double)x[j + 8].re * u0.re + (double)x[j + 8].im * u0.im + (double)x[j1 + 8].re * u1.re +
           (double)x[j1 + 8].im * u1.im;
  }
  return acc;
}
// Re<lambda| diag(d0, d1) on register bit A |psi>; A = -1: one factor (d0) for all.
template <typename R, int A>
__device__ __forceinline__ double grad_d(const cpx<R>* x, R d0r, R d0i, R d1r, R d1i, uint32_t smask) {
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    if (!((smask >> j) & 1)) continue;
    const bool one = A >= 0 && ((j >> (A < 0 ? 0 : A)) & 1);
    cpx<R> u = cmul<R>(one ? d1r : d0r, one ? d1i : d0i, x[j]);
    acc += (double)x[j + 8].re * u.re + (double)x[j + 8].im * u.im;
  }
  return acc;
}

// Warp-sum v and add it to the CTA's gradient accumulator for (slot, warp).
__device__ __forceinline__ void grad_accum(double* sgrad, int slot, int warp, int lane, double v) {
  v = warp_sum(v);
  if (lane == 0) sgrad[slot * 8 + warp] += v;
}

// ---------------------------------------------------------------- phase fans
// FO_CPHASE on register bit A for the TT tiles of a thread; tile t's context is
// ctx0 | (t ? pairq : 0).
// tid: the thread (which lanes add which terms); ltid: the logical thread id
// whose bits the thread factor reads (tid but for deferred lane X gates).
template <typename R, int A, int TT, int NS>
__device__ __forceinline__ void phase_fan(cpx<R> (&x)[TT][NS], const FOp* op, uint32_t nterms, uint64_t ctx0,
                                          uint64_t pairq, int tid, int ltid) {
  // record 0 after the op: H[0..7]; records 1..: (angle, mask) pairs; each
  // record's data starts after its 16-byte no-op header
  const double2* H = reinterpret_cast<const double2*>(reinterpret_cast<const char*>(op + 1) + 16);
  // the out-of-tile angles: lane l adds terms l, l + 32, ...; then a warp sum
  // (the whole warp runs this: the op has no thread-bit controls)
  double th0 = 0.0, thp = 0.0;
  for (uint32_t i = tid & 31; i < nterms; i += 32) {
    const uint32_t r = i / KET_CPHASE_TERMS_PER_RECORD, w = i - r * KET_CPHASE_TERMS_PER_RECORD;
    const double2 t = __ldg(reinterpret_cast<const double2*>(reinterpret_cast<const char*>(op + 2 + r) + 16) + w);
    const uint64_t mk = (uint64_t)__double_as_longlong(t.y);
    if (ctx0 & mk) th0 += t.x;
    if (pairq & mk) thp += t.x;
  }
  th0 = warp_sum(th0);
  if (TT > 1) thp = warp_sum(thp);
  const double2* mp = reinterpret_cast<const double2*>(op->m);
  // thread factor: H[s] for every thread-id bit s that is set
  double fr = 1.0, fi = 0.0;
#pragma unroll
  for (int sb = 0; sb < 8; sb++) {
    const double2 h = __ldg(H + sb);
    const bool on = (ltid >> sb) & 1;
    const double hr = on ? h.x : 1.0, hi = on ? h.y : 0.0;
    const double r = fr * hr - fi * hi;
    fi = fr * hi + fi * hr;
    fr = r;
  }
#pragma unroll
  for (int t = 0; t < TT; t++) {
    double sn, cs;
    sincos(th0 + (t ? thp : 0.0), &sn, &cs);
    const double gr = cs * fr - sn * fi, gi = cs * fi + sn * fr;
#pragma unroll
    for (int k = 0; k < NS / 2; k++) {
      const int j = ((k >> A) << (A + 1)) | (1 << A) | (k & ((1 << A) - 1));
      const double2 tk = __ldg(mp + k);
      const R pr = (R)(tk.x * gr - tk.y * gi), pi = (R)(tk.x * gi + tk.y * gr);
      cmul_in<R>(x[t][j], pr, pi);
    }
  }
}

// FO_PPOLY: the phases of a run of controlled-phase gates (the layout is
// described in fused_abi.h), for the TT tiles of a thread (the second at
// ctx0 | pairq).  Lane g (of tid) multiplies the phases of group g's terms
// that match the tile; each thread then multiplies, per register bit, the
// products of the groups whose thread mask its logical id ltid matches (tid
// but for deferred lane X gates), and its slots take them.  The
// whole warp runs this (no thread-bit controls on the op).
template <typename R, int TT, int NS>
__device__ __forceinline__ void phase_poly(cpx<R> (&x)[TT][NS], const FOp* op, uint64_t ctx0, uint64_t pairq,
                                           int tid, int ltid) {
  const char* m = reinterpret_cast<const char*>(op->m);
  const uint4 c0 = __ldg(reinterpret_cast<const uint4*>(m));
  const uint2 c1 = __ldg(reinterpret_cast<const uint2*>(m + 16));
  const uint32_t cnt[KET_NR_MAX + 1] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y};
  const uint32_t ngrp = __ldg(reinterpret_cast<const uint32_t*>(op) + 4);  // FOp::lmask
  const int lane = tid & 31;
  uint4 d = make_uint4(0u, 0u, 0u, 0u);  // this lane's group: {tm, terms, record}
  if ((uint32_t)lane < ngrp) d = __ldg(reinterpret_cast<const uint4*>(m + 32) + lane);
  // the group products for each tile
  cpx<double> K[TT];
#pragma unroll
  for (int t = 0; t < TT; t++) {
    K[t].re = 1.0;
    K[t].im = 0.0;
  }
  {
    const char* p = reinterpret_cast<const char*>(op + d.z) + 16;
    uint32_t w = 0;
    for (uint32_t k = 0; k < d.y; k++) {
      const double2 ph = __ldg(reinterpret_cast<const double2*>(p));
      const uint64_t cm = __ldg(reinterpret_cast<const unsigned long long*>(p + 16));
#pragma unroll
      for (int t = 0; t < TT; t++) {
        const uint64_t ctx = ctx0 | (t ? pairq : 0);
        if ((ctx & cm) == cm) cmul_in<double>(K[t], ph.x, ph.y);
      }
      if (++w == KET_PPOLY_TERMS_PER_RECORD) {
        w = 0;
        p += sizeof(FOp) - (KET_PPOLY_TERMS_PER_RECORD - 1) * sizeof(PPolyTerm);
      } else {
        p += sizeof(PPolyTerm);
      }
    }
  }
  uint32_t g = 0;
#pragma unroll
  for (int seg = 0; seg <= KET_NR_MAX; seg++) {
    if (seg > 0 && (1 << (seg - 1)) >= NS) break;  // register bits beyond the slots name no group
    if (cnt[seg] == 0) continue;
    cpx<double> F[TT];
#pragma unroll
    for (int t = 0; t < TT; t++) {
      F[t].re = 1.0;
      F[t].im = 0.0;
    }
    for (uint32_t k = 0; k < cnt[seg]; k++, g++) {
      const uint32_t tm = __shfl_sync(0xffffffffu, d.x, (int)g);
#pragma unroll
      for (int t = 0; t < TT; t++) {
        const double kr = __shfl_sync(0xffffffffu, K[t].re, (int)g);
        const double ki = __shfl_sync(0xffffffffu, K[t].im, (int)g);
        if (((uint32_t)ltid & tm) == tm) cmul_in<double>(F[t], kr, ki);
      }
    }
#pragma unroll
    for (int t = 0; t < TT; t++) {
      const R fr = (R)F[t].re, fi = (R)F[t].im;
#pragma unroll
      for (int j = 0; j < NS; j++)
        if (seg == 0 || ((j >> (seg - 1)) & 1)) cmul_in<R>(x[t][j], fr, fi);
    }
  }
}

}  // namespace ket
