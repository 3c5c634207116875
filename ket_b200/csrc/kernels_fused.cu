// kernels_fused.cu -- the register-tiled fused gate pass.
//
// One CTA of 256 threads owns a tile of 2^12 amplitudes at a time: the L
// lowest qubits (contiguous in HBM) plus 12-L high qubits chosen by the
// planner.  Each thread keeps 16 amplitudes in registers.  The tile's 12 bits
// are split into 5 lane bits, 3 warp bits and 4 register bits; a gate whose
// target is a register bit is applied inside each thread, a gate on a lane
// bit uses warp shuffles, and a gate on a warp bit first re-lays the tile out
// through shared memory (FO_EXCH, XOR-swizzled so lanes hit distinct banks).
// Diagonal gates need no pairing and apply on any qubit, in or out of the
// tile.  The global load and store use a layout whose lane bits are the
// tile's low bits, so every warp touches whole 128-byte lines.  A pass costs
// one read and one write of the state however many gates it holds; the
// persistent grid keeps two CTAs per SM so one CTA's loads overlap the
// other's arithmetic.
//
// Arithmetic is branch-free inside an op (controls become selects), so the
// eight independent amplitude pairs of a register-bit gate interleave; the
// per-gate pruning of the reference (|a|^2 < 1e-14 -> 0) is one integer test
// on the exponent words of all 16 amplitudes, with the exact FP64 check only
// in the rare case that some amplitude is below 1e-7 in magnitude.
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace ket {

namespace {

__constant__ uint16_t c_slotmask[16];  // slots j with (j & creg) == creg

template <typename R>
struct SwzT;
template <>
struct SwzT<double> {  // 16-byte elements: 8 per 128-byte bank row
  static __device__ __forceinline__ uint32_t f(uint32_t i) { return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9)) & 7u); }
};
template <>
struct SwzT<float> {  // 8-byte elements: 16 per bank row
  static __device__ __forceinline__ uint32_t f(uint32_t i) { return i ^ (((i >> 4) ^ (i >> 8)) & 15u); }
};

// Magnitude word of a component for the quick pruning test.
__device__ __forceinline__ uint32_t magw(double v) { return (uint32_t)__double2hiint(v) & 0x7fffffffu; }
__device__ __forceinline__ uint32_t magw(float v) { return __float_as_uint(v) & 0x7fffffffu; }
template <typename R> struct Tiny;
template <> struct Tiny<double> { static constexpr uint32_t w = 0x3E7AD7F3u; };  // > hi word of 1e-7
template <> struct Tiny<float> { static constexpr uint32_t w = 0x33D6BF96u; };   // > bits of 1e-7f

template <typename R>
__device__ __forceinline__ void prune16(cpx<R>* x, double thr, double qthr) {
  uint32_t any = 0;
#pragma unroll
  for (int j = 0; j < 16; j++) any |= (uint32_t)(max(magw(x[j].re), magw(x[j].im)) < Tiny<R>::w);
  if (any) {
#pragma unroll
    for (int j = 0; j < 16; j++) prune_amp(x[j], thr, qthr);
  }
}

struct Layout {
  uint32_t tbase;   // tile index bits contributed by this thread's lane and warp
  uint32_t rp[4];   // tile bit of each register bit (as a mask)
};

__device__ __forceinline__ Layout make_layout(const uint8_t* pos, int lane, int warp) {
  Layout L;
  uint32_t t = 0;
#pragma unroll
  for (int l = 0; l < 5; l++) t |= (uint32_t)((lane >> l) & 1) << pos[l];
#pragma unroll
  for (int w = 0; w < 3; w++) t |= (uint32_t)((warp >> w) & 1) << pos[5 + w];
  L.tbase = t;
#pragma unroll
  for (int k = 0; k < 4; k++) L.rp[k] = 1u << pos[8 + k];
  return L;
}

__device__ __forceinline__ uint32_t rofs(const Layout& L, int j) {
  uint32_t o = 0;
  if (j & 1) o |= L.rp[0];
  if (j & 2) o |= L.rp[1];
  if (j & 4) o |= L.rp[2];
  if (j & 8) o |= L.rp[3];
  return o;
}

// Global index of tile bit p: p < L -> qubit p, else hbits[p - L].
__device__ __forceinline__ uint64_t gbit(const Pass2Args& a, int p) {
  return uint64_t(1) << (p < a.L ? p : a.hbits[p - a.L]);
}

struct GLayout {
  uint64_t gthr;
  uint64_t gr[4];
};

__device__ __forceinline__ GLayout make_glayout(const Pass2Args& a, const uint8_t* pos, int lane, int warp) {
  GLayout G;
  uint64_t t = 0;
#pragma unroll
  for (int l = 0; l < 5; l++)
    if ((lane >> l) & 1) t |= gbit(a, pos[l]);
#pragma unroll
  for (int w = 0; w < 3; w++)
    if ((warp >> w) & 1) t |= gbit(a, pos[5 + w]);
  G.gthr = t;
#pragma unroll
  for (int k = 0; k < 4; k++) G.gr[k] = gbit(a, pos[8 + k]);
  return G;
}

__device__ __forceinline__ uint64_t grofs(const GLayout& G, int j) {
  uint64_t o = 0;
  if (j & 1) o |= G.gr[0];
  if (j & 2) o |= G.gr[1];
  if (j & 4) o |= G.gr[2];
  if (j & 8) o |= G.gr[3];
  return o;
}

template <typename R>
__device__ __forceinline__ cpx<R> shfl_xor_c(cpx<R> v, int mask) {
  cpx<R> o;
  o.re = __shfl_xor_sync(0xffffffffu, v.re, mask);
  o.im = __shfl_xor_sync(0xffffffffu, v.im, mask);
  return o;
}

template <typename R>
__device__ __forceinline__ cpx<R> sel(bool p, cpx<R> a, cpx<R> b) {
  cpx<R> o;
  o.re = p ? a.re : b.re;
  o.im = p ? a.im : b.im;
  return o;
}

// y0 = m00 x0 + m01 x1, y1 = m10 x0 + m11 x1.  FORM 1: all entries real;
// FORM 2: m00, m11 real and m01, m10 imaginary (Rx-like); 0: general.
template <typename R, int FORM>
__device__ __forceinline__ void mat2x2(cpx<R>& x0, cpx<R>& x1, const R* m) {
  cpx<R> y0, y1;
  if (FORM == 2) {
    // (a + i b)(xr + i xi) with a = 0: (-b xi, b xr)
    y0.re = fma(m[0], x0.re, -m[3] * x1.im);
    y0.im = fma(m[0], x0.im, m[3] * x1.re);
    y1.re = fma(m[6], x1.re, -m[5] * x0.im);
    y1.im = fma(m[6], x1.im, m[5] * x0.re);
  } else if (FORM == 1) {
    y0.re = fma(m[0], x0.re, m[2] * x1.re);
    y0.im = fma(m[0], x0.im, m[2] * x1.im);
    y1.re = fma(m[4], x0.re, m[6] * x1.re);
    y1.im = fma(m[4], x0.im, m[6] * x1.im);
  } else {
    y0 = mac2<R>(m[0], m[1], x0, m[2], m[3], x1);
    y1 = mac2<R>(m[4], m[5], x0, m[6], m[7], x1);
  }
  x0 = y0;
  x1 = y1;
}

template <typename R, int A, int FORM>
__device__ __forceinline__ void mat1_reg(cpx<R>* x, const R* m, uint32_t smask) {
  if (smask == 0xffffu) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
      if (j & (1 << A)) continue;
      mat2x2<R, FORM>(x[j], x[j | (1 << A)], m);
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; j++) {
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

template <typename R, int A>
__device__ __forceinline__ void x1_reg(cpx<R>* x, uint32_t smask) {
  if (smask == 0xffffu) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
      if (j & (1 << A)) continue;
      cpx<R> t = x[j];
      x[j] = x[j | (1 << A)];
      x[j | (1 << A)] = t;
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < 16; j++) {
    if (j & (1 << A)) continue;
    const int j1 = j | (1 << A);
    const bool p = (smask >> j) & 1;
    cpx<R> t0 = x[j], t1 = x[j1];
    x[j] = sel<R>(p, t1, t0);
    x[j1] = sel<R>(p, t0, t1);
  }
}

// diag(d0, d1) on register bit A; D0ONE: d0 == 1, so bit-0 slots are untouched.
template <typename R, int A, bool D0ONE>
__device__ __forceinline__ void diag_reg(cpx<R>* x, R d0r, R d0i, R d1r, R d1i, uint32_t smask) {
  if (smask == 0xffffu) {
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const bool one = (j >> A) & 1;
      if (D0ONE && !one) continue;
      x[j] = cmul<R>(one ? d1r : d0r, one ? d1i : d0i, x[j]);
    }
    return;
  }
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const bool one = (j >> A) & 1;
    if (D0ONE && !one) continue;
    const R dr = one ? d1r : d0r, di = one ? d1i : d0i;
    cpx<R> y = cmul<R>(dr, di, x[j]);
    x[j] = sel<R>((smask >> j) & 1, y, x[j]);
  }
}

template <typename R>
__device__ __forceinline__ void phase_all(cpx<R>* x, R dr, R di, uint32_t smask) {
#pragma unroll
  for (int j = 0; j < 16; j++) {
    cpx<R> y = cmul<R>(dr, di, x[j]);
    x[j] = sel<R>((smask >> j) & 1, y, x[j]);
  }
}

// ---------------------------------------------------------------- TMA staging
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bulk copy (TMA engine, no tensor map): global -> shared, completion on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait: false when the iteration limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < (1u << 26); it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Issue the bulk copies of one tile (2^(12-L) contiguous chunks of 2^L amplitudes) into buf.
template <typename R>
__device__ __forceinline__ void issue_tile(const Pass2Args& a, const typename Vec2<R>::T* amp, uint64_t tile,
                                           cpx<R>* buf, uint64_t* bar, int tid) {
  const uint32_t nch = 1u << (KET_T2_BITS - a.L);
  const uint32_t cbytes = (uint32_t)sizeof(cpx<R>) << a.L;
  if (tid < 32) {
    uint64_t ctx = 0;
    for (int j = 0; j < a.nctx; j++)
      if ((tile >> j) & 1) ctx |= uint64_t(1) << a.ctxbits[j];
    if (tid == 0) mbar_expect_tx(bar, nch * cbytes);
    __syncwarp();
    for (uint32_t c = tid; c < nch; c += 32) {
      uint64_t g = ctx;
      for (int j = 0; j < a.nh; j++)
        if ((c >> j) & 1) g |= uint64_t(1) << a.hbits[j];
      bulk_g2s(buf + ((size_t)c << a.L), amp + g, cbytes, bar);
    }
  }
}

// Adjoint probes.  Register bit 3 selects psi (0) / lambda (1).
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

template <typename R, int NT, bool GRAD>
__global__ void __launch_bounds__(NT, GRAD ? 1 : 2) k_fused2(Pass2Args a) {
  typedef typename Vec2<R>::T V;
  extern __shared__ __align__(128) unsigned char smraw[];
  cpx<R>* sm = reinterpret_cast<cpx<R>*>(smraw);  // exchange buffer (swizzled)
  double* sgrad = reinterpret_cast<double*>(smraw + (sizeof(cpx<R>) << KET_T2_BITS));  // [slot][warp]
  if (GRAD) {
    for (int i = threadIdx.x; i < a.nslots * 8; i += NT) sgrad[i] = 0.0;
    __syncthreads();
  }
  V* amp = reinterpret_cast<V*>(a.amp);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t ntiles = uint64_t(1) << (a.n - KET_T2_BITS);
  constexpr double thr = 1e-14, qthr = 1e-7;  // accumulate()'s threshold (statevector.ts:24) and its root
  cpx<R> x[16];

  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    uint64_t ctxbase = 0;
    for (int j = 0; j < a.nctx; j++)
      if ((tile >> j) & 1) ctxbase |= uint64_t(1) << a.ctxbits[j];
    {
      // global addresses are rebuilt here and at the store rather than kept
      // live through the op loop (register pressure); lane l holds tile bit l,
      // so each warp load covers whole 128-byte lines
      const GLayout gl = make_glayout(a, a.load_pos, lane, warp);
#pragma unroll
      for (int j = 0; j < 16; j++) x[j] = ld_amp<R>(amp + (ctxbase | gl.gthr | grofs(gl, j)));
    }
    Layout L = make_layout(a.load_pos, lane, warp);
    for (int k = 0; k < a.nops; k++) {
      const FOp* op = a.ops + k;
      const uint4 h0 = __ldg(reinterpret_cast<const uint4*>(op));
      const int type = h0.x & 0xff, oa = (h0.x >> 8) & 0xff, ob = (h0.x >> 16) & 0xff, fl = h0.x >> 24;
      if (type == FO_EXCH || type == FO_RELABEL) {
        uint8_t pos[KET_T2_BITS];
        const uint32_t pw[3] = {h0.y, h0.z, h0.w};
#pragma unroll
        for (int q = 0; q < KET_T2_BITS; q++) pos[q] = (uint8_t)(pw[q >> 2] >> (8 * (q & 3)));
        if (type == FO_RELABEL) {
          L = make_layout(pos, lane, warp);
          continue;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 16; j++) sm[SwzT<R>::f(L.tbase | rofs(L, j))] = x[j];
        __syncthreads();
        L = make_layout(pos, lane, warp);
#pragma unroll
        for (int j = 0; j < 16; j++) x[j] = sm[SwzT<R>::f(L.tbase | rofs(L, j))];
        continue;
      }
      const uint4 h1 = __ldg(reinterpret_cast<const uint4*>(op) + 1);  // creg, cthr, ctile, d0|d1
      const uint64_t cctx = __ldg(reinterpret_cast<const unsigned long long*>(op) + 4);
      if ((ctxbase & cctx) != cctx) continue;  // uniform over the CTA
      const bool pr = fl & FOF_PRUNE;
      const uint32_t creg = h1.x, cthr = h1.y;
      const uint32_t smask = ((uint32_t)(tid & cthr) == cthr) ? (uint32_t)c_slotmask[creg & 15] : 0u;
      const double* M = op->m;
      switch (type) {
        case FO_MAT1R: {
          R m[8];
#pragma unroll
          for (int q = 0; q < 8; q++) m[q] = (R)__ldg(M + q);
          const int form = (fl & FOF_REAL) ? 1 : ((fl & FOF_RXFORM) ? 2 : 0);
#define KET_MAT1R(F)                                        \
  switch (oa) {                                             \
    case 0: mat1_reg<R, 0, F>(x, m, smask); break;          \
    case 1: mat1_reg<R, 1, F>(x, m, smask); break;          \
    case 2: mat1_reg<R, 2, F>(x, m, smask); break;          \
    default: mat1_reg<R, 3, F>(x, m, smask); break;         \
  }
          if (form == 1) { KET_MAT1R(1) } else if (form == 2) { KET_MAT1R(2) } else { KET_MAT1R(0) }
#undef KET_MAT1R
          break;
        }
        case FO_MAT1L: {
          const int bitv = (lane >> oa) & 1;
          // own output = c0 * own + c1 * partner
          const R c0r = (R)__ldg(M + (bitv ? 6 : 0)), c0i = (R)__ldg(M + (bitv ? 7 : 1));
          const R c1r = (R)__ldg(M + (bitv ? 4 : 2)), c1i = (R)__ldg(M + (bitv ? 5 : 3));
          const int msk = 1 << oa;
          if (fl & FOF_REAL) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
              cpx<R> p = shfl_xor_c<R>(x[j], msk);
              cpx<R> y;
              y.re = fma(c0r, x[j].re, c1r * p.re);
              y.im = fma(c0r, x[j].im, c1r * p.im);
              x[j] = sel<R>((smask >> j) & 1, y, x[j]);
            }
          } else if (fl & FOF_RXFORM) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
              cpx<R> p = shfl_xor_c<R>(x[j], msk);
              cpx<R> y;
              y.re = fma(c0r, x[j].re, -c1i * p.im);
              y.im = fma(c0r, x[j].im, c1i * p.re);
              x[j] = sel<R>((smask >> j) & 1, y, x[j]);
            }
          } else {
#pragma unroll
            for (int j = 0; j < 16; j++) {
              cpx<R> p = shfl_xor_c<R>(x[j], msk);
              cpx<R> y = mac2<R>(c0r, c0i, x[j], c1r, c1i, p);
              x[j] = sel<R>((smask >> j) & 1, y, x[j]);
            }
          }
          break;
        }
        case FO_X1R:
          switch (oa) {
            case 0: x1_reg<R, 0>(x, smask); break;
            case 1: x1_reg<R, 1>(x, smask); break;
            case 2: x1_reg<R, 2>(x, smask); break;
            default: x1_reg<R, 3>(x, smask); break;
          }
          break;
        case FO_X1L: {
          const int msk = 1 << oa;
#pragma unroll
          for (int j = 0; j < 16; j++) {
            cpx<R> p = shfl_xor_c<R>(x[j], msk);
            x[j] = sel<R>((smask >> j) & 1, p, x[j]);
          }
          break;
        }
        case FO_SWAPS: case FO_MAT2S: {
          // Rare ops (controlled swaps, dense 4x4s) run on the shared-memory
          // copy of the tile, in the current layout, with small code.
          __syncthreads();
#pragma unroll
          for (int j = 0; j < 16; j++) sm[SwzT<R>::f(L.tbase | rofs(L, j))] = x[j];
          __syncthreads();
          const uint32_t ct = h1.z;
          const int ta = oa, tb = ob, lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
          for (uint32_t g = tid; g < (1u << (KET_T2_BITS - 2)); g += NT) {
            uint32_t b0 = insert0_32(insert0_32(g, lo), hi);
            if ((b0 & ct) != ct) continue;
            const uint32_t i1 = b0 | (1u << tb), i2 = b0 | (1u << ta), i3 = b0 | (1u << ta) | (1u << tb);
            if (type == FO_SWAPS) {
              cpx<R> t = sm[SwzT<R>::f(i1)];
              sm[SwzT<R>::f(i1)] = sm[SwzT<R>::f(i2)];
              sm[SwzT<R>::f(i2)] = t;
              continue;
            }
            cpx<R> v[4] = {sm[SwzT<R>::f(b0)], sm[SwzT<R>::f(i1)], sm[SwzT<R>::f(i2)], sm[SwzT<R>::f(i3)]};
            const uint32_t idx[4] = {b0, i1, i2, i3};
            for (int r = 0; r < 4; r++) {
              cpx<R> s0 = mac2<R>((R)__ldg(M + 8 * r), (R)__ldg(M + 8 * r + 1), v[0], (R)__ldg(M + 8 * r + 2),
                                  (R)__ldg(M + 8 * r + 3), v[1]);
              cpx<R> s1 = mac2<R>((R)__ldg(M + 8 * r + 4), (R)__ldg(M + 8 * r + 5), v[2], (R)__ldg(M + 8 * r + 6),
                                  (R)__ldg(M + 8 * r + 7), v[3]);
              cpx<R> y;
              y.re = s0.re + s1.re;
              y.im = s0.im + s1.im;
              if (pr) prune_amp(y, thr, qthr);
              sm[SwzT<R>::f(idx[r])] = y;
            }
          }
          __syncthreads();
#pragma unroll
          for (int j = 0; j < 16; j++) x[j] = sm[SwzT<R>::f(L.tbase | rofs(L, j))];
          continue;  // pruning already done
        }
        case FO_DIAGR: {
          const R d0r = (R)__ldg(M + 0), d0i = (R)__ldg(M + 1), d1r = (R)__ldg(M + 2), d1i = (R)__ldg(M + 3);
          if (fl & FOF_D0ONE) {
            switch (oa) {
              case 0: diag_reg<R, 0, true>(x, d0r, d0i, d1r, d1i, smask); break;
              case 1: diag_reg<R, 1, true>(x, d0r, d0i, d1r, d1i, smask); break;
              case 2: diag_reg<R, 2, true>(x, d0r, d0i, d1r, d1i, smask); break;
              default: diag_reg<R, 3, true>(x, d0r, d0i, d1r, d1i, smask); break;
            }
          } else {
            switch (oa) {
              case 0: diag_reg<R, 0, false>(x, d0r, d0i, d1r, d1i, smask); break;
              case 1: diag_reg<R, 1, false>(x, d0r, d0i, d1r, d1i, smask); break;
              case 2: diag_reg<R, 2, false>(x, d0r, d0i, d1r, d1i, smask); break;
              default: diag_reg<R, 3, false>(x, d0r, d0i, d1r, d1i, smask); break;
            }
          }
          break;
        }
        case FO_DIAGT: case FO_DIAGX: {
          bool one;
          if (type == FO_DIAGT) one = (tid >> oa) & 1;
          else one = (ctxbase & __ldg(reinterpret_cast<const unsigned long long*>(op) + 5)) != 0;
          if ((fl & FOF_D0ONE) && !one) break;
          const R dr = (R)__ldg(M + (one ? 2 : 0)), di = (R)__ldg(M + (one ? 3 : 1));
          phase_all<R>(x, dr, di, smask);
          break;
        }
        case FO_DIAG: {
          const int d0 = (int16_t)(h1.w & 0xffff), d1 = (int16_t)(h1.w >> 16);
          const uint32_t ct = h1.z;
          const uint64_t dg0 = __ldg(reinterpret_cast<const unsigned long long*>(op) + 5);
          const uint64_t dg1 = __ldg(reinterpret_cast<const unsigned long long*>(op) + 6);
          const int u0 = d0 < 0 ? (int)((ctxbase & dg0) != 0) : 0;
          const int u1 = d1 == -1 ? (int)((ctxbase & dg1) != 0) : 0;
          R dm[8];
#pragma unroll
          for (int q = 0; q < 8; q++) dm[q] = (R)__ldg(M + q);
#pragma unroll
          for (int j = 0; j < 16; j++) {
            const uint32_t idx = L.tbase | rofs(L, j);
            const int k0 = d0 >= 0 ? (int)((idx >> d0) & 1) : u0;
            const int k1 = d1 >= 0 ? (int)((idx >> d1) & 1) : u1;
            const int kk = d1 != -2 ? 2 * k0 + k1 : k0;
            R dr = dm[0], di = dm[1];
            dr = kk == 1 ? dm[2] : dr;
            di = kk == 1 ? dm[3] : di;
            dr = kk == 2 ? dm[4] : dr;
            di = kk == 2 ? dm[5] : di;
            dr = kk == 3 ? dm[6] : dr;
            di = kk == 3 ? dm[7] : di;
            cpx<R> y = cmul<R>(dr, di, x[j]);
            x[j] = sel<R>((idx & ct) == ct, y, x[j]);
          }
          break;
        }
        case FO_GRADM: case FO_GRADD: {
          if (!GRAD) break;
          // <lambda|D|psi> over this thread's amplitudes: register bit 3 of the
          // slot index selects psi (0) or lambda (1) -- the planner pins the
          // ancilla there
          const int slot = (int16_t)(h1.w >> 16);
          double acc = 0.0;
          if (type == FO_GRADM) {
            R d[8];
#pragma unroll
            for (int q = 0; q < 8; q++) d[q] = (R)__ldg(M + q);
            switch (oa) {
              case 0: acc = grad_m<R, 0>(x, d, smask); break;
              case 1: acc = grad_m<R, 1>(x, d, smask); break;
              default: acc = grad_m<R, 2>(x, d, smask); break;
            }
          } else {
            const R d0r = (R)__ldg(M + 0), d0i = (R)__ldg(M + 1), d1r = (R)__ldg(M + 2), d1i = (R)__ldg(M + 3);
            if (fl & (FOF_TGT_THR | FOF_TGT_CTX)) {
              const bool one = (fl & FOF_TGT_CTX)
                                   ? (ctxbase & __ldg(reinterpret_cast<const unsigned long long*>(op) + 5)) != 0
                                   : (bool)((tid >> oa) & 1);
              acc = grad_d<R, -1>(x, one ? d1r : d0r, one ? d1i : d0i, one ? d1r : d0r, one ? d1i : d0i, smask);
            } else {
              switch (oa) {
                case 0: acc = grad_d<R, 0>(x, d0r, d0i, d1r, d1i, smask); break;
                case 1: acc = grad_d<R, 1>(x, d0r, d0i, d1r, d1i, smask); break;
                default: acc = grad_d<R, 2>(x, d0r, d0i, d1r, d1i, smask); break;
              }
            }
          }
          grad_accum(sgrad, slot, warp, lane, acc);
          break;
        }
        case FO_GRADM2: {
          if (!GRAD) break;
          __syncthreads();
#pragma unroll
          for (int j = 0; j < 16; j++) sm[SwzT<R>::f(L.tbase | rofs(L, j))] = x[j];
          __syncthreads();
          const int slot = (int16_t)(h1.w >> 16), anc = (int16_t)(h1.w & 0xffff);
          const uint32_t ct = h1.z;
          const int ta = oa, tb = ob;
          int b3[3] = {ta, tb, anc};
          for (int u = 1; u < 3; u++)
            for (int v = u; v > 0 && b3[v - 1] > b3[v]; v--) { int t = b3[v]; b3[v] = b3[v - 1]; b3[v - 1] = t; }
          double acc = 0.0;
          for (uint32_t g = tid; g < (1u << (KET_T2_BITS - 3)); g += NT) {
            uint32_t b0 = insert0_32(insert0_32(insert0_32(g, b3[0]), b3[1]), b3[2]);
            if ((b0 & ct) != ct) continue;
            const uint32_t idx[4] = {b0, b0 | (1u << tb), b0 | (1u << ta), b0 | (1u << ta) | (1u << tb)};
            cpx<R> v[4];
            for (int c = 0; c < 4; c++) v[c] = sm[SwzT<R>::f(idx[c])];
            for (int r = 0; r < 4; r++) {
              cpx<R> s0 = mac2<R>((R)__ldg(M + 8 * r), (R)__ldg(M + 8 * r + 1), v[0], (R)__ldg(M + 8 * r + 2),
                                  (R)__ldg(M + 8 * r + 3), v[1]);
              cpx<R> s1 = mac2<R>((R)__ldg(M + 8 * r + 4), (R)__ldg(M + 8 * r + 5), v[2], (R)__ldg(M + 8 * r + 6),
                                  (R)__ldg(M + 8 * r + 7), v[3]);
              cpx<R> lam = sm[SwzT<R>::f(idx[r] | (1u << anc))];
              acc += (double)lam.re * (s0.re + s1.re) + (double)lam.im * (s0.im + s1.im);
            }
          }
          grad_accum(sgrad, slot, warp, lane, acc);
          continue;
        }
        default: break;
      }
      if (pr) prune16<R>(x, thr, qthr);  // mixing ops only (the planner clears the flag elsewhere)
    }
    // the planner leaves the store layout in force here
    {
      const GLayout gl = make_glayout(a, a.store_pos, lane, warp);
#pragma unroll
      for (int j = 0; j < 16; j++) st_amp<R>(amp + (ctxbase | gl.gthr | grofs(gl, j)), x[j]);
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

template <typename R, bool GRAD>
cudaError_t launch_t(const Pass2Args& a, cudaStream_t s) {
  const int NT = 256;
  static bool init = false;
  if (!init) {
    uint16_t sm[16];
    for (int c = 0; c < 16; c++) {
      uint16_t v = 0;
      for (int j = 0; j < 16; j++)
        if ((j & c) == c) v |= (uint16_t)(1u << j);
      sm[c] = v;
    }
    cudaMemcpyToSymbol(c_slotmask, sm, sizeof(sm));
    cudaFuncSetAttribute(k_fused2<R, NT, GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    init = true;
  }
  size_t smem = (sizeof(cpx<R>) << KET_T2_BITS) + (GRAD ? sizeof(double) * 8 * (size_t)a.nslots : 0);
  uint64_t ntiles = uint64_t(1) << (a.n - KET_T2_BITS);
  unsigned blocks = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)fused2_grid());
  k_fused2<R, NT, GRAD><<<blocks, NT, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

int fused2_grid() { return num_sms() * 2; }

cudaError_t launch_fused2(const Pass2Args& a, int precision, cudaStream_t s) {
  if (a.nslots > 0) return precision == KET_C64 ? launch_t<float, true>(a, s) : launch_t<double, true>(a, s);
  return precision == KET_C64 ? launch_t<float, false>(a, s) : launch_t<double, false>(a, s);
}

cudaError_t launch_grad_reduce(const double* gpart, int nctas, int nslots, double* out, cudaStream_t s) {
  k_grad_reduce<<<(nslots + 127) / 128, 128, 0, s>>>(gpart, nctas, nslots, out);
  return cudaGetLastError();
}

}  // namespace ket
