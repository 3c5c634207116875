// common.cuh -- device-side helpers shared by the engine's kernels.
#pragma once

#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>
#endif

namespace ket {

// Amplitude storage: complex128 as double2, complex64 as float2.
template <typename R> struct Vec2;
template <> struct Vec2<double> { typedef double2 T; };
template <> struct Vec2<float> { typedef float2 T; };

template <typename R>
struct cpx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ cpx<R> ld_amp(const typename Vec2<R>::T* p) {
  typename Vec2<R>::T v = *p;
  return cpx<R>{v.x, v.y};
}
template <typename R>
__device__ __forceinline__ void st_amp(typename Vec2<R>::T* p, cpx<R> a) {
  typename Vec2<R>::T v;
  v.x = a.re;
  v.y = a.im;
  *p = v;
}

// out = m0*x0 + m1*x1 (complex), FMA form.
template <typename R>
__device__ __forceinline__ cpx<R> mac2(R m0r, R m0i, cpx<R> x0, R m1r, R m1i, cpx<R> x1) {
  cpx<R> o;
  o.re = fma(m0r, x0.re, fma(-m0i, x0.im, fma(m1r, x1.re, -m1i * x1.im)));
  o.im = fma(m0r, x0.im, fma(m0i, x0.re, fma(m1r, x1.im, m1i * x1.re)));
  return o;
}

template <typename R>
__device__ __forceinline__ cpx<R> cmul(R mr, R mi, cpx<R> x) {
  cpx<R> o;
  o.re = fma(mr, x.re, -mi * x.im);
  o.im = fma(mr, x.im, mi * x.re);
  return o;
}

// |a|^2 exactly as the reference computes it (re*re + im*im, two rounded
// products then a rounded sum: JavaScript never contracts to FMA).
__device__ __forceinline__ double norm2_ref(double re, double im) {
  return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}
__device__ __forceinline__ double norm2_ref(float re, float im) {
  double r = re, i = im;
  return __dadd_rn(__dmul_rn(r, r), __dmul_rn(i, i));
}

// accumulate() pruning (statevector.ts:19-27): |a|^2 < thr -> 0.  thr is
// 1e-14 scaled by any deferred factor; 0 disables.  The quick integer test on
// the exponent field skips the exact check for all but tiny amplitudes.
__device__ __forceinline__ void prune_amp(cpx<double>& a, double thr, double qthr) {
  if (fabs(a.re) < qthr && fabs(a.im) < qthr) {
    if (norm2_ref(a.re, a.im) < thr) {
      a.re = 0.0;
      a.im = 0.0;
    }
  }
}
__device__ __forceinline__ void prune_amp(cpx<float>& a, double thr, double qthr) {
  if (fabsf(a.re) < (float)qthr && fabsf(a.im) < (float)qthr) {
    if (norm2_ref(a.re, a.im) < thr) {
      a.re = 0.0f;
      a.im = 0.0f;
    }
  }
}

// Insert a zero bit at position b into x.
__device__ __forceinline__ uint64_t insert0(uint64_t x, int b) {
  uint64_t lo = x & ((uint64_t(1) << b) - 1);
  return ((x ^ lo) << 1) | lo;
}
__device__ __forceinline__ uint32_t insert0_32(uint32_t x, int b) {
  uint32_t lo = x & ((1u << b) - 1);
  return ((x ^ lo) << 1) | lo;
}

// Warp reduction of a double.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide deterministic sum (fixed tree order); all threads get the result.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = (l < NT / 32) ? red[l] : 0.0;
    t = warp_sum(t);
    if (l == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

}  // namespace ket
