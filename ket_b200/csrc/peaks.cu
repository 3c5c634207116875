// peaks.cu -- ket_measure_fp64: the FP64 FMA rate of the device, measured.
//
// The fused-pass kernels are HBM-bound and are held against the measured copy
// bandwidth; the small batched circuits run from shared memory and are bound
// by the FP64 pipe instead.  This kernel gives that denominator on the GPU at
// hand: every thread runs 8 independent FMA chains in registers, enough
// independent work per warp to keep the pipe busy, over a grid of several
// CTAs per SM, timed with CUDA events on the context's stream.
#include "common.cuh"
#include "ctx.h"
#include "read.h"

namespace ket {
namespace {

constexpr int kChains = 8;
constexpr int kIters = 1 << 14;

__global__ void __launch_bounds__(256) k_fma_rate(double seed, double* sink) {
  double v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; c++) v[c] = seed + 1e-3 * (threadIdx.x + c);
  const double m = 0.999999999, b = 1e-9;
  for (int i = 0; i < kIters; i++) {
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = fma(v[c], m, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; c++) s += v[c];
  if (s == 12345.678) sink[blockIdx.x] = s;  // never true: keeps the chains alive
}

}  // namespace
}  // namespace ket

using namespace ket;

extern "C" int ket_measure_fp64(ket_ctx* c, double* fma_per_s) {
  if (!c || !fma_per_s) return fail(KET_ERR_TYPE, "null argument");
  cudaSetDevice(c->device);
  void* sink = nullptr;
  int rc = ctx_scratch(c, 8 * 4096, &sink);
  if (rc) return rc;
  const int grid = num_sms() * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_rate<<<grid, 256, 0, c->stream>>>(1.0, (double*)sink);  // warm-up
  cudaEventRecord(e0, c->stream);
  const int reps = 4;
  for (int r = 0; r < reps; r++) k_fma_rate<<<grid, 256, 0, c->stream>>>(1.0 + r, (double*)sink);
  cudaEventRecord(e1, c->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->launches += reps + 1;
  if (e != cudaSuccess) return cuda_fail(e, "ket_measure_fp64");
  const double fmas = (double)reps * grid * 256.0 * kChains * kIters;
  *fma_per_s = fmas / (ms * 1e-3);
  return KET_OK;
}
