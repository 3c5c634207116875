// matrix.cu -- circuitMatrix() (circuit.ts:1462-1485) and blochAngles()
// (:4102-4129).
//
// circuitMatrix simulates the circuit once per basis column.  Here all 2^n
// columns run as one 2n-qubit state: the low n qubits are the circuit's, the
// high n hold the column, and the state starts as the identity (amplitude 1
// at index flip(col) + col * 2^n, flip = n-bit reversal, because rows and
// columns use q0 as the most significant bit).  Gates touch only the low
// qubits, so the columns never mix and the reference's per-amplitude pruning
// is per column, exactly as the reference's one-column simulations prune.
// One permutation pass then writes the matrix row-major in that order.
//
// blochAngles reduces rho00, rho11 and rho01 = sum psi(i) psi(i|q)* over the
// pairs of qubit q in one pass (fixed-order partial sums), and the host takes
// the angles.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "engine.h"
#include "launch.h"

using namespace ket;

namespace {

__host__ __device__ inline uint64_t flip_bits(uint64_t i, int n) {
  uint64_t r = 0;
  for (int b = 0; b < n; b++)
    if ((i >> b) & 1) r |= uint64_t(1) << (n - 1 - b);
  return r;
}

// the identity as a 2n-qubit state: |flip(col)> (x) |col>
__global__ void k_identity_state(double2* a, int n) {
  const uint64_t dim = uint64_t(1) << n;
  for (uint64_t col = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; col < dim;
       col += (uint64_t)gridDim.x * blockDim.x)
    a[flip_bits(col, n) | (col << n)] = make_double2(1.0, 0.0);
}

// out[flip(r) * dim + col] = a[r + col * dim]
__global__ void k_matrix_order(const double2* a, int n, double2* out) {
  const uint64_t dim = uint64_t(1) << n, N = dim * dim;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i & (dim - 1), col = i >> n;
    out[flip_bits(r, n) * dim + col] = a[i];
  }
}

constexpr int BNT = 256;

// per block: rho00, rho11, Re rho01, Im rho01 over its slice of the pairs
template <typename R>
__global__ void __launch_bounds__(BNT) k_bloch(const typename Vec2<R>::T* a, uint64_t half, int q, uint64_t chunk,
                                               double* partial) {
  __shared__ double sh[4][BNT];
  const uint64_t lo = (uint64_t)blockIdx.x * chunk;
  const uint64_t hi = lo + chunk < half ? lo + chunk : half;
  const uint64_t low = (uint64_t(1) << q) - 1;
  double r00 = 0, r11 = 0, re = 0, im = 0;
  for (uint64_t j = lo + threadIdx.x; j < hi; j += BNT) {
    const uint64_t i0 = ((j & ~low) << 1) | (j & low), i1 = i0 | (uint64_t(1) << q);
    const typename Vec2<R>::T v0 = a[i0], v1 = a[i1];
    const double a0r = v0.x, a0i = v0.y, a1r = v1.x, a1i = v1.y;
    r00 += a0r * a0r + a0i * a0i;
    r11 += a1r * a1r + a1i * a1i;
    re += a0r * a1r + a0i * a1i;
    im += a0i * a1r - a0r * a1i;
  }
  sh[0][threadIdx.x] = r00;
  sh[1][threadIdx.x] = r11;
  sh[2][threadIdx.x] = re;
  sh[3][threadIdx.x] = im;
  __syncthreads();
  for (int w = BNT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < 4; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) partial[(uint64_t)blockIdx.x * 4 + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_bloch_sum(const double* partial, int nb, double* out) {
  if (threadIdx.x >= 4) return;
  double s = 0;
  for (int b = 0; b < nb; b++) s += partial[(uint64_t)b * 4 + threadIdx.x];
  out[threadIdx.x] = s;
}

#define TRY(x) do { int _rc = (x); if (_rc) return _rc; } while (0)

}  // namespace

extern "C" {

int ket_circuit_matrix(ket_ctx* ctx, int nqubits, const ket_op* ops, size_t nops, const double* mats, size_t nmat,
                       const ket_exec_opts* opts, double* out) {
  if (!ctx || !out) return fail(KET_ERR_TYPE, "null argument");
  if (nops && !ops) return fail(KET_ERR_TYPE, "null op list");
  if (nqubits < 0) return fail(KET_ERR_RANGE, "negative qubit count");
  if (nqubits > 12)
    return fail(KET_ERR_RANGE, "circuitMatrix(): circuit too large (" + std::to_string(nqubits) + " qubits = " +
                                   std::to_string(1 << nqubits) + "x" + std::to_string(1 << nqubits) + " matrix)");
  {  // every op on the circuit's own qubits (a wider state would accept the column qubits too)
    std::vector<Gate> lowered;
    std::string err;
    const int rc = lower_ops(nqubits, ops, nops, mats, nmat, opts ? opts->prune != 0 : true, lowered, err);
    if (rc) return fail(rc, err);
  }
  if (nqubits == 0) {
    out[0] = 1.0;
    out[1] = 0.0;
    return KET_OK;
  }
  cudaSetDevice(ctx->device);
  ket_state* st = nullptr;
  TRY(ket_state_alloc(ctx, 2 * nqubits, KET_C128, &st));
  const uint64_t dim = uint64_t(1) << nqubits, N = dim * dim;
  int rc = KET_OK;
  double2* ordered = nullptr;
  do {
    cudaError_t e = cudaMemsetAsync(st->amp, 0, 16 * N, ctx->stream);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemsetAsync(state)"); break; }
    prof_begin(ctx);
    k_identity_state<<<(unsigned)((dim + 255) / 256), 256, 0, ctx->stream>>>((double2*)st->amp, nqubits);
    prof_end(ctx, PK_READ);
    if ((e = cudaGetLastError()) != cudaSuccess) { rc = cuda_fail(e, "identity launch"); break; }
    if ((rc = ket_apply_ops(st, ops, nops, mats, nmat, opts)) != KET_OK) break;
    if ((rc = dev_alloc((void**)&ordered, 16 * N)) != KET_OK) break;
    prof_begin(ctx);
    k_matrix_order<<<(unsigned)std::min<uint64_t>((N + 255) / 256, 148 * 32), 256, 0, ctx->stream>>>(
        (const double2*)st->amp, nqubits, ordered);
    prof_end(ctx, PK_READ);
    if ((e = cudaGetLastError()) != cudaSuccess) { rc = cuda_fail(e, "matrix order launch"); break; }
    ctx->d2h_bytes += 16 * N;
    e = cudaMemcpyAsync(out, ordered, 16 * N, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) { rc = cuda_fail(e, "cudaMemcpyAsync(matrix)"); break; }
    rc = ctx_wait(ctx);
  } while (0);
  if (ordered) cudaFree(ordered);
  ket_state_free(st);
  return rc;
}

int ket_bloch(const ket_state* st, int q, double* out) {
  if (!st || !out) return fail(KET_ERR_TYPE, "null argument");
  if (q < 0 || q >= st->n)
    return fail(KET_ERR_RANGE, "qubit index " + std::to_string(q) + " is out of range for a " +
                                   std::to_string(st->n) + "-qubit circuit");
  ket_ctx* c = st->ctx;
  cudaSetDevice(c->device);
  const uint64_t half = uint64_t(1) << (st->n - 1);
  const uint64_t chunk = half > 4096 * 1024 ? (half + 4095) / 4096 : 1024;
  const int nb = (int)((half + chunk - 1) / chunk);
  void* scr;
  TRY(ctx_scratch(c, 32 * (size_t)nb + 64, &scr));
  double* part = (double*)scr;
  double* sums = part + 4 * (size_t)nb;
  prof_begin(c);
  if (st->precision == KET_C64)
    k_bloch<float><<<nb, BNT, 0, c->stream>>>((const float2*)st->amp, half, q, chunk, part);
  else
    k_bloch<double><<<nb, BNT, 0, c->stream>>>((const double2*)st->amp, half, q, chunk, part);
  k_bloch_sum<<<1, 32, 0, c->stream>>>(part, nb, sums);
  prof_end(c, PK_READ);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "bloch launch");
  double s[4];
  c->d2h_bytes += 32;
  e = cudaMemcpyAsync(s, sums, 32, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(bloch)");
  TRY(ctx_wait(c));
  // Bloch vector rz = rho00 - rho11, rx = 2 Re rho01, ry = -2 Im rho01 (circuit.ts:4122-4128)
  const double rz = s[0] - s[1], rx = 2 * s[2], ry = -2 * s[3];
  for (int k = 0; k < 4; k++) out[k] = s[k];
  out[4] = std::acos(std::fmax(-1.0, std::fmin(1.0, rz)));
  out[5] = std::atan2(ry, rx);
  return KET_OK;
}

}  // extern "C"
