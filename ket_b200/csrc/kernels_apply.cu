// kernels_apply.cu -- gate application kernels.
//
// Two families:
//   * single-gate passes (one launch per gate, grid-stride over amplitude
//     pairs / groups) -- the unfused path and the home of wide unitaries;
//   * the fused tile pass: each CTA streams tiles of 2^m amplitudes (the L
//     lowest qubits plus m-L chosen high qubits) through shared memory and
//     applies every gate of the pass to the tile before writing it back, so
//     a pass costs one read and one write of the state however many gates
//     it holds.
//
// Semantics follow src/statevector.ts: 2x2 on pairs (x0 with bit t = 0,
// x1 = x0 | 2^t), 4x4 on (a = MSB, b), controls must all be 1, and with
// pruning on every computed amplitude with |a|^2 < 1e-14 becomes exactly 0
// (accumulate(), statevector.ts:19-27).
#include <algorithm>

#include "common.cuh"
#include "launch.h"

namespace ket {

int num_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

namespace {

struct M2 { double m[8]; };
struct M4 { double m[32]; };

template <typename R>
__device__ __forceinline__ void apply2(cpx<R>& x0, cpx<R>& x1, const double* m) {
  const R m0r = (R)m[0], m0i = (R)m[1], m1r = (R)m[2], m1i = (R)m[3];
  const R m2r = (R)m[4], m2i = (R)m[5], m3r = (R)m[6], m3i = (R)m[7];
  cpx<R> y0 = mac2<R>(m0r, m0i, x0, m1r, m1i, x1);
  cpx<R> y1 = mac2<R>(m2r, m2i, x0, m3r, m3i, x1);
  x0 = y0;
  x1 = y1;
}

template <typename R>
__device__ __forceinline__ void apply4(cpx<R>* x, const double* m) {
  cpx<R> y[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    cpx<R> a = mac2<R>((R)m[8 * r + 0], (R)m[8 * r + 1], x[0], (R)m[8 * r + 2], (R)m[8 * r + 3], x[1]);
    cpx<R> b = mac2<R>((R)m[8 * r + 4], (R)m[8 * r + 5], x[2], (R)m[8 * r + 6], (R)m[8 * r + 7], x[3]);
    y[r].re = a.re + b.re;
    y[r].im = a.im + b.im;
  }
#pragma unroll
  for (int r = 0; r < 4; r++) x[r] = y[r];
}

// ------------------------------------------------------------------ single-gate kernels
template <typename R>
__global__ void k_mat1(typename Vec2<R>::T* a, uint64_t npairs, int t, uint64_t cmask, M2 m, int prune,
                       double thr, double qthr) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i0 = insert0(p, t);
    if ((i0 & cmask) != cmask) continue;
    uint64_t i1 = i0 | (uint64_t(1) << t);
    cpx<R> x0 = ld_amp<R>(a + i0), x1 = ld_amp<R>(a + i1);
    apply2<R>(x0, x1, m.m);
    if (prune) { prune_amp(x0, thr, qthr); prune_amp(x1, thr, qthr); }
    st_amp<R>(a + i0, x0);
    st_amp<R>(a + i1, x1);
  }
}

template <typename R>
__global__ void k_x1(typename Vec2<R>::T* a, uint64_t npairs, int t, uint64_t cmask) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i0 = insert0(p, t);
    if ((i0 & cmask) != cmask) continue;
    uint64_t i1 = i0 | (uint64_t(1) << t);
    typename Vec2<R>::T v0 = a[i0], v1 = a[i1];
    a[i0] = v1;
    a[i1] = v0;
  }
}

template <typename R>
__global__ void k_diag(typename Vec2<R>::T* a, uint64_t N, int t0, int t1, uint64_t cmask, M4 d, int prune,
                       double thr, double qthr) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
    if ((i & cmask) != cmask) continue;
    int k = (int)((i >> t0) & 1);
    if (t1 >= 0) k = 2 * k + (int)((i >> t1) & 1);
    cpx<R> x = ld_amp<R>(a + i);
    x = cmul<R>((R)d.m[2 * k], (R)d.m[2 * k + 1], x);
    if (prune) prune_amp(x, thr, qthr);
    st_amp<R>(a + i, x);
  }
}

template <typename R>
__global__ void k_swap(typename Vec2<R>::T* a, uint64_t nq, int lo, int hi, uint64_t cmask) {
  // enumerate indices with bit lo = 0 and bit hi = 0, then swap (lo=1,hi=0) <-> (lo=0,hi=1)
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < nq; p += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = insert0(insert0(p, lo), hi);
    if ((base & cmask) != cmask) continue;
    uint64_t i01 = base | (uint64_t(1) << lo), i10 = base | (uint64_t(1) << hi);
    typename Vec2<R>::T v = a[i01];
    a[i01] = a[i10];
    a[i10] = v;
  }
}

template <typename R>
__global__ void k_mat2(typename Vec2<R>::T* a, uint64_t nq, int ta, int tb, uint64_t cmask, M4 m, int prune,
                       double thr, double qthr) {
  const int lo = ta < tb ? ta : tb, hi = ta < tb ? tb : ta;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < nq; p += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = insert0(insert0(p, lo), hi);
    if ((base & cmask) != cmask) continue;
    uint64_t ia = uint64_t(1) << ta, ib = uint64_t(1) << tb;
    uint64_t idx[4] = {base, base | ib, base | ia, base | ia | ib};
    cpx<R> x[4];
#pragma unroll
    for (int j = 0; j < 4; j++) x[j] = ld_amp<R>(a + idx[j]);
    apply4<R>(x, m.m);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (prune) prune_amp(x[j], thr, qthr);
      st_amp<R>(a + idx[j], x[j]);
    }
  }
}

// Dense k-qubit unitary: one CTA per group of 2^k amplitudes, staged in smem
// (inputs xs, outputs ys, global indices idx).
template <typename R>
__global__ void k_matk(typename Vec2<R>::T* a, uint64_t ngroups, int k, const int* tq, const double* mat, int prune,
                       double thr, double qthr) {
  extern __shared__ unsigned char smraw[];
  const uint32_t D = 1u << k;
  cpx<R>* xs = reinterpret_cast<cpx<R>*>(smraw);
  cpx<R>* ys = xs + D;
  uint64_t* idx = reinterpret_cast<uint64_t*>(ys + D);
  int sorted[KET_MAX_OP_QUBITS];
  for (int j = 0; j < k; j++) sorted[j] = tq[j];
  for (int x = 1; x < k; x++)
    for (int y = x; y > 0 && sorted[y - 1] > sorted[y]; y--) { int t = sorted[y]; sorted[y] = sorted[y - 1]; sorted[y - 1] = t; }
  for (uint64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    uint64_t ctx = g;
    for (int j = 0; j < k; j++) ctx = insert0(ctx, sorted[j]);
    for (uint32_t i = threadIdx.x; i < D; i += blockDim.x) {
      uint64_t b = ctx;
      for (int bit = 0; bit < k; bit++)
        if ((i >> (k - 1 - bit)) & 1) b |= uint64_t(1) << tq[bit];
      idx[i] = b;
      xs[i] = ld_amp<R>(a + b);
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < D; r += blockDim.x) {
      double sr = 0, si = 0;
      const double* row = mat + 2 * (size_t)r * D;
      for (uint32_t c = 0; c < D; c++) {
        double mr = row[2 * c], mi = row[2 * c + 1];
        double xr = xs[c].re, xi = xs[c].im;
        sr = fma(mr, xr, fma(-mi, xi, sr));
        si = fma(mr, xi, fma(mi, xr, si));
      }
      cpx<R> o{(R)sr, (R)si};
      if (prune) prune_amp(o, thr, qthr);
      ys[r] = o;
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < D; r += blockDim.x) st_amp<R>(a + idx[r], ys[r]);
    __syncthreads();
  }
}

// ------------------------------------------------------------------ fused tile pass
template <typename R, int NT>
__global__ void __launch_bounds__(NT) k_fused(PassArgs args) {
  typedef typename Vec2<R>::T V;
  extern __shared__ unsigned char smraw[];
  cpx<R>* s = reinterpret_cast<cpx<R>*>(smraw);
  V* amp = reinterpret_cast<V*>(args.amp);
  const int m = args.m, L = args.L;
  const uint32_t T = 1u << m;
  const uint32_t lowmask = (1u << L) - 1;
  const uint64_t ntiles = uint64_t(1) << (args.n - m);
  const int tid = threadIdx.x;

  for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    uint64_t base = 0;
    for (int j = 0; j < args.nctx; j++)
      if ((tile >> j) & 1) base |= uint64_t(1) << args.ctxbits[j];

    for (uint32_t i = tid; i < T; i += NT) {
      uint64_t g = base | (i & lowmask);
      uint32_t hi = i >> L;
      for (int j = 0; j < args.nh; j++)
        if ((hi >> j) & 1) g |= uint64_t(1) << args.hbits[j];
      s[i] = ld_amp<R>(amp + g);
    }
    __syncthreads();

    for (int k = 0; k < args.nops; k++) {
      const DevOp& op = args.ops[k];
      if ((base & op.cctx) != op.cctx) continue;  // uniform: a context control is off for this tile
      const int type = op.type;
      const uint32_t ct = op.ctile;
      const bool pr = op.flags & 1;
      if (type == G_MAT1) {
        const int b = op.b0;
        double mm[8];
#pragma unroll
        for (int j = 0; j < 8; j++) mm[j] = op.m[j];
        for (uint32_t p = tid; p < T / 2; p += NT) {
          uint32_t i0 = insert0_32(p, b);
          if ((i0 & ct) != ct) continue;
          uint32_t i1 = i0 | (1u << b);
          cpx<R> x0 = s[i0], x1 = s[i1];
          apply2<R>(x0, x1, mm);
          if (pr) { prune_amp(x0, args.thr, args.qthr); prune_amp(x1, args.thr, args.qthr); }
          s[i0] = x0;
          s[i1] = x1;
        }
      } else if (type == G_X1) {
        const int b = op.b0;
        for (uint32_t p = tid; p < T / 2; p += NT) {
          uint32_t i0 = insert0_32(p, b);
          if ((i0 & ct) != ct) continue;
          uint32_t i1 = i0 | (1u << b);
          cpx<R> x0 = s[i0];
          s[i0] = s[i1];
          s[i1] = x0;
        }
      } else if (type == G_DIAG1 || type == G_DIAG2) {
        int u0 = op.b0 < 0 ? (int)((base & op.g0) != 0) : -1;
        int u1 = (type == G_DIAG2 && op.b1 < 0) ? (int)((base & op.g1) != 0) : -1;
        for (uint32_t i = tid; i < T; i += NT) {
          if ((i & ct) != ct) continue;
          int k0 = u0 >= 0 ? u0 : (int)((i >> op.b0) & 1);
          int kk = k0;
          if (type == G_DIAG2) {
            int k1 = u1 >= 0 ? u1 : (int)((i >> op.b1) & 1);
            kk = 2 * k0 + k1;
          }
          cpx<R> x = cmul<R>((R)op.m[2 * kk], (R)op.m[2 * kk + 1], s[i]);
          if (pr) prune_amp(x, args.thr, args.qthr);
          s[i] = x;
        }
      } else if (type == G_SWAP) {
        const int lo = op.b0 < op.b1 ? op.b0 : op.b1, hi = op.b0 < op.b1 ? op.b1 : op.b0;
        for (uint32_t p = tid; p < T / 4; p += NT) {
          uint32_t bb = insert0_32(insert0_32(p, lo), hi);
          if ((bb & ct) != ct) continue;
          uint32_t i01 = bb | (1u << lo), i10 = bb | (1u << hi);
          cpx<R> v = s[i01];
          s[i01] = s[i10];
          s[i10] = v;
        }
      } else if (type == G_MAT2) {
        const int ba = op.b0, bbit = op.b1;
        const int lo = ba < bbit ? ba : bbit, hi = ba < bbit ? bbit : ba;
        for (uint32_t p = tid; p < T / 4; p += NT) {
          uint32_t bb = insert0_32(insert0_32(p, lo), hi);
          if ((bb & ct) != ct) continue;
          uint32_t idx[4] = {bb, bb | (1u << bbit), bb | (1u << ba), bb | (1u << ba) | (1u << bbit)};
          cpx<R> x[4];
#pragma unroll
          for (int j = 0; j < 4; j++) x[j] = s[idx[j]];
          apply4<R>(x, op.m);
#pragma unroll
          for (int j = 0; j < 4; j++) {
            if (pr) prune_amp(x[j], args.thr, args.qthr);
            s[idx[j]] = x[j];
          }
        }
      }
      __syncthreads();
    }

    for (uint32_t i = tid; i < T; i += NT) {
      uint64_t g = base | (i & lowmask);
      uint32_t hi = i >> L;
      for (int j = 0; j < args.nh; j++)
        if ((hi >> j) & 1) g |= uint64_t(1) << args.hbits[j];
      st_amp<R>(amp + g, s[i]);
    }
    __syncthreads();
  }
}

inline unsigned grid_for(uint64_t work, int nt) {
  uint64_t blocks = (work + nt - 1) / nt;
  uint64_t cap = (uint64_t)num_sms() * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (unsigned)blocks;
}

template <typename R>
cudaError_t launch_gate_t(const Gate& g, void* ampv, int n, const void* dev_matk, cudaStream_t s) {
  typedef typename Vec2<R>::T V;
  V* a = reinterpret_cast<V*>(ampv);
  const uint64_t N = uint64_t(1) << n;
  const int NT = 256;
  const double thr = 1e-14, qthr = 1e-7;
  const int pr = g.prune ? 1 : 0;
  switch (g.type) {
    case G_MAT1: {
      M2 m;
      for (int k = 0; k < 4; k++) { m.m[2 * k] = g.m[k].re; m.m[2 * k + 1] = g.m[k].im; }
      k_mat1<R><<<grid_for(N / 2, NT), NT, 0, s>>>(a, N / 2, g.t0, g.cmask, m, pr, thr, qthr);
      break;
    }
    case G_X1:
      k_x1<R><<<grid_for(N / 2, NT), NT, 0, s>>>(a, N / 2, g.t0, g.cmask);
      break;
    case G_DIAG1: case G_DIAG2: {
      M4 d;
      int cnt = g.type == G_DIAG1 ? 2 : 4;
      for (int k = 0; k < cnt; k++) { d.m[2 * k] = g.m[k].re; d.m[2 * k + 1] = g.m[k].im; }
      k_diag<R><<<grid_for(N, NT), NT, 0, s>>>(a, N, g.t0, g.type == G_DIAG2 ? g.t1 : -1, g.cmask, d, pr, thr, qthr);
      break;
    }
    case G_SWAP: {
      int lo = std::min(g.t0, g.t1), hi = std::max(g.t0, g.t1);
      k_swap<R><<<grid_for(N / 4, NT), NT, 0, s>>>(a, N / 4, lo, hi, g.cmask);
      break;
    }
    case G_MAT2: {
      M4 m;
      for (int k = 0; k < 16; k++) { m.m[2 * k] = g.m[k].re; m.m[2 * k + 1] = g.m[k].im; }
      k_mat2<R><<<grid_for(N / 4, NT), NT, 0, s>>>(a, N / 4, g.t0, g.t1, g.cmask, m, pr, thr, qthr);
      break;
    }
    case G_MATK: {
      int k = (int)g.tk.size();
      const int* dq = reinterpret_cast<const int*>(dev_matk);
      const double* dm = reinterpret_cast<const double*>(reinterpret_cast<const char*>(dev_matk) + 64);
      size_t smem = (2 * sizeof(cpx<R>) + sizeof(uint64_t)) * (size_t(1) << k);
      if (smem > 48 * 1024) cudaFuncSetAttribute(k_matk<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      uint64_t ngroups = N >> k;
      unsigned blocks = (unsigned)std::min<uint64_t>(ngroups, (uint64_t)num_sms() * 8);
      k_matk<R><<<blocks, NT, smem, s>>>(a, ngroups, k, dq, dm, pr, thr, qthr);
      break;
    }
  }
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_fused_t(const PassArgs& a, cudaStream_t s) {
  const int NT = 256;
  size_t smem = sizeof(cpx<R>) * (size_t(1) << a.m);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_fused<R, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  uint64_t ntiles = uint64_t(1) << (a.n - a.m);
  int per_sm = std::max(1, (int)((200 * 1024) / std::max<size_t>(smem, 1)));
  if (per_sm > 4) per_sm = 4;
  unsigned blocks = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)num_sms() * per_sm);
  k_fused<R, NT><<<blocks, NT, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

DevOp encode_devop(const Gate& g, const Pass& p, bool prune) {
  DevOp d;
  memset(&d, 0, sizeof(d));
  d.type = g.type;
  // tile-local position of a global qubit, -1 when outside the tile
  auto tpos = [&](int q) -> int {
    if (q < 0) return -1;
    if (q < p.L) return q;
    for (size_t j = 0; j < p.hbits.size(); j++)
      if (p.hbits[j] == q) return p.L + (int)j;
    return -1;
  };
  d.b0 = tpos(g.t0);
  d.b1 = tpos(g.t1);
  d.flags = (g.prune && prune) ? 1 : 0;
  for (int q = 0; q < 64; q++) {
    if (!((g.cmask >> q) & 1)) continue;
    int t = tpos(q);
    if (t >= 0) d.ctile |= 1u << t;
    else d.cctx |= uint64_t(1) << q;
  }
  if (g.t0 >= 0 && d.b0 < 0) d.g0 = uint64_t(1) << g.t0;
  if (g.t1 >= 0 && d.b1 < 0) d.g1 = uint64_t(1) << g.t1;
  int cnt = g.type == G_MAT2 ? 16 : (g.type == G_DIAG1 ? 2 : 4);
  for (int k = 0; k < cnt; k++) { d.m[2 * k] = g.m[k].re; d.m[2 * k + 1] = g.m[k].im; }
  return d;
}

cudaError_t launch_gate(const Gate& g, int precision, void* amp, int n, const void* dev_matk, cudaStream_t s) {
  return precision == KET_C64 ? launch_gate_t<float>(g, amp, n, dev_matk, s)
                              : launch_gate_t<double>(g, amp, n, dev_matk, s);
}

cudaError_t launch_fused(const PassArgs& a, int precision, cudaStream_t s) {
  return precision == KET_C64 ? launch_fused_t<float>(a, s) : launch_fused_t<double>(a, s);
}

}  // namespace ket
