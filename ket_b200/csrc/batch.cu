// batch.cu -- thousands of QAOA MaxCut circuits of uneven width in one
// persistent launch (ket_batch_qaoa).
//
// Each instance: H on all n qubits, then per layer exp(-i gamma Z_u Z_v) on
// every edge and Rx(2 beta) on every qubit; output <C> = sum_e (1 - <Z_u Z_v>)/2.
// The reference builds the same circuit as qaoa(n, E, -2 gamma, beta)
// (algorithms.ts:260-276: cnot . rz . cnot per edge) and measures it with
// vqe(., maxCutHamiltonian(n, E)) (algorithms.ts:231-241, 301-336).
//
// Work items are pulled from a global queue by a persistent grid:
//   * an instance of n <= TILE qubits is one item, simulated entirely in
//     shared memory (all layers and the <C> reduction);
//   * a wider instance is split into 2p passes of tiles of 2^TILE amplitudes
//     (pass A of a layer: the cost phase, which is diagonal, plus Rx on qubits
//     0..TILE-1; pass B: Rx on the remaining qubits).  A tile of pass k waits
//     (bounded spin, error flag on timeout) until every tile of pass k-1 of
//     its instance has been written back; the queue hands items out in an
//     order where everything a tile waits on was handed out earlier, so the
//     fully resident grid cannot deadlock.
// The cost phase exp(-i gamma (|E| - 2 cut(x))) takes cut(x) from the edge
// masks and a per-layer table of |E|+1 phases.  <C> partials are written per
// (instance, tile) and reduced in a fixed order.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "launch.h"

namespace ket {

namespace {

#define KQ_MAX_EDGES 64
#define KQ_MAX_P 16

struct QInst {
  int n, ne, p, ntiles;     // ntiles = 2^(n - tile) for split instances, 1 otherwise
  int64_t state;            // offset (amplitudes) of the instance's state in the workspace (split only)
  int64_t cut;              // offset (bytes) of the instance's cut values in the cut area (split only)
  int64_t edge_off;         // first edge in the edge array
  int64_t part_off;         // first <C> partial of the instance
};

struct QItem {
  int inst;
  int pass;   // -1: whole instance in shared memory; else pass index 0..2p-1
  int tile;
};

struct QArgs {
  const QInst* inst;
  const QItem* items;
  const uint64_t* emask;    // edge masks (1<<u | 1<<v)
  const double* gamma;      // [inst * p + l]
  const double* beta;
  double2* work;            // split-instance states
  uint8_t* cutw;            // split-instance cut(x) per amplitude, written by pass 0
  double* part;             // <C> partials
  unsigned int* next;       // queue head
  unsigned int* done;       // per instance: tiles finished (pass-major)
  int* status;
  uint32_t spin_limit;      // polls before a wait gives up (status KET_ERR_TIMEOUT)
  int nitems;
  int tile;                 // tile qubits
};

__device__ __forceinline__ int cut_of(uint64_t x, const uint64_t* em, int ne) {
  int c = 0;
  for (int e = 0; e < ne; e++) c += __popcll(x & em[e]) & 1;
  return c;
}

template <int NT>
__device__ void fill_phase(double2* tab, double gamma, int ne) {
  for (int c = threadIdx.x; c <= ne; c += NT) {
    double s, co;
    sincos(-gamma * (double)(ne - 2 * c), &s, &co);
    tab[c] = make_double2(co, s);
  }
}

// Shared-memory position of local amplitude i: the three low index bits are
// XORed with bits 3-5.  For every group of rotated bits below, the eight
// threads of a quarter warp then touch eight distinct 16-byte slots of a
// 128-byte row (conflict-free), whichever bits the group holds.
__device__ __forceinline__ uint32_t sw(uint32_t i) { return i ^ ((i >> 3) & 7u); }

// Rx(2 beta) = [[c, -i s], [-i s, c]] on one pair, in registers.
__device__ __forceinline__ void rx_pair(double2& a, double2& b, double cb, double sb) {
  const double2 x = a, y = b;
  a = make_double2(fma(cb, x.x, sb * y.y), fma(cb, x.y, -sb * y.x));
  b = make_double2(fma(cb, y.x, sb * x.y), fma(cb, y.y, -sb * x.x));
}

// Rx(2 beta) on the K local bits g[0] < ... < g[K-1] of a shared-memory block
// of 2^m amplitudes: each thread loads the 2^K amplitudes of a subcube into
// registers, rotates every bit of the group there (lowest first), and stores
// them back -- one shared-memory round trip per group instead of one per
// bit.  Per amplitude the rotations run in the same order as bit by bit, so
// results are the same.
template <int NT, int K>
__device__ void rx_group(double2* s, int m, uint32_t gp, double cb, double sb) {
  int g[K];  // the group's bits, packed one per byte of gp (kept in registers)
#pragma unroll
  for (int q = 0; q < K; q++) g[q] = (int)((gp >> (8 * q)) & 0xffu);
  const uint32_t nsub = 1u << (m - K);
  for (uint32_t u = threadIdx.x; u < nsub; u += NT) {
    uint32_t b = u;
#pragma unroll
    for (int q = 0; q < K; q++) b = insert0_32(b, g[q]);
    double2 v[1 << K];
#pragma unroll
    for (int j = 0; j < (1 << K); j++) {
      uint32_t o = b;
#pragma unroll
      for (int q = 0; q < K; q++)
        if ((j >> q) & 1) o |= 1u << g[q];
      v[j] = s[sw(o)];
    }
#pragma unroll
    for (int q = 0; q < K; q++)
#pragma unroll
      for (int j = 0; j < (1 << K); j++)
        if (!((j >> q) & 1)) rx_pair(v[j], v[j | (1 << q)], cb, sb);
#pragma unroll
    for (int j = 0; j < (1 << K); j++) {
      uint32_t o = b;
#pragma unroll
      for (int q = 0; q < K; q++)
        if ((j >> q) & 1) o |= 1u << g[q];
      s[sw(o)] = v[j];
    }
  }
}

// Bits per group: three at 256 threads per CTA, so that the registers of three
// resident CTAs (the shared-memory limit) hold a group's 8 amplitudes without
// spills; four at 128 and 512 threads.
template <int NT>
constexpr int rx_group_bits() { return NT == 256 ? 3 : 4; }
template <int NT>
constexpr int batch_min_blocks() { return NT == 512 ? 1 : 3; }

// Rx(2 beta) on every local bit set in `bits`, in ascending order, a group of
// bits per shared-memory round trip.
template <int NT>
__device__ void rx_bits(double2* s, int m, uint32_t bits, double cb, double sb) {
  constexpr int KM = rx_group_bits<NT>();
  while (bits) {
    uint32_t gp = 0;
    int k = 0;
    while (bits && k < KM) {
      gp |= (uint32_t)(__ffs(bits) - 1) << (8 * k++);
      bits &= bits - 1;
    }
    __syncthreads();
    if constexpr (KM == 4) {
      if (k == 4) { rx_group<NT, 4>(s, m, gp, cb, sb); continue; }
    }
    switch (k) {
      case 3: rx_group<NT, 3>(s, m, gp, cb, sb); break;
      case 2: rx_group<NT, 2>(s, m, gp, cb, sb); break;
      default: rx_group<NT, 1>(s, m, gp, cb, sb); break;
    }
  }
}

// 16-byte asynchronous copy global -> shared (through L2 only: the data was
// written by other CTAs of the same launch).
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n cp.async.wait_group 0;" ::: "memory");
}

template <int NT>
__global__ void __launch_bounds__(NT, batch_min_blocks<NT>()) k_batch_qaoa(QArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* s = reinterpret_cast<double2*>(smraw);
  double2* tab = s + (1u << a.tile);                             // phase table (<= 65 entries)
  uint64_t* em = reinterpret_cast<uint64_t*>(tab + KQ_MAX_EDGES + 1);
  double* red = reinterpret_cast<double*>(em + KQ_MAX_EDGES);     // 32 doubles
  uint8_t* cutb = reinterpret_cast<uint8_t*>(red + 32);           // cut(x) per amplitude (whole instance / tile)
  static_assert((16 * (KQ_MAX_EDGES + 1) + 8 * KQ_MAX_EDGES + 8 * 32) % 16 == 0, "cut bytes 16-byte aligned");
  __shared__ int item_sh;
  const int T = a.tile;
  for (;;) {
    if (threadIdx.x == 0) item_sh = (int)atomicAdd(a.next, 1u);
    __syncthreads();
    const int it = item_sh;
    __syncthreads();
    if (it >= a.nitems) break;
    const QItem w = a.items[it];
    const QInst I = a.inst[w.inst];
    for (int e = threadIdx.x; e < I.ne; e += NT) em[e] = a.emask[I.edge_off + e];
    const int n = I.n;
    if (w.pass < 0) {
      // ---- whole instance in shared memory
      const uint32_t N = 1u << n;
      const double amp0 = 1.0 / sqrt((double)N);
      __syncthreads();  // edge masks in
      // cut(x) depends on x only: computed once, read by every layer and <C>
      for (uint32_t i = threadIdx.x; i < N; i += NT) {
        s[sw(i)] = make_double2(amp0, 0.0);
        cutb[i] = (uint8_t)cut_of(i, em, I.ne);
      }
      for (int l = 0; l < I.p; l++) {
        __syncthreads();
        fill_phase<NT>(tab, a.gamma[w.inst * I.p + l], I.ne);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < N; i += NT) {
          const double2 ph = tab[cutb[i]];
          const double2 v = s[sw(i)];
          s[sw(i)] = make_double2(fma(ph.x, v.x, -ph.y * v.y), fma(ph.x, v.y, ph.y * v.x));
        }
        double sb, cb;
        sincos(a.beta[w.inst * I.p + l], &sb, &cb);
        rx_bits<NT>(s, n, (1u << n) - 1u, cb, sb);
      }
      __syncthreads();
      double acc = 0.0;
      for (uint32_t i = threadIdx.x; i < N; i += NT) {
        const double2 v = s[sw(i)];
        acc += (v.x * v.x + v.y * v.y) * (double)cutb[i];
      }
      acc = block_sum<NT>(acc, red);
      if (threadIdx.x == 0) a.part[I.part_off] = acc;
      __syncthreads();
      continue;
    }
    // ---- one tile of one pass of a wide instance
    const int layer = w.pass >> 1;
    const bool passA = (w.pass & 1) == 0;
    // tile bits: pass A = qubits 0..T-1; pass B = low (T - (n - T)) qubits + qubits T..n-1
    const int nhigh = n - T;               // qubits >= T
    const int lowB = T - nhigh;            // low qubits kept in pass-B tiles
    if (w.pass > 0) {
      // wait until every tile of the previous pass has been written back; a
      // wait that ran out anywhere (status set) ends every later wait at once
      const unsigned int need = (unsigned int)w.pass * (unsigned int)I.ntiles;
      if (threadIdx.x == 0) {
        volatile unsigned int* d = a.done + w.inst;
        volatile int* st = a.status;
        uint32_t spins = 0;
        while (*d < need) {
          if (*st != 0) break;
          if (++spins > a.spin_limit) { atomicExch(a.status, (int)KET_ERR_TIMEOUT); break; }
          __nanosleep(200);
        }
        __threadfence();
        item_sh = *st;
      }
      __syncthreads();
      const bool failed = item_sh != 0;
      __syncthreads();
      if (failed) {
        // the call reports the timeout; drain the queue without the tile's work
        if (threadIdx.x == 0) atomicAdd(a.done + w.inst, 1u);
        continue;
      }
    }
    double2* g = a.work + I.state;
    // global index of tile element i
    auto gidx = [&](uint32_t i) -> uint64_t {
      if (passA) return ((uint64_t)w.tile << T) | i;
      const uint64_t lo = i & ((1u << lowB) - 1);
      const uint64_t hi = (uint64_t)(i >> lowB) << T;                 // qubits T..n-1
      const uint64_t mid = (uint64_t)w.tile << lowB;                  // qubits lowB..T-1 from the tile id
      return hi | mid | lo;
    };
    const uint32_t TN = 1u << T;
    if (w.pass == 0) {
      const double amp0 = 1.0 / sqrt((double)(uint64_t(1) << n));
      for (uint32_t i = threadIdx.x; i < TN; i += NT) s[sw(i)] = make_double2(amp0, 0.0);
    } else {
      // the whole tile in flight at once, straight into shared memory, and
      // for pass A of later layers its cut values (kept by layer 0; pass-A
      // tiles are contiguous)
      for (uint32_t i = threadIdx.x; i < TN; i += NT) cp_async16(s + sw(i), g + gidx(i));
      if (passA && layer > 0) {
        const uint8_t* cw = a.cutw + I.cut + ((uint64_t)w.tile << T);
        for (uint32_t i = 16 * threadIdx.x; i < TN; i += 16 * NT) cp_async16(cutb + i, cw + i);
      }
      cp_async_wait_all();
    }
    double sb, cb;
    sincos(a.beta[w.inst * I.p + layer], &sb, &cb);
    if (passA) {
      __syncthreads();
      fill_phase<NT>(tab, a.gamma[w.inst * I.p + layer], I.ne);
      __syncthreads();
      // pass A tiles are contiguous: layer 0 computes cut(x) and keeps it,
      // later layers copied it into shared memory with the tile
      uint8_t* cw = a.cutw + I.cut;
      for (uint32_t i = threadIdx.x; i < TN; i += NT) {
        const uint64_t x = gidx(i);
        int cx;
        if (layer == 0) {
          cx = cut_of(x, em, I.ne);
          cw[x] = (uint8_t)cx;
        } else {
          cx = cutb[i];
        }
        const double2 ph = tab[cx];
        const double2 v = s[sw(i)];
        s[sw(i)] = make_double2(fma(ph.x, v.x, -ph.y * v.y), fma(ph.x, v.y, ph.y * v.x));
      }
      rx_bits<NT>(s, T, (1u << T) - 1u, cb, sb);
    } else {
      rx_bits<NT>(s, T, ((1u << T) - 1u) & ~((1u << lowB) - 1u), cb, sb);
    }
    __syncthreads();
    const bool last = w.pass == 2 * I.p - 1;
    if (last) {
      double acc = 0.0;
      for (uint32_t i = threadIdx.x; i < TN; i += NT) {
        const double2 v = s[sw(i)];
        acc += (v.x * v.x + v.y * v.y) * (double)cut_of(gidx(i), em, I.ne);
      }
      acc = block_sum<NT>(acc, red);
      if (threadIdx.x == 0) a.part[I.part_off + w.tile] = acc;
    } else {
      for (uint32_t i = threadIdx.x; i < TN; i += NT) g[gidx(i)] = s[sw(i)];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(a.done + w.inst, 1u);
    }
    __syncthreads();
  }
}

__global__ void k_qaoa_reduce(const QInst* inst, int ninst, const double* part, double* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ninst) return;
  const QInst I = inst[i];
  double acc = 0.0;
  for (int t = 0; t < I.ntiles; t++) acc += part[I.part_off + t];
  out[i] = acc;
}

// Test hook (ket_debug_batch_hook): drop one work item from the queue and
// shorten the waits, so that the tiles depending on it time out.
int g_drop_item = -1;
uint32_t g_spin_limit = 1u << 24;

}  // namespace
}  // namespace ket

using namespace ket;

// Launch the persistent batch kernel with NT threads per CTA (every CTA
// resident at once) and its fixed-order reduction, captured in a CUDA graph
// when use_graph is set.
template <int NT>
static cudaError_t run_batch(ket_ctx* c, const QArgs& a, size_t smem, int ninst, double* dout, int use_graph) {
  // the shared-memory limit is a per-device attribute of the kernel
  static std::atomic<uint64_t> attr_set{0};
  const uint64_t bit = uint64_t(1) << (c->device & 63);
  if (!(attr_set.load() & bit)) {
    const size_t smax = (17u << 12) + 16 * (KQ_MAX_EDGES + 1) + 8 * KQ_MAX_EDGES + 8 * 32;
    cudaError_t e = cudaFuncSetAttribute(k_batch_qaoa<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    if (e != cudaSuccess) return e;
    attr_set.fetch_or(bit);
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_qaoa<NT>, NT, smem);
  per_sm = std::max(1, per_sm);
  const int grid = num_sms() * per_sm;
  auto record = [&]() -> cudaError_t {
    cudaMemsetAsync(a.next, 0, 4 * ((size_t)ninst + 2), c->stream);
    k_batch_qaoa<NT><<<grid, NT, smem, c->stream>>>(a);
    k_qaoa_reduce<<<(ninst + 127) / 128, 128, 0, c->stream>>>(a.inst, ninst, a.part, dout);
    return cudaGetLastError();
  };
  if (!use_graph) return record();
  // A batch of the same shape reuses the executable graph: its inputs were
  // re-uploaded to the same addresses, so only a changed launch (sizes,
  // buffers, shape) is captured and instantiated again.
  uint64_t key = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t nb) {
    for (size_t i = 0; i < nb; i++) key = (key ^ ((const unsigned char*)p)[i]) * 1099511628211ull;
  };
  const int nt = NT;
  mix(&a, sizeof(a));
  mix(&smem, sizeof(smem));
  mix(&ninst, sizeof(ninst));
  mix(&dout, sizeof(dout));
  mix(&nt, sizeof(nt));
  mix(&grid, sizeof(grid));
  if (c->graph_exec && c->graph_key == key) return cudaGraphLaunch(c->graph_exec, c->stream);
  cudaGraph_t graph;
  cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  e = record();
  cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
  if (e != cudaSuccess) return e;
  if (e2 != cudaSuccess) return e2;
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  c->graph_key = 0;
  e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return e;
  c->graph_key = key;
  return cudaGraphLaunch(c->graph_exec, c->stream);
}

extern "C" int ket_batch_config(ket_ctx* c, int block_threads, int tile_bits) {
  if (!c) return fail(KET_ERR_TYPE, "null context");
  if (block_threads == 0) block_threads = 256;
  if (tile_bits == 0) tile_bits = 12;
  if (block_threads != 128 && block_threads != 256 && block_threads != 512)
    return fail(KET_ERR_TYPE, "block_threads must be 128, 256 or 512");
  if (tile_bits != 11 && tile_bits != 12) return fail(KET_ERR_TYPE, "tile_bits must be 11 or 12");
  c->batch_threads = block_threads;
  c->batch_tile = tile_bits;
  return KET_OK;
}

extern "C" int ket_debug_batch_hook(int drop_item, uint32_t spin_limit) {
  g_drop_item = drop_item;
  g_spin_limit = spin_limit ? spin_limit : (1u << 24);
  return KET_OK;
}

extern "C" int ket_batch_qaoa(ket_ctx* c, int ninst, const int* n, const int* ne, const int64_t* eoff,
                              const int* edges, int p, const double* gamma, const double* beta, int use_graph,
                              double* out) {
  if (!c || (ninst > 0 && (!n || !ne || !eoff || !edges || !gamma || !beta || !out)))
    return fail(KET_ERR_TYPE, "null argument");
  if (ninst < 0 || p < 0 || p > KQ_MAX_P) return fail(KET_ERR_TYPE, "bad instance count or layer count");
  if (ninst == 0) return KET_OK;
  cudaSetDevice(c->device);
  const int T = c->batch_tile;
  std::vector<QInst> inst(ninst);
  std::vector<uint64_t> masks;
  int64_t work = 0, parts = 0, nedges = 0;
  for (int i = 0; i < ninst; i++) {
    if (n[i] < 1 || n[i] > 30) return fail(KET_ERR_RANGE, "instance qubit count out of range (1..30)");
    if (ne[i] < 0 || ne[i] > KQ_MAX_EDGES) return fail(KET_ERR_TYPE, "instance edge count out of range (0..64)");
    if (n[i] > T && n[i] - T > T)
      return fail(KET_ERR_UNSUPPORTED, "instance wider than twice the tile width (" + std::to_string(2 * T) + " qubits)");
    QInst& I = inst[i];
    I.n = n[i];
    I.ne = ne[i];
    I.p = p;
    I.edge_off = (int64_t)masks.size();
    for (int e = 0; e < ne[i]; e++) {
      int u = edges[2 * (eoff[i] + e)], v = edges[2 * (eoff[i] + e) + 1];
      if (u < 0 || v < 0 || u >= n[i] || v >= n[i]) return fail(KET_ERR_RANGE, "edge endpoint out of range");
      if (u == v) return fail(KET_ERR_TYPE, "self-loop edge");
      masks.push_back((uint64_t(1) << u) | (uint64_t(1) << v));
    }
    nedges += ne[i];
    const bool split = I.n > T && p > 0;
    I.ntiles = split ? (1 << (I.n - T)) : 1;
    I.state = split ? work : 0;
    I.cut = split ? work : 0;  // the cut bytes sit at the same index offset in their own area
    if (split) work += int64_t(1) << I.n;
    I.part_off = parts;
    parts += I.ntiles;
  }
  // Work order: wide instances pass by pass (largest first, interleaved so a
  // tile rarely waits), then the shared-memory instances (largest first).
  std::vector<int> order(ninst);
  for (int i = 0; i < ninst; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return inst[x].n > inst[y].n; });
  std::vector<QItem> items;
  for (int k = 0; k < 2 * p; k++)
    for (int i : order) {
      const QInst& I = inst[i];
      if (!(I.n > T && p > 0)) continue;
      for (int t = 0; t < I.ntiles; t++) items.push_back(QItem{i, k, t});
    }
  for (int i : order)
    if (!(inst[i].n > T && p > 0)) items.push_back(QItem{i, -1, 0});
  if (g_drop_item >= 0 && (size_t)g_drop_item < items.size()) items.erase(items.begin() + g_drop_item);
  // device buffers in the second scratch pool
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  size_t off_inst = 0, off_items = al(sizeof(QInst) * ninst), off_mask = off_items + al(sizeof(QItem) * items.size());
  size_t off_g = off_mask + al(8 * std::max<size_t>(masks.size(), 1));
  size_t off_b = off_g + al(8 * (size_t)ninst * p + 8);
  size_t off_part = off_b + al(8 * (size_t)ninst * p + 8);
  size_t off_out = off_part + al(8 * (size_t)parts);
  size_t off_cnt = off_out + al(8 * (size_t)ninst);
  size_t off_work = off_cnt + al(4 * ((size_t)ninst + 2));
  size_t off_cut = off_work + al(16 * (size_t)work);
  size_t total = off_cut + (size_t)work + 256;
  if (c->scratch2_bytes < total) {
    int rc = ctx_wait(c);
    if (rc) return rc;
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    c->graph_key = 0;
    if (c->scratch2) cudaFree(c->scratch2);
    c->scratch2 = nullptr;
    c->scratch2_bytes = 0;
    rc = dev_alloc(&c->scratch2, total);
    if (rc) return rc;
    c->scratch2_bytes = total;
  }
  char* base = (char*)c->scratch2;
  std::vector<double> gv(gamma, gamma + (size_t)ninst * p), bv(beta, beta + (size_t)ninst * p);
  cudaMemcpyAsync(base + off_inst, inst.data(), sizeof(QInst) * ninst, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(base + off_items, items.data(), sizeof(QItem) * items.size(), cudaMemcpyHostToDevice, c->stream);
  if (!masks.empty()) cudaMemcpyAsync(base + off_mask, masks.data(), 8 * masks.size(), cudaMemcpyHostToDevice, c->stream);
  if (p > 0) {
    cudaMemcpyAsync(base + off_g, gv.data(), 8 * gv.size(), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(base + off_b, bv.data(), 8 * bv.size(), cudaMemcpyHostToDevice, c->stream);
  }
  c->h2d_bytes += sizeof(QInst) * ninst + sizeof(QItem) * items.size() + 8 * masks.size() + 16 * gv.size();
  QArgs a;
  a.inst = (const QInst*)(base + off_inst);
  a.items = (const QItem*)(base + off_items);
  a.emask = (const uint64_t*)(base + off_mask);
  a.gamma = (const double*)(base + off_g);
  a.beta = (const double*)(base + off_b);
  a.part = (double*)(base + off_part);
  a.next = (unsigned int*)(base + off_cnt);
  a.done = a.next + 2;
  a.status = c->d_status;
  a.spin_limit = g_spin_limit;
  a.work = (double2*)(base + off_work);
  a.cutw = (uint8_t*)(base + off_cut);
  a.nitems = (int)items.size();
  a.tile = T;
  const size_t smem = (17u << T) + 16 * (KQ_MAX_EDGES + 1) + 8 * KQ_MAX_EDGES + 8 * 32;  // state, table, masks, sums, cuts
  double* dout = (double*)(base + off_out);
  prof_begin(c);
  cudaError_t e;
  switch (c->batch_threads) {
    case 128: e = run_batch<128>(c, a, smem, ninst, dout, use_graph); break;
    case 512: e = run_batch<512>(c, a, smem, ninst, dout, use_graph); break;
    default: e = run_batch<256>(c, a, smem, ninst, dout, use_graph); break;
  }
  prof_end(c, PK_BATCH);
  c->launches += 1;  // the reduction (prof_end counted the batch kernel)
  if (e != cudaSuccess) return cuda_fail(e, "batch launch");
  e = cudaMemcpyAsync(out, dout, 8 * (size_t)ninst, cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(out)");
  c->d2h_bytes += 8 * (size_t)ninst;
  int rc = ctx_wait(c);
  if (rc) return rc;
  return check_status(c);
}
