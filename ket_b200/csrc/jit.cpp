// jit.cpp -- register-tiled pass kernels compiled at run time, one per program shape.
//
// The interpreter k_fused2 pays, on every op of every tile, an op fetch, a
// dispatch and, for X and CNOT on register bits, register moves.  This file
// writes, for the program of one pass, a kernel with one compile-time step per
// op (jit_ops.cuh) and compiles it with NVRTC for sm_100a.  A kernel depends
// only on the program's shape -- each op's code, pruning flag and controls --
// while the data (matrices, layouts, qubits, masks) stays in the op records
// the interpreter reads, so the cache (keyed by shape) serves every circuit
// and every parameter set with the same structure.
//
// Policy (ket_exec_opts.specialize):
//  -1   interpreter only;
//   1   compile what is missing, waiting for it, then run compiled kernels;
//   0   (default) run compiled kernels that are ready (from earlier runs or
//       ket_jit_compile); passes of states of 26 qubits or more whose kernel
//       is missing run on the interpreter and queue the compile on background
//       threads, so a repeated circuit speeds up without a first call that
//       waits for the compiler.
//
// NVRTC is loaded with dlopen on first use and the driver entry points come
// from the runtime (cudaGetDriverEntryPoint): the library links neither.
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda.h>

#include "launch.h"
#include "jit.h"
#include "jit_sources.inc"  // kJitHeaders: the device headers as strings (written by build.py)
#include "jit_ops.cuh"

namespace ket {
namespace {

// ---------------------------------------------------------------- NVRTC
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
  bool ok = false;
  std::string err;
  int major = 0, minor = 0;
  nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*);
  nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*cubin)(nvrtcProgram_t, char*);
  nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*log)(nvrtcProgram_t, char*);
  nvrtcResult_t (*destroy)(nvrtcProgram_t*);
};

Nvrtc load_nvrtc() {
  Nvrtc n;
  // The toolkit's NVRTC first, by path: after `import torch` the soname
  // resolves to torch's bundled (possibly older) copy already in the process.
  const char* names[] = {"/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so.12", "libnvrtc.so"};
  void* h = nullptr;
  for (const char* nm : names)
    if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
  if (!h) {
    n.err = "NVRTC (libnvrtc.so.12) not found";
    return n;
  }
  auto sym = [&](const char* s) { return dlsym(h, s); };
  n.create = (decltype(n.create))sym("nvrtcCreateProgram");
  n.compile = (decltype(n.compile))sym("nvrtcCompileProgram");
  n.cubin_size = (decltype(n.cubin_size))sym("nvrtcGetCUBINSize");
  n.cubin = (decltype(n.cubin))sym("nvrtcGetCUBIN");
  n.log_size = (decltype(n.log_size))sym("nvrtcGetProgramLogSize");
  n.log = (decltype(n.log))sym("nvrtcGetProgramLog");
  n.destroy = (decltype(n.destroy))sym("nvrtcDestroyProgram");
  n.ok = n.create && n.compile && n.cubin_size && n.cubin && n.log_size && n.log && n.destroy;
  if (!n.ok) n.err = "NVRTC is missing an entry point";
  if (auto ver = (nvrtcResult_t(*)(int*, int*))sym("nvrtcVersion")) ver(&n.major, &n.minor);
  return n;
}

Nvrtc& nvrtc() {
  static Nvrtc n = load_nvrtc();
  return n;
}

// Compile one kernel source to an sm_100a cubin; false and a log on failure.
bool compile_cubin(const std::string& src, std::vector<char>& cubin, std::string& log) {
  Nvrtc& N = nvrtc();
  if (!N.ok) {
    log = N.err;
    return false;
  }
  std::vector<const char*> hs, hn;
  for (const JitHeader& h : kJitHeaders) {
    hn.push_back(h.name);
    hs.push_back(h.text);
  }
  nvrtcProgram_t prog = nullptr;
  if (N.create(&prog, src.c_str(), "ket_pass.cu", (int)hs.size(), hs.data(), hn.data()) != 0) {
    log = "nvrtcCreateProgram failed";
    return false;
  }
  std::vector<const char*> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "-DNDEBUG"};
  // three-input min.f32 needs the PTX of CUDA 12.9 or later
  if (N.major < 12 || (N.major == 12 && N.minor < 9)) opts.push_back("-DKET_NO_MIN3");
  if (getenv("KET_JIT_VERBOSE")) opts.push_back("-Xptxas=-v");  // register and spill report in the log
  const int rc = N.compile(prog, (int)opts.size(), opts.data());
  size_t ls = 0;
  N.log_size(prog, &ls);
  if (ls > 1) {
    log.resize(ls);
    N.log(prog, &log[0]);
  }
  bool ok = rc == 0;
  if (ok) {
    size_t cs = 0;
    ok = N.cubin_size(prog, &cs) == 0 && cs > 0;
    if (ok) {
      cubin.resize(cs);
      ok = N.cubin(prog, cubin.data()) == 0;
    }
  }
  N.destroy(&prog);
  return ok;
}

// ---------------------------------------------------------------- driver entry points
struct Driver {
  bool ok = false;
  CUresult (*load)(CUmodule*, const void*);
  CUresult (*get)(CUfunction*, CUmodule, const char*);
  CUresult (*attr)(CUfunction, CUfunction_attribute, int);
  CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                     void**, void**);
  CUresult (*global)(CUdeviceptr*, size_t*, CUmodule, const char*);
  CUresult (*copy2d)(const CUDA_MEMCPY2D*, CUstream);
  CUresult (*encode)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                     const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                     CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
};

Driver& driver() {
  static Driver d = [] {
    Driver r;
    void* p[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const char* names[7] = {"cuModuleLoadData", "cuModuleGetFunction", "cuFuncSetAttribute", "cuLaunchKernel",
                            "cuModuleGetGlobal", "cuMemcpy2DAsync", "cuTensorMapEncodeTiled"};
    bool ok = true;
    for (int i = 0; i < 7; i++) {
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPoint(names[i], &p[i], cudaEnableDefault, &q) != cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !p[i])
        ok = false;
    }
    r.load = (decltype(r.load))p[0];
    r.get = (decltype(r.get))p[1];
    r.attr = (decltype(r.attr))p[2];
    r.launch = (decltype(r.launch))p[3];
    r.global = (decltype(r.global))p[4];
    r.copy2d = (decltype(r.copy2d))p[5];
    r.encode = (decltype(r.encode))p[6];
    r.ok = ok;
    return r;
  }();
  return d;
}

// ---------------------------------------------------------------- source
const char* real_name(int precision) { return precision == KET_C64 ? "float" : "double"; }

// The lane or thread-id bit that lane ops and thread diagonals take as a
// template argument (0 for other ops).
int static_lane(const FOp& f) {
  return (f.opc >= OC_MAT1L && f.opc < OC_MAT1L + 3) || f.opc == OC_X1L || f.opc == OC_DIAGT ? f.a : 0;
}

// Stages of the staged form: one per tile group and one in flight (64 KB
// each at complex128, 32 KB at complex64).
int stage_count(int) { return 3; }

// A program with adjoint probes: its kernel keeps per-CTA probe sums.
bool has_probes(const FOp* prog, int nops) {
  for (int k = 0; k < nops; k++)
    if (prog[k].type != FO_CONT && prog[k].opc >= OC_GRADM && prog[k].opc <= OC_GRADM2) return true;
  return false;
}

std::string make_source(const FOp* prog, int nops, int precision, int NR, bool staged) {
  const char* R = real_name(precision);
  const int NT = 32 << (7 - NR);
  std::string s;
  s.reserve(300 + 96 * (size_t)nops);
  if (staged) s += "#define KET_STAGED_THREADS " + std::to_string(NT) + "\n";
  s += "#include \"jit_ops.cuh\"\n";
  s += "__constant__ ket::jit::COp c_ops[" + std::to_string(nops > 0 ? nops : 1) + "];\n";
  if (staged) {
    s += "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(2 * NT) +
         ", 1) ket_pass(const ket::Pass2Args a, const __grid_constant__ ket::jit::TMap tm) {\n";
  } else {
    s += "extern \"C\" __global__ void __launch_bounds__(" + std::to_string(NT) +
         (has_probes(prog, nops) ? ", 2) ket_probe_pass(const ket::Pass2Args a) {\n"
                                 : ", 2) ket_pass(const ket::Pass2Args a) {\n");
  }
  s += "  using namespace ket;\n";
  s += "  const FOp* g = a.ops;\n";
  if (staged)
    s += std::string("  jit::run_tiles_staged<") + R + ", " + std::to_string(NR) + ", " +
         std::to_string(stage_count(precision)) + ">(a, &tm, [&](cpx<" + R + "> (&x)[" + std::to_string(1 << NR) +
         "], SLay<" + std::to_string(NR) + ">& sl, jit::Tile& t) {\n";
  else
    s += std::string("  jit::run_tiles<") + R + ", " + std::to_string(NR) +
         (has_probes(prog, nops) ? ", true" : ", false") + ">(a, [&](cpx<" + R + "> (&x)[" + std::to_string(1 << NR) +
         "], SLay<" + std::to_string(NR) + ">& sl, jit::Tile& t) {\n";
  for (int k = 0; k < nops; k++) {
    const FOp& f = prog[k];
    if (f.type == FO_CONT || f.opc == OC_NOP) continue;
    const unsigned fl = f.flags & (FOF_PRUNE | FOF_D0ONE | FOF_SW);
    s += std::string("    jit::step<") + R + ", " + std::to_string(NR) + ", " + std::to_string((int)f.opc) + ", " +
         std::to_string(fl) + ", " + std::to_string((int)f.creg) + ", " + std::to_string((unsigned)f.cthr) + "u, " +
         (f.cctx ? "true" : "false") + ", " + std::to_string(static_lane(f)) + ">(x, sl, c_ops[" + std::to_string(k) +
         "], g + " + std::to_string(k) + ", t);\n";
  }
  s += "  });\n}\n";
  return s;
}

// The shape of a program: what selects code in make_source.
std::string shape_key(const FOp* prog, int nops, int precision, int nreg, bool staged) {
  std::string k = std::string(precision == KET_C64 ? "f" : "d") + std::to_string(nreg) + (staged ? "s" : "r");
  k.reserve(8 * (size_t)nops + 1);
  for (int i = 0; i < nops; i++) {
    const FOp& f = prog[i];
    if (f.type == FO_CONT || f.opc == OC_NOP) {
      k += '.';
      continue;
    }
    const unsigned fl = f.flags & (FOF_PRUNE | FOF_D0ONE | FOF_SW);
    char buf[32];
    snprintf(buf, sizeof buf, "%x,%x,%x,%x,%d,%d;", (unsigned)f.opc, fl, (unsigned)f.creg, (unsigned)f.cthr,
             f.cctx ? 1 : 0, static_lane(f));
    k += buf;
  }
  return k;
}

// A kernel's state: queued / compiling / compiled (cubin) / failed, and its
// module instances.
struct Entry {
  enum { QUEUED, BUSY, READY, FAILED } st = QUEUED;
  bool staged = false;
  bool grad = false;  // adjoint probe pass (per-CTA probe sums after the exchange buffer)
  std::string src, log;
  std::vector<char> cubin;
  // (device, stream) -> the kernel loaded for it: each stream owns a module
  // instance, because a launch fills the module's constant array
  std::map<std::pair<int, void*>, JitFn> fn;
};

struct Cache {
  std::mutex mu;
  std::condition_variable cv;       // a compile finished
  std::condition_variable work;     // a job was queued
  std::unordered_map<std::string, Entry> map;
  std::deque<std::string> queue;
  std::vector<std::thread> pool;
  bool stop = false;
  int busy = 0;
  int64_t compiled = 0, failed = 0, launches = 0;
  double compile_s = 0;

  ~Cache() {
    {
      std::lock_guard<std::mutex> g(mu);
      stop = true;
      queue.clear();
    }
    work.notify_all();
    for (auto& t : pool) t.join();
  }

  void start_pool() {  // under mu
    if (!pool.empty()) return;
    unsigned n = std::thread::hardware_concurrency();
    n = n < 2 ? 2 : (n > 32 ? 32 : n);
    for (unsigned i = 0; i < n; i++) pool.emplace_back([this] { worker(); });
  }

  void worker() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      work.wait(lk, [this] { return stop || !queue.empty(); });
      if (stop) return;
      const std::string key = queue.front();
      queue.pop_front();
      Entry& e = map[key];
      if (e.st != Entry::QUEUED) continue;
      e.st = Entry::BUSY;
      busy++;
      const std::string src = e.src;
      lk.unlock();
      std::vector<char> cubin;
      std::string log;
      const auto t0 = std::chrono::steady_clock::now();
      const bool ok = compile_cubin(src, cubin, log);
      const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      lk.lock();
      Entry& e2 = map[key];
      e2.st = ok ? Entry::READY : Entry::FAILED;
      e2.cubin.swap(cubin);
      e2.log.swap(log);
      busy--;
      compile_s += dt;
      (ok ? compiled : failed)++;
      cv.notify_all();
    }
  }
};

Cache& cache() {
  // NVRTC is opened before the cache exists, so the cache (and its threads) is
  // torn down before NVRTC's own statics at exit
  nvrtc();
  static Cache c;
  return c;
}

}  // namespace

namespace {

// Queue the kernels of passes that are not known yet (under C.mu); keys[i] is
// the shape of pass i, empty for a pass without a kernel, or without a known
// one on a state below min_qubits.
std::vector<std::string> enqueue(Cache& C, const std::vector<JitPass>& passes, int precision, int min_qubits) {
  std::vector<std::string> keys(passes.size());
  bool queued = false;
  for (size_t i = 0; i < passes.size(); i++) {
    const JitPass& p = passes[i];
    // the constant op array holds at most 64 KB (512 records)
    if (!p.prog || (size_t)p.nops * sizeof(jit::COp) > 60000) continue;
    keys[i] = shape_key(p.prog, p.nops, precision, p.nreg, p.staged);
    if (C.map.find(keys[i]) == C.map.end()) {
      // below min_qubits a ready kernel is used but none is compiled
      if (p.nqubits < min_qubits) {
        keys[i].clear();
        continue;
      }
      // a process compiles at most KET_JIT_MAX_KERNELS shapes (modules stay
      // loaded); beyond that new shapes run on the interpreter
      if (C.map.size() >= KET_JIT_MAX_KERNELS) {
        keys[i].clear();
        continue;
      }
      Entry& e = C.map[keys[i]];
      e.src = make_source(p.prog, p.nops, precision, p.nreg, p.staged);
      e.staged = p.staged;
      e.grad = !p.staged && has_probes(p.prog, p.nops);
      if (const char* dir = getenv("KET_JIT_DUMP")) {  // kernel sources, for inspection
        const std::string path = std::string(dir) + "/ket_pass_" + std::to_string(C.map.size()) + ".cu";
        if (FILE* fp = fopen(path.c_str(), "w")) {
          fputs(e.src.c_str(), fp);
          // the layouts (role -> tile bit): the load layout, then each exchange's
          auto lay = [&](const char* what, int k, const uint8_t* pos) {
            fprintf(fp, "// %s %d:", what, k);
            for (int r = 0; r < KET_T2_BITS; r++) fprintf(fp, " %d", pos[r]);
            fputc('\n', fp);
          };
          if (p.load_pos) lay("load", -1, p.load_pos);
          for (int k = 0; k < p.nops; k++)
            if (p.prog[k].type == FO_EXCH) lay("exch", k, p.prog[k].pos);
          fclose(fp);
        }
      }
      C.queue.push_back(keys[i]);
      queued = true;
    }
  }
  if (queued) {
    C.start_pool();
    C.work.notify_all();
  }
  return keys;
}

// Wait until every listed kernel is compiled; false and its log if one failed.
bool wait_keys(Cache& C, std::unique_lock<std::mutex>& lk, const std::vector<std::string>& keys, std::string& log) {
  for (const std::string& k : keys) {
    if (k.empty()) continue;
    C.cv.wait(lk, [&] {
      const Entry& e = C.map[k];
      return e.st == Entry::READY || e.st == Entry::FAILED;
    });
    const Entry& e = C.map[k];
    if (e.st == Entry::FAILED) {
      log = e.log;
      return false;
    }
  }
  return true;
}

}  // namespace

int jit_compile(const std::vector<JitPass>& passes, int precision, int64_t* distinct, std::string& log) {
  Cache& C = cache();
  std::unique_lock<std::mutex> lk(C.mu);
  const std::vector<std::string> keys = enqueue(C, passes, precision, 0);
  if (distinct) {
    std::vector<std::string> u;
    for (const std::string& k : keys)
      if (!k.empty()) u.push_back(k);
    std::sort(u.begin(), u.end());
    *distinct = (int64_t)(std::unique(u.begin(), u.end()) - u.begin());
  }
  return wait_keys(C, lk, keys, log) ? KET_OK : KET_ERR_CUDA;
}

int jit_prepare(const std::vector<JitPass>& passes, int precision, int mode, cudaStream_t stream,
                std::vector<JitFn>& out, std::string& err) {
  out.assign(passes.size(), JitFn{});
  if (mode < 0) return KET_OK;
  if (!driver().ok) {
    if (mode == 1) return err = "driver entry points for run-time kernels are unavailable", KET_ERR_UNSUPPORTED;
    return KET_OK;
  }
  Cache& C = cache();
  std::unique_lock<std::mutex> lk(C.mu);
  const std::vector<std::string> keys = enqueue(C, passes, precision, mode == 1 ? 0 : KET_JIT_AUTO_QUBITS);
  if (mode == 1) {  // wait for every kernel this plan needs
    std::string log;
    if (!wait_keys(C, lk, keys, log)) return err = "run-time compile of a pass kernel failed: " + log, KET_ERR_CUDA;
  }
  Driver& D = driver();
  int device = 0;
  cudaGetDevice(&device);
  for (size_t i = 0; i < passes.size(); i++) {
    if (keys[i].empty()) continue;
    Entry& e = C.map[keys[i]];
    if (e.st != Entry::READY) continue;
    const std::pair<int, void*> where(device, (void*)stream);
    auto f = e.fn.find(where);
    if (f == e.fn.end()) {
      CUmodule mod;
      CUfunction fn;
      CUdeviceptr cops = 0;
      size_t cbytes = 0;
      if (D.load(&mod, e.cubin.data()) != CUDA_SUCCESS || D.get(&fn, mod, e.grad ? "ket_probe_pass" : "ket_pass") != CUDA_SUCCESS ||
          D.global(&cops, &cbytes, mod, "c_ops") != CUDA_SUCCESS) {
        if (mode == 1) return err = "loading a run-time compiled pass kernel failed", KET_ERR_CUDA;
        continue;
      }
      const int smem = pass_smem(precision, e.staged) + (e.grad ? 64 * KET_JIT_MAX_PROBES : 0);
      if (D.attr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, smem) != CUDA_SUCCESS) {
        if (mode == 1) return err = "setting the shared memory of a pass kernel failed", KET_ERR_CUDA;
        continue;
      }
      JitFn j;
      j.staged = e.staged;
      j.grad = e.grad;
      j.fn = (void*)fn;
      j.cops = (unsigned long long)cops;
      j.cops_bytes = cbytes;
      f = e.fn.emplace(where, j).first;
    }
    out[i] = f->second;
  }
  return KET_OK;
}

int tiled_nreg(int nqubits, int reg_bits) {
  if (reg_bits == 4 || reg_bits == 5) return reg_bits;
  static const int large = [] {
    const char* e = getenv("KET_JIT_NREG");
    return e && atoi(e) == 5 ? 5 : 4;
  }();
  return nqubits >= KET_JIT_AUTO_QUBITS ? large : KET_FUSED_NREG;
}

static_assert(jit::kStageTimeout == KET_ERR_TIMEOUT && jit::kStageMisaligned == KET_ERR_CUDA,
              "status words of the staged loop");
static_assert(sizeof(jit::TMap) == sizeof(CUtensorMap), "tensor map size");

unsigned jit_grid(int n) {
  return (unsigned)std::min<uint64_t>(uint64_t(1) << (n - KET_T2_BITS), (uint64_t)2 * num_sms());
}

int pass_smem(int precision, bool staged) {
  const int tile = (precision == KET_C64 ? 8 : 16) << KET_T2_BITS;
  return staged ? stage_count(precision) * tile + 16 * stage_count(precision) : tile;
}

namespace {
int64_t g_stage_drop = -1;  // ket_debug_stage_drop

// The staged form's tensor map over the state (see jit_ops.cuh): rank 2,
// {64 reals of a row of 2^5 amplitudes, rows}, one row per box.
bool encode_tile_map(const Pass2Args& a, int precision, jit::TMap& out) {
  const bool c64 = precision == KET_C64;
  const uint64_t asz = c64 ? 8 : 16;
  CUtensorMap m;
  const CUtensorMapDataType dt = c64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const cuuint32_t es[2] = {1, 1};
  const cuuint64_t dim[2] = {64, cuuint64_t(1) << (a.n - 5)};
  const cuuint64_t str[1] = {32 * asz};
  const cuuint32_t box[2] = {64, 1};
  if (driver().encode(&m, dt, 2, a.amp, dim, str, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  memcpy(&out, &m, sizeof(m));
  return true;
}
}  // namespace

void jit_debug_stage_drop(int64_t tile) { g_stage_drop = tile; }

bool use_staged(int n, int stage) {
  if (n < KET_T2_BITS) return false;
  if (stage != 0) return stage > 0;
  static const int env = getenv("KET_STAGE") ? atoi(getenv("KET_STAGE")) : 0;
  return env > 0;
}

cudaError_t jit_launch(const JitFn& f, const Pass2Args& in, int precision, cudaStream_t s) {
  Pass2Args a = in;
  fill_pass2_offsets(a, precision);
  // the ops' first 128 bytes into the kernel's constant array (stream-ordered
  // after the program's upload and the previous pass's kernel)
  if ((size_t)a.nops * sizeof(jit::COp) > f.cops_bytes) return cudaErrorInvalidValue;
  CUDA_MEMCPY2D cp;
  memset(&cp, 0, sizeof(cp));
  cp.srcMemoryType = CU_MEMORYTYPE_DEVICE;
  cp.srcDevice = (CUdeviceptr)a.ops;
  cp.srcPitch = sizeof(FOp);
  cp.dstMemoryType = CU_MEMORYTYPE_DEVICE;
  cp.dstDevice = (CUdeviceptr)f.cops;
  cp.dstPitch = sizeof(jit::COp);
  cp.WidthInBytes = sizeof(jit::COp);
  cp.Height = (size_t)a.nops;
  if (a.nops > 0 && driver().copy2d(&cp, (CUstream)s) != CUDA_SUCCESS) return cudaErrorLaunchFailure;
  const int smem = pass_smem(precision, f.staged);
  const uint64_t ntiles = uint64_t(1) << (a.n - KET_T2_BITS);
  CUresult r;
  if (f.staged) {
    // one CTA per SM: two tile groups
    jit::TMap tm;
    if (!encode_tile_map(a, precision, tm)) return cudaErrorInvalidValue;
    a.drop_tile = g_stage_drop;
    const unsigned blocks = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)num_sms());
    void* params[2] = {&a, &tm};
    r = driver().launch((CUfunction)f.fn, blocks, 1, 1, 2 * (32 << (7 - a.nreg)), 1, 1, smem, (CUstream)s, params,
                        nullptr);
  } else {
    // two CTAs per SM at either register-bit count (__launch_bounds__(NT, 2));
    // probe passes add their per-(slot, warp) sums after the exchange buffer
    if (f.grad && (a.nslots < 1 || a.nslots > KET_JIT_MAX_PROBES)) return cudaErrorInvalidValue;
    const unsigned blocks = jit_grid(a.n);
    void* params[1] = {&a};
    r = driver().launch((CUfunction)f.fn, blocks, 1, 1, 32 << (7 - a.nreg), 1, 1, smem + (f.grad ? 64 * a.nslots : 0),
                        (CUstream)s, params, nullptr);
  }
  {
    std::lock_guard<std::mutex> g(cache().mu);
    cache().launches++;
  }
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

void jit_shutdown() {
  Cache& C = cache();
  std::unique_lock<std::mutex> lk(C.mu);
  for (const std::string& k : C.queue) {
    Entry& e = C.map[k];
    if (e.st == Entry::QUEUED) {
      e.st = Entry::FAILED;
      e.log = "compile cancelled at shutdown";
    }
  }
  C.queue.clear();
  C.cv.notify_all();
  C.cv.wait(lk, [&] { return C.busy == 0; });
}

int jit_wait_all() {
  Cache& C = cache();
  std::unique_lock<std::mutex> lk(C.mu);
  C.cv.wait(lk, [&] { return C.queue.empty() && C.busy == 0; });
  return C.failed ? KET_ERR_CUDA : KET_OK;
}

void jit_stats(int64_t out[4], double* compile_s) {
  Cache& C = cache();
  std::lock_guard<std::mutex> g(C.mu);
  out[0] = (int64_t)C.map.size();
  out[1] = C.compiled;
  out[2] = C.failed;
  out[3] = C.launches;
  if (compile_s) *compile_s = C.compile_s;
}

}  // namespace ket
