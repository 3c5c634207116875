// noalloc.cu -- ket_marginals_noalloc: marginals() for callers that cannot
// allocate device memory.
//
// Some callers must not call cudaMalloc: code running inside another
// framework's memory pool or under its allocator hooks, where an allocation
// behind the pool's back would break its accounting; and callers that only
// hand over buffers they already own (a device state from their own
// allocator and a device output array).  Every other entry point of this
// library draws its reduction scratch from a context pool that grows with
// cudaMalloc, so this one keeps its scratch in a fixed array instead:
// g_noalloc_scratch below, KET_NOALLOC_SCRATCH_BYTES (640 KiB) of device
// memory that every GPU which loads the library holds until the process
// exits.
//
// Sharing: every call on a device uses the same array and leaves the last
// call's partial sums in it.  Calls whose kernels overlap on the GPU (two
// streams, or two threads without ordering between them) race on the array
// and produce wrong results; order them on one stream.
//
// The array's address is looked up once per device and kept for the life of
// the process.  cudaDeviceReset unloads the library's device code, so this
// entry point must not be called on a device after cudaDeviceReset has run
// on it: the kept address would then point at freed memory.
#include <mutex>

#include "ctx.h"
#include "read.h"

namespace ket {
namespace {

constexpr size_t kNoallocBytes = KET_NOALLOC_SCRATCH_BYTES;
// Per-block partial sums of the marginals reduction: at most 2048 blocks x 40
// qubits doubles (marg_chunk() never makes more than 2048 blocks).
static __device__ __align__(256) double g_noalloc_scratch[kNoallocBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};  // device address of g_noalloc_scratch, per device

// Set-up, once per device, with that device current: look up the address of
// the array.  In host code g_noalloc_scratch only names the symbol; the
// address the kernels need comes from cudaGetSymbolAddress.
int scratch_for_current_device(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(KET_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return KET_OK;
}

// The caller's buffers must be device (or managed) memory of the current
// device: a host pointer, or one on another device, would fault the kernel.
// cudaPointerGetAttributes only queries; it allocates nothing.
int check_device_pointer(const void* p, int dev, const char* what) {
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the sticky query error
    return fail(KET_ERR_TYPE, std::string(what) + " is not a device pointer");
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
    return fail(KET_ERR_TYPE, std::string(what) + " is not device or managed memory");
  if (at.type == cudaMemoryTypeDevice && at.device != dev)
    return fail(KET_ERR_TYPE, std::string(what) + " lives on another device than the current one");
  return KET_OK;
}

}  // namespace
}  // namespace ket

using namespace ket;

extern "C" int ket_marginals_noalloc(const void* amp, int nqubits, int precision, double* out, void* stream) {
  if (!amp || !out) return fail(KET_ERR_TYPE, "null argument");
  if (nqubits < 1 || nqubits > KET_MAX_QUBITS) return fail(KET_ERR_RANGE, "qubit count out of range (1..40)");
  if (precision != KET_C128 && precision != KET_C64) return fail(KET_ERR_TYPE, "precision must be KET_C128 or KET_C64");
  const uint64_t N = uint64_t(1) << nqubits;
  const uint64_t nb = (N + marg_chunk(nqubits) - 1) / marg_chunk(nqubits);
  const uint64_t need = sizeof(double) * nb * (uint64_t)nqubits;
  if (need > kNoallocBytes)
    return fail(KET_ERR_RANGE, "marginals of this state need " + std::to_string(need) +
                                   " bytes of scratch, more than the fixed " + std::to_string(kNoallocBytes) +
                                   "-byte array of ket_marginals_noalloc");
  int dev = -1;
  cudaError_t ge = cudaGetDevice(&dev);
  if (ge != cudaSuccess) return cuda_fail(ge, "cudaGetDevice");
  int rc = check_device_pointer(amp, dev, "amp");
  if (!rc) rc = check_device_pointer(out, dev, "out");
  if (rc) return rc;
  void* scratch = nullptr;
  rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  // every partial the reduction reads is written by this call's first kernel,
  // so the array needs no clearing
  cudaError_t e = launch_marginals(amp, nqubits, precision, (double*)scratch, out, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "ket_marginals_noalloc launch");
  return KET_OK;
}
