// BFV multiplication with library-owned static scratch: the one entry point
// that never allocates device memory.
//
// Who needs it: callers that cannot call cudaMalloc on the path that
// multiplies -- a serving runtime or host framework that reserves all device
// memory up front and forbids allocation afterwards, code that must not take
// the implicit device synchronisation cudaMalloc/cudaFree can cause, or a
// plugin host that gives the library no allocator.  cp_bfv_mul needs a
// caller-provided workspace; cp_bfv_mul_noalloc uses the fixed array below
// instead.
//
// The scratch is a file-scope __device__ array of CP_NOALLOC_SCRATCH_BYTES
// (8 MiB).  It exists on a GPU once this library's device code is loaded
// there: with CUDA's default lazy module loading that happens at the first
// use of the module on that device, typically this entry point's first call,
// and then it stays until the process exits.  That first call per device is a
// warm-up: loading the module (and the 8 MiB with it) may itself allocate and
// synchronise; every later call allocates nothing.  In host code
// `g_noalloc_scratch` names a host-side stand-in, not a device address: it must
// never be passed to a kernel.  The device address is obtained with
// cudaGetSymbolAddress once per device, with that device current, on the first
// call made on that device; that first call should therefore come before any
// stream capture.  The current device must be the engine's device.
//
// All calls share the one array and it keeps whatever the last call left
// there.  Nothing in it needs to start at zero: every region the chain uses
// is written before it is read.  Calls whose executions overlap on the GPU
// (different streams, or different threads without ordering) race on the
// array and corrupt each other's results; serialise them.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/cupoly_b200.h"
#include "launch.cuh"

namespace {

constexpr size_t kScratchBytes = CP_NOALLOC_SCRATCH_BYTES;
static_assert(kScratchBytes == (size_t)8 << 20, "header and library disagree on the scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_dev_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up on first use).
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return cpoly::cuda_fail("cp_bfv_mul_noalloc: cudaGetDevice", err);
  if (dev < 0 || dev >= kMaxDevices) {
    cpoly::set_error("cp_bfv_mul_noalloc: device index out of range");
    return CP_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_dev_ptr[dev]) {
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess || !p) return cpoly::cuda_fail("cp_bfv_mul_noalloc: cudaGetSymbolAddress", err);
    g_dev_ptr[dev] = p;
  }
  *out = g_dev_ptr[dev];
  return CP_OK;
}

}  // namespace

extern "C" int cp_bfv_mul_noalloc(const cp_engine* e, void* c0, void* c1, void* c2, const void* a0, const void* a1,
                                  const void* b0, const void* b1, void* stream) {
  if (!e || !c0 || !c1 || !c2 || !a0 || !a1 || !b0 || !b1) {
    cpoly::set_error("cp_bfv_mul_noalloc: NULL argument");
    return CP_ERR_INVALID;
  }
  const size_t need = cp_workspace_bytes(e);
  if (need > kScratchBytes) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "cp_bfv_mul_noalloc: this parameter set needs %zu bytes of scratch; the static scratch holds %zu "
                  "bytes (use cp_bfv_mul with a caller workspace)",
                  need, kScratchBytes);
    cpoly::set_error(msg);
    return CP_ERR_UNSUPPORTED;
  }
  int dev = -1;
  if (cudaError_t err = cudaGetDevice(&dev)) return cpoly::cuda_fail("cp_bfv_mul_noalloc: cudaGetDevice", err);
  if (dev != e->e.device) {
    char msg[160];
    std::snprintf(msg, sizeof msg,
                  "cp_bfv_mul_noalloc: the current device (%d) is not the engine's device (%d); the static scratch "
                  "is per device",
                  dev, e->e.device);
    cpoly::set_error(msg);
    return CP_ERR_INVALID;
  }
  void* ws = nullptr;
  if (int rc = scratch_address(&ws)) return rc;
  return cp_bfv_mul(e, c0, c1, c2, a0, a1, b0, b1, ws, stream);
}
