// Launch helpers shared by the kernel files.
#pragma once
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <string>

#include "engine.cuh"

namespace cpoly {

// NVTX range for the duration of a scope: names the composite calls and the stages
// of the batched chain on a profiler timeline (header-only NVTX 3; without a tool
// attached a push / pop is a check of one function pointer).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Status codes of the C ABI (mirrored in include/cupoly_b200.h).
enum : int {
  CP_OK_ = 0,
  CP_ERR_INVALID_ = 1,
  CP_ERR_CUDA_ = 2,
  CP_ERR_UNSUPPORTED_ = 3,
  CP_ERR_OOM_ = 4,
  CP_ERR_TIMEOUT_ = 5,
};

inline int cuda_fail(const char* what, cudaError_t err = cudaGetLastError()) {
  set_error(std::string(what) + ": " + cudaGetErrorString(err));
  return CP_ERR_CUDA_;
}

inline int check_launch(const char* what) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return cuda_fail(what, err);
  return CP_OK_;
}

// Raise a kernel's dynamic shared-memory limit once per device.
template <typename K>
inline int ensure_smem(K kernel, int bytes, std::atomic<unsigned long long>& done_mask) {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ULL << (dev & 63);
  if (done_mask.load() & bit) return CP_OK_;
  cudaError_t err = cudaSuccess;
  if (bytes > 48 * 1024) err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (err == cudaSuccess)  // favour shared memory: several CTAs per SM
    err = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (err != cudaSuccess) return cuda_fail("cudaFuncSetAttribute", err);
  done_mask.fetch_or(bit);
  return CP_OK_;
}

// Kernel entry points implemented in the .cu files.
int launch_dgt(const Engine& e, void* data, int base, int npolys, long long poly_stride, bool inverse,
               cudaStream_t st);
// Out-of-place forms: forward reads `fsrc` (nullptr = in place); inverse reads
// per `isrc` (nullptr = in place).  Output always to `dst`.
int launch_dgt_ex(const Engine& e, void* dst, const void* fsrc, const InvSrc* isrc, int base, int npolys,
                  long long poly_stride, bool inverse, cudaStream_t st);
int launch_dgt_list(const Engine& e, void* data, const int* rid_list, int nlist, bool inverse, cudaStream_t st);
int launch_dgt_list_ex(const Engine& e, void* data, const void* fsrc, const InvSrc* isrc, const int* rid_list,
                       int nlist, bool inverse, cudaStream_t st);
// Residues rid_off .. rid_off + nres - 1 only (src nullptr: in place).
int launch_dgt_part(const Engine& e, void* dst, const void* src, int rid_off, int nres, int npolys,
                    long long poly_stride, bool inverse, cudaStream_t st);

}  // namespace cpoly
