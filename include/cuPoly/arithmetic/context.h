// cuPoly's Context (include/cuPoly/arithmetic/context.h:34-109): one CUDA
// stream plus the device scratch the poly_* calls need.  Every poly_* call
// taking this context is enqueued on its stream; coefficient I/O synchronises
// it, as in cuPoly.  Scratch is sized from the current CUDAEngine parameter
// set and regrown (after a stream synchronise) when a later set needs more.
// Like cuPoly's, a Context is not thread safe.
#ifndef CONTEXT_H
#define CONTEXT_H
#include <cuPoly/settings.h>

#include <cstddef>
#include <vector>

class Context {
 public:
  Context();
  ~Context();
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;

  cudaStream_t get_stream() { return stream; }

  // Device scratch of cp_workspace_bytes() bytes for the composite HPS calls.
  void* workspace();
  // One QB-sized polynomial of device scratch (cuPoly's d_aux_coefs).
  GaussianInteger* aux();
  // General device scratch of at least `bytes` (coefficient limbs, xi / rho outputs).
  void* scratch(size_t bytes);
  // Host staging of at least `words` 64-bit words.
  uint64_t* host_scratch(size_t words);

  GaussianInteger* d_aux_coefs = nullptr;  // valid after the first aux()

 private:
  cudaStream_t stream = nullptr;
  void* d_workspace = nullptr;
  size_t workspace_bytes = 0;
  size_t aux_bytes = 0;
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  std::vector<uint64_t> h_scratch;
  void grow(void** p, size_t* have, size_t need);
};
#endif
