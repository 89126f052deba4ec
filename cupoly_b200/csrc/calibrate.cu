// Integer-throughput calibration: the measured peak of the modular primitives
// on this GPU, used as the denominator of the integer roofline (the DGT and
// HPS kernels are bound by integer issue, not by HBM).
//
// Each thread runs 8 independent chains of the primitive for `iters`
// iterations; the grid fills every SM several times over.  Results are folded
// into one word per thread so the work cannot be optimised away.
#include "../../include/cupoly_b200.h"
#include "launch.cuh"

namespace {

using namespace cpoly;

template <int KIND>
__global__ void __launch_bounds__(256) k_calibrate(uint64_t* __restrict__ sink, int iters, uint64_t p, uint64_t w,
                                                   uint64_t ws, ModConst mc) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = (tid * 0x9E3779B97F4A7C15ULL + i * 0x632BE59BD9B4E019ULL) % p;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (KIND == 0) x[i] = shoup_mul(x[i], w, ws, p);               // constant multiply
      if (KIND == 1) x[i] = mul_mod(x[i], x[(i + 1) & 7], mc);       // data x data (pseudo-Mersenne)
      if (KIND == 2) x[i] = add_mod(x[i], x[(i + 3) & 7], p);        // modular add
      if (KIND == 3) x[i] = (uint64_t)((uint32_t)x[i] * (uint32_t)w + (uint32_t)(x[i] >> 32));  // 32-bit IMAD
    }
  }
  uint64_t acc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc ^= x[i];
  sink[tid] = acc;
}

}  // namespace

extern "C" int cp_calibrate_int(int kind, int iters, void* sink, long long nthreads, float* ms, void* stream) {
  if (kind < 0 || kind > 3 || iters <= 0 || !sink || !ms || nthreads <= 0 || nthreads % 256) {
    set_error("cp_calibrate_int: bad argument");
    return CP_ERR_INVALID;
  }
  const uint64_t p = 9223372036801560577ULL;  // the first prime of the table
  const uint64_t w = 1234567890123456789ULL % p;
  const uint64_t ws = h_shoup(w, p);
  const ModConst mc = h_modconst(p);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, st);
  const unsigned blocks = (unsigned)(nthreads / 256);
  uint64_t* s = reinterpret_cast<uint64_t*>(sink);
  switch (kind) {
    case 0: k_calibrate<0><<<blocks, 256, 0, st>>>(s, iters, p, w, ws, mc); break;
    case 1: k_calibrate<1><<<blocks, 256, 0, st>>>(s, iters, p, w, ws, mc); break;
    case 2: k_calibrate<2><<<blocks, 256, 0, st>>>(s, iters, p, w, ws, mc); break;
    default: k_calibrate<3><<<blocks, 256, 0, st>>>(s, iters, p, w, ws, mc); break;
  }
  cudaEventRecord(b, st);
  cudaError_t err = cudaEventSynchronize(b);
  if (err == cudaSuccess) err = cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (err != cudaSuccess) return cuda_fail("cp_calibrate_int", err);
  return check_launch("cp_calibrate_int");
}
