// cuPoly's DGTEngine (include/cuPoly/cuda/dgt.h:106-283): the transform and the
// DGT-domain pointwise operations on raw GaussianInteger device arrays of one
// polynomial over `base`, over the C ABI (cp_dgt, cp_add, cp_mul, ...).
#ifndef DGT_H
#define DGT_H
#include <cuPoly/settings.h>

class Context;

class DGTEngine {
 public:
  static bool is_init;
  static void init() { is_init = true; }  // tables live in the engine: nothing to do
  static void destroy() { is_init = false; }

  static void execute_dgt(GaussianInteger* data, const int base, const int direction, Context* ctx);
  static void execute_add_dgt(GaussianInteger* c, const GaussianInteger* a, const GaussianInteger* b,
                              const int base, const cudaStream_t stream);
  static void execute_sub_dgt(GaussianInteger* c, const GaussianInteger* a, const GaussianInteger* b,
                              const int base, const cudaStream_t stream);
  static void execute_double_add_dgt(GaussianInteger* c1, const GaussianInteger* a1, const GaussianInteger* b1,
                                     GaussianInteger* c2, const GaussianInteger* a2, const GaussianInteger* b2,
                                     const int base, const cudaStream_t stream);
  static void execute_dr2_dgt(GaussianInteger* ct21, GaussianInteger* ct22, GaussianInteger* ct23,
                              const GaussianInteger* ct01, const GaussianInteger* ct02,
                              const GaussianInteger* ct11, const GaussianInteger* ct12, const int base,
                              const cudaStream_t stream);
  static void execute_mul_dgt_gi(GaussianInteger* c, const GaussianInteger* a, const GaussianInteger* b,
                                 const int base, const cudaStream_t stream);
  static void execute_mul_dgt_u64(GaussianInteger* c, const GaussianInteger* a, const uint64_t* b,
                                  const int base, const cudaStream_t stream);
  static void execute_muladd_dgt(GaussianInteger* d, const GaussianInteger* a, const GaussianInteger* b,
                                 const GaussianInteger* c, const int base, const cudaStream_t stream);
};
#endif
