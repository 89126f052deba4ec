// Declarations of the host launchers for pointwise, HPS and sampler kernels.
#pragma once
#include <cuda_runtime.h>

#include "engine.cuh"

namespace cpoly {

int pw_add(const Engine& e, void* c, const void* a, const void* b, int base, cudaStream_t st);
int pw_sub(const Engine& e, void* c, const void* a, const void* b, int base, cudaStream_t st);
int pw_double_add(const Engine& e, void* c1, const void* a1, const void* b1, void* c2, const void* a2,
                  const void* b2, int base, cudaStream_t st);
int pw_mul(const Engine& e, void* c, const void* a, const void* b, int base, cudaStream_t st, int npolys = 1);
int pw_mul_u64(const Engine& e, void* c, const void* a, const uint64_t* b, int base, cudaStream_t st);
int pw_mul_list(const Engine& e, void* c, const void* a, const void* b, const int* rid_list, int nlist,
                cudaStream_t st);
int pw_muladd(const Engine& e, void* d, const void* a, const void* b, const void* c, int base, cudaStream_t st);
// Operand pairs per dot-product launch; longer sums take several launches.
constexpr int kDotTerms = 64;
int pw_dot(const Engine& e, void* c, const void* const* a, const void* const* b, int n, int base,
           cudaStream_t st);
int pw_dot_batch(const Engine& e, void* c, const void* a, const void* b, int n, int npolys, bool b_shared, int base,
                 cudaStream_t st);
int pw_dr2(const Engine& e, void* c21, void* c22, void* c23, const void* c01, const void* c02, const void* c11,
           const void* c12, int base, cudaStream_t st, int npolys = 1);
int pw_negate(const Engine& e, void* b, const void* a, int base, cudaStream_t st);
int pw_op_by_int(const Engine& e, void* b, const void* a, int base, uint64_t x, int op, cudaStream_t st);
int pw_double_op_by_int(const Engine& e, void* b1, const void* a1, void* b2, const void* a2, int base, uint64_t x1,
                        uint64_t x2, int op, cudaStream_t st);

// HPS (coefficient domain, folded Gaussian layout)
int hps_basis_ext(const Engine& e, void* out, const void* in, bool q_to_b, int npolys, cudaStream_t st);
// prescaled inputs y_i = x_i (S/s_i)^-1 (an inverse DGT with untwist table off_untwist_pre[0])
int hps_basis_ext_pre(const Engine& e, void* out, const void* in, bool q_to_b, int npolys, cudaStream_t st);
// complex scaling and B -> Q of prescaled inputs (inverse DGTs with untwist tables
// off_untwist_pre[1] over Q and off_untwist_pre[0] over B)
int hps_scale_to_q_pre(const Engine& e, void* out_q, const void* in_q, const void* in_b, void* scratch_b, int npolys,
                       cudaStream_t st);
int hps_complex_scaling(const Engine& e, void* out_b, const void* in_q, const void* in_b, int npolys,
                        cudaStream_t st);
int hps_scale_to_q(const Engine& e, void* out_q, const void* in_q, const void* in_b, void* scratch_b, int npolys,
                   cudaStream_t st);
int hps_simple_scaling(const Engine& e, void* out_t, const void* in_q, cudaStream_t st);
int rns_xi_rho(const Engine& e, void* out, const void* in, bool rho, cudaStream_t st, int npolys = 1);

// Sampler
int sample_poly(const Engine& e, void* out, int base, int kind, uint64_t seed, uint32_t stream_id, int npolys,
                cudaStream_t st, const uint32_t* ids = nullptr);

}  // namespace cpoly
