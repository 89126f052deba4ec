// CKKS-mode RNS operations on the same DGT engine.
//
// Replaces cuPoly's CKKS kernels (src/cuda/cudaengine.cu:800-981 and
// 1086-1184) and their polynomial wrappers (src/arithmetic/polynomial.cu:
// 530-608, 696-800):
//  * approximate modulus raising Q_l -> B (fast_conv_Q_to_B):
//      y_j = sum_{i<=l} [x_i (Q_l/q_i)^-1]_{q_i} (Q_l/q_i) mod b_j;
//  * approximate modulus reduction QB -> Q_l (fast_conv_B_to_Q):
//      z_i = (x_i - sum_j [y_j (B/b_j)^-1]_{b_j} (B/b_j)) B^-1 mod q_i;
//  * rescale (ckks_rescale): x_i <- (x_i - x_l) q_l^-1 mod q_i, i < l;
//  * xi / rho: x_i B^-1 mod q_i and x_i B mod q_i (xi_ckks_rns_rid,
//    rho_ckks_rns_rid).
// Q_l = q_0 ... q_l; Q is the first 63-bit prime followed by primes of the
// precision bucket in descending order, so x_l < q_l < q_i for i < l.  Every
// multiply is by a constant (Shoup product with a precomputed quotient), so
// nothing here depends on the prime's form.  The definitions above are
// integer-exact; the results are the same whatever the reduction order.
#include "../../include/cupoly_b200.h"
#include "launch.cuh"

namespace cpoly {

namespace {

constexpr int kMaxCk = 24;

struct CkArgs {
  const ModConst* mc;
  const uint64_t* H;
  int N, k, kl, level;
};

// B residues of the coefficient-domain Q residues 0..level (rows of N elements).
// Polynomial blockIdx.y at strides out_stride / in_stride (elements).
__global__ void __launch_bounds__(128) k_ckks_raise(ulonglong2* __restrict__ outB, const ulonglong2* __restrict__ inQ,
                                                    CkArgs a, int o_inv, int o_inv_s, int o_m, int o_m_s,
                                                    long long out_stride, long long in_stride) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  outB += blockIdx.y * out_stride;
  inQ += blockIdx.y * in_stride;
  const int l = a.level;
  uint64_t tr[kMaxCk], ti[kMaxCk];
  for (int i = 0; i <= l; ++i) {
    const uint64_t q = a.mc[i].p;
    const ulonglong2 x = inQ[(size_t)i * a.N + j];
    const uint64_t c = __ldg(a.H + o_inv + l * a.k + i), cs = __ldg(a.H + o_inv_s + l * a.k + i);
    tr[i] = shoup_mul(x.x, c, cs, q);
    ti[i] = shoup_mul(x.y, c, cs, q);
  }
  for (int jb = 0; jb < a.kl; ++jb) {
    const uint64_t b = a.mc[a.k + jb].p;
    uint64_t ar = 0, ai = 0;
    for (int i = 0; i <= l; ++i) {
      const size_t w = ((size_t)l * a.k + i) * a.kl + jb;
      const uint64_t c = __ldg(a.H + o_m + w), cs = __ldg(a.H + o_m_s + w);
      ar = add_mod(ar, shoup_mul(tr[i], c, cs, b), b);  // tr[i] < q_i < 2^64: any input
      ai = add_mod(ai, shoup_mul(ti[i], c, cs, b), b);
    }
    outB[(size_t)jb * a.N + j] = make_ulonglong2(ar, ai);
  }
}

// Q residues 0..level of the coefficient-domain QB polynomial; higher Q rows untouched.
// Polynomial blockIdx.y at strides out_stride / in_stride (elements).
__global__ void __launch_bounds__(128) k_ckks_reduce(ulonglong2* __restrict__ outQ, const ulonglong2* __restrict__ inQB,
                                                     CkArgs a, int o_bi, int o_bi_s, int o_bq, int o_bq_s, int o_ib,
                                                     int o_ib_s, long long out_stride, long long in_stride) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  outQ += blockIdx.y * out_stride;
  inQB += blockIdx.y * in_stride;
  uint64_t sr[kMaxCk], si[kMaxCk];
  for (int jb = 0; jb < a.kl; ++jb) {
    const uint64_t b = a.mc[a.k + jb].p;
    const ulonglong2 y = inQB[(size_t)(a.k + jb) * a.N + j];
    const uint64_t c = __ldg(a.H + o_bi + jb), cs = __ldg(a.H + o_bi_s + jb);
    sr[jb] = shoup_mul(y.x, c, cs, b);
    si[jb] = shoup_mul(y.y, c, cs, b);
  }
  for (int i = 0; i <= a.level; ++i) {
    const uint64_t q = a.mc[i].p;
    uint64_t vr = 0, vi = 0;
    for (int jb = 0; jb < a.kl; ++jb) {
      const uint64_t c = __ldg(a.H + o_bq + jb * a.k + i), cs = __ldg(a.H + o_bq_s + jb * a.k + i);
      vr = add_mod(vr, shoup_mul(sr[jb], c, cs, q), q);
      vi = add_mod(vi, shoup_mul(si[jb], c, cs, q), q);
    }
    const ulonglong2 x = inQB[(size_t)i * a.N + j];
    const uint64_t c = __ldg(a.H + o_ib + i), cs = __ldg(a.H + o_ib_s + i);
    outQ[(size_t)i * a.N + j] = make_ulonglong2(shoup_mul(x.x + q - vr, c, cs, q), shoup_mul(x.y + q - vi, c, cs, q));
  }
}

// x_i <- (x_i - x_l) q_l^-1 mod q_i for i < level; polynomial blockIdx.y.
__global__ void __launch_bounds__(256) k_ckks_rescale(ulonglong2* __restrict__ x, long long poly_stride, CkArgs a,
                                                      int o_inv, int o_inv_s) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  ulonglong2* xp = x + blockIdx.y * poly_stride;
  const int l = a.level;
  const ulonglong2 xl = xp[(size_t)l * a.N + j];
  for (int i = 0; i < l; ++i) {
    const uint64_t q = a.mc[i].p;
    const uint64_t c = __ldg(a.H + o_inv + l * a.k + i), cs = __ldg(a.H + o_inv_s + l * a.k + i);
    const ulonglong2 v = xp[(size_t)i * a.N + j];
    xp[(size_t)i * a.N + j] = make_ulonglong2(shoup_mul(v.x + q - xl.x, c, cs, q), shoup_mul(v.y + q - xl.y, c, cs, q));
  }
}

// out_i = x_i c_i mod q_i over the Q residues.
__global__ void __launch_bounds__(256) k_ckks_scale(ulonglong2* __restrict__ out, const ulonglong2* __restrict__ in,
                                                    CkArgs a, int o_c, int o_c_s) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  const int i = blockIdx.y;
  const uint64_t q = a.mc[i].p;
  const uint64_t c = __ldg(a.H + o_c + i), cs = __ldg(a.H + o_c_s + i);
  const ulonglong2 v = in[(size_t)i * a.N + j];
  out[(size_t)i * a.N + j] = make_ulonglong2(shoup_mul(v.x, c, cs, q), shoup_mul(v.y, c, cs, q));
}

CkArgs args(const Engine& e, int level) { return CkArgs{e.d_mc, e.d_hps, e.N, e.k, e.kl, level}; }

}  // namespace

}  // namespace cpoly

using namespace cpoly;

#define CK_REQUIRE(cond, msg) \
  do {                        \
    if (!(cond)) {            \
      set_error(msg);         \
      return CP_ERR_INVALID;  \
    }                         \
  } while (0)
#define CK_ENGINE(h, name)                                       \
  do {                                                           \
    CK_REQUIRE(h, name ": NULL engine");                         \
    if (!(h)->e.ckks_prec) {                                     \
      set_error(name ": needs an engine from cp_ckks_engine_create"); \
      return CP_ERR_UNSUPPORTED;                                 \
    }                                                            \
  } while (0)

extern "C" {

// Batched implementations: npolys polynomials back to back; the workspace holds
// npolys QB polynomials.  The single-polynomial calls are npolys = 1.
static int ckks_raise(const cp_engine* h, void* out_qb, const void* in_q, int level, int npolys, void* ws,
                      void* stream, const char* name) {
  CK_ENGINE(h, "cp_ckks_modulus_raising");
  CK_REQUIRE(out_qb && in_q && ws && npolys >= 0, "cp_ckks_modulus_raising: NULL argument or negative count");
  const Engine& e = h->e;
  CK_REQUIRE(level >= 0 && level < e.k, "cp_ckks_modulus_raising: level must be in [0, k)");
  if (npolys == 0) return CP_OK;
  CK_REQUIRE(npolys <= 65535, "cp_ckks_modulus_raising: at most 65535 polynomials per call");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ulonglong2* out = reinterpret_cast<ulonglong2*>(out_qb);
  ulonglong2* w = reinterpret_cast<ulonglong2*>(ws);
  const long long qsz = (long long)e.k * e.N, qbsz = (long long)(e.k + e.kl) * e.N;
  cudaError_t err = cudaMemcpy2DAsync(out, qbsz * 16, in_q, qsz * 16, qsz * 16, npolys, cudaMemcpyDeviceToDevice, st);
  if (err != cudaSuccess) return cuda_fail(name, err);
  if (int rc = launch_dgt_part(e, w, in_q, 0, level + 1, npolys, qsz, true, st)) return rc;  // Q_l, coefficients
  const auto& o = e.ho;
  k_ckks_raise<<<dim3((e.N + 127) / 128, npolys), 128, 0, st>>>(out + qsz, w, args(e, level), o.ck_qlqi_inv,
                                                                 o.ck_qlqi_inv_s, o.ck_qlqi_b, o.ck_qlqi_b_s, qbsz, qsz);
  if (int rc = check_launch(name)) return rc;
  return launch_dgt_part(e, out + qsz, nullptr, e.k, e.kl, npolys, qbsz, false, st);
}

static int ckks_reduce(const cp_engine* h, void* out_q, const void* in_qb, int level, int npolys, void* ws,
                       void* stream, const char* name) {
  CK_ENGINE(h, "cp_ckks_modulus_reduction");
  CK_REQUIRE(out_q && in_qb && ws && npolys >= 0, "cp_ckks_modulus_reduction: NULL argument or negative count");
  const Engine& e = h->e;
  CK_REQUIRE(level >= 0 && level < e.k, "cp_ckks_modulus_reduction: level must be in [0, k)");
  if (npolys == 0) return CP_OK;
  CK_REQUIRE(npolys <= 65535, "cp_ckks_modulus_reduction: at most 65535 polynomials per call");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  ulonglong2* w = reinterpret_cast<ulonglong2*>(ws);
  const ulonglong2* in = reinterpret_cast<const ulonglong2*>(in_qb);
  const long long qsz = (long long)e.k * e.N, qbsz = (long long)(e.k + e.kl) * e.N;
  // coefficients of Q_l and of B into the workspace (same QB layout)
  if (int rc = launch_dgt_part(e, w, in, 0, level + 1, npolys, qbsz, true, st)) return rc;
  if (int rc = launch_dgt_part(e, w + qsz, in + qsz, e.k, e.kl, npolys, qbsz, true, st)) return rc;
  const auto& o = e.ho;
  ulonglong2* out = reinterpret_cast<ulonglong2*>(out_q);
  k_ckks_reduce<<<dim3((e.N + 127) / 128, npolys), 128, 0, st>>>(out, w, args(e, level), o.ck_bbj_inv, o.ck_bbj_inv_s,
                                                                  o.ck_bbj_q, o.ck_bbj_q_s, o.ck_binv_q, o.ck_binv_q_s,
                                                                  qsz, qbsz);
  if (int rc = check_launch(name)) return rc;
  return launch_dgt_part(e, out, nullptr, 0, level + 1, npolys, qsz, false, st);
}

static int ckks_rescale(const cp_engine* h, void* x, int npolys, int level, void* stream) {
  const Engine& e = h->e;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const long long qsz = (long long)e.k * e.N;
  ulonglong2* p = reinterpret_cast<ulonglong2*>(x);
  if (int rc = launch_dgt_part(e, p, nullptr, 0, level + 1, npolys, qsz, true, st)) return rc;
  k_ckks_rescale<<<dim3((e.N + 255) / 256, npolys), 256, 0, st>>>(p, qsz, args(e, level), e.ho.ck_inv_ql,
                                                                   e.ho.ck_inv_ql_s);
  if (int rc = check_launch("cp_ckks_rescale")) return rc;
  return launch_dgt_part(e, p, nullptr, 0, level + 1, npolys, qsz, false, st);
}

int cp_ckks_modulus_raising(const cp_engine* h, void* out_qb, const void* in_q, int level, void* ws, void* stream) {
  return ckks_raise(h, out_qb, in_q, level, 1, ws, stream, "cp_ckks_modulus_raising");
}

int cp_ckks_modulus_reduction(const cp_engine* h, void* out_q, const void* in_qb, int level, void* ws, void* stream) {
  return ckks_reduce(h, out_q, in_qb, level, 1, ws, stream, "cp_ckks_modulus_reduction");
}

int cp_ckks_rescale(const cp_engine* h, void* a, void* b, int level, void* stream) {
  CK_ENGINE(h, "cp_ckks_rescale");
  CK_REQUIRE(a, "cp_ckks_rescale: NULL argument");
  CK_REQUIRE(level >= 1 && level < h->e.k, "cp_ckks_rescale: level must be in [1, k)");
  void* polys[2] = {a, b};
  for (void* x : polys)
    if (x)
      if (int rc = ckks_rescale(h, x, 1, level, stream)) return rc;
  return CP_OK;
}

size_t cp_ckks_batch_workspace_bytes(const cp_engine* h, int npolys) {
  if (!h || npolys < 0) return 0;
  return (size_t)npolys * (h->e.k + h->e.kl) * h->e.N * 16;
}

int cp_ckks_modulus_raising_batch(const cp_engine* h, void* out_qb, const void* in_q, int level, int npolys, void* ws,
                                  void* stream) {
  return ckks_raise(h, out_qb, in_q, level, npolys, ws, stream, "cp_ckks_modulus_raising_batch");
}

int cp_ckks_modulus_reduction_batch(const cp_engine* h, void* out_q, const void* in_qb, int level, int npolys,
                                    void* ws, void* stream) {
  return ckks_reduce(h, out_q, in_qb, level, npolys, ws, stream, "cp_ckks_modulus_reduction_batch");
}

int cp_ckks_rescale_batch(const cp_engine* h, void* x, int npolys, int level, void* stream) {
  CK_ENGINE(h, "cp_ckks_rescale_batch");
  CK_REQUIRE(x && npolys >= 0, "cp_ckks_rescale_batch: NULL argument or negative count");
  CK_REQUIRE(level >= 1 && level < h->e.k, "cp_ckks_rescale_batch: level must be in [1, k)");
  CK_REQUIRE(npolys <= 65535, "cp_ckks_rescale_batch: at most 65535 polynomials per call");
  if (npolys == 0) return CP_OK;
  return ckks_rescale(h, x, npolys, level, stream);
}

static int ckks_scale(const cp_engine* h, void* out, const void* in, bool xi, void* stream, const char* name) {
  CK_REQUIRE(h && out && in, "cp_ckks_xi/rho: NULL argument");
  if (!h->e.ckks_prec) {
    set_error("cp_ckks_xi/rho: needs an engine from cp_ckks_engine_create");
    return CP_ERR_UNSUPPORTED;
  }
  const Engine& e = h->e;
  dim3 grid((e.N + 255) / 256, e.k);
  k_ckks_scale<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<ulonglong2*>(out), reinterpret_cast<const ulonglong2*>(in), args(e, 0),
      xi ? e.ho.ck_binv_q : e.ho.ck_b_q, xi ? e.ho.ck_binv_q_s : e.ho.ck_b_q_s);
  return check_launch(name);
}

int cp_ckks_xi(const cp_engine* h, void* out, const void* in, void* stream) {
  return ckks_scale(h, out, in, true, stream, "cp_ckks_xi");
}

int cp_ckks_rho(const cp_engine* h, void* out, const void* in, void* stream) {
  return ckks_scale(h, out, in, false, stream, "cp_ckks_rho");
}

}  // extern "C"
