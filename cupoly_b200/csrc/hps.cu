// Exact RNS base conversion and HPS scaling (replaces cuPoly's
// polynomial_basis_ext_Q_aux / _Q_compute_v / _Q_to_B, the B-side trio,
// polynomial_complex_scaling and simple_scaling; src/cuda/cudaengine.cu:
// 304-798).
//
// cuPoly estimates the CRT overflow v with doubles (FPERROR = 1e-9) and the
// HPS rounding with a 64-bit fraction sum in double.  Here both are exact and
// use only word-size modular arithmetic:
//  * base conversion: mixed-radix digits d_i of X (MRC), then X mod m as the
//    dot product sum_i d_i (prod_{l<i} s_l mod m), accumulated in 192 bits
//    and reduced once per target;
//  * complex scaling: with r the centred lift of (t x_i mod q_i) over Q,
//    round(t X / Q) = (t X - r) / Q, hence
//    round(t X / Q) mod b_j = (t y_j - [r]_{b_j}) Q^-1 mod b_j;
//  * simple scaling: round(t X / Q) mod t = -[r]_t Q^-1 mod t.
// The centring test compares MRC digits with those of (Q - 1) / 2.
#include "launch.cuh"
#include "pointwise.cuh"

namespace cpoly {

namespace {

constexpr int kMaxBase = 24;  // largest |Q| or |B| with a compiled kernel

__device__ __forceinline__ uint64_t red1(uint64_t x, uint64_t m) { return red2p(x, m); }  // x < 2m

// Garner form of the mixed-radix conversion for larger bases:
// d_i = (x_i - sum_{l<i} d_l W[i][l]) Pinv_i mod s_i, W[i][l] = prod_{j<l} s_j
// mod s_i, Pinv_i = (prod_{j<i} s_j)^-1 mod s_i; the sums are lazy (192-bit).
template <int NS>
__device__ __forceinline__ void mrc_garner(uint64_t (&d)[NS], const ModConst* __restrict__ mcs,
                                           const uint64_t* __restrict__ W, const uint64_t* __restrict__ pinv,
                                           const uint64_t* __restrict__ pinv_s) {
#pragma unroll
  for (int i = 1; i < NS; ++i) {
    uint64_t l = 0, h = 0, t = 0;
#pragma unroll
    for (int j = 0; j < i; ++j) mac192(l, h, t, d[j], __ldg(W + i * NS + j));
    const ModConst m = mcs[i];
    const uint64_t sum = red192(l, h, t, m.p, m.r1, m.r2);
    d[i] = shoup_mul(d[i] + m.p - sum, __ldg(pinv + i), __ldg(pinv_s + i), m.p);
  }
}

// Mixed-radix digits of the value with residues z over primes s.
template <int NS>
__device__ __forceinline__ void mrc(uint64_t (&d)[NS], const uint64_t (&s)[NS], const uint64_t* __restrict__ inv,
                                    const uint64_t* __restrict__ inv_s) {
#pragma unroll
  for (int i = 1; i < NS; ++i) {
    uint64_t y = d[i];
#pragma unroll
    for (int l = 0; l < i; ++l) {
      const uint64_t dl = red1(d[l], s[i]);
      const int c = i * (i - 1) / 2 + l;
      y = shoup_mul(y + s[i] - dl, __ldg(inv + c), __ldg(inv_s + c), s[i]);
    }
    d[i] = y;
  }
}

// Sequential MRC for small bases (k(k-1)/2 dependent Shoup steps), Garner with
// lazy sums from 8 primes on (fewer instructions once the sums are long).
template <int NS>
__device__ __forceinline__ void mrc_any(uint64_t (&d)[NS], const uint64_t (&s)[NS], const uint64_t* inv,
                                        const uint64_t* inv_s, const ModConst* mcs, const uint64_t* W,
                                        const uint64_t* pinv, const uint64_t* pinv_s) {
  if constexpr (NS >= 8)
    mrc_garner<NS>(d, mcs, W, pinv, pinv_s);
  else
    mrc<NS>(d, s, inv, inv_s);
}

// X mod t for an arbitrary modulus t < 2^63 (digits reduced by a Shoup step).
template <int NS>
__device__ __forceinline__ uint64_t horner_small(const uint64_t (&d)[NS], uint64_t t, uint64_t one_s,
                                                 const uint64_t* __restrict__ hor,
                                                 const uint64_t* __restrict__ hor_s) {
  uint64_t acc = shoup_mul(d[NS - 1], 1 % t, one_s, t);
#pragma unroll
  for (int i = NS - 2; i >= 0; --i) {
    acc = shoup_mul(acc, __ldg(hor + i), __ldg(hor_s + i), t);
    acc = add_mod(acc, shoup_mul(d[i], 1 % t, one_s, t), t);
  }
  return acc;
}

// X mod m = sum_i d_i w_i with w_i = prod_{l<i} s_l mod m, accumulated in three
// words and reduced once (every target prime has 2^64 mod m < 2^32).
template <int NS>
__device__ __forceinline__ uint64_t dot_mod(const uint64_t (&d)[NS], const uint64_t* __restrict__ w,
                                            const ModConst& mt) {
  uint64_t l = 0, h = 0, t = 0;
#pragma unroll
  for (int i = 0; i < NS; ++i) mac192(l, h, t, d[i], __ldg(w + i));
  return red192(l, h, t, mt.p, mt.r1, mt.r2);
}

// digits > (prod - 1) / 2 ?
template <int NS>
__device__ __forceinline__ bool above_half(const uint64_t (&d)[NS], const uint64_t* __restrict__ half) {
  int state = 0;  // 0 equal so far, 1 greater, -1 less
#pragma unroll
  for (int i = NS - 1; i >= 0; --i) {
    const uint64_t h = __ldg(half + i);
    if (state == 0) state = d[i] > h ? 1 : (d[i] < h ? -1 : 0);
  }
  return state > 0;
}

struct ConvArgs {
  const ModConst* mc;
  const uint64_t* inv;
  const uint64_t* inv_s;
  const uint64_t* hor;
  const uint64_t* hor_s;
  const uint64_t* pm;  // mixed-radix weights [target][source]
  const uint64_t *W, *pinv, *pinv_s;  // Garner constants of the source base
  int src_off, dst_off, ndst, N;
  long long in_stride, out_stride;  // per polynomial, in elements
};

// X mod m_j for every target j; one thread per Gaussian element (2 coefficients).
template <int NS>
__global__ void __launch_bounds__(128) k_basis_ext(ulonglong2* __restrict__ out, const ulonglong2* __restrict__ in,
                                                   ConvArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  in += blockIdx.y * a.in_stride;
  out += blockIdx.y * a.out_stride;
  if constexpr (NS < 8) {  // small bases: both coefficients at once (more ILP)
    uint64_t s[NS], dr[NS], di[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      s[i] = a.mc[a.src_off + i].p;
      const ulonglong2 x = in[(size_t)i * a.N + j];
      dr[i] = x.x;
      di[i] = x.y;
    }
    mrc_any<NS>(dr, s, a.inv, a.inv_s, a.mc + a.src_off, a.W, a.pinv, a.pinv_s);
    mrc_any<NS>(di, s, a.inv, a.inv_s, a.mc + a.src_off, a.W, a.pinv, a.pinv_s);
    for (int t = 0; t < a.ndst; ++t) {
      const ModConst mt = a.mc[a.dst_off + t];
      const uint64_t* w = a.pm + t * NS;
      out[(size_t)t * a.N + j] = make_ulonglong2(dot_mod<NS>(dr, w, mt), dot_mod<NS>(di, w, mt));
    }
  } else {  // large bases: one coefficient at a time keeps the digits in registers
    const uint64_t* iw = reinterpret_cast<const uint64_t*>(in);
    uint64_t* ow = reinterpret_cast<uint64_t*>(out);
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t s[NS], d[NS];
#pragma unroll
      for (int i = 0; i < NS; ++i) d[i] = iw[2 * ((size_t)i * a.N + j) + comp];
      mrc_any<NS>(d, s, a.inv, a.inv_s, a.mc + a.src_off, a.W, a.pinv, a.pinv_s);
      for (int t = 0; t < a.ndst; ++t)
        ow[2 * ((size_t)t * a.N + j) + comp] = dot_mod<NS>(d, a.pm + t * NS, a.mc[a.dst_off + t]);
    }
  }
}

struct ScaleArgs {
  const ModConst* mc;
  const uint64_t *inv, *inv_s, *hor, *hor_s, *half, *pm;
  const uint64_t *W, *pinv, *pinv_s;  // Garner constants of Q
  const uint64_t *t_q, *t_q_s, *t_b, *t_b_s, *q_mod_b, *qinv_b, *qinv_b_s;
  int k, kl, N;
  long long q_stride, b_stride, out_stride;
};

// round(t X / Q) mod b_j for X given by Q and B residues (coefficient domain).
template <int NQ>
__global__ void __launch_bounds__(128) k_complex_scaling(ulonglong2* __restrict__ out_b,
                                                         const ulonglong2* __restrict__ in_q,
                                                         const ulonglong2* __restrict__ in_b, ScaleArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  in_q += blockIdx.y * a.q_stride;
  in_b += blockIdx.y * a.b_stride;
  out_b += blockIdx.y * a.out_stride;
  if constexpr (NQ >= 8) {  // large bases: one coefficient at a time (register pressure)
    const uint64_t* qw = reinterpret_cast<const uint64_t*>(in_q);
    const uint64_t* bw = reinterpret_cast<const uint64_t*>(in_b);
    uint64_t* ow = reinterpret_cast<uint64_t*>(out_b);
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t s[NQ], d[NQ];
#pragma unroll
      for (int i = 0; i < NQ; ++i) {
        const uint64_t p = a.mc[i].p;
        d[i] = shoup_mul(qw[2 * ((size_t)i * a.N + j) + comp], __ldg(a.t_q + i), __ldg(a.t_q_s + i), p);
      }
      mrc_any<NQ>(d, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
      const bool neg = above_half<NQ>(d, a.half);
      for (int t = 0; t < a.kl; ++t) {
        const ModConst mt = a.mc[a.k + t];
        const uint64_t b = mt.p;
        uint64_t r = dot_mod<NQ>(d, a.pm + t * NQ, mt);
        if (neg) r = sub_mod(r, __ldg(a.q_mod_b + t), b);
        const uint64_t ty = shoup_mul(bw[2 * ((size_t)t * a.N + j) + comp], __ldg(a.t_b + t), __ldg(a.t_b_s + t), b);
        ow[2 * ((size_t)t * a.N + j) + comp] = shoup_mul(ty + b - r, __ldg(a.qinv_b + t), __ldg(a.qinv_b_s + t), b);
      }
    }
    return;
  }
  uint64_t s[NQ], dr[NQ], di[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    s[i] = a.mc[i].p;
    const ulonglong2 x = in_q[(size_t)i * a.N + j];
    const uint64_t tq = __ldg(a.t_q + i), tqs = __ldg(a.t_q_s + i);
    dr[i] = shoup_mul(x.x, tq, tqs, s[i]);
    di[i] = shoup_mul(x.y, tq, tqs, s[i]);
  }
  mrc_any<NQ>(dr, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
  mrc_any<NQ>(di, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
  const bool nr = above_half<NQ>(dr, a.half);
  const bool ni = above_half<NQ>(di, a.half);
  for (int t = 0; t < a.kl; ++t) {
    const ModConst mt = a.mc[a.k + t];
    const uint64_t b = mt.p;
    const uint64_t qb = __ldg(a.q_mod_b + t);
    uint64_t rr = dot_mod<NQ>(dr, a.pm + t * NQ, mt);
    uint64_t ri = dot_mod<NQ>(di, a.pm + t * NQ, mt);
    if (nr) rr = sub_mod(rr, qb, b);
    if (ni) ri = sub_mod(ri, qb, b);
    const ulonglong2 y = in_b[(size_t)t * a.N + j];
    const uint64_t tb = __ldg(a.t_b + t), tbs = __ldg(a.t_b_s + t);
    const uint64_t qi = __ldg(a.qinv_b + t), qis = __ldg(a.qinv_b_s + t);
    const uint64_t ur = shoup_mul(shoup_mul(y.x, tb, tbs, b) + b - rr, qi, qis, b);
    const uint64_t ui = shoup_mul(shoup_mul(y.y, tb, tbs, b) + b - ri, qi, qis, b);
    out_b[(size_t)t * a.N + j] = make_ulonglong2(ur, ui);
  }
}

// Complex scaling fused with the exact B -> Q conversion of its result:
// out_q = (round(t X / Q) mod B) mod q_i; the kl B-residues stay in registers.
// One thread per Gaussian element; the two coefficients are done in turn.
template <int NQ, int NB>
__global__ void __launch_bounds__(128) k_scale_to_q(ulonglong2* __restrict__ out_q, const ulonglong2* __restrict__ in_q,
                                                    const ulonglong2* __restrict__ in_b, ScaleArgs a, ConvArgs c) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  in_q += blockIdx.y * a.q_stride;
  in_b += blockIdx.y * a.b_stride;
  uint64_t* o = reinterpret_cast<uint64_t*>(out_q + blockIdx.y * a.q_stride);
  // primes are re-read from the (cached) constant table instead of living in
  // registers: the digit arrays are what must stay resident
  uint64_t s[NQ], sb[NB];
  if constexpr (NQ < 8) {
#pragma unroll
    for (int i = 0; i < NQ; ++i) s[i] = a.mc[i].p;
  }
  if constexpr (NB < 8) {
#pragma unroll
    for (int i = 0; i < NB; ++i) sb[i] = a.mc[NQ + i].p;
  }
#pragma unroll 1
  for (int comp = 0; comp < 2; ++comp) {
    uint64_t d[NQ], u[NB];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
      const uint64_t* x = reinterpret_cast<const uint64_t*>(in_q + (size_t)i * a.N + j);
      d[i] = shoup_mul(x[comp], __ldg(a.t_q + i), __ldg(a.t_q_s + i), a.mc[i].p);
    }
    mrc_any<NQ>(d, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
    const bool neg = above_half<NQ>(d, a.half);
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      const uint64_t b = a.mc[NQ + t].p;
      uint64_t r = dot_mod<NQ>(d, a.pm + t * NQ, a.mc[NQ + t]);
      if (neg) r = sub_mod(r, __ldg(a.q_mod_b + t), b);
      const uint64_t* y = reinterpret_cast<const uint64_t*>(in_b + (size_t)t * a.N + j);
      const uint64_t ty = shoup_mul(y[comp], __ldg(a.t_b + t), __ldg(a.t_b_s + t), b);
      u[t] = shoup_mul(ty + b - r, __ldg(a.qinv_b + t), __ldg(a.qinv_b_s + t), b);
    }
    mrc_any<NB>(u, sb, c.inv, c.inv_s, c.mc + c.src_off, c.W, c.pinv, c.pinv_s);
#pragma unroll
    for (int i = 0; i < NQ; ++i)
      o[2 * ((size_t)i * a.N + j) + comp] = dot_mod<NB>(u, c.pm + i * NB, a.mc[i]);
  }
}

struct SimpleArgs {
  const ModConst* mc;
  const uint64_t *inv, *inv_s, *hor, *hor_s, *half, *t_q, *t_q_s;
  const uint64_t *W, *pinv, *pinv_s;  // Garner constants of Q
  uint64_t t, one_s, q_mod_t, qinv_t, qinv_t_s;
  int N;
};

// round(t X / Q) mod t, written to one Gaussian residue.
template <int NQ>
__global__ void __launch_bounds__(128) k_simple_scaling(ulonglong2* __restrict__ out,
                                                        const ulonglong2* __restrict__ in_q, SimpleArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  if constexpr (NQ >= 8) {  // large bases: one coefficient at a time (register pressure)
    const uint64_t* qw = reinterpret_cast<const uint64_t*>(in_q);
    uint64_t res[2];
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t s[NQ], d[NQ];
#pragma unroll
      for (int i = 0; i < NQ; ++i)
        d[i] = shoup_mul(qw[2 * ((size_t)i * a.N + j) + comp], __ldg(a.t_q + i), __ldg(a.t_q_s + i), a.mc[i].p);
      mrc_any<NQ>(d, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
      const bool neg = above_half<NQ>(d, a.half);
      uint64_t r = horner_small<NQ>(d, a.t, a.one_s, a.hor, a.hor_s);
      if (neg) r = sub_mod(r, a.q_mod_t, a.t);
      res[comp] = shoup_mul(neg_mod(r, a.t), a.qinv_t, a.qinv_t_s, a.t);
    }
    out[j] = make_ulonglong2(res[0], res[1]);
    return;
  }
  uint64_t s[NQ], dr[NQ], di[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    s[i] = a.mc[i].p;
    const ulonglong2 x = in_q[(size_t)i * a.N + j];
    const uint64_t tq = __ldg(a.t_q + i), tqs = __ldg(a.t_q_s + i);
    dr[i] = shoup_mul(x.x, tq, tqs, s[i]);
    di[i] = shoup_mul(x.y, tq, tqs, s[i]);
  }
  mrc_any<NQ>(dr, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
  mrc_any<NQ>(di, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
  const bool nr = above_half<NQ>(dr, a.half);
  const bool ni = above_half<NQ>(di, a.half);
  uint64_t rr = horner_small<NQ>(dr, a.t, a.one_s, a.hor, a.hor_s);
  uint64_t ri = horner_small<NQ>(di, a.t, a.one_s, a.hor, a.hor_s);
  if (nr) rr = sub_mod(rr, a.q_mod_t, a.t);
  if (ni) ri = sub_mod(ri, a.q_mod_t, a.t);
  out[j] = make_ulonglong2(shoup_mul(neg_mod(rr, a.t), a.qinv_t, a.qinv_t_s, a.t),
                           shoup_mul(neg_mod(ri, a.t), a.qinv_t, a.qinv_t_s, a.t));
}

template <int NS>
int launch_basis_ext_n(ulonglong2* out, const ulonglong2* in, const ConvArgs& a, int npolys, cudaStream_t st) {
  dim3 grid((a.N + 127) / 128, npolys);
  k_basis_ext<NS><<<grid, 128, 0, st>>>(out, in, a);
  return check_launch("basis_ext");
}
template <int NQ>
int launch_cs_n(ulonglong2* out, const ulonglong2* q, const ulonglong2* b, const ScaleArgs& a, int npolys,
                cudaStream_t st) {
  dim3 grid((a.N + 127) / 128, npolys);
  k_complex_scaling<NQ><<<grid, 128, 0, st>>>(out, q, b, a);
  return check_launch("complex_scaling");
}
template <int NQ>
int launch_ss_n(ulonglong2* out, const ulonglong2* q, const SimpleArgs& a, cudaStream_t st) {
  k_simple_scaling<NQ><<<(a.N + 127) / 128, 128, 0, st>>>(out, q, a);
  return check_launch("simple_scaling");
}

#define CP_SWITCH_NS(n, CALL)                                                                             \
  switch (n) {                                                                                            \
    case 1: return CALL(1); case 2: return CALL(2); case 3: return CALL(3); case 4: return CALL(4);       \
    case 5: return CALL(5); case 6: return CALL(6); case 7: return CALL(7); case 8: return CALL(8);       \
    case 9: return CALL(9); case 10: return CALL(10); case 11: return CALL(11); case 12: return CALL(12); \
    case 13: return CALL(13); case 14: return CALL(14); case 15: return CALL(15);                        \
    case 16: return CALL(16); case 17: return CALL(17); case 18: return CALL(18);                        \
    case 19: return CALL(19); case 20: return CALL(20); case 21: return CALL(21);                        \
    case 22: return CALL(22); case 23: return CALL(23); case 24: return CALL(24);                        \
    default: set_error("base larger than 24 primes is not compiled"); return CP_ERR_UNSUPPORTED_;        \
  }

}  // namespace

int hps_basis_ext(const Engine& e, void* out, const void* in, bool q_to_b, int npolys, cudaStream_t st) {
  ConvArgs a;
  a.mc = e.d_mc;
  a.N = e.N;
  if (q_to_b) {
    a.inv = e.d_hps + e.ho.qb_inv;
    a.inv_s = e.d_hps + e.ho.qb_inv_s;
    a.W = e.d_hps + e.ho.qq_w;
    a.pinv = e.d_hps + e.ho.q_pinv;
    a.pinv_s = e.d_hps + e.ho.q_pinv_s;
    a.hor = e.d_hps + e.ho.qb_hor;
    a.hor_s = e.d_hps + e.ho.qb_hor_s;
    a.pm = e.d_hps + e.ho.qb_pm;
    a.src_off = 0;
    a.dst_off = e.k;
    a.ndst = e.kl;
  } else {
    a.inv = e.d_hps + e.ho.bq_inv;
    a.inv_s = e.d_hps + e.ho.bq_inv_s;
    a.W = e.d_hps + e.ho.bb_w;
    a.pinv = e.d_hps + e.ho.b_pinv;
    a.pinv_s = e.d_hps + e.ho.b_pinv_s;
    a.hor = e.d_hps + e.ho.bq_hor;
    a.hor_s = e.d_hps + e.ho.bq_hor_s;
    a.pm = e.d_hps + e.ho.bq_pm;
    a.src_off = e.k;
    a.dst_off = 0;
    a.ndst = e.k;
  }
  const int ns = q_to_b ? e.k : e.kl;
  a.in_stride = (long long)ns * e.N;
  a.out_stride = (long long)a.ndst * e.N;
  auto* o = reinterpret_cast<ulonglong2*>(out);
  auto* i = reinterpret_cast<const ulonglong2*>(in);
#define CALL(n) launch_basis_ext_n<n>(o, i, a, npolys, st)
  CP_SWITCH_NS(ns, CALL)
#undef CALL
}

static ScaleArgs scale_args(const Engine& e) {
  ScaleArgs a;
  a.mc = e.d_mc;
  a.inv = e.d_hps + e.ho.qb_inv;
  a.inv_s = e.d_hps + e.ho.qb_inv_s;
  a.W = e.d_hps + e.ho.qq_w;
  a.pinv = e.d_hps + e.ho.q_pinv;
  a.pinv_s = e.d_hps + e.ho.q_pinv_s;
  a.hor = e.d_hps + e.ho.qb_hor;
  a.pm = e.d_hps + e.ho.qb_pm;
  a.hor_s = e.d_hps + e.ho.qb_hor_s;
  a.half = e.d_hps + e.ho.qb_half;
  a.t_q = e.d_hps + e.ho.t_q;
  a.t_q_s = e.d_hps + e.ho.t_q_s;
  a.t_b = e.d_hps + e.ho.t_b;
  a.t_b_s = e.d_hps + e.ho.t_b_s;
  a.q_mod_b = e.d_hps + e.ho.q_mod_b;
  a.qinv_b = e.d_hps + e.ho.qinv_b;
  a.qinv_b_s = e.d_hps + e.ho.qinv_b_s;
  a.k = e.k;
  a.kl = e.kl;
  a.N = e.N;
  a.q_stride = (long long)e.k * e.N;
  a.b_stride = (long long)e.kl * e.N;
  a.out_stride = (long long)e.kl * e.N;
  return a;
}

int hps_complex_scaling(const Engine& e, void* out_b, const void* in_q, const void* in_b, int npolys,
                        cudaStream_t st) {
  ScaleArgs a = scale_args(e);
  auto* o = reinterpret_cast<ulonglong2*>(out_b);
  auto* q = reinterpret_cast<const ulonglong2*>(in_q);
  auto* b = reinterpret_cast<const ulonglong2*>(in_b);
#define CALL(n) launch_cs_n<n>(o, q, b, a, npolys, st)
  CP_SWITCH_NS(e.k, CALL)
#undef CALL
}

namespace {
template <int NQ>
int launch_scale_to_q_n(ulonglong2* o, const ulonglong2* q, const ulonglong2* b, const ScaleArgs& a,
                        const ConvArgs& c, int npolys, cudaStream_t st) {
  dim3 grid((a.N + 127) / 128, npolys);
  k_scale_to_q<NQ, NQ + 1><<<grid, 128, 0, st>>>(o, q, b, a, c);
  return check_launch("scale_to_q");
}
}  // namespace

int hps_scale_to_q(const Engine& e, void* out_q, const void* in_q, const void* in_b, void* scratch_b, int npolys,
                   cudaStream_t st) {
  // fused kernel for small bases (the B residues never leave registers); from
  // 8 primes on the two separate kernels keep more warps resident and win
  if (e.kl == e.k + 1 && e.k < 8) {
    ScaleArgs a = scale_args(e);
    ConvArgs c;
    c.mc = e.d_mc;
    c.N = e.N;
    c.inv = e.d_hps + e.ho.bq_inv;
    c.inv_s = e.d_hps + e.ho.bq_inv_s;
    c.W = e.d_hps + e.ho.bb_w;
    c.pinv = e.d_hps + e.ho.b_pinv;
    c.pinv_s = e.d_hps + e.ho.b_pinv_s;
    c.hor = e.d_hps + e.ho.bq_hor;
    c.hor_s = e.d_hps + e.ho.bq_hor_s;
    c.pm = e.d_hps + e.ho.bq_pm;
    c.src_off = e.k;
    c.dst_off = 0;
    c.ndst = e.k;
    auto* o = reinterpret_cast<ulonglong2*>(out_q);
    auto* q = reinterpret_cast<const ulonglong2*>(in_q);
    auto* b = reinterpret_cast<const ulonglong2*>(in_b);
    switch (e.k) {
#define CP_SQ(n) \
  case n: return launch_scale_to_q_n<n>(o, q, b, a, c, npolys, st);
      CP_SQ(1) CP_SQ(2) CP_SQ(3) CP_SQ(4) CP_SQ(5) CP_SQ(6) CP_SQ(7) CP_SQ(8)
      CP_SQ(9) CP_SQ(10) CP_SQ(11) CP_SQ(12) CP_SQ(13) CP_SQ(14) CP_SQ(15) CP_SQ(16)
#undef CP_SQ
    }
  }
  int rc = hps_complex_scaling(e, scratch_b, in_q, in_b, npolys, st);
  if (rc) return rc;
  return hps_basis_ext(e, out_q, scratch_b, false, npolys, st);
}

int hps_simple_scaling(const Engine& e, void* out_t, const void* in_q, cudaStream_t st) {
  SimpleArgs a;
  a.mc = e.d_mc;
  a.inv = e.d_hps + e.ho.qb_inv;
  a.inv_s = e.d_hps + e.ho.qb_inv_s;
  a.W = e.d_hps + e.ho.qq_w;
  a.pinv = e.d_hps + e.ho.q_pinv;
  a.pinv_s = e.d_hps + e.ho.q_pinv_s;
  a.hor = e.d_hps + e.ho.qt_hor;
  a.hor_s = e.d_hps + e.ho.qt_hor_s;
  a.half = e.d_hps + e.ho.qb_half;
  a.t_q = e.d_hps + e.ho.t_q;
  a.t_q_s = e.d_hps + e.ho.t_q_s;
  a.t = e.t;
  a.one_s = e.t_shoup_one;
  a.q_mod_t = e.h_q_mod_t;
  a.qinv_t = e.h_qinv_t;
  a.qinv_t_s = e.h_qinv_t_s;
  a.N = e.N;
  auto* o = reinterpret_cast<ulonglong2*>(out_t);
  auto* q = reinterpret_cast<const ulonglong2*>(in_q);
#define CALL(n) launch_ss_n<n>(o, q, a, st)
  CP_SWITCH_NS(e.k, CALL)
#undef CALL
}

// xi / rho decomposition (cuPoly src/cuda/cudaengine.cu:992-1062): residue i of
// output polynomial i is a_i * (Q/q_i)^-1 (xi) or a_i * (Q/q_i) (rho) mod q_i;
// every other residue of output polynomial i is zero.
namespace {
__global__ void __launch_bounds__(256) k_xi_rho(ulonglong2* __restrict__ out, const ulonglong2* __restrict__ in,
                                                const ModConst* __restrict__ mc, const uint64_t* __restrict__ w,
                                                const uint64_t* __restrict__ ws, int k, int N) {
  const int i = blockIdx.y;  // output polynomial
  const int r = blockIdx.z;  // residue
  ulonglong2* o = out + ((size_t)i * k + r) * N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    if (r != i) {
      o[j] = make_ulonglong2(0, 0);
    } else {
      const ulonglong2 x = in[(size_t)r * N + j];
      const uint64_t p = mc[r].p;
      o[j] = make_ulonglong2(shoup_mul(x.x, w[r], ws[r], p), shoup_mul(x.y, w[r], ws[r], p));
    }
  }
}
}  // namespace

int rns_xi_rho(const Engine& e, void* out, const void* in, bool rho, cudaStream_t st) {
  const uint64_t* w = e.d_hps + (rho ? e.ho.rho_q : e.ho.xi_q);
  const uint64_t* ws = e.d_hps + (rho ? e.ho.rho_q_s : e.ho.xi_q_s);
  int bx = (e.N + 255) / 256;
  if (bx > 1024) bx = 1024;
  dim3 grid(bx, e.k, e.k);
  k_xi_rho<<<grid, 256, 0, st>>>(reinterpret_cast<ulonglong2*>(out), reinterpret_cast<const ulonglong2*>(in), e.d_mc,
                                 w, ws, e.k, e.N);
  return check_launch("xi_rho");
}

}  // namespace cpoly
