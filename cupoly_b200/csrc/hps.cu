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
//    and reduced once per target.  The lift is cuPoly's, decided exactly:
//    X in [0, S) is read as X - S when S - X <= S FPERROR (cuPoly's v rounds
//    up there), which makes the small negative values that the scaled BFV
//    tensor produces come out negative, as in cuPoly;
//  * complex scaling: with r the centred lift of (t x_i mod q_i) over Q,
//    round(t X / Q) = (t X - r) / Q, hence
//    round(t X / Q) mod b_j = (t y_j - [r]_{b_j}) Q^-1 mod b_j;
//  * simple scaling: round(t X / Q) mod t = -[r]_t Q^-1 mod t.
// The centring test compares MRC digits with those of (Q - 1) / 2.
//
// Fast path (every kernel below except simple scaling): with
// y_i = x_i (S/s_i)^-1 mod s_i, sum_i y_i / s_i = v + X/S for X in [0, S), so
// X mod m = sum_i y_i (S/s_i) - v S (mod m) -- s Shoup products instead of the
// s(s-1)/2 of the mixed-radix digits.  v and the side of 1/2 of X/S (the
// centring) come from an FP64 sum on the FP64 pipe, whose error is below
// 2^-43; they are used only when the fraction lies at least 2^-36 from the cut
// the caller applies (1/2 for the centring, 1 - FPERROR for cuPoly's lift; see
// fast_v).  Otherwise that coefficient takes the exact mixed-radix path, so
// every result is exact either way.
#include "launch.cuh"
#include "pointwise.cuh"

namespace cpoly {

namespace {

constexpr int kMaxBase = 24;  // largest |Q| or |B| with a compiled kernel
constexpr int kFastMin = 7;   // smallest source base that takes the fast path (measured: below it the digits are cheaper)

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
    for (int j = 0; j < i; ++j) mac192_w(l, h, t, d[j], __ldg(W + i * NS + j));
    const ModConst m = mcs[i];
    const uint64_t sum = red192_w(l, h, t, m.p, m.r1, m.r2);
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
  for (int i = 0; i < NS; ++i) mac192_w(l, h, t, d[i], __ldg(w + i));
  return red192_w(l, h, t, mt.p, mt.r1, mt.r2);
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

// Fast base conversion constants of one source base S = prod s_i.
struct Fast {
  const uint64_t *hinv, *hinv_s;  // per source i: (S/s_i)^-1 mod s_i (times t for the scaling)
  const uint64_t* hmod;           // [target][i]: (S/s_i) mod m_target
  const uint64_t* negv;           // [target][v], v in [0, NS]: (-v S) mod m_target
  const uint64_t* invd;           // per source: 1/s_i as IEEE-754 double bits
};

// FP64 overflow count: sum_i y_i / s_i = v + X/S.  Returns whether v (and,
// with `half`, the side of 1/2 of X/S) is certain.
__device__ __forceinline__ double u32_to_double(uint32_t x) {  // exact, FP64 pipe only
  return __hiloint2double(0x43300000, (int)x) - 4503599627370496.0;
}

// cuPoly's lift: X in [0, S) is read as X - S when X / S >= 1 - FPERROR (see
// lift_threshold_digits in tables.cu); this is the fraction side of that test.
constexpr double kLiftFrac = 1.0 - 1e-9;

// Which integer the callers take from the sum f = v + X/S: w = v + [X/S >= c] with the cut
// c = 1/2 (centring, `half`) or c = kLiftFrac (cuPoly's lift).  Either way w is the integer
// floor(f + 1 - c), so an error in f moves w only where f + 1 - c lies near an integer, that
// is where the fraction of f lies near c.  Near 0 and near 1 it does not: a fraction just
// below 1 read where the true one is just above 0 (or the reverse) changes floor(f) by one
// and the side of c the other way, and w is the same.  The BFV chain's B -> Q conversion,
// whose values are small signed integers (fractions within 2^-40 of 0 or 1), therefore takes
// the fast path.

template <int NS>
__device__ __forceinline__ bool fast_v(const uint64_t (&y)[NS], const uint64_t* __restrict__ invd, bool half, int& v,
                                       bool& above, bool lift = false, bool* neg = nullptr) {
  double f = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) {  // y = yh 2^32 + yl, both halves exact in FP64
    const double c = __longlong_as_double(__ldg(invd + i));
    f = __fma_rn(u32_to_double((uint32_t)y[i]), c, f);
    f = __fma_rn(u32_to_double((uint32_t)(y[i] >> 32)), c * 4294967296.0, f);
  }
  const double fl = floor(f);
  const double fr = f - fl;  // exact
  v = (int)fl;
  above = fr >= 0.5;
  const double d = 0x1p-36;
  if (lift) *neg = fr > kLiftFrac;
  if (!half && !lift) return fr > d && fr < 1.0 - d;  // a plain floor is uncertain near integers
  return (!half || fabs(fr - 0.5) > d) && (!lift || fabs(fr - kLiftFrac) > d);
}

// (sum_i y_i hmod_i + negv) mod m: lazy 192-bit sum (< 25 * 2^126), one reduction.
template <int NS>
__device__ __forceinline__ uint64_t fast_dot(const uint64_t (&y)[NS], const uint64_t* __restrict__ hmod, uint64_t negv,
                                             const ModConst& mt) {
  uint64_t l = negv, h = 0, t = 0;
#pragma unroll
  for (int i = 0; i < NS; ++i) mac192_w(l, h, t, y[i], __ldg(hmod + i));
  return red192_w(l, h, t, mt.p, mt.r1, mt.r2);
}

struct ConvArgs {
  Fast f;
  const ModConst* mc;
  const uint64_t* inv;
  const uint64_t* inv_s;
  const uint64_t* hor;
  const uint64_t* hor_s;
  const uint64_t* pm;  // mixed-radix weights [target][source]
  const uint64_t *W, *pinv, *pinv_s;  // Garner constants of the source base
  const uint64_t* lift;               // MRC digits of the source base's lift threshold minus one
  const uint64_t *rec, *rec_s;        // prescaled inputs y_i = x_i (S/s_i)^-1: x_i = y_i (S/s_i)
  int force_exact;                    // 1: every coefficient takes the exact path
  int src_off, dst_off, ndst, N;
  long long in_stride, out_stride;  // per polynomial, in elements
};

// Exact path of one coefficient (component comp of element j): mixed-radix
// digits, then one dot product per target.
// With `prescaled`, the inputs are y_i = x_i (S/s_i)^-1 and x_i is recovered first.
template <int NS>
__device__ __noinline__ void ext_exact(uint64_t* ow, const uint64_t* iw, int j, int comp, const ConvArgs& a,
                                       bool prescaled = false) {
  uint64_t s[NS], d[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    s[i] = a.mc[a.src_off + i].p;
    d[i] = iw[2 * ((size_t)i * a.N + j) + comp];
    if (prescaled) d[i] = shoup_mul(d[i], __ldg(a.rec + i), __ldg(a.rec_s + i), s[i]);
  }
  mrc_any<NS>(d, s, a.inv, a.inv_s, a.mc + a.src_off, a.W, a.pinv, a.pinv_s);
  const bool neg = above_half<NS>(d, a.lift);  // cuPoly's lift: X - S
  for (int t = 0; t < a.ndst; ++t) {
    const ModConst mt = a.mc[a.dst_off + t];
    uint64_t r = dot_mod<NS>(d, a.pm + t * NS, mt);
    if (neg) r = add_mod(r, __ldg(a.f.negv + t * (NS + 1) + 1), mt.p);
    ow[2 * ((size_t)t * a.N + j) + comp] = r;
  }
}

// X mod m_j for every target j; one thread per Gaussian element (2 coefficients).
template <int NS>
__global__ void __launch_bounds__(128) k_basis_ext(ulonglong2* __restrict__ out, const ulonglong2* __restrict__ in,
                                                   const __grid_constant__ ConvArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  const uint64_t* iw = reinterpret_cast<const uint64_t*>(in + blockIdx.y * a.in_stride);
  uint64_t* ow = reinterpret_cast<uint64_t*>(out + blockIdx.y * a.out_stride);
  if constexpr (NS <= kFastMin - 1) {  // tiny bases: the mixed-radix digits cost no more than the fast path
    uint64_t s[NS], dr[NS], di[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      s[i] = a.mc[a.src_off + i].p;
      const ulonglong2 x = in[blockIdx.y * a.in_stride + (size_t)i * a.N + j];
      dr[i] = x.x;
      di[i] = x.y;
    }
    mrc_any<NS>(dr, s, a.inv, a.inv_s, a.mc + a.src_off, a.W, a.pinv, a.pinv_s);
    mrc_any<NS>(di, s, a.inv, a.inv_s, a.mc + a.src_off, a.W, a.pinv, a.pinv_s);
    const bool nr = above_half<NS>(dr, a.lift), ni = above_half<NS>(di, a.lift);  // cuPoly's lift: X - S
    for (int t = 0; t < a.ndst; ++t) {
      const ModConst mt = a.mc[a.dst_off + t];
      const uint64_t* w = a.pm + t * NS;
      const uint64_t ns = __ldg(a.f.negv + t * (NS + 1) + 1);  // -S mod m
      uint64_t rr = dot_mod<NS>(dr, w, mt), ri = dot_mod<NS>(di, w, mt);
      if (nr) rr = add_mod(rr, ns, mt.p);
      if (ni) ri = add_mod(ri, ns, mt.p);
      out[blockIdx.y * a.out_stride + (size_t)t * a.N + j] = make_ulonglong2(rr, ri);
    }
  } else if constexpr (NS < 8) {  // small bases: both coefficients together (ILP)
    uint64_t yr[NS], yi[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      const ulonglong2 x = in[blockIdx.y * a.in_stride + (size_t)i * a.N + j];
      const uint64_t h = __ldg(a.f.hinv + i), hs = __ldg(a.f.hinv_s + i), p = a.mc[a.src_off + i].p;
      yr[i] = shoup_mul(x.x, h, hs, p);
      yi[i] = shoup_mul(x.y, h, hs, p);
    }
    int vr, vi;
    bool ab, nr, ni;
    const bool okr = fast_v<NS>(yr, a.f.invd, false, vr, ab, true, &nr);
    const bool oki = fast_v<NS>(yi, a.f.invd, false, vi, ab, true, &ni);
    if (okr && oki && !a.force_exact) {
      vr += nr ? 1 : 0;  // cuPoly's lift: X - S
      vi += ni ? 1 : 0;
      for (int t = 0; t < a.ndst; ++t) {
        const ModConst mt = a.mc[a.dst_off + t];
        const uint64_t* hm = a.f.hmod + t * NS;
        const uint64_t* nv = a.f.negv + t * (NS + 1);
        out[blockIdx.y * a.out_stride + (size_t)t * a.N + j] =
            make_ulonglong2(fast_dot<NS>(yr, hm, __ldg(nv + vr), mt), fast_dot<NS>(yi, hm, __ldg(nv + vi), mt));
      }
    } else {
      ext_exact<NS>(ow, iw, j, 0, a);
      ext_exact<NS>(ow, iw, j, 1, a);
    }
  } else {  // large bases: one coefficient at a time (registers)
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t y[NS];
#pragma unroll
      for (int i = 0; i < NS; ++i)
        y[i] = shoup_mul(iw[2 * ((size_t)i * a.N + j) + comp], __ldg(a.f.hinv + i), __ldg(a.f.hinv_s + i),
                         a.mc[a.src_off + i].p);
      int v;
      bool above, neg;
      if (!a.force_exact && fast_v<NS>(y, a.f.invd, false, v, above, true, &neg)) {
        v += neg ? 1 : 0;  // cuPoly's lift: X - S
        for (int t = 0; t < a.ndst; ++t)
          ow[2 * ((size_t)t * a.N + j) + comp] =
              fast_dot<NS>(y, a.f.hmod + t * NS, __ldg(a.f.negv + t * (NS + 1) + v), a.mc[a.dst_off + t]);
      } else {
        ext_exact<NS>(ow, iw, j, comp, a);
      }
    }
  }
}

// X mod m_j from prescaled inputs y_i = x_i (S/s_i)^-1 mod s_i, which an inverse DGT with
// an off_untwist_pre table leaves: the fast path starts at its FP64 sum for every base
// size (no constant product before it, and no mixed-radix digits for small bases); a
// coefficient it cannot decide recovers x_i and takes the exact path.
template <int NS>
__global__ void __launch_bounds__(128) k_basis_ext_pre(ulonglong2* __restrict__ out, const ulonglong2* __restrict__ in,
                                                       const __grid_constant__ ConvArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  const uint64_t* iw = reinterpret_cast<const uint64_t*>(in + blockIdx.y * a.in_stride);
  uint64_t* ow = reinterpret_cast<uint64_t*>(out + blockIdx.y * a.out_stride);
  if constexpr (NS < 8) {  // small bases: both coefficients together (ILP)
    uint64_t yr[NS], yi[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      const ulonglong2 x = in[blockIdx.y * a.in_stride + (size_t)i * a.N + j];
      yr[i] = x.x;
      yi[i] = x.y;
    }
    int vr, vi;
    bool ab, nr, ni;
    const bool okr = fast_v<NS>(yr, a.f.invd, false, vr, ab, true, &nr);
    const bool oki = fast_v<NS>(yi, a.f.invd, false, vi, ab, true, &ni);
    if (okr && oki && !a.force_exact) {
      vr += nr ? 1 : 0;  // cuPoly's lift: X - S
      vi += ni ? 1 : 0;
      for (int t = 0; t < a.ndst; ++t) {
        const ModConst mt = a.mc[a.dst_off + t];
        const uint64_t* hm = a.f.hmod + t * NS;
        const uint64_t* nv = a.f.negv + t * (NS + 1);
        out[blockIdx.y * a.out_stride + (size_t)t * a.N + j] =
            make_ulonglong2(fast_dot<NS>(yr, hm, __ldg(nv + vr), mt), fast_dot<NS>(yi, hm, __ldg(nv + vi), mt));
      }
    } else {
      ext_exact<NS>(ow, iw, j, 0, a, true);
      ext_exact<NS>(ow, iw, j, 1, a, true);
    }
  } else {  // large bases: one coefficient at a time (registers)
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t y[NS];
#pragma unroll
      for (int i = 0; i < NS; ++i) y[i] = iw[2 * ((size_t)i * a.N + j) + comp];
      int v;
      bool above, neg;
      if (!a.force_exact && fast_v<NS>(y, a.f.invd, false, v, above, true, &neg)) {
        v += neg ? 1 : 0;  // cuPoly's lift: X - S
        for (int t = 0; t < a.ndst; ++t)
          ow[2 * ((size_t)t * a.N + j) + comp] =
              fast_dot<NS>(y, a.f.hmod + t * NS, __ldg(a.f.negv + t * (NS + 1) + v), a.mc[a.dst_off + t]);
      } else {
        ext_exact<NS>(ow, iw, j, comp, a, true);
      }
    }
  }
}

struct ScaleArgs {
  Fast fq;  // Q side of the fast path, t folded into hinv
  const ModConst* mc;
  const uint64_t *inv, *inv_s, *hor, *hor_s, *half, *pm;
  const uint64_t *W, *pinv, *pinv_s;  // Garner constants of Q
  const uint64_t *t_q, *t_q_s, *t_b, *t_b_s, *q_mod_b, *qinv_b, *qinv_b_s;
  // prescaled inputs (k_complex_scaling_pre): Q side y_i = t x_i (Q/q_i)^-1, B side
  // y'_j = t Q^-1 (B/b_j)^-1 y_j; the output is z_j (B/b_j)^-1, the B -> Q conversion's
  // prescaled input
  const uint64_t *trec, *trec_s, *brec, *brec_s, *bhinv, *bhinv_s, *hm2, *negw2;
  int force_exact;
  int k, kl, N;
  long long q_stride, b_stride, out_stride;
};

// Exact path of complex scaling for one coefficient, written straight out.
template <int NQ>
__device__ __noinline__ void scale_exact_write(uint64_t* ow, const uint64_t* qw, const uint64_t* bw, int j, int comp,
                                               const ScaleArgs& a) {
  uint64_t s[NQ], d[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    s[i] = a.mc[i].p;
    d[i] = shoup_mul(qw[2 * ((size_t)i * a.N + j) + comp], __ldg(a.t_q + i), __ldg(a.t_q_s + i), s[i]);
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

// round(t X / Q) mod b_j for X given by Q and B residues (coefficient domain).
template <int NQ>
__global__ void __launch_bounds__(128) k_complex_scaling(ulonglong2* __restrict__ out_b,
                                                         const ulonglong2* __restrict__ in_q,
                                                         const ulonglong2* __restrict__ in_b,
                                                         const __grid_constant__ ScaleArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  const uint64_t* qw = reinterpret_cast<const uint64_t*>(in_q + blockIdx.y * a.q_stride);
  const uint64_t* bw = reinterpret_cast<const uint64_t*>(in_b + blockIdx.y * a.b_stride);
  uint64_t* ow = reinterpret_cast<uint64_t*>(out_b + blockIdx.y * a.out_stride);
  if constexpr (NQ <= kFastMin - 1) {  // small bases: mixed-radix digits, both coefficients together
    const ulonglong2* q2 = reinterpret_cast<const ulonglong2*>(qw);
    const ulonglong2* b2 = reinterpret_cast<const ulonglong2*>(bw);
    uint64_t s[NQ], dr[NQ], di[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
      s[i] = a.mc[i].p;
      const ulonglong2 x = q2[(size_t)i * a.N + j];
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
      const ulonglong2 y = b2[(size_t)t * a.N + j];
      const uint64_t tb = __ldg(a.t_b + t), tbs = __ldg(a.t_b_s + t);
      const uint64_t qi = __ldg(a.qinv_b + t), qis = __ldg(a.qinv_b_s + t);
      reinterpret_cast<ulonglong2*>(ow)[(size_t)t * a.N + j] =
          make_ulonglong2(shoup_mul(shoup_mul(y.x, tb, tbs, b) + b - rr, qi, qis, b),
                          shoup_mul(shoup_mul(y.y, tb, tbs, b) + b - ri, qi, qis, b));
    }
  } else if constexpr (NQ < 8) {  // small bases: both coefficients together (ILP)
    uint64_t yr[NQ], yi[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
      const ulonglong2 x = reinterpret_cast<const ulonglong2*>(qw)[(size_t)i * a.N + j];
      const uint64_t h = __ldg(a.fq.hinv + i), hs = __ldg(a.fq.hinv_s + i), p = a.mc[i].p;
      yr[i] = shoup_mul(x.x, h, hs, p);
      yi[i] = shoup_mul(x.y, h, hs, p);
    }
    int vr, vi;
    bool ar, ai;
    const bool okr = fast_v<NQ>(yr, a.fq.invd, true, vr, ar);
    const bool oki = fast_v<NQ>(yi, a.fq.invd, true, vi, ai);
    if (okr && oki && !a.force_exact) {
      const int wr = vr + (ar ? 1 : 0), wi = vi + (ai ? 1 : 0);
      for (int t = 0; t < a.kl; ++t) {
        const ModConst mt = a.mc[a.k + t];
        const uint64_t b = mt.p;
        const uint64_t* hm = a.fq.hmod + t * NQ;
        const uint64_t* nv = a.fq.negv + t * (NQ + 1);
        const uint64_t rr = fast_dot<NQ>(yr, hm, __ldg(nv + wr), mt);
        const uint64_t ri = fast_dot<NQ>(yi, hm, __ldg(nv + wi), mt);
        const ulonglong2 y = reinterpret_cast<const ulonglong2*>(bw)[(size_t)t * a.N + j];
        const uint64_t tb = __ldg(a.t_b + t), tbs = __ldg(a.t_b_s + t);
        const uint64_t qi = __ldg(a.qinv_b + t), qis = __ldg(a.qinv_b_s + t);
        reinterpret_cast<ulonglong2*>(ow)[(size_t)t * a.N + j] =
            make_ulonglong2(shoup_mul(shoup_mul(y.x, tb, tbs, b) + b - rr, qi, qis, b),
                            shoup_mul(shoup_mul(y.y, tb, tbs, b) + b - ri, qi, qis, b));
      }
    } else {
      scale_exact_write<NQ>(ow, qw, bw, j, 0, a);
      scale_exact_write<NQ>(ow, qw, bw, j, 1, a);
    }
  } else {
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t y[NQ];
#pragma unroll
      for (int i = 0; i < NQ; ++i)
        y[i] = shoup_mul(qw[2 * ((size_t)i * a.N + j) + comp], __ldg(a.fq.hinv + i), __ldg(a.fq.hinv_s + i), a.mc[i].p);
      int v;
      bool above;
      if (!a.force_exact && fast_v<NQ>(y, a.fq.invd, true, v, above)) {
        const int w = v + (above ? 1 : 0);
        for (int t = 0; t < a.kl; ++t) {
          const ModConst mt = a.mc[a.k + t];
          const uint64_t b = mt.p;
          const uint64_t r = fast_dot<NQ>(y, a.fq.hmod + t * NQ, __ldg(a.fq.negv + t * (NQ + 1) + w), mt);
          const uint64_t ty = shoup_mul(bw[2 * ((size_t)t * a.N + j) + comp], __ldg(a.t_b + t), __ldg(a.t_b_s + t), b);
          ow[2 * ((size_t)t * a.N + j) + comp] = shoup_mul(ty + b - r, __ldg(a.qinv_b + t), __ldg(a.qinv_b_s + t), b);
        }
      } else {
        scale_exact_write<NQ>(ow, qw, bw, j, comp, a);
      }
    }
  }
}

// Exact path of the prescaled complex scaling for one coefficient: recover x_i and y_j,
// round(t X / Q) mod b_j as scale_exact_write, then times (B/b_j)^-1.
template <int NQ>
__device__ __noinline__ void scale_exact_pre_write(uint64_t* ow, const uint64_t* qw, const uint64_t* bw, int j,
                                                   int comp, const ScaleArgs& a) {
  uint64_t s[NQ], d[NQ];
#pragma unroll
  for (int i = 0; i < NQ; ++i) {
    s[i] = a.mc[i].p;
    const uint64_t x = shoup_mul(qw[2 * ((size_t)i * a.N + j) + comp], __ldg(a.trec + i), __ldg(a.trec_s + i), s[i]);
    d[i] = shoup_mul(x, __ldg(a.t_q + i), __ldg(a.t_q_s + i), s[i]);
  }
  mrc_any<NQ>(d, s, a.inv, a.inv_s, a.mc, a.W, a.pinv, a.pinv_s);
  const bool neg = above_half<NQ>(d, a.half);
  for (int t = 0; t < a.kl; ++t) {
    const ModConst mt = a.mc[a.k + t];
    const uint64_t b = mt.p;
    uint64_t r = dot_mod<NQ>(d, a.pm + t * NQ, mt);
    if (neg) r = sub_mod(r, __ldg(a.q_mod_b + t), b);
    const uint64_t y = shoup_mul(bw[2 * ((size_t)t * a.N + j) + comp], __ldg(a.brec + t), __ldg(a.brec_s + t), b);
    const uint64_t ty = shoup_mul(y, __ldg(a.t_b + t), __ldg(a.t_b_s + t), b);
    const uint64_t z = shoup_mul(ty + b - r, __ldg(a.qinv_b + t), __ldg(a.qinv_b_s + t), b);
    ow[2 * ((size_t)t * a.N + j) + comp] = shoup_mul(z, __ldg(a.bhinv + t), __ldg(a.bhinv_s + t), b);
  }
}

// round(t X / Q) (B/b_j)^-1 mod b_j from prescaled inputs (see ScaleArgs): with w the
// centred overflow count, [t X mod Q centred] Q^-1 (B/b_j)^-1 = sum_i y_i q_i^-1 (B/b_j)^-1 -
// w (B/b_j)^-1, so each output is y'_j minus one dot product -- no constant products.
template <int NQ>
__global__ void __launch_bounds__(128) k_complex_scaling_pre(ulonglong2* __restrict__ out_b,
                                                             const ulonglong2* __restrict__ in_q,
                                                             const ulonglong2* __restrict__ in_b,
                                                             const __grid_constant__ ScaleArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.N) return;
  const uint64_t* qw = reinterpret_cast<const uint64_t*>(in_q + blockIdx.y * a.q_stride);
  const uint64_t* bw = reinterpret_cast<const uint64_t*>(in_b + blockIdx.y * a.b_stride);
  uint64_t* ow = reinterpret_cast<uint64_t*>(out_b + blockIdx.y * a.out_stride);
  if constexpr (NQ < 8) {  // small bases: both coefficients together (ILP)
    uint64_t yr[NQ], yi[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) {
      const ulonglong2 x = reinterpret_cast<const ulonglong2*>(qw)[(size_t)i * a.N + j];
      yr[i] = x.x;
      yi[i] = x.y;
    }
    int vr, vi;
    bool ar, ai;
    const bool okr = fast_v<NQ>(yr, a.fq.invd, true, vr, ar);
    const bool oki = fast_v<NQ>(yi, a.fq.invd, true, vi, ai);
    if (okr && oki && !a.force_exact) {
      const int wr = vr + (ar ? 1 : 0), wi = vi + (ai ? 1 : 0);
      for (int t = 0; t < a.kl; ++t) {
        const ModConst mt = a.mc[a.k + t];
        const uint64_t b = mt.p;
        const uint64_t* hm = a.hm2 + t * NQ;
        const uint64_t* nw = a.negw2 + t * (NQ + 1);
        const uint64_t rr = fast_dot<NQ>(yr, hm, __ldg(nw + wr), mt);
        const uint64_t ri = fast_dot<NQ>(yi, hm, __ldg(nw + wi), mt);
        const ulonglong2 y = reinterpret_cast<const ulonglong2*>(bw)[(size_t)t * a.N + j];
        reinterpret_cast<ulonglong2*>(ow)[(size_t)t * a.N + j] = make_ulonglong2(sub_mod(y.x, rr, b), sub_mod(y.y, ri, b));
      }
    } else {
      scale_exact_pre_write<NQ>(ow, qw, bw, j, 0, a);
      scale_exact_pre_write<NQ>(ow, qw, bw, j, 1, a);
    }
  } else {
#pragma unroll 1
    for (int comp = 0; comp < 2; ++comp) {
      uint64_t y[NQ];
#pragma unroll
      for (int i = 0; i < NQ; ++i) y[i] = qw[2 * ((size_t)i * a.N + j) + comp];
      int v;
      bool above;
      if (!a.force_exact && fast_v<NQ>(y, a.fq.invd, true, v, above)) {
        const int w = v + (above ? 1 : 0);
        for (int t = 0; t < a.kl; ++t) {
          const ModConst mt = a.mc[a.k + t];
          const uint64_t r = fast_dot<NQ>(y, a.hm2 + t * NQ, __ldg(a.negw2 + t * (NQ + 1) + w), mt);
          ow[2 * ((size_t)t * a.N + j) + comp] = sub_mod(bw[2 * ((size_t)t * a.N + j) + comp], r, mt.p);
        }
      } else {
        scale_exact_pre_write<NQ>(ow, qw, bw, j, comp, a);
      }
    }
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
template <int NS>
int launch_basis_ext_pre_n(ulonglong2* out, const ulonglong2* in, const ConvArgs& a, int npolys, cudaStream_t st) {
  dim3 grid((a.N + 127) / 128, npolys);
  k_basis_ext_pre<NS><<<grid, 128, 0, st>>>(out, in, a);
  return check_launch("basis_ext_pre");
}
template <int NQ>
int launch_cs_pre_n(ulonglong2* out, const ulonglong2* q, const ulonglong2* b, const ScaleArgs& a, int npolys,
                    cudaStream_t st) {
  dim3 grid((a.N + 127) / 128, npolys);
  k_complex_scaling_pre<NQ><<<grid, 128, 0, st>>>(out, q, b, a);
  return check_launch("complex_scaling_pre");
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

static ConvArgs conv_args(const Engine& e, bool q_to_b) {
  ConvArgs a;
  a.mc = e.d_mc;
  a.force_exact = e.hps_force_exact;
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
    a.f = Fast{e.d_hps + e.ho.fq_hinv, e.d_hps + e.ho.fq_hinv_s, e.d_hps + e.ho.fq_hmod, e.d_hps + e.ho.fq_negv,
               e.d_hps + e.ho.fq_invd};
    a.lift = e.d_hps + e.ho.q_lift;
    a.rec = e.d_hps + e.ho.rho_q;  // (Q/q_i) mod q_i
    a.rec_s = e.d_hps + e.ho.rho_q_s;
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
    a.f = Fast{e.d_hps + e.ho.fb_hinv, e.d_hps + e.ho.fb_hinv_s, e.d_hps + e.ho.fb_hmod, e.d_hps + e.ho.fb_negv,
               e.d_hps + e.ho.fb_invd};
    a.lift = e.d_hps + e.ho.b_lift;
    a.rec = e.d_hps + e.ho.fb_rec;  // (B/b_j) mod b_j
    a.rec_s = e.d_hps + e.ho.fb_rec_s;
    a.src_off = e.k;
    a.dst_off = 0;
    a.ndst = e.k;
  }
  const int ns = q_to_b ? e.k : e.kl;
  a.in_stride = (long long)ns * e.N;
  a.out_stride = (long long)a.ndst * e.N;
  return a;
}

int hps_basis_ext(const Engine& e, void* out, const void* in, bool q_to_b, int npolys, cudaStream_t st) {
  const ConvArgs a = conv_args(e, q_to_b);
  const int ns = q_to_b ? e.k : e.kl;
  auto* o = reinterpret_cast<ulonglong2*>(out);
  auto* i = reinterpret_cast<const ulonglong2*>(in);
#define CALL(n) launch_basis_ext_n<n>(o, i, a, npolys, st)
  CP_SWITCH_NS(ns, CALL)
#undef CALL
}

int hps_basis_ext_pre(const Engine& e, void* out, const void* in, bool q_to_b, int npolys, cudaStream_t st) {
  const ConvArgs a = conv_args(e, q_to_b);
  const int ns = q_to_b ? e.k : e.kl;
  auto* o = reinterpret_cast<ulonglong2*>(out);
  auto* i = reinterpret_cast<const ulonglong2*>(in);
#define CALL(n) launch_basis_ext_pre_n<n>(o, i, a, npolys, st)
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
  a.fq = Fast{e.d_hps + e.ho.fq_thinv, e.d_hps + e.ho.fq_thinv_s, e.d_hps + e.ho.fq_hmod, e.d_hps + e.ho.fq_negv,
              e.d_hps + e.ho.fq_invd};
  a.trec = e.d_hps + e.ho.fq_trec;
  a.trec_s = e.d_hps + e.ho.fq_trec_s;
  a.brec = e.d_hps + e.ho.cs_brec;
  a.brec_s = e.d_hps + e.ho.cs_brec_s;
  a.bhinv = e.d_hps + e.ho.fb_hinv;
  a.bhinv_s = e.d_hps + e.ho.fb_hinv_s;
  a.hm2 = e.d_hps + e.ho.cs_hm2;
  a.negw2 = e.d_hps + e.ho.cs_negw2;
  a.force_exact = e.hps_force_exact;
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
}  // namespace

int hps_scale_to_q(const Engine& e, void* out_q, const void* in_q, const void* in_b, void* scratch_b, int npolys,
                   cudaStream_t st) {
  // complex scaling into scratch_b, then the exact B -> Q conversion.  (A fused
  // single kernel that kept the B residues in registers measured 2-4 % slower
  // on B200 for |Q| = 2..7: its register footprint halves the resident warps.)
  int rc = hps_complex_scaling(e, scratch_b, in_q, in_b, npolys, st);
  if (rc) return rc;
  return hps_basis_ext(e, out_q, scratch_b, false, npolys, st);
}

// The chain's form on prescaled inputs (the off_untwist_pre tables): in_q holds
// t x_i (Q/q_i)^-1 mod q_i and in_b t Q^-1 (B/b_j)^-1 y_j mod b_j; out_q is round(t X / Q)
// over Q in the coefficient domain.
int hps_scale_to_q_pre(const Engine& e, void* out_q, const void* in_q, const void* in_b, void* scratch_b, int npolys,
                       cudaStream_t st) {
  const ScaleArgs a = scale_args(e);
  auto* o = reinterpret_cast<ulonglong2*>(scratch_b);
  auto* q = reinterpret_cast<const ulonglong2*>(in_q);
  auto* b = reinterpret_cast<const ulonglong2*>(in_b);
  int rc;
#define CALL(n) launch_cs_pre_n<n>(o, q, b, a, npolys, st)
  rc = [&]() -> int { CP_SWITCH_NS(e.k, CALL) }();
#undef CALL
  if (rc) return rc;
  return hps_basis_ext_pre(e, out_q, scratch_b, false, npolys, st);
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
  const int i = blockIdx.y;      // output polynomial of the decomposition
  const int r = blockIdx.z % k;  // residue
  const int pl = blockIdx.z / k;  // input polynomial of the batch
  in += (size_t)pl * k * N;
  out += (size_t)pl * k * k * N;
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

int rns_xi_rho(const Engine& e, void* out, const void* in, bool rho, cudaStream_t st, int npolys) {
  const uint64_t* w = e.d_hps + (rho ? e.ho.rho_q : e.ho.xi_q);
  const uint64_t* ws = e.d_hps + (rho ? e.ho.rho_q_s : e.ho.xi_q_s);
  if (npolys <= 0) return 0;
  if ((long long)npolys * e.k > 65535) {
    set_error("xi_rho: at most 65535 / k polynomials per call");
    return 1;
  }
  int bx = (e.N + 255) / 256;
  if (bx > 1024) bx = 1024;
  dim3 grid(bx, e.k, e.k * npolys);
  k_xi_rho<<<grid, 256, 0, st>>>(reinterpret_cast<ulonglong2*>(out), reinterpret_cast<const ulonglong2*>(in), e.d_mc,
                                 w, ws, e.k, e.N);
  return check_launch("xi_rho");
}

}  // namespace cpoly
