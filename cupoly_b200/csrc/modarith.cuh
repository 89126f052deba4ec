// Modular arithmetic for 63-bit primes on sm_100a.
//
// Replaces cuPoly's Barrett `mod`/`mulmod`/`addmod`/`submod` and the
// Gaussian-integer helpers (cuPoly src/cuda/dgt.cu:285-675,
// include/cuPoly/cuda/dgt.h:74-82).  Every result is canonical in [0, p).
//
// p < 2^63, so a + b < 2^64 for reduced a, b but 4p > 2^64: lazy [0, 4p)
// butterflies are impossible and every add/sub is corrected immediately.
//
//  * shoup_mul(a, w, w', p): a * w mod p for a constant w with
//    w' = floor(w 2^64 / p); valid for any a < 2^64 (Shoup / Harvey).
//  * mont_redc(hi:lo): (hi:lo) * 2^-64 mod p for hi:lo < p 2^64 (Montgomery).
//  * pm_red(hi:lo): hi:lo mod p for hi:lo < 2^127 by pseudo-Mersenne folding
//    (every prime of the table is p = 2^63 - c with c < 2^31 - 1, so
//    2^63 == c mod p); about 3 wide multiplies, against about 15 for a
//    Montgomery step followed by the Shoup correction by 2^64 mod p.
//  * mul_mod(a, b) and the Gaussian products use pm_red.
#pragma once
#include <cstdint>

#ifndef CP_HD
#define CP_HD __host__ __device__ __forceinline__
#endif

namespace cpoly {

// Per-residue constants, one entry per prime of an engine (Q then B).
struct ModConst {
  uint64_t p;       // the prime
  uint64_t pneg;    // -p^-1 mod 2^64
  uint64_t r1;      // 2^64 mod p (below 2^32 for every 63-bit prime of the table)
  uint64_t r1s;     // shoup companion of r1
  uint64_t r2;      // 2^128 mod p
  uint64_t pm;      // 1: p = 2^63 - c with c < 2^31 - 1 (pm_red applies); 0: generic path
};

#ifdef __CUDA_ARCH__
// hi:lo = a * b as four 32 x 32 -> 64 multiply-adds, each folding the previous carry
// in (a 32 x 32 product plus one 32-bit addend, or plus two for the top word, stays
// below 2^64): the low and high words of one product share their partial products.
__device__ __forceinline__ void mul128(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
  asm("{\n\t.reg .u32 a0, a1, b0, b1, r0, r1, s1, c0, c1, c2;\n\t.reg .u64 t0, t1, t2, t3, x;\n\t"
      "mov.b64 {a0, a1}, %2;\n\tmov.b64 {b0, b1}, %3;\n\t"
      "mul.wide.u32 t0, a0, b0;\n\tmov.b64 {r0, c0}, t0;\n\t"
      "cvt.u64.u32 x, c0;\n\tmad.wide.u32 t1, a0, b1, x;\n\tmov.b64 {s1, c1}, t1;\n\t"
      "cvt.u64.u32 x, s1;\n\tmad.wide.u32 t2, a1, b0, x;\n\tmov.b64 {r1, c2}, t2;\n\t"
      "cvt.u64.u32 x, c1;\n\tmad.wide.u32 t3, a1, b1, x;\n\t"
      "cvt.u64.u32 x, c2;\n\tadd.u64 %1, t3, x;\n\tmov.b64 %0, {r0, r1};\n\t}"
      : "=l"(lo), "=l"(hi)
      : "l"(a), "l"(b));
}
#endif

// Three-word accumulation (t:h:l) += a * b, for lazily reduced dot products.
CP_HD void mac192(uint64_t& l, uint64_t& h, uint64_t& t, uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  const uint64_t pl = a * b, ph = __umul64hi(a, b);
  asm("add.cc.u64 %0, %0, %3;\n\taddc.cc.u64 %1, %1, %4;\n\taddc.u64 %2, %2, 0;"
      : "+l"(l), "+l"(h), "+l"(t)
      : "l"(pl), "l"(ph));
#else
  unsigned __int128 pr = (unsigned __int128)a * b;
  unsigned __int128 lo = (unsigned __int128)l + (uint64_t)pr;
  unsigned __int128 hi = (unsigned __int128)h + (uint64_t)(pr >> 64) + (uint64_t)(lo >> 64);
  l = (uint64_t)lo;
  h = (uint64_t)hi;
  t += (uint64_t)(hi >> 64);
#endif
}

// mac192 with the product formed by mul128: fewer 32-bit multiplies; used by the base
// conversions, whose dot products are bound by the integer multiply pipe.
CP_HD void mac192_w(uint64_t& l, uint64_t& h, uint64_t& t, uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  uint64_t pl, ph;
  mul128(a, b, pl, ph);
  asm("add.cc.u64 %0, %0, %3;\n\taddc.cc.u64 %1, %1, %4;\n\taddc.u64 %2, %2, 0;"
      : "+l"(l), "+l"(h), "+l"(t)
      : "l"(pl), "l"(ph));
#else
  mac192(l, h, t, a, b);
#endif
}

// (t 2^128 + h 2^64 + l) mod p for t < 2^8, using r1 = 2^64 mod p < 2^32 and
// r2 = 2^128 mod p: fold the high words down three times, then at most two
// subtractions (the value is below 2^64 < 3p).
CP_HD uint64_t red192(uint64_t l, uint64_t h, uint64_t t, uint64_t p, uint64_t r1, uint64_t r2) {
  const uint32_t r = (uint32_t)r1;  // r1 < 2^32: 64 x 32-bit products below
  // y = l + h r1 + t r2 < 2^97
  unsigned __int128 y = (unsigned __int128)l + (unsigned __int128)h * r + (unsigned __int128)t * r2;
  // z = lo(y) + hi(y) r1 < 2^66
  unsigned __int128 z = (unsigned __int128)(uint64_t)y + (unsigned __int128)(uint64_t)(y >> 64) * r;
  // w = lo(z) + hi(z) r1 < 2^64 + 2^34; one carry at most
  const uint64_t zl = (uint64_t)z, zh = (uint64_t)(z >> 64);
  uint64_t w = zl + zh * r1;
  if (w < zl) w += r1;
  w = w >= p ? w - p : w;
  w = w >= p ? w - p : w;
  return w;
}

// red192 with every product written as 32 x 32 -> 64 multiplies (r1 < 2^32, t < 2^8):
// seven wide multiplies; used by the base conversions.
CP_HD uint64_t red192_w(uint64_t l, uint64_t h, uint64_t t, uint64_t p, uint64_t r1, uint64_t r2) {
  const uint64_t r = (uint32_t)r1;
  // y = l + h r1 + t r2 < 2^97
  const uint64_t a0 = (uint64_t)(uint32_t)h * r, a1 = (h >> 32) * r;       // h r1 = a0 + a1 2^32
  const uint64_t b0 = (uint64_t)(uint32_t)t * (uint32_t)r2;                 // t r2 = b0 + b1 2^32
  const uint64_t b1 = (uint64_t)(uint32_t)t * (uint32_t)(r2 >> 32);
  const unsigned __int128 y = (unsigned __int128)l + a0 + b0 + ((unsigned __int128)a1 << 32) +
                              ((unsigned __int128)b1 << 32);
  // z = lo(y) + hi(y) r1 < 2^67, hi(y) < 2^34
  const uint64_t yh = (uint64_t)(y >> 64);
  const unsigned __int128 z = (unsigned __int128)(uint64_t)y + (uint64_t)(uint32_t)yh * r +
                              ((unsigned __int128)((yh >> 32) * r) << 32);
  // w = lo(z) + hi(z) r1 < 2^64 + 2^35: one carry at most
  const uint64_t zl = (uint64_t)z, zh = (uint64_t)(z >> 64);
  uint64_t w = zl + (uint64_t)(uint32_t)zh * r;
  if (w < zl) w += r1;
  w = w >= p ? w - p : w;
  w = w >= p ? w - p : w;
  return w;
}

CP_HD uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// The corrections below select on the sign of a 64-bit difference: every
// intermediate lies in (-p, 2p) with p < 2^63, so its sign bit decides.
CP_HD uint64_t red2p(uint64_t s, uint64_t p) {  // s in [0, 2p) -> [0, p)
  const int64_t t = (int64_t)(s - p);
  return t < 0 ? s : (uint64_t)t;
}

CP_HD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t p) { return red2p(a + b, p); }

CP_HD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t p) {
  const int64_t d = (int64_t)(a - b);
  return d < 0 ? (uint64_t)d + p : (uint64_t)d;
}

CP_HD uint64_t neg_mod(uint64_t a, uint64_t p) { return a == 0 ? 0 : p - a; }

// a * w mod p, w < p constant, ws = floor(w * 2^64 / p); any a < 2^64.
CP_HD uint64_t shoup_mul(uint64_t a, uint64_t w, uint64_t ws, uint64_t p) {
  const uint64_t q = mulhi64(a, ws);
  return red2p(a * w - q * p, p);  // a w - q p in [0, 2p)
}

// Montgomery reduction of hi:lo < p * 2^64 -> hi:lo * 2^-64 mod p.
CP_HD uint64_t mont_redc(uint64_t hi, uint64_t lo, uint64_t p, uint64_t pneg) {
  uint64_t m = lo * pneg;
  return red2p(hi + mulhi64(m, p) + (lo != 0), p);
}

// a * b * 2^-64 mod p for a * b < p * 2^64.
CP_HD uint64_t mont_mul(uint64_t a, uint64_t b, uint64_t p, uint64_t pneg) {
  return mont_redc(mulhi64(a, b), a * b, p, pneg);
}

// hi:lo mod p for hi:lo < 2^127, p = 2^63 - c with c < 2^31 - 1:
//   X = H 2^63 + L == L + H c,        H < 2^64, L < 2^63;
//   Z = L + H c = Zh 2^63 + Zl == Zl + Zh c,   Zh <= 2c + 1;
//   r = Zl + Zh c < 2^63 + c + 2c^2 <= 2p, then one correction.
CP_HD uint64_t pm_red(uint64_t hi, uint64_t lo, uint64_t p) {
  const uint64_t c = (1ull << 63) - p;
  const uint64_t H = (hi << 1) | (lo >> 63);
  const uint64_t L = lo & 0x7FFFFFFFFFFFFFFFull;
  const uint64_t y0 = (H & 0xFFFFFFFFull) * c;  // < 2^63
  const uint64_t y1 = (H >> 32) * c;             // < 2^63; H c = y0 + y1 2^32
  const uint64_t t = y1 << 32;
  uint64_t zl = L + y0;                          // < 2^64
  zl += t;
  const uint64_t zh = (y1 >> 32) + (zl < t);     // Z = zh 2^64 + zl
  const uint64_t Zh = (zh << 1) | (zl >> 63);
  return red2p((zl & 0x7FFFFFFFFFFFFFFFull) + Zh * c, p);
}

// hi:lo mod p for hi:lo < p 2^64, any p < 2^63: Montgomery step, then the
// factor 2^64 restored by a Shoup product with r1 = 2^64 mod p.
CP_HD uint64_t gen_red(uint64_t hi, uint64_t lo, const ModConst& m) {
  return shoup_mul(mont_redc(hi, lo, m.p, m.pneg), m.r1, m.r1s, m.p);
}

// hi:lo mod p: pseudo-Mersenne folding for the 63-bit primes, the generic
// Montgomery path for the others (the CKKS precision buckets).  Callers keep
// hi:lo < min(2^127, p 2^64).  The branch is uniform across a residue.
CP_HD uint64_t red128(uint64_t hi, uint64_t lo, const ModConst& m) {
  return m.pm ? pm_red(hi, lo, m.p) : gen_red(hi, lo, m);
}

// Exact a * b mod p for a < p, b < 2^64.
CP_HD uint64_t mul_mod(uint64_t a, uint64_t b, const ModConst& m) {
#ifdef __CUDA_ARCH__
  uint64_t lo, hi;
  mul128(a, b, lo, hi);
  return red128(hi, lo, m);
#else
  return red128(mulhi64(a, b), a * b, m);
#endif
}

// 128-bit accumulate helpers (hi:lo += a * b).
CP_HD void mac128(uint64_t& hi, uint64_t& lo, uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  uint64_t pl, ph;
  mul128(a, b, pl, ph);
#else
  uint64_t pl = a * b, ph = mulhi64(a, b);
#endif
  lo += pl;
  hi += ph + (lo < pl);
}

// Gaussian integer (re + im i) mod p: exact product, result canonical.
// re = a0 b0 + a1 (p - b1), im = a0 b1 + a1 b0, each < 2 p^2 < min(2^127, p 2^64),
// reduced by red128.
CP_HD void gi_mul(uint64_t& cr, uint64_t& ci, uint64_t a0, uint64_t a1, uint64_t b0,
                  uint64_t b1, const ModConst& m) {
  uint64_t rh = 0, rl = 0, ih = 0, il = 0;
  mac128(rh, rl, a0, b0);
  mac128(rh, rl, a1, b1 == 0 ? 0 : m.p - b1);
  mac128(ih, il, a0, b1);
  mac128(ih, il, a1, b0);
  cr = red128(rh, rl, m);
  ci = red128(ih, il, m);
}

// Gaussian times a Gaussian constant with Shoup companions (4 shoup products).
CP_HD void gi_mul_const(uint64_t& xr, uint64_t& xi, uint64_t wr, uint64_t wrs, uint64_t wi,
                        uint64_t wis, uint64_t p) {
  uint64_t a = shoup_mul(xr, wr, wrs, p);
  uint64_t b = shoup_mul(xi, wi, wis, p);
  uint64_t c = shoup_mul(xr, wi, wis, p);
  uint64_t d = shoup_mul(xi, wr, wrs, p);
  xr = sub_mod(a, b, p);
  xi = add_mod(c, d, p);
}

// ---------------------------------------------------------------------------
// Host-side helpers (table construction)
// ---------------------------------------------------------------------------
inline uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t p) {
  return (uint64_t)((unsigned __int128)a * b % p);
}
inline uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t p) {
  uint64_t r = 1 % p;
  a %= p;
  while (e) {
    if (e & 1) r = h_mulmod(r, a, p);
    a = h_mulmod(a, a, p);
    e >>= 1;
  }
  return r;
}
inline uint64_t h_invmod(uint64_t a, uint64_t p) { return h_powmod(a, p - 2, p); }
inline uint64_t h_shoup(uint64_t w, uint64_t p) {
  return (uint64_t)(((unsigned __int128)w << 64) / p);
}
inline ModConst h_modconst(uint64_t p) {
  ModConst m;
  m.p = p;
  uint64_t inv = 1;  // Newton iteration for p^-1 mod 2^64
  for (int i = 0; i < 7; ++i) inv *= 2 - p * inv;
  m.pneg = (uint64_t)0 - inv;
  m.r1 = (uint64_t)(((unsigned __int128)1 << 64) % p);
  m.r1s = h_shoup(m.r1, p);
  m.r2 = h_mulmod(m.r1, m.r1, p);
  m.pm = (p >> 63) == 0 && (1ull << 63) - p < (1ull << 31) - 1;
  return m;
}

}  // namespace cpoly
