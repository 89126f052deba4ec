// TEST INFRASTRUCTURE, not product code.  Part of the recipe that compiles
// cuPoly's own sources (pdroalves/cupoly 0.3.5) into oracle/_ref/ so that
// their outputs pin the oracle and the CUDA path.
//
// NTL is not installed here.  cuPoly's library sources use a small part of
// NTL's ZZ (src/cuda/cudaengine.cu:1234-1510, src/cuda/dgt.cu:1657-1766,
// src/arithmetic/polynomial.cu:190-296): construction, + - * / % << >>,
// comparisons, stream output, conv<uint64_t>, to_ZZ, NumBits, power, InvMod.
// This header supplies that subset with NTL's documented meaning, on the
// in-repo big integer (include/cuPoly/zz.h) placed in namespace NTL:
//   * / and % round the quotient toward minus infinity (NTL's floor rule);
//   * conv<unsigned long>(a) keeps the low-order 64 bits of a;
//   * InvMod(a, n) is the inverse of a mod n in [0, n), an error when
//     gcd(a, n) != 1.
#pragma once
#define CUPOLY_ZZ_NAMESPACE NTL
#define CUPOLY_ZZ_LOW_WORD_CONV 1
#include "../../../../include/cuPoly/zz.h"

#include <stdexcept>

namespace NTL {

// Inverse of a modulo n (n > 1), by the extended Euclidean algorithm.
inline ZZ InvMod(const ZZ& a, const ZZ& n) {
  if (n <= ZZ(1)) throw std::invalid_argument("InvMod: modulus must exceed 1");
  ZZ r0 = n, r1 = a % n, s0(0), s1(1);
  while (!IsZero(r1)) {
    const ZZ q = r0 / r1;
    ZZ t = r0 - q * r1;
    r0 = r1;
    r1 = t;
    t = s0 - q * s1;
    s0 = s1;
    s1 = t;
  }
  if (r0 != ZZ(1)) throw std::invalid_argument("InvMod: not invertible");
  return s0 % n;
}

inline ZZ PowerMod(const ZZ& a, const ZZ& e, const ZZ& n) {
  ZZ r(1), b = a % n, x = e;
  while (!IsZero(x)) {
    if (!IsZero(x % ZZ(2))) r = r * b % n;
    b = b * b % n;
    x = x >> 1;
  }
  return r % n;
}

inline ZZ to_ZZ(const ZZ& a) { return a; }

// NTL's remainder by a machine word is itself a machine word (rem(a, b) in
// [0, b) for b > 0): cuPoly assigns `ZZ % uint64_t` straight to uint64_t
// fields (src/arithmetic/polynomial.cu:210-216, src/cuda/cudaengine.cu:1408).
inline long operator%(const ZZ& a, long b) {
  unsigned long w;
  conv(w, a % ZZ(b));
  return (long)w;
}
inline long operator%(const ZZ& a, unsigned long b) { return a % (long)b; }
inline long operator%(const ZZ& a, int b) { return a % (long)b; }
inline ZZ operator/(const ZZ& a, long b) { return a / ZZ(b); }
inline ZZ operator/(const ZZ& a, unsigned long b) { return a / ZZ(b); }
inline ZZ operator/(const ZZ& a, int b) { return a / ZZ((long)b); }
inline void conv(unsigned long& x, long a) { x = (unsigned long)a; }

inline long to_long_low(const ZZ& a) {
  unsigned long w;
  conv(w, a);
  return (long)w;
}
inline void conv(unsigned long long& x, const ZZ& a) {
  unsigned long w;
  conv(w, a);
  x = w;
}
inline void conv(int& x, const ZZ& a) { x = (int)to_long_low(a); }
inline void conv(unsigned& x, const ZZ& a) { x = (unsigned)to_long_low(a); }

}  // namespace NTL

#ifndef NTL_CLIENT
#define NTL_CLIENT \
  using namespace std; \
  using namespace NTL;
#endif
