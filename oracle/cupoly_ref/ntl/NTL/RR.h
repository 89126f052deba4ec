// TEST INFRASTRUCTURE, not product code.  Part of the recipe that compiles
// cuPoly's own sources into oracle/_ref/ (see ZZ.h beside this file).
//
// The subset of NTL's RR that cuPoly's precomputation uses: RR::SetPrecision,
// to_RR of integers, + - * /, floor, FloorToZZ, conversion to ZZ and to
// uint64_t (src/cuda/cudaengine.cu:1463-1510, src/cuda/dgt.cu:1755-1766), and
// sqrt for poly_norm_2 (src/arithmetic/polynomial.cu:1472-1487).
//
// Semantics follow NTL's documentation of RR: a value is x * 2^e with x a ZZ;
// every arithmetic result and every conversion into RR is the exact value
// rounded to the current precision p (bits of x), to nearest with ties to even.
// Conversion of an RR to ZZ (conv, to_ZZ, FloorToZZ) takes the floor.
// The precision matters to cuPoly: its HPS fractions are the fractional parts
// of t (QB/q_i)^-1 B / q_i rounded at 512 bits, so when that quotient has more
// than 384 integer bits, the low bits of its 128-bit fraction are the rounded
// quotient's, not the exact value's.
#pragma once
#include <NTL/ZZ.h>

#include <cmath>
#include <iostream>

namespace NTL {

class RR {
 public:
  RR() = default;

  static void SetPrecision(long p) { prec_ref() = p < 53 ? 53 : p; }
  static long precision() { return prec_ref(); }
  static void SetOutputPrecision(long) {}

  // Exact value m 2^e rounded to the current precision.
  static RR make(const ZZ& m, long e, bool sticky = false) {
    RR r;
    r.x_ = m;
    r.e_ = e;
    r.round_to(precision(), sticky);
    return r;
  }
  const ZZ& mantissa() const { return x_; }
  long exponent() const { return e_; }

  friend RR operator+(const RR& a, const RR& b) {
    if (IsZero(a.x_)) return make(b.x_, b.e_);
    if (IsZero(b.x_)) return make(a.x_, a.e_);
    const long e = a.e_ < b.e_ ? a.e_ : b.e_;
    return make((a.x_ << (a.e_ - e)) + (b.x_ << (b.e_ - e)), e);
  }
  friend RR operator-(const RR& a) {
    RR r = a;
    r.x_ = -r.x_;
    return r;
  }
  friend RR operator-(const RR& a, const RR& b) { return a + (-b); }
  friend RR operator*(const RR& a, const RR& b) { return make(a.x_ * b.x_, a.e_ + b.e_); }
  // Quotient to precision + 2 bits plus a sticky bit for the remainder, then
  // rounded once: the correctly rounded quotient.
  friend RR operator/(const RR& a, const RR& b) {
    if (IsZero(b.x_)) throw std::domain_error("RR: division by zero");
    if (IsZero(a.x_)) return RR();
    const ZZ na = abs(a.x_), nb = abs(b.x_);
    long s = precision() + 2 + NumBits(nb) - NumBits(na);
    if (s < 0) s = 0;
    const ZZ num = na << s;
    const ZZ q = num / nb, r = num - q * nb;
    const bool neg = (sign(a.x_) < 0) != (sign(b.x_) < 0);
    return make(neg ? -q : q, a.e_ - b.e_ - s, !IsZero(r));
  }
  RR& operator+=(const RR& b) { return *this = *this + b; }
  RR& operator-=(const RR& b) { return *this = *this - b; }
  RR& operator*=(const RR& b) { return *this = *this * b; }
  RR& operator/=(const RR& b) { return *this = *this / b; }

  friend bool operator==(const RR& a, const RR& b) { return a.x_ == b.x_ && a.e_ == b.e_; }
  friend bool operator!=(const RR& a, const RR& b) { return !(a == b); }
  friend bool operator<(const RR& a, const RR& b) { return sign((a - b).x_) < 0; }
  friend bool operator>(const RR& a, const RR& b) { return b < a; }

  // floor(x 2^e) as an integer.
  ZZ floor_zz() const {
    if (e_ >= 0) return x_ << e_;
    const ZZ one(1);
    const ZZ m = abs(x_);
    ZZ q = m >> (-e_);
    if (sign(x_) < 0) {
      const bool exact = (q << (-e_)) == m;
      q = -q;
      if (!exact) q = q - one;
    }
    return q;
  }
  double to_double() const {
    // Nearest double, computed from the top 64 bits of the mantissa.
    if (IsZero(x_)) return 0.0;
    const long nb = NumBits(x_);
    const long sh = nb > 64 ? nb - 64 : 0;
    unsigned long w;
    conv(w, abs(x_) >> sh);
    const double v = std::ldexp((double)w, (int)(e_ + sh));
    return sign(x_) < 0 ? -v : v;
  }

 private:
  static long& prec_ref() {
    static long p = 150;  // NTL's default precision
    return p;
  }
  // Round the magnitude of x to p bits, nearest, ties to even; `sticky` says
  // that nonzero bits below x were already dropped (a division's remainder).
  void round_to(long p, bool sticky) {
    if (IsZero(x_)) {
      e_ = 0;
      return;
    }
    const bool neg = sign(x_) < 0;
    ZZ m = abs(x_);
    const long nb = NumBits(m);
    if (nb > p) {
      const long drop = nb - p;
      const ZZ kept = m >> drop;
      const ZZ rest = m - (kept << drop);
      const ZZ half = ZZ(1) << (drop - 1);
      bool up = false;
      if (rest > half) {
        up = true;
      } else if (rest == half) {
        up = sticky || !IsZero(kept % ZZ(2));
      }
      m = up ? kept + ZZ(1) : kept;
      e_ += drop;
    } else if (sticky) {
      // Fewer than p bits with a nonzero tail cannot occur: the quotient
      // carries p + 2 bits before rounding.
    }
    // Normalise: odd mantissa (zero is (0, 0)).
    while (!IsZero(m) && IsZero(m % ZZ(2))) {
      m = m >> 1;
      ++e_;
    }
    x_ = neg ? -m : m;
  }

  ZZ x_;
  long e_ = 0;
};

inline RR to_RR(const ZZ& a) { return RR::make(a, 0); }
inline RR to_RR(long a) { return RR::make(ZZ(a), 0); }
inline RR to_RR(int a) { return RR::make(ZZ(a), 0); }
inline RR to_RR(unsigned long a) { return RR::make(ZZ(a), 0); }
inline RR to_RR(unsigned long long a) { return RR::make(ZZ(a), 0); }
inline RR to_RR(unsigned a) { return RR::make(ZZ(a), 0); }
inline RR to_RR(double d) {
  if (d == 0.0) return RR();
  int ex;
  const double f = std::frexp(d, &ex);
  const long long m = (long long)std::ldexp(f, 53);
  return RR::make(ZZ(m), (long)ex - 53);
}

inline RR floor(const RR& a) { return RR::make(a.floor_zz(), 0); }
inline ZZ FloorToZZ(const RR& a) { return a.floor_zz(); }
inline ZZ to_ZZ(const RR& a) { return a.floor_zz(); }
inline void conv(ZZ& z, const RR& a) { z = a.floor_zz(); }
inline void conv(unsigned long& x, const RR& a) { conv(x, a.floor_zz()); }
inline void conv(long& x, const RR& a) { x = to_long_low(a.floor_zz()); }
inline void conv(double& x, const RR& a) { x = a.to_double(); }
inline void conv(RR& z, const ZZ& a) { z = to_RR(a); }
inline double to_double(const RR& a) { return a.to_double(); }

// Square root rounded to the current precision (used only by cuPoly's norm
// helper): isqrt of the mantissa scaled to 2p + 2 bits, then one rounding.
inline RR sqrt(const RR& a) {
  if (IsZero(a.mantissa())) return RR();
  if (sign(a.mantissa()) < 0) throw std::domain_error("RR: sqrt of a negative value");
  ZZ m = a.mantissa();
  long e = a.exponent();
  long shift = 2 * RR::precision() + 4 - NumBits(m);
  if (shift < 0) shift = 0;
  if ((e - shift) % 2) ++shift;
  m = m << shift;
  e -= shift;
  // Newton iteration for floor(sqrt(m)).
  ZZ y = ZZ(1) << ((NumBits(m) + 1) / 2);
  for (;;) {
    const ZZ z = (y + m / y) >> 1;
    if (z >= y) break;
    y = z;
  }
  return RR::make(y, e / 2, y * y != m);
}

inline std::ostream& operator<<(std::ostream& os, const RR& a) { return os << a.to_double(); }

}  // namespace NTL
