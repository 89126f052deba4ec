// Arbitrary-precision signed integer for the cuPoly compatibility layer.
//
// cuPoly's public API carries NTL's ZZ (poly_set_coeff / poly_get_coeff,
// CUDAEngine::RNSProduct; include/cuPoly/arithmetic/polynomial.h:461-470,
// include/cuPoly/cuda/cudaengine.h:87-95).  NTL is not a dependency here:
// this header supplies the subset of ZZ those signatures and cuPoly-style
// test code use (construction from machine integers and decimal strings,
// + - * / %, comparisons, shifts, stream I/O, NumBits, power, conv<...>,
// to_ZZ).  Division and remainder follow NTL's floor convention: the
// remainder takes the sign of the divisor.  Shifts act on the magnitude and
// keep the sign.
//
// Representation: sign and magnitude, magnitude as little-endian 64-bit
// limbs with no leading zero limb (zero = no limbs, never negative).
// Division is Knuth's Algorithm D (TAOCP vol. 2, 4.3.1) on 64-bit digits.
#pragma once
#include <algorithm>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

// The class lives in namespace cupoly unless the includer defines
// CUPOLY_ZZ_NAMESPACE first (the build of cuPoly's own sources under oracle/
// places it in namespace NTL, beside its RR).
#ifndef CUPOLY_ZZ_NAMESPACE
#define CUPOLY_ZZ_NAMESPACE cupoly
#endif

namespace CUPOLY_ZZ_NAMESPACE {

class ZZ {
 public:
  using limb = uint64_t;
  using mag_t = std::vector<limb>;

  ZZ() = default;
  ZZ(int v) : ZZ((long long)v) {}
  ZZ(long v) : ZZ((long long)v) {}
  ZZ(long long v) {
    if (v < 0) {
      neg_ = true;
      mag_.push_back(limb(0) - limb(v));
    } else if (v > 0) {
      mag_.push_back(limb(v));
    }
  }
  ZZ(unsigned v) : ZZ((unsigned long long)v) {}
  ZZ(unsigned long v) : ZZ((unsigned long long)v) {}
  ZZ(unsigned long long v) {
    if (v) mag_.push_back(limb(v));
  }

  // Magnitude from n little-endian limbs, with a sign.
  static ZZ from_limbs(const limb* w, size_t n, bool negative = false) {
    ZZ r;
    r.mag_.assign(w, w + n);
    trim(r.mag_);
    r.neg_ = negative && !r.mag_.empty();
    return r;
  }
  static ZZ from_string(const std::string& s) {
    size_t i = 0;
    bool negative = false;
    while (i < s.size() && isspace((unsigned char)s[i])) ++i;
    if (i < s.size() && (s[i] == '-' || s[i] == '+')) negative = s[i++] == '-';
    if (i >= s.size() || !isdigit((unsigned char)s[i])) throw std::invalid_argument("ZZ: not a decimal integer: " + s);
    ZZ r;
    while (i < s.size() && isdigit((unsigned char)s[i])) {
      limb chunk = 0, scale = 1;
      for (int d = 0; d < 19 && i < s.size() && isdigit((unsigned char)s[i]); ++d, ++i) {
        chunk = chunk * 10 + limb(s[i] - '0');
        scale *= 10;
      }
      mul_small_add(r.mag_, scale, chunk);
    }
    r.neg_ = negative && !r.mag_.empty();
    return r;
  }

  const mag_t& limbs() const { return mag_; }
  bool is_negative() const { return neg_; }
  bool is_zero() const { return mag_.empty(); }
  int sign() const { return mag_.empty() ? 0 : (neg_ ? -1 : 1); }
  long num_bits() const {
    if (mag_.empty()) return 0;
    return long(64 * (mag_.size() - 1)) + (64 - __builtin_clzll(mag_.back()));
  }

  std::string to_string() const {
    if (mag_.empty()) return "0";
    mag_t m = mag_;
    std::vector<limb> chunks;  // base 10^19, least significant first
    while (!m.empty()) chunks.push_back(div_small(m, 10000000000000000000ull));
    std::string s = neg_ ? "-" : "";
    s += std::to_string(chunks.back());
    for (size_t i = chunks.size() - 1; i-- > 0;) {
      std::string c = std::to_string(chunks[i]);
      s += std::string(19 - c.size(), '0') + c;
    }
    return s;
  }

  // ---- arithmetic ----
  friend ZZ operator-(const ZZ& a) {
    ZZ r = a;
    r.neg_ = !r.mag_.empty() && !a.neg_;
    return r;
  }
  friend ZZ operator+(const ZZ& a, const ZZ& b) { return add_signed(a, b.neg_, b.mag_); }
  friend ZZ operator-(const ZZ& a, const ZZ& b) { return add_signed(a, !b.neg_ && !b.mag_.empty(), b.mag_); }
  friend ZZ operator*(const ZZ& a, const ZZ& b) {
    ZZ r;
    r.mag_ = mul(a.mag_, b.mag_);
    r.neg_ = !r.mag_.empty() && (a.neg_ != b.neg_);
    return r;
  }
  // Floor division: q = floor(a / b), r = a - q b (sign of b).
  static void divide(ZZ& q, ZZ& r, const ZZ& a, const ZZ& b) {
    if (b.mag_.empty()) throw std::domain_error("ZZ: division by zero");
    mag_t qm, rm;
    divmod(a.mag_, b.mag_, qm, rm);
    ZZ qq, rr;
    qq.mag_ = std::move(qm);
    qq.neg_ = !qq.mag_.empty() && (a.neg_ != b.neg_);
    rr.mag_ = std::move(rm);
    rr.neg_ = !rr.mag_.empty() && a.neg_;
    if (!rr.mag_.empty() && rr.neg_ != b.neg_) {  // truncated -> floor
      qq = qq - ZZ(1);
      rr = rr + b;
    }
    q = std::move(qq);
    r = std::move(rr);
  }
  friend ZZ operator/(const ZZ& a, const ZZ& b) {
    ZZ q, r;
    divide(q, r, a, b);
    return q;
  }
  friend ZZ operator%(const ZZ& a, const ZZ& b) {
    ZZ q, r;
    divide(q, r, a, b);
    return r;
  }
  friend ZZ operator<<(const ZZ& a, long n) {
    if (n < 0) return a >> -n;
    ZZ r;
    r.mag_ = shl(a.mag_, (size_t)n);
    r.neg_ = a.neg_ && !r.mag_.empty();
    return r;
  }
  friend ZZ operator>>(const ZZ& a, long n) {
    if (n < 0) return a << -n;
    ZZ r;
    r.mag_ = shr(a.mag_, (size_t)n);
    r.neg_ = a.neg_ && !r.mag_.empty();
    return r;
  }
  ZZ& operator+=(const ZZ& b) { return *this = *this + b; }
  ZZ& operator-=(const ZZ& b) { return *this = *this - b; }
  ZZ& operator*=(const ZZ& b) { return *this = *this * b; }
  ZZ& operator/=(const ZZ& b) { return *this = *this / b; }
  ZZ& operator%=(const ZZ& b) { return *this = *this % b; }
  ZZ& operator<<=(long n) { return *this = *this << n; }
  ZZ& operator>>=(long n) { return *this = *this >> n; }
  ZZ& operator++() { return *this = *this + ZZ(1); }
  ZZ& operator--() { return *this = *this - ZZ(1); }

  // ---- comparison ----
  static int compare(const ZZ& a, const ZZ& b) {
    if (a.neg_ != b.neg_) return a.neg_ ? -1 : 1;
    const int c = cmp(a.mag_, b.mag_);
    return a.neg_ ? -c : c;
  }
  friend bool operator==(const ZZ& a, const ZZ& b) { return a.neg_ == b.neg_ && a.mag_ == b.mag_; }
  friend bool operator!=(const ZZ& a, const ZZ& b) { return !(a == b); }
  friend bool operator<(const ZZ& a, const ZZ& b) { return compare(a, b) < 0; }
  friend bool operator>(const ZZ& a, const ZZ& b) { return compare(a, b) > 0; }
  friend bool operator<=(const ZZ& a, const ZZ& b) { return compare(a, b) <= 0; }
  friend bool operator>=(const ZZ& a, const ZZ& b) { return compare(a, b) >= 0; }

  friend std::ostream& operator<<(std::ostream& os, const ZZ& a) { return os << a.to_string(); }
  friend std::istream& operator>>(std::istream& is, ZZ& a) {
    std::string s;
    if (is >> s) a = from_string(s);
    return is;
  }

 private:
  bool neg_ = false;
  mag_t mag_;

  static void trim(mag_t& m) {
    while (!m.empty() && m.back() == 0) m.pop_back();
  }
  static int cmp(const mag_t& a, const mag_t& b) {
    if (a.size() != b.size()) return a.size() < b.size() ? -1 : 1;
    for (size_t i = a.size(); i-- > 0;)
      if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
  }
  static mag_t add(const mag_t& a, const mag_t& b) {
    const mag_t& x = a.size() >= b.size() ? a : b;
    const mag_t& y = a.size() >= b.size() ? b : a;
    mag_t r(x.size() + 1, 0);
    unsigned __int128 c = 0;
    for (size_t i = 0; i < x.size(); ++i) {
      c += (unsigned __int128)x[i] + (i < y.size() ? y[i] : 0);
      r[i] = (limb)c;
      c >>= 64;
    }
    r[x.size()] = (limb)c;
    trim(r);
    return r;
  }
  static mag_t sub(const mag_t& a, const mag_t& b) {  // requires a >= b
    mag_t r(a.size(), 0);
    limb borrow = 0;
    for (size_t i = 0; i < a.size(); ++i) {
      const unsigned __int128 d = (unsigned __int128)a[i] - (i < b.size() ? b[i] : 0) - borrow;
      r[i] = (limb)d;
      borrow = (limb)(d >> 64) ? 1 : 0;
    }
    trim(r);
    return r;
  }
  static ZZ add_signed(const ZZ& a, bool bneg, const mag_t& bm) {
    ZZ r;
    if (a.neg_ == bneg) {
      r.mag_ = add(a.mag_, bm);
      r.neg_ = a.neg_;
    } else if (cmp(a.mag_, bm) >= 0) {
      r.mag_ = sub(a.mag_, bm);
      r.neg_ = a.neg_;
    } else {
      r.mag_ = sub(bm, a.mag_);
      r.neg_ = bneg;
    }
    r.neg_ = r.neg_ && !r.mag_.empty();
    return r;
  }
  static mag_t mul(const mag_t& a, const mag_t& b) {
    if (a.empty() || b.empty()) return {};
    mag_t r(a.size() + b.size(), 0);
    for (size_t i = 0; i < a.size(); ++i) {
      unsigned __int128 c = 0;
      for (size_t j = 0; j < b.size(); ++j) {
        c += (unsigned __int128)a[i] * b[j] + r[i + j];
        r[i + j] = (limb)c;
        c >>= 64;
      }
      r[i + b.size()] = (limb)c;
    }
    trim(r);
    return r;
  }
  static void mul_small_add(mag_t& m, limb s, limb add) {
    unsigned __int128 c = add;
    for (auto& w : m) {
      c += (unsigned __int128)w * s;
      w = (limb)c;
      c >>= 64;
    }
    if (c) m.push_back((limb)c);
    trim(m);
  }
  static limb div_small(mag_t& m, limb d) {  // m <- m / d, returns m mod d
    unsigned __int128 rem = 0;
    for (size_t i = m.size(); i-- > 0;) {
      const unsigned __int128 cur = (rem << 64) | m[i];
      m[i] = (limb)(cur / d);
      rem = cur % d;
    }
    trim(m);
    return (limb)rem;
  }
  static mag_t shl(const mag_t& a, size_t n) {
    if (a.empty()) return {};
    const size_t w = n / 64, b = n % 64;
    mag_t r(a.size() + w + 1, 0);
    for (size_t i = 0; i < a.size(); ++i) {
      r[i + w] |= a[i] << b;
      if (b) r[i + w + 1] |= a[i] >> (64 - b);
    }
    trim(r);
    return r;
  }
  static mag_t shr(const mag_t& a, size_t n) {
    const size_t w = n / 64, b = n % 64;
    if (w >= a.size()) return {};
    mag_t r(a.size() - w, 0);
    for (size_t i = 0; i < r.size(); ++i) {
      r[i] = a[i + w] >> b;
      if (b && i + w + 1 < a.size()) r[i] |= a[i + w + 1] << (64 - b);
    }
    trim(r);
    return r;
  }
  // |u| = q |v| + r, 0 <= r < |v| (Knuth D with 64-bit digits).
  static void divmod(const mag_t& u_in, const mag_t& v_in, mag_t& q, mag_t& r) {
    if (cmp(u_in, v_in) < 0) {
      q.clear();
      r = u_in;
      return;
    }
    if (v_in.size() == 1) {
      q = u_in;
      const limb rem = div_small(q, v_in[0]);
      r.clear();
      if (rem) r.push_back(rem);
      return;
    }
    const int s = __builtin_clzll(v_in.back());
    mag_t v = shl(v_in, (size_t)s);
    mag_t u = shl(u_in, (size_t)s);
    u.resize(u_in.size() + 1, 0);
    const size_t n = v.size(), m = u.size() - n;
    q.assign(m, 0);
    for (size_t j = m; j-- > 0;) {
      const unsigned __int128 num = ((unsigned __int128)u[j + n] << 64) | u[j + n - 1];
      unsigned __int128 qhat = num / v[n - 1];
      unsigned __int128 rhat = num % v[n - 1];
      while ((qhat >> 64) != 0 || qhat * v[n - 2] > ((rhat << 64) | u[j + n - 2])) {
        --qhat;
        rhat += v[n - 1];
        if ((rhat >> 64) != 0) break;
      }
      limb carry = 0, borrow = 0;
      for (size_t i = 0; i < n; ++i) {
        const unsigned __int128 p = qhat * v[i] + carry;
        carry = (limb)(p >> 64);
        const unsigned __int128 d = (unsigned __int128)u[i + j] - (limb)p - borrow;
        u[i + j] = (limb)d;
        borrow = (limb)(d >> 64) ? 1 : 0;
      }
      const unsigned __int128 d = (unsigned __int128)u[j + n] - carry - borrow;
      u[j + n] = (limb)d;
      if ((limb)(d >> 64) != 0) {  // qhat was one too large: add v back
        --qhat;
        unsigned __int128 c = 0;
        for (size_t i = 0; i < n; ++i) {
          c += (unsigned __int128)u[i + j] + v[i];
          u[i + j] = (limb)c;
          c >>= 64;
        }
        u[j + n] += (limb)c;
      }
      q[j] = (limb)qhat;
    }
    trim(q);
    u.resize(n);
    r = shr(u, (size_t)s);
  }
};

inline ZZ to_ZZ(long long v) { return ZZ(v); }
inline ZZ to_ZZ(int v) { return ZZ(v); }
inline ZZ to_ZZ(long v) { return ZZ(v); }
inline ZZ to_ZZ(unsigned v) { return ZZ(v); }
inline ZZ to_ZZ(unsigned long v) { return ZZ(v); }
inline ZZ to_ZZ(unsigned long long v) { return ZZ(v); }
inline ZZ to_ZZ(const char* s) { return ZZ::from_string(s); }
inline ZZ to_ZZ(const std::string& s) { return ZZ::from_string(s); }

inline long NumBits(const ZZ& a) { return a.num_bits(); }
inline bool IsZero(const ZZ& a) { return a.is_zero(); }
inline long sign(const ZZ& a) { return a.sign(); }
inline ZZ abs(const ZZ& a) { return a.is_negative() ? -a : a; }
inline ZZ power2_ZZ(long n) { return ZZ(1) << n; }
inline ZZ power(const ZZ& a, long e) {
  if (e < 0) throw std::domain_error("ZZ: negative exponent");
  ZZ r(1), b = a;
  for (; e; e >>= 1) {
    if (e & 1) r *= b;
    if (e > 1) b *= b;
  }
  return r;
}
// Value of a in (-2^63, 2^64) as a machine integer; throws outside.
inline long to_long(const ZZ& a) {
  if (a.limbs().size() > 1 || (!a.limbs().empty() && a.limbs()[0] >> 63))
    throw std::overflow_error("ZZ: value does not fit a long");
  const long m = a.limbs().empty() ? 0 : (long)a.limbs()[0];
  return a.is_negative() ? -m : m;
}
inline unsigned long to_ulong(const ZZ& a) {
  if (a.is_negative() || a.limbs().size() > 1) throw std::overflow_error("ZZ: value does not fit an unsigned long");
  return a.limbs().empty() ? 0ul : (unsigned long)a.limbs()[0];
}

// NTL-style conversions: conv(x, a) and T x = conv<T>(a).
inline void conv(ZZ& x, long a) { x = ZZ(a); }
inline void conv(ZZ& x, int a) { x = ZZ(a); }
inline void conv(ZZ& x, unsigned long a) { x = ZZ(a); }
inline void conv(ZZ& x, unsigned long long a) { x = ZZ(a); }
inline void conv(ZZ& x, long long a) { x = ZZ(a); }
inline void conv(ZZ& x, const char* s) { x = ZZ::from_string(s); }
inline void conv(ZZ& x, const std::string& s) { x = ZZ::from_string(s); }
inline void conv(ZZ& x, const ZZ& a) { x = a; }
inline void conv(long& x, const ZZ& a) { x = to_long(a); }
#ifdef CUPOLY_ZZ_LOW_WORD_CONV
// NTL's rule for a machine-word conversion: the low-order 64 bits of a (two's
// complement for a negative a), whatever a's size.
inline void conv(unsigned long& x, const ZZ& a) {
  const unsigned long w = a.limbs().empty() ? 0ul : (unsigned long)a.limbs()[0];
  x = a.is_negative() ? 0ul - w : w;
}
#else
inline void conv(unsigned long& x, const ZZ& a) { x = to_ulong(a); }
#endif
template <class T, class S>
inline T conv(const S& a) {
  T x;
  conv(x, a);
  return x;
}

}  // namespace CUPOLY_ZZ_NAMESPACE
