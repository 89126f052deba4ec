// Host-side construction of an engine's device tables.
//
// Replaces cuPoly's DGTEngine::init / compute_gjk / compute_nthroot
// (src/cuda/dgt.cu:1501-1982) and CUDAEngine::precompute
// (src/cuda/cudaengine.cu:1337-1673).  All constants are computed here from
// the primes and their primitive roots with 128-bit integer arithmetic; no
// multi-precision library is needed because the HPS step is done by exact
// mixed-radix conversion, whose constants are single-word residues.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>

#include "engine.cuh"
#include "prime_table.h"

namespace cpoly {

namespace {
thread_local std::string g_last_error;

uint64_t omega(uint64_t p, uint64_t g, uint64_t n) { return h_powmod(g, (p - 1) / n, p); }

int brev(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) {
    r = (r << 1) | (x & 1);
    x >>= 1;
  }
  return r;
}

// Gaussian arithmetic on the host.
struct G {
  uint64_t re, im;
};
G gmul(G a, G b, uint64_t p) {
  uint64_t r = (uint64_t)(((unsigned __int128)a.re * b.re + (unsigned __int128)a.im * (b.im ? p - b.im : 0)) % p);
  uint64_t i = (uint64_t)(((unsigned __int128)a.re * b.im + (unsigned __int128)a.im * b.re) % p);
  return {r, i};
}
G gpow(G a, uint64_t e, uint64_t p) {
  G r{1, 0};
  while (e) {
    if (e & 1) r = gmul(r, a, p);
    a = gmul(a, a, p);
    e >>= 1;
  }
  return r;
}

// Extended Euclid inverse of a modulo m (m need not be prime); 0 if none.
uint64_t inv_general(uint64_t a, uint64_t m) {
  __int128 t = 0, nt = 1, r = m, nr = a % m;
  while (nr != 0) {
    __int128 q = r / nr;
    __int128 tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  if (r != 1) return 0;
  if (t < 0) t += m;
  return (uint64_t)t;
}

uint64_t shoup_general(uint64_t w, uint64_t m) {
  return (uint64_t)(((unsigned __int128)w << 64) / m);
}

// Mixed-radix digits of the value with residues r_i over primes s_i.
std::vector<uint64_t> mrc_digits(const std::vector<uint64_t>& r, const std::vector<uint64_t>& s) {
  size_t n = s.size();
  std::vector<uint64_t> d(n);
  for (size_t i = 0; i < n; ++i) {
    uint64_t y = r[i] % s[i];
    for (size_t l = 0; l < i; ++l) {
      uint64_t dl = d[l] % s[i];
      y = (y + s[i] - dl) % s[i];
      y = h_mulmod(y, h_invmod(s[l] % s[i], s[i]), s[i]);
    }
    d[i] = y;
  }
  return d;
}

// Mixed-radix digits of T - 1 for the lift threshold T = S - floor(S F) of the
// base s (S = prod s_i; F = 4835703278458517 / 2^82, the double nearest 1e-9,
// cuPoly's FPERROR).  cuPoly lifts X in [0, S) to X - S exactly when its double
// sum of X / S lands within FPERROR of 1 (src/cuda/cudaengine.cu:513-534,
// 690-703), i.e. when S - X <= S F: X >= T.  The kernels test X > T - 1 on the
// digits.
std::vector<uint64_t> lift_threshold_digits(const std::vector<uint64_t>& s) {
  std::vector<uint64_t> S{1};
  auto mul_word = [](std::vector<uint64_t>& a, uint64_t w) {
    unsigned __int128 carry = 0;
    for (auto& x : a) {
      const unsigned __int128 t = (unsigned __int128)x * w + carry;
      x = (uint64_t)t;
      carry = t >> 64;
    }
    if (carry) a.push_back((uint64_t)carry);
  };
  for (auto p : s) mul_word(S, p);
  mul_word(S, 4835703278458517ull);  // S F 2^82
  // U = floor(S F): shift right by 82 bits
  std::vector<uint64_t> U;
  const size_t w = 82 / 64, b = 82 % 64;
  for (size_t i = w; i < S.size(); ++i) {
    uint64_t v = S[i] >> b;
    if (i + 1 < S.size()) v |= S[i + 1] << (64 - b);
    U.push_back(v);
  }
  std::vector<uint64_t> r(s.size());
  for (size_t i = 0; i < s.size(); ++i) {
    unsigned __int128 acc = 0;  // U mod s_i, most significant limb first
    for (size_t l = U.size(); l-- > 0;) acc = ((acc << 64) | U[l]) % s[i];
    r[i] = s[i] - 1 - (uint64_t)acc;  // (T - 1) mod s_i = (-U - 1) mod s_i
  }
  return mrc_digits(r, s);
}

void parallel_for(int n, const std::function<void(int)>& f) {
  unsigned hw = std::thread::hardware_concurrency();
  int nt = (int)std::min<unsigned>(hw ? hw : 1, 16);
  if (n < 2 || nt < 2) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  std::atomic<int> next{0};
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&]() {
      for (int i = next++; i < n; i = next++) f(i);
    });
  for (auto& x : th) x.join();
}
}  // namespace

uint64_t primitive_root_of(uint64_t p) {
  for (int i = 0; i < kNumPrimes; ++i)
    if (kPrimes[i] == p) return kPrimitiveRoots[i];
  return 0;
}

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

int Engine::n_residues(int base) const {
  switch (base) {
    case 0: return k;          // Q
    case 1: return kl;         // B
    case 2: return k + kl;     // QB
    case 3: return 1;          // T
    default: return -1;
  }
}
int Engine::rid_offset(int base) const { return base == 1 ? k : 0; }

DgtPlan make_plan(int logN, int logR, int logCta) {
  DgtPlan P;
  P.logN = logN;
  if (logCta <= 0 || logCta > kMaxLogNc) logCta = kMaxLogNc;
  P.logNc = logN < logCta ? logN : logCta;
  P.S = logN - P.logNc;
  P.logR = logR < P.logNc ? logR : P.logNc;
  while ((P.logNc - P.logR) > 10) ++P.logR;  // at most 1024 threads per CTA
  P.npass = (P.logNc + P.logR - 1) / P.logR;
  P.w[0] = P.logNc - (P.npass - 1) * P.logR;
  P.p[0] = P.logNc - P.w[0];
  for (int i = 1; i < P.npass; ++i) {
    P.w[i] = P.logR;
    P.p[i] = P.p[i - 1] - P.logR;
  }
  return P;
}

// Place a plan's radix, pass and split tables from entry `off` of a residue block;
// returns the next free entry.
static int place_plan(const DgtPlan& P, int N, DgtTableLayout& L, int off) {
  L.off_rad = off;
  off += 1 << P.logR;
  for (int i = 0; i < P.npass; ++i) {
    if (P.p[i] > 0) {
      L.off_fwd[i] = off;
      off += 1 << (P.p[i] + P.w[i]);
      L.off_inv[i] = off;
      off += 1 << (P.p[i] + P.w[i]);
    }
  }
  if (P.S > 0) {
    L.off_split_fwd = off;
    off += N;
    L.off_split_inv = off;
    off += N;
  }
  return off;
}

int build_tables(Engine& e) {
  const int nres = e.k + e.kl;
  const int N = e.N;
  const bool narrow = e.narrow_units > 0;
  DgtTableLayout& L = e.layout;
  DgtTableLayout& L2 = e.layout_narrow;
  L = DgtTableLayout{};
  L2 = DgtTableLayout{};
  int off = place_plan(e.plan, N, L, 0);
  if (narrow) off = place_plan(e.plan_narrow, N, L2, off);
  L.off_twist = off;
  off += 3 * N;
  L.off_untwist = off;
  off += 3 * N;
  for (int v = 0; v < 2; ++v) {
    L.off_untwist_pre[v] = off;
    off += 3 * N;
  }
  L.stride = (off + 1) & ~1;
  L2.off_twist = L.off_twist;
  L2.off_untwist = L.off_untwist;
  L2.off_untwist_pre[0] = L.off_untwist_pre[0];
  L2.off_untwist_pre[1] = L.off_untwist_pre[1];
  L2.stride = L.stride;

  // Per-residue factors of the prescaled untwist tables (off_untwist_pre):
  //   Q residue i: (Q/q_i)^-1 and t (Q/q_i)^-1 mod q_i;  B residue j: t Q^-1 (B/b_j)^-1 mod b_j and 1.
  std::vector<uint64_t> pre0(nres, 1), pre1(nres, 1);
  for (int r = 0; r < nres; ++r) {
    const uint64_t p = e.primes[r];
    const bool in_q = r < e.k;
    const int lo = in_q ? 0 : e.k, hi = in_q ? e.k : nres;
    uint64_t hat = 1 % p;  // S / s_r mod s_r, S the product of r's base
    for (int u = lo; u < hi; ++u)
      if (u != r) hat = h_mulmod(hat, e.primes[u] % p, p);
    const uint64_t hinv = h_invmod(hat, p), tp = e.t % p;
    if (in_q) {
      pre0[r] = hinv;
      pre1[r] = h_mulmod(tp, hinv, p);
    } else {
      uint64_t qm = 1 % p;
      for (int u = 0; u < e.k; ++u) qm = h_mulmod(qm, e.primes[u] % p, p);
      pre0[r] = h_mulmod(h_mulmod(tp, h_invmod(qm, p), p), hinv, p);
    }
  }

  std::vector<ulonglong2> tab((size_t)L.stride * nres);
  parallel_for(nres, [&](int r) {
    const uint64_t p = e.primes[r];
    ulonglong2* T = tab.data() + (size_t)r * L.stride;
    const uint64_t gen = e.roots[r];
    const uint64_t wN = omega(p, gen, (uint64_t)N);
    const uint64_t wNi = h_invmod(wN, p);
    // powers of w_N and w_N^-1
    std::vector<uint64_t> pw(N), pwi(N);
    pw[0] = pwi[0] = 1;
    for (int i = 1; i < N; ++i) {
      pw[i] = h_mulmod(pw[i - 1], wN, p);
      pwi[i] = h_mulmod(pwi[i - 1], wNi, p);
    }
    auto put = [&](int idx, uint64_t w) { T[idx] = make_ulonglong2(w, h_shoup(w, p)); };
    auto fill_plan = [&](const DgtPlan& P, const DgtTableLayout& Lp) {
      const int R = 1 << P.logR;
      const int Nc = 1 << P.logNc;
      for (int j = 0; j < R; ++j) put(Lp.off_rad + j, pw[(size_t)j * (N / R)]);
      for (int i = 0; i < P.npass; ++i) {
        if (P.p[i] == 0) continue;
        const int pp = P.p[i], ww = P.w[i];
        const int M = 1 << (pp + ww);
        const int step = N / M;  // w_M = w_N^step
        for (int pos = 0; pos < (1 << ww); ++pos) {
          const int kk = brev(pos, ww);
          for (int Lw = 0; Lw < (1 << pp); ++Lw) {
            const size_t e_ = (size_t)Lw * kk % M * step;
            put(Lp.off_fwd[i] + pos * (1 << pp) + Lw, pw[e_]);
            put(Lp.off_inv[i] + pos * (1 << pp) + Lw, pwi[e_]);
          }
        }
      }
      if (P.S > 0) {
        for (int pos = 0; pos < (1 << P.S); ++pos) {
          const int kk = brev(pos, P.S);
          for (int Lw = 0; Lw < Nc; ++Lw) {
            const size_t e_ = (size_t)Lw * kk % N;
            put(Lp.off_split_fwd + pos * Nc + Lw, pw[e_]);
            put(Lp.off_split_inv + pos * Nc + Lw, pwi[e_]);
          }
        }
      }
    };
    fill_plan(e.plan, L);
    if (narrow) fill_plan(e.plan_narrow, L2);
    // twist by xi^n and untwist by xi^-n * N^-1
    G xi{e.xi[r].first, e.xi[r].second};
    G xii = gpow(xi, 4 * (uint64_t)N - 1, p);
    const uint64_t ninv = h_invmod((uint64_t)N, p);
    G a{1, 0}, b{ninv, 0};
    // Karatsuba triples (w_re, w_im - w_re, w_re + w_im): three constant
    // products per Gaussian element instead of four.
    auto put_gauss = [&](int idx, G w) {
      put(idx, w.re);
      put(idx + 1, (w.im + p - w.re) % p);
      put(idx + 2, (uint64_t)(((unsigned __int128)w.re + w.im) % p));
    };
    const uint64_t f0 = pre0[r], f1 = pre1[r];
    for (int n = 0; n < N; ++n) {
      put_gauss(L.off_twist + 3 * n, a);
      put_gauss(L.off_untwist + 3 * n, b);
      put_gauss(L.off_untwist_pre[0] + 3 * n, G{h_mulmod(b.re, f0, p), h_mulmod(b.im, f0, p)});
      put_gauss(L.off_untwist_pre[1] + 3 * n, G{h_mulmod(b.re, f1, p), h_mulmod(b.im, f1, p)});
      a = gmul(a, xi, p);
      b = gmul(b, xii, p);
    }
  });

  // ---------------- HPS / mixed-radix constants ----------------
  std::vector<uint64_t> Q(e.primes.begin(), e.primes.begin() + e.k);
  std::vector<uint64_t> B(e.primes.begin() + e.k, e.primes.end());
  std::vector<uint64_t> H;  // packed words
  auto mark = [&]() { return (int)H.size(); };
  auto push_pair = [&](uint64_t w, uint64_t m, std::vector<uint64_t>& vals, std::vector<uint64_t>& comp) {
    vals.push_back(w);
    comp.push_back(shoup_general(w, m));
  };
  auto append = [&](const std::vector<uint64_t>& v) {
    int o = mark();
    H.insert(H.end(), v.begin(), v.end());
    return o;
  };
  // MRC inverse constants of a base s: inv[i*(i-1)/2 + l] = s_l^-1 mod s_i
  auto mrc_inv = [&](const std::vector<uint64_t>& s, std::vector<uint64_t>& v, std::vector<uint64_t>& c) {
    for (size_t i = 1; i < s.size(); ++i)
      for (size_t l = 0; l < i; ++l) push_pair(h_invmod(s[l] % s[i], s[i]), s[i], v, c);
  };
  // Horner constants: hor[j*(n-1) + i] = s_i mod m_j
  auto horner = [&](const std::vector<uint64_t>& s, const std::vector<uint64_t>& m, std::vector<uint64_t>& v,
                    std::vector<uint64_t>& c) {
    for (size_t j = 0; j < m.size(); ++j)
      for (size_t i = 0; i + 1 < s.size(); ++i) push_pair(s[i] % m[j], m[j], v, c);
  };
  auto prod_mod = [&](const std::vector<uint64_t>& s, uint64_t m) {
    uint64_t r = 1 % m;
    for (auto x : s) r = h_mulmod(r, x % m, m);
    return r;
  };
  {
    std::vector<uint64_t> v, c;
    mrc_inv(Q, v, c);
    e.ho.qb_inv = append(v);
    e.ho.qb_inv_s = append(c);
  }
  {
    std::vector<uint64_t> v, c;
    horner(Q, B, v, c);
    e.ho.qb_hor = append(v);
    e.ho.qb_hor_s = append(c);
  }
  {
    std::vector<uint64_t> half(Q.size());
    for (size_t i = 0; i < Q.size(); ++i) half[i] = (Q[i] - 1) / 2;  // (Q-1)/2 mod q_i
    e.ho.qb_half = append(mrc_digits(half, Q));
    e.ho.q_lift = append(lift_threshold_digits(Q));
    e.ho.b_lift = append(lift_threshold_digits(B));
  }
  {
    std::vector<uint64_t> v, c;
    mrc_inv(B, v, c);
    e.ho.bq_inv = append(v);
    e.ho.bq_inv_s = append(c);
  }
  {
    std::vector<uint64_t> v, c;
    horner(B, Q, v, c);
    e.ho.bq_hor = append(v);
    e.ho.bq_hor_s = append(c);
  }
  {
    // mixed-radix weights: X mod m = sum_i d_i (prod_{l<i} s_l mod m)
    auto weights = [&](const std::vector<uint64_t>& s, const std::vector<uint64_t>& m) {
      std::vector<uint64_t> w;
      for (size_t j = 0; j < m.size(); ++j) {
        uint64_t acc = 1 % m[j];
        for (size_t i = 0; i < s.size(); ++i) {
          w.push_back(acc);
          acc = h_mulmod(acc, s[i] % m[j], m[j]);
        }
      }
      return w;
    };
    e.ho.qb_pm = append(weights(Q, B));
    e.ho.bq_pm = append(weights(B, Q));
    // Garner constants of each base: W[i][l] = prod_{j<l} s_j mod s_i, Pinv_i
    e.ho.qq_w = append(weights(Q, Q));
    e.ho.bb_w = append(weights(B, B));
    auto pinv = [&](const std::vector<uint64_t>& s, int& off_v, int& off_s) {
      std::vector<uint64_t> v, c;
      for (size_t i = 0; i < s.size(); ++i) {
        uint64_t pr = 1 % s[i];
        for (size_t j = 0; j < i; ++j) pr = h_mulmod(pr, s[j] % s[i], s[i]);
        push_pair(h_invmod(pr, s[i]), s[i], v, c);
      }
      off_v = append(v);
      off_s = append(c);
    };
    pinv(Q, e.ho.q_pinv, e.ho.q_pinv_s);
    pinv(B, e.ho.b_pinv, e.ho.b_pinv_s);
  }
  {
    std::vector<uint64_t> v, c;
    horner(Q, std::vector<uint64_t>{e.t}, v, c);
    e.ho.qt_hor = append(v);
    e.ho.qt_hor_s = append(c);
  }
  {
    std::vector<uint64_t> v, c, v2, c2, v3, c3, v4, c4;
    for (auto b : B) {
      uint64_t qm = prod_mod(Q, b);
      push_pair(qm, b, v, c);
      push_pair(h_invmod(qm, b), b, v2, c2);
      push_pair(e.t % b, b, v4, c4);
    }
    for (auto q : Q) push_pair(e.t % q, q, v3, c3);
    e.ho.q_mod_b = append(v);
    e.ho.q_mod_b_s = append(c);
    e.ho.qinv_b = append(v2);
    e.ho.qinv_b_s = append(c2);
    e.ho.t_q = append(v3);
    e.ho.t_q_s = append(c3);
    e.ho.t_b = append(v4);
    e.ho.t_b_s = append(c4);
  }
  {
    uint64_t qt = prod_mod(Q, e.t);
    uint64_t qi = inv_general(qt, e.t);
    std::vector<uint64_t> v{qt}, c{shoup_general(qt, e.t)}, v2{qi}, c2{shoup_general(qi, e.t)};
    e.ho.q_mod_t = append(v);
    e.ho.q_mod_t_s = append(c);
    e.ho.qinv_t = append(v2);
    e.ho.qinv_t_s = append(c2);
    e.t_shoup_one = shoup_general(1 % e.t, e.t);
    e.h_q_mod_t = qt;
    e.h_qinv_t = qi;
    e.h_qinv_t_s = shoup_general(qi, e.t);
  }
  {
    std::vector<uint64_t> v, c, v2, c2;
    for (size_t i = 0; i < Q.size(); ++i) {
      uint64_t qq = 1 % Q[i];
      for (size_t l = 0; l < Q.size(); ++l)
        if (l != i) qq = h_mulmod(qq, Q[l] % Q[i], Q[i]);
      push_pair(h_invmod(qq, Q[i]), Q[i], v, c);
      push_pair(qq, Q[i], v2, c2);
    }
    e.ho.xi_q = append(v);
    e.ho.xi_q_s = append(c);
    e.ho.rho_q = append(v2);
    e.ho.rho_q_s = append(c2);
  }
  {
    // fast base conversion: S = prod(src); hat_i = S / s_i
    auto fast = [&](const std::vector<uint64_t>& src, const std::vector<uint64_t>& dst, bool with_t, int& o_hinv,
                    int& o_hinv_s, int* o_thinv, int* o_thinv_s, int& o_hmod, int& o_negv, int& o_invd) {
      const size_t n = src.size();
      std::vector<uint64_t> hinv, hinv_s, thinv, thinv_s, hmod, negv, invd;
      for (size_t i = 0; i < n; ++i) {
        uint64_t hat = 1 % src[i];
        for (size_t l = 0; l < n; ++l)
          if (l != i) hat = h_mulmod(hat, src[l] % src[i], src[i]);
        const uint64_t hi = h_invmod(hat, src[i]);
        push_pair(hi, src[i], hinv, hinv_s);
        if (with_t) push_pair(h_mulmod(e.t % src[i], hi, src[i]), src[i], thinv, thinv_s);
        const double d = 1.0 / (double)src[i];
        uint64_t bits;
        std::memcpy(&bits, &d, 8);
        invd.push_back(bits);
      }
      for (size_t j = 0; j < dst.size(); ++j) {
        const uint64_t m = dst[j];
        for (size_t i = 0; i < n; ++i) {
          uint64_t hat = 1 % m;
          for (size_t l = 0; l < n; ++l)
            if (l != i) hat = h_mulmod(hat, src[l] % m, m);
          hmod.push_back(hat);
        }
        const uint64_t Sm = prod_mod(src, m);
        for (size_t v = 0; v <= n; ++v) negv.push_back((m - h_mulmod(v % m, Sm, m)) % m);
      }
      o_hinv = append(hinv);
      o_hinv_s = append(hinv_s);
      if (with_t) {
        *o_thinv = append(thinv);
        *o_thinv_s = append(thinv_s);
      }
      o_hmod = append(hmod);
      o_negv = append(negv);
      o_invd = append(invd);
    };
    fast(Q, B, true, e.ho.fq_hinv, e.ho.fq_hinv_s, &e.ho.fq_thinv, &e.ho.fq_thinv_s, e.ho.fq_hmod, e.ho.fq_negv,
         e.ho.fq_invd);
    fast(B, Q, false, e.ho.fb_hinv, e.ho.fb_hinv_s, nullptr, nullptr, e.ho.fb_hmod, e.ho.fb_negv, e.ho.fb_invd);
  }
  {
    // conversions of prescaled inputs (the off_untwist_pre tables): recovery factors and the
    // complex scaling's dot constants with Q^-1 (B/b_j)^-1 folded in
    const size_t k = Q.size(), kl = B.size();
    auto hat_mod = [&](const std::vector<uint64_t>& s, size_t i) {
      uint64_t h = 1 % s[i];
      for (size_t l = 0; l < s.size(); ++l)
        if (l != i) h = h_mulmod(h, s[l] % s[i], s[i]);
      return h;
    };
    std::vector<uint64_t> trec, trec_s, rec, rec_s, brec, brec_s, hm2, negw2;
    for (size_t i = 0; i < k; ++i) {  // x_i = y_i (t (Q/q_i)^-1)^-1
      const uint64_t q = Q[i];
      const uint64_t th = h_mulmod(e.t % q, h_invmod(hat_mod(Q, i), q), q);
      push_pair(h_invmod(th, q), q, trec, trec_s);
    }
    for (size_t j = 0; j < kl; ++j) {
      const uint64_t b = B[j];
      const uint64_t bh = hat_mod(B, j), bhi = h_invmod(bh, b);
      push_pair(bh, b, rec, rec_s);  // z_j = zhat_j (B/b_j)
      const uint64_t qinv = h_invmod(prod_mod(Q, b), b);
      const uint64_t f = h_mulmod(h_mulmod(e.t % b, qinv, b), bhi, b);  // t Q^-1 (B/b_j)^-1
      push_pair(h_invmod(f, b), b, brec, brec_s);
      for (size_t i = 0; i < k; ++i) hm2.push_back(h_mulmod(h_invmod(Q[i] % b, b), bhi, b));
      for (size_t w = 0; w <= k; ++w) negw2.push_back((b - h_mulmod(w % b, bhi, b)) % b);
    }
    e.ho.fq_trec = append(trec);
    e.ho.fq_trec_s = append(trec_s);
    e.ho.fb_rec = append(rec);
    e.ho.fb_rec_s = append(rec_s);
    e.ho.cs_brec = append(brec);
    e.ho.cs_brec_s = append(brec_s);
    e.ho.cs_hm2 = append(hm2);
    e.ho.cs_negw2 = append(negw2);
  }
  {
    std::vector<uint64_t> v;  // 2^(64 l) mod p_r for the limb-to-residue conversion
    for (auto p : e.primes) {
      const uint64_t r1 = (uint64_t)(((unsigned __int128)1 << 64) % p);
      uint64_t acc = 1;
      for (int l = 0; l < kMaxLimbs; ++l) {
        v.push_back(acc);
        acc = h_mulmod(acc, r1, p);
      }
    }
    e.ho.pow64 = append(v);
    std::vector<uint64_t> vm;  // the same powers times 2^64 (for the Montgomery path)
    for (auto p : e.primes) {
      const uint64_t r1 = (uint64_t)(((unsigned __int128)1 << 64) % p);
      uint64_t acc = r1;
      for (int l = 0; l < kMaxLimbs; ++l) {
        vm.push_back(acc);
        acc = h_mulmod(acc, r1, p);
      }
    }
    e.ho.pow64m = append(vm);
  }
  if (e.ckks_prec) {
    const int k = e.k, kl = e.kl;
    std::vector<uint64_t> a, as, b, bs, c, cs, d, ds, f, fs, g, gs, h, hs;
    for (int l = 0; l < k; ++l)
      for (int i = 0; i < k; ++i) {
        const uint64_t qi = Q[i];
        const uint64_t inv_ql = i < l ? h_invmod(Q[l] % qi, qi) : 0;
        push_pair(inv_ql, qi, a, as);
        uint64_t m = 1 % qi;  // Q_l / q_i mod q_i
        for (int u = 0; u <= l; ++u)
          if (u != i) m = h_mulmod(m, Q[u] % qi, qi);
        push_pair(i <= l ? h_invmod(m, qi) : 0, qi, b, bs);
        for (int j = 0; j < kl; ++j) {
          uint64_t mb = 1 % B[j];  // Q_l / q_i mod b_j
          for (int u = 0; u <= l; ++u)
            if (u != i) mb = h_mulmod(mb, Q[u] % B[j], B[j]);
          push_pair(i <= l ? mb : 0, B[j], c, cs);
        }
      }
    for (int j = 0; j < kl; ++j) {
      uint64_t m = 1 % B[j];
      for (int u = 0; u < kl; ++u)
        if (u != j) m = h_mulmod(m, B[u] % B[j], B[j]);
      push_pair(h_invmod(m, B[j]), B[j], d, ds);
      for (int i = 0; i < k; ++i) {
        uint64_t mq = 1 % Q[i];
        for (int u = 0; u < kl; ++u)
          if (u != j) mq = h_mulmod(mq, B[u] % Q[i], Q[i]);
        push_pair(mq, Q[i], f, fs);
      }
    }
    for (int i = 0; i < k; ++i) {
      const uint64_t bq = prod_mod(B, Q[i]);
      push_pair(h_invmod(bq, Q[i]), Q[i], g, gs);
      push_pair(bq, Q[i], h, hs);
    }
    e.ho.ck_inv_ql = append(a);
    e.ho.ck_inv_ql_s = append(as);
    e.ho.ck_qlqi_inv = append(b);
    e.ho.ck_qlqi_inv_s = append(bs);
    e.ho.ck_qlqi_b = append(c);
    e.ho.ck_qlqi_b_s = append(cs);
    e.ho.ck_bbj_inv = append(d);
    e.ho.ck_bbj_inv_s = append(ds);
    e.ho.ck_bbj_q = append(f);
    e.ho.ck_bbj_q_s = append(fs);
    e.ho.ck_binv_q = append(g);
    e.ho.ck_binv_q_s = append(gs);
    e.ho.ck_b_q = append(h);
    e.ho.ck_b_q_s = append(hs);
  }
  e.hps_words = H.size();

  // ---------------- upload ----------------
  cudaError_t err;
  if ((err = cudaMalloc(&e.d_tab, tab.size() * sizeof(ulonglong2))) != cudaSuccess ||
      (err = cudaMalloc(&e.d_mc, e.mconst.size() * sizeof(ModConst))) != cudaSuccess ||
      (err = cudaMalloc(&e.d_hps, (H.size() + 1) * sizeof(uint64_t))) != cudaSuccess ||
      (err = cudaMalloc(&e.d_err, sizeof(int))) != cudaSuccess) {
    set_error(std::string("cudaMalloc failed for engine tables: ") + cudaGetErrorString(err));
    free_tables(e);
    return 4;
  }
  if ((err = cudaMemcpy(e.d_tab, tab.data(), tab.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (err = cudaMemcpy(e.d_mc, e.mconst.data(), e.mconst.size() * sizeof(ModConst), cudaMemcpyHostToDevice)) !=
          cudaSuccess ||
      (err = cudaMemcpy(e.d_hps, H.data(), H.size() * sizeof(uint64_t), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (err = cudaMemset(e.d_err, 0, sizeof(int))) != cudaSuccess) {
    set_error(std::string("table upload failed: ") + cudaGetErrorString(err));
    free_tables(e);
    return 2;
  }
  return 0;
}

void free_tables(Engine& e) {
  if (e.d_tab) cudaFree(e.d_tab);
  if (e.d_mc) cudaFree(e.d_mc);
  if (e.d_hps) cudaFree(e.d_hps);
  if (e.d_err) cudaFree(e.d_err);
  e.d_err = nullptr;
  e.d_tab = nullptr;
  e.d_mc = nullptr;
  e.d_hps = nullptr;
}

}  // namespace cpoly
