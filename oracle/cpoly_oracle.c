/*
 * C restatement of cuPoly's hot path -- TEST INFRASTRUCTURE AND CPU BASELINE ONLY.
 *
 * Not part of the product: only tests/, __graft_entry__.smoke() and the CPU
 * legs of bench.py load this library (through oracle/coracle.py).
 *
 * Restates, from the mathematics, in portable C with unsigned __int128:
 *  - cuPoly's hierarchical DGT (src/cuda/dgt.cu:819-1006, tables :1501-1982):
 *    pass 1 = Nb-point Gentleman-Sande DIF on the twisted columns (stride Na),
 *    pass 2 = inter-pass twiddle g_N^(t brev_Nb(c)) then Na-point DIF;
 *    inverse = the mirror with Cooley-Tukey DIT and N^-1 folded in;
 *  - pointwise Gaussian products (dgt.cu:547-570, 1251-1437);
 *  - exact basis extension X mod m for X in [0, P) by mixed-radix conversion
 *    (the value cuPoly's polynomial_basis_ext_* targets,
 *    src/cuda/cudaengine.cu:483-796);
 *  - exact HPS complex scaling round(t X / Q) (cudaengine.cu:382-469) and the
 *    BFV multiplication chain composed as in polynomial.cu:350-527, 951-999.
 * Constant multiplications use Shoup's precomputed quotients; OpenMP
 * parallelises over polynomials x residues.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }
static inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t p) { uint64_t s = a + b; return s >= p ? s - p : s; }
static inline uint64_t submod(uint64_t a, uint64_t b, uint64_t p) { return a >= b ? a - b : a + p - b; }
static inline uint64_t shoup_c(uint64_t w, uint64_t p) { return (uint64_t)(((u128)w << 64) / p); }
static inline uint64_t shoup(uint64_t a, uint64_t w, uint64_t ws, uint64_t p) {
  uint64_t q = (uint64_t)(((u128)a * ws) >> 64);
  uint64_t r = a * w - q * p;
  return r >= p ? r - p : r;
}
static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
  uint64_t r = 1 % p;
  a %= p;
  while (e) {
    if (e & 1) r = mulmod(r, a, p);
    a = mulmod(a, a, p);
    e >>= 1;
  }
  return r;
}
static uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a, p - 2, p); }
static int ilog2(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }
static int brev(int x, int bits) { int r = 0; for (int i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; } return r; }

static inline void gmul(uint64_t* cr, uint64_t* ci, uint64_t ar, uint64_t ai, uint64_t br, uint64_t bi, uint64_t p) {
  u128 re = (u128)ar * br + (u128)ai * (bi ? p - bi : 0);
  u128 im = (u128)ar * bi + (u128)ai * br;
  *cr = (uint64_t)(re % p);
  *ci = (uint64_t)(im % p);
}

/* (Na, Nb) of cuPoly's hierarchical split (include/cuPoly/cuda/dgt.h:41-50); 0 for single block */
static void split_of(int N, int* Na, int* Nb) {
  switch (N) {
    case 1024: *Na = 32; *Nb = 32; return;
    case 2048: *Na = 64; *Nb = 32; return;
    case 4096: *Na = 64; *Nb = 64; return;
    case 8192: *Na = 128; *Nb = 64; return;
    case 16384: *Na = 128; *Nb = 128; return;
    case 32768: *Na = 256; *Nb = 128; return;
    default: *Na = 0; *Nb = 0;
  }
}

/* Per-(prime, N) tables. */
typedef struct {
  int N, Na, Nb;
  uint64_t p;
  uint64_t *tw_a, *tw_as, *itw_a, *itw_as; /* S-point roots w_S^j, j < S, for S = Na */
  uint64_t *tw_b, *tw_bs, *itw_b, *itw_bs; /* S = Nb (or N when single block) */
  uint64_t *gN, *gNs, *giN, *giNs;         /* inter-pass twiddles */
  uint64_t *xr, *xi, *ixr, *ixi;           /* xi^n and xi^-n N^-1 */
} tables_t;

static void roots(uint64_t p, uint64_t g, int S, uint64_t** w, uint64_t** ws, uint64_t** iw, uint64_t** iws) {
  uint64_t r = powmod(g, (p - 1) / S, p), ri = invmod(r, p);
  *w = malloc(S * 8); *ws = malloc(S * 8); *iw = malloc(S * 8); *iws = malloc(S * 8);
  uint64_t a = 1, b = 1;
  for (int j = 0; j < S; ++j) {
    (*w)[j] = a; (*ws)[j] = shoup_c(a, p); (*iw)[j] = b; (*iws)[j] = shoup_c(b, p);
    a = mulmod(a, r, p); b = mulmod(b, ri, p);
  }
}

static tables_t* make_tables(uint64_t p, uint64_t g, int N, uint64_t xir, uint64_t xii) {
  tables_t* T = calloc(1, sizeof(tables_t));
  T->N = N; T->p = p;
  split_of(N, &T->Na, &T->Nb);
  if (T->Na) {
    roots(p, g, T->Na, &T->tw_a, &T->tw_as, &T->itw_a, &T->itw_as);
    roots(p, g, T->Nb, &T->tw_b, &T->tw_bs, &T->itw_b, &T->itw_bs);
    uint64_t w = powmod(g, (p - 1) / N, p), wi = invmod(w, p), ninv = invmod(N, p);
    int lb = ilog2(T->Nb);
    T->gN = malloc(N * 8); T->gNs = malloc(N * 8); T->giN = malloc(N * 8); T->giNs = malloc(N * 8);
    for (int c = 0; c < N; ++c) {
      /* forward: tmp[t Nb + c'] * g_N^(t brev(c')) ; index c = t*Nb + c' */
      uint64_t f = powmod(w, (uint64_t)(c / T->Nb) * brev(c % T->Nb, lb), p);
      /* inverse: row c' = c / Na, column t = c % Na */
      uint64_t v = mulmod(powmod(wi, (uint64_t)brev(c / T->Na, lb) * (c % T->Na), p), ninv, p);
      T->gN[c] = f; T->gNs[c] = shoup_c(f, p); T->giN[c] = v; T->giNs[c] = shoup_c(v, p);
    }
  } else {
    roots(p, g, N, &T->tw_b, &T->tw_bs, &T->itw_b, &T->itw_bs);
  }
  T->xr = malloc(N * 8); T->xi = malloc(N * 8); T->ixr = malloc(N * 8); T->ixi = malloc(N * 8);
  /* xi^-1 = xi^(4N - 1) */
  uint64_t br = xir, bi = xii, er = 1, ei = 0;
  uint64_t e = 4 * (uint64_t)N - 1;
  while (e) {
    if (e & 1) gmul(&er, &ei, er, ei, br, bi, p);
    gmul(&br, &bi, br, bi, br, bi, p);
    e >>= 1;
  }
  /* single-block inverse folds N^-1 into the untwist; the hierarchical one
     applies (Na Nb)^-1 with the inter-pass twiddle (cuPoly dgt.cu:1654-1662, 1940-1945) */
  uint64_t ar = 1, ai = 0, cr = T->Na ? 1 : invmod(N, p), ci = 0;
  for (int n = 0; n < N; ++n) {
    T->xr[n] = ar; T->xi[n] = ai; T->ixr[n] = cr; T->ixi[n] = ci;
    gmul(&ar, &ai, ar, ai, xir, xii, p);
    gmul(&cr, &ci, cr, ci, er, ei, p);
  }
  return T;
}

static void free_tables(tables_t* T) {
  free(T->tw_a); free(T->tw_as); free(T->itw_a); free(T->itw_as);
  free(T->tw_b); free(T->tw_bs); free(T->itw_b); free(T->itw_bs);
  free(T->gN); free(T->gNs); free(T->giN); free(T->giNs);
  free(T->xr); free(T->xi); free(T->ixr); free(T->ixi);
  free(T);
}

/* S-point GS DIF on interleaved (re, im) x[2S] (cuPoly dgt.cu:681-714). */
static void dif(uint64_t* x, int S, const uint64_t* w, const uint64_t* ws, uint64_t p) {
  for (int m = S >> 1, st = 1; m >= 1; m >>= 1, st <<= 1)
    for (int i0 = 0; i0 < S; i0 += 2 * m)
      for (int j = 0; j < m; ++j) {
        uint64_t* a = x + 2 * (i0 + j);
        uint64_t* b = x + 2 * (i0 + j + m);
        uint64_t ar = a[0], ai = a[1], br = b[0], bi = b[1];
        a[0] = addmod(ar, br, p); a[1] = addmod(ai, bi, p);
        uint64_t dr = submod(ar, br, p), di = submod(ai, bi, p);
        int e = j * st;
        b[0] = shoup(dr, w[e], ws[e], p); b[1] = shoup(di, w[e], ws[e], p);
      }
}

/* S-point CT DIT with inverse roots (cuPoly dgt.cu:716-753). */
static void dit(uint64_t* x, int S, const uint64_t* w, const uint64_t* ws, uint64_t p) {
  for (int m = 1, st = S >> 1; m < S; m <<= 1, st >>= 1)
    for (int i0 = 0; i0 < S; i0 += 2 * m)
      for (int j = 0; j < m; ++j) {
        uint64_t* a = x + 2 * (i0 + j);
        uint64_t* b = x + 2 * (i0 + j + m);
        int e = j * st;
        uint64_t br = shoup(b[0], w[e], ws[e], p), bi = shoup(b[1], w[e], ws[e], p);
        uint64_t ar = a[0], ai = a[1];
        a[0] = addmod(ar, br, p); a[1] = addmod(ai, bi, p);
        b[0] = submod(ar, br, p); b[1] = submod(ai, bi, p);
      }
}

/* forward DGT of one residue, in place, x[2N] interleaved */
static void dgt_fwd(uint64_t* x, const tables_t* T, uint64_t* tmp) {
  const int N = T->N;
  const uint64_t p = T->p;
  if (!T->Na) {
    for (int n = 0; n < N; ++n) gmul(&x[2 * n], &x[2 * n + 1], x[2 * n], x[2 * n + 1], T->xr[n], T->xi[n], p);
    dif(x, N, T->tw_b, T->tw_bs, p);
    return;
  }
  const int Na = T->Na, Nb = T->Nb;
  uint64_t col[2 * 256];
  for (int b = 0; b < Na; ++b) {
    for (int t = 0; t < Nb; ++t) {
      int n = t * Na + b;
      gmul(&col[2 * t], &col[2 * t + 1], x[2 * n], x[2 * n + 1], T->xr[n], T->xi[n], p);
    }
    dif(col, Nb, T->tw_b, T->tw_bs, p);
    memcpy(tmp + 2 * (size_t)b * Nb, col, 16 * Nb);
  }
  for (int c = 0; c < Nb; ++c) {
    for (int t = 0; t < Na; ++t) {
      int idx = t * Nb + c;
      col[2 * t] = shoup(tmp[2 * idx], T->gN[idx], T->gNs[idx], p);
      col[2 * t + 1] = shoup(tmp[2 * idx + 1], T->gN[idx], T->gNs[idx], p);
    }
    dif(col, Na, T->tw_a, T->tw_as, p);
    memcpy(x + 2 * (size_t)c * Na, col, 16 * Na);
  }
}

static void dgt_inv(uint64_t* x, const tables_t* T, uint64_t* tmp) {
  const int N = T->N;
  const uint64_t p = T->p;
  if (!T->Na) {
    dit(x, N, T->itw_b, T->itw_bs, p);
    for (int n = 0; n < N; ++n) gmul(&x[2 * n], &x[2 * n + 1], x[2 * n], x[2 * n + 1], T->ixr[n], T->ixi[n], p);
    return;
  }
  const int Na = T->Na, Nb = T->Nb;
  uint64_t col[2 * 256];
  for (int c = 0; c < Nb; ++c) {
    memcpy(col, x + 2 * (size_t)c * Na, 16 * Na);
    dit(col, Na, T->itw_a, T->itw_as, p);
    for (int t = 0; t < Na; ++t) {
      int idx = c * Na + t;
      tmp[2 * idx] = shoup(col[2 * t], T->giN[idx], T->giNs[idx], p);
      tmp[2 * idx + 1] = shoup(col[2 * t + 1], T->giN[idx], T->giNs[idx], p);
    }
  }
  for (int b = 0; b < Na; ++b) {
    for (int t = 0; t < Nb; ++t) {
      int idx = t * Na + b;
      col[2 * t] = tmp[2 * idx];
      col[2 * t + 1] = tmp[2 * idx + 1];
    }
    dit(col, Nb, T->itw_b, T->itw_bs, p);
    for (int t = 0; t < Nb; ++t) {
      int n = t * Na + b;
      gmul(&x[2 * n], &x[2 * n + 1], col[2 * t], col[2 * t + 1], T->ixr[n], T->ixi[n], p);
    }
  }
}

/* ------------------------------------------------------------------ */
/* public API                                                          */
/* ------------------------------------------------------------------ */

int oc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* DGT of npolys x nres residues of N Gaussian elements (data [npolys][nres][N][2]) in place.
 * primes[nres], gens[nres] (primitive roots), xi[nres][2]. */
void oc_dgt(uint64_t* data, int npolys, int nres, int N, const uint64_t* primes, const uint64_t* gens,
            const uint64_t* xi, int inverse) {
  tables_t** T = malloc(sizeof(tables_t*) * nres);
  for (int r = 0; r < nres; ++r) T[r] = make_tables(primes[r], gens[r], N, xi[2 * r], xi[2 * r + 1]);
#pragma omp parallel
  {
    uint64_t* tmp = malloc(16 * (size_t)N);
#pragma omp for schedule(static)
    for (long u = 0; u < (long)npolys * nres; ++u) {
      int r = (int)(u % nres);
      uint64_t* x = data + 2 * (size_t)N * u;
      if (inverse) dgt_inv(x, T[r], tmp); else dgt_fwd(x, T[r], tmp);
    }
    free(tmp);
  }
  for (int r = 0; r < nres; ++r) free_tables(T[r]);
  free(T);
}

/* ---- exact base conversion by mixed-radix conversion ---- */
static void mrc_digits(uint64_t* d, const uint64_t* z, const uint64_t* s, int n, const uint64_t* inv) {
  for (int i = 0; i < n; ++i) {
    uint64_t y = z[i] % s[i];
    for (int l = 0; l < i; ++l) {
      y = submod(y, d[l] % s[i], s[i]);
      y = mulmod(y, inv[i * n + l], s[i]);
    }
    d[i] = y;
  }
}
static uint64_t horner(const uint64_t* d, const uint64_t* s, int n, uint64_t m) {
  uint64_t acc = d[n - 1] % m;
  for (int i = n - 2; i >= 0; --i) acc = addmod(mulmod(acc, s[i] % m, m), d[i] % m, m);
  return acc;
}
static uint64_t* mrc_inverses(const uint64_t* s, int n) {
  uint64_t* inv = calloc((size_t)n * n, 8);
  for (int i = 0; i < n; ++i)
    for (int l = 0; l < i; ++l) inv[i * n + l] = invmod(s[l] % s[i], s[i]);
  return inv;
}

/* mixed-radix digits d > h, compared from the most significant */
static int digits_gt(const uint64_t* d, const uint64_t* h, int n) {
  for (int i = n - 1; i >= 0; --i)
    if (d[i] != h[i]) return d[i] > h[i];
  return 0;
}
static uint64_t prod_mod(const uint64_t* s, int n, uint64_t m) {
  uint64_t r = 1 % m;
  for (int i = 0; i < n; ++i) r = mulmod(r, s[i] % m, m);
  return r;
}
/* X mod m with cuPoly's lift: X - S when X > lift (the digits of the threshold minus
 * one, pyoracle.lift_digits) -- cuPoly's FPERROR rounding of the overflow count,
 * src/cuda/cudaengine.cu:513-534, 690-703. */
static uint64_t lifted(const uint64_t* d, const uint64_t* s, int n, uint64_t m, const uint64_t* lift) {
  uint64_t r = horner(d, s, n, m);
  if (lift && digits_gt(d, lift, n)) r = submod(r, prod_mod(s, n, m), m);
  return r;
}

/* out[j][c] = lift(X_c) mod dst_j for X_c = crt(in[.][c]) in [0, prod(src)); count coefficients per
 * residue; lift = digits of the lift threshold minus one (NULL: no lift). */
void oc_basis_ext(uint64_t* out, const uint64_t* in, long count, const uint64_t* src, int ns, const uint64_t* dst,
                  int nd, const uint64_t* lift) {
  uint64_t* inv = mrc_inverses(src, ns);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < count; ++c) {
    uint64_t z[64], d[64];
    for (int i = 0; i < ns; ++i) z[i] = in[(size_t)i * count + c];
    mrc_digits(d, z, src, ns, inv);
    for (int j = 0; j < nd; ++j) out[(size_t)j * count + c] = lifted(d, src, ns, dst[j], lift);
  }
  free(inv);
}

/* out[j][c] = round(t X_c / Q) mod B-prime j; X from Q and B residues (coefficient rows). */
void oc_complex_scaling(uint64_t* out_b, const uint64_t* in_q, const uint64_t* in_b, long count, const uint64_t* Q,
                        int k, const uint64_t* B, int kl, uint64_t t) {
  uint64_t* inv = mrc_inverses(Q, k);
  uint64_t half[64], hd[64], qb[64], qbi[64];
  for (int i = 0; i < k; ++i) half[i] = (Q[i] - 1) / 2;
  mrc_digits(hd, half, Q, k, inv);
  for (int j = 0; j < kl; ++j) {
    qb[j] = 1;
    for (int i = 0; i < k; ++i) qb[j] = mulmod(qb[j], Q[i] % B[j], B[j]);
    qbi[j] = invmod(qb[j], B[j]);
  }
#pragma omp parallel for schedule(static)
  for (long c = 0; c < count; ++c) {
    uint64_t z[64], d[64];
    for (int i = 0; i < k; ++i) z[i] = mulmod(in_q[(size_t)i * count + c], t % Q[i], Q[i]);
    mrc_digits(d, z, Q, k, inv);
    int neg = 0;
    for (int i = k - 1; i >= 0; --i) {
      if (d[i] != hd[i]) { neg = d[i] > hd[i]; break; }
    }
    for (int j = 0; j < kl; ++j) {
      uint64_t b = B[j];
      uint64_t r = horner(d, Q, k, b);
      if (neg) r = submod(r, qb[j], b);
      uint64_t ty = mulmod(in_b[(size_t)j * count + c], t % b, b);
      out_b[(size_t)j * count + c] = mulmod(submod(ty, r, b), qbi[j], b);
    }
  }
  free(inv);
}

/* round(t X / Q) mod t for X from Q residues (simple scaling). */
void oc_simple_scaling(uint64_t* out, const uint64_t* in_q, long count, const uint64_t* Q, int k, uint64_t t) {
  uint64_t* inv = mrc_inverses(Q, k);
  uint64_t half[64], hd[64];
  for (int i = 0; i < k; ++i) half[i] = (Q[i] - 1) / 2;
  mrc_digits(hd, half, Q, k, inv);
  uint64_t qt = 1;
  for (int i = 0; i < k; ++i) qt = (uint64_t)((u128)qt * (Q[i] % t) % t);
  /* Q^-1 mod t by extended Euclid (t need not be prime) */
  __int128 r0 = t, r1 = qt, s0 = 0, s1 = 1;
  while (r1) { __int128 q = r0 / r1, tmp = r0 - q * r1; r0 = r1; r1 = tmp; tmp = s0 - q * s1; s0 = s1; s1 = tmp; }
  uint64_t qinv = (uint64_t)((s0 % (__int128)t + t) % t);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < count; ++c) {
    uint64_t z[64], d[64];
    for (int i = 0; i < k; ++i) z[i] = mulmod(in_q[(size_t)i * count + c], t % Q[i], Q[i]);
    mrc_digits(d, z, Q, k, inv);
    int neg = 0;
    for (int i = k - 1; i >= 0; --i) {
      if (d[i] != hd[i]) { neg = d[i] > hd[i]; break; }
    }
    uint64_t rt = horner(d, Q, k, t);
    if (neg) rt = submod(rt, qt, t);
    out[c] = (uint64_t)((u128)((t - rt) % t) * qinv % t);
  }
  free(inv);
}

/* Negacyclic products through the DGT: c = a * b mod (x^nphi + 1, p_r) for
 * npolys x nres coefficient rows ([npolys][nres][nphi]). */
void oc_polymul(uint64_t* c, const uint64_t* a, const uint64_t* b, int npolys, int nres, int nphi,
                const uint64_t* primes, const uint64_t* gens, const uint64_t* xi) {
  const int N = nphi / 2;
  tables_t** T = malloc(sizeof(tables_t*) * nres);
  for (int r = 0; r < nres; ++r) T[r] = make_tables(primes[r], gens[r], N, xi[2 * r], xi[2 * r + 1]);
#pragma omp parallel
  {
    uint64_t* tmp = malloc(16 * (size_t)N);
    uint64_t* x = malloc(16 * (size_t)N);
    uint64_t* y = malloc(16 * (size_t)N);
#pragma omp for schedule(static)
    for (long u = 0; u < (long)npolys * nres; ++u) {
      int r = (int)(u % nres);
      uint64_t p = primes[r];
      const uint64_t* ar = a + (size_t)u * nphi;
      const uint64_t* br = b + (size_t)u * nphi;
      for (int j = 0; j < N; ++j) {
        x[2 * j] = ar[j]; x[2 * j + 1] = ar[j + N];
        y[2 * j] = br[j]; y[2 * j + 1] = br[j + N];
      }
      dgt_fwd(x, T[r], tmp);
      dgt_fwd(y, T[r], tmp);
      for (int j = 0; j < N; ++j) gmul(&x[2 * j], &x[2 * j + 1], x[2 * j], x[2 * j + 1], y[2 * j], y[2 * j + 1], p);
      dgt_inv(x, T[r], tmp);
      uint64_t* cr = c + (size_t)u * nphi;
      for (int j = 0; j < N; ++j) { cr[j] = x[2 * j]; cr[j + N] = x[2 * j + 1]; }
    }
    free(tmp); free(x); free(y);
  }
  for (int r = 0; r < nres; ++r) free_tables(T[r]);
  free(T);
}

/* BFV multiplication chain in the coefficient domain for npairs ciphertext
 * pairs: inputs a0, a1, b0, b1 as [npairs][k][nphi] rows mod Q; outputs
 * c0, c1, c2 as [npairs][k][nphi] = ((round(t/Q * tensor) mod B) mod q_i), both base
 * conversions with cuPoly's lift (lift_q, lift_b: threshold digits of Q and B).
 * primes = Q ++ B (k + kl), gens their primitive roots, xi[k + kl][2]. */
void oc_bfv_mul(uint64_t* c0, uint64_t* c1, uint64_t* c2, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
                const uint64_t* b1, int npairs, int k, int kl, int nphi, const uint64_t* primes, const uint64_t* gens,
                const uint64_t* xi, uint64_t t, const uint64_t* lift_q, const uint64_t* lift_b) {
  const int N = nphi / 2, nr = k + kl;
  const uint64_t* Q = primes;
  const uint64_t* B = primes + k;
  tables_t** T = malloc(sizeof(tables_t*) * nr);
  for (int r = 0; r < nr; ++r) T[r] = make_tables(primes[r], gens[r], N, xi[2 * r], xi[2 * r + 1]);
  uint64_t* inv = mrc_inverses(Q, k);
  uint64_t* invb = mrc_inverses(B, kl);
  for (int pr = 0; pr < npairs; ++pr) {
    const size_t off = (size_t)pr * k * nphi;
    /* extended inputs over Q u B: in[4][nr][nphi] */
    uint64_t* ext = malloc(8 * (size_t)4 * nr * nphi);
    const uint64_t* ins[4] = {a0 + off, a1 + off, b0 + off, b1 + off};
    for (int v = 0; v < 4; ++v) {
      memcpy(ext + (size_t)v * nr * nphi, ins[v], 8 * (size_t)k * nphi);
#pragma omp parallel for schedule(static)
      for (long c = 0; c < nphi; ++c) {
        uint64_t z[64], d[64];
        for (int i = 0; i < k; ++i) z[i] = ins[v][(size_t)i * nphi + c];
        mrc_digits(d, z, Q, k, inv);
        for (int j = 0; j < kl; ++j) ext[((size_t)v * nr + k + j) * nphi + c] = lifted(d, Q, k, B[j], lift_q);
      }
    }
    /* tensor product over every prime via the DGT */
    uint64_t* ten = malloc(8 * (size_t)3 * nr * nphi);
#pragma omp parallel
    {
      uint64_t* tmp = malloc(16 * (size_t)N);
      uint64_t* X[4];
      for (int v = 0; v < 4; ++v) X[v] = malloc(16 * (size_t)N);
#pragma omp for schedule(static)
      for (int r = 0; r < nr; ++r) {
        uint64_t p = primes[r];
        for (int v = 0; v < 4; ++v) {
          const uint64_t* row = ext + ((size_t)v * nr + r) * nphi;
          for (int j = 0; j < N; ++j) { X[v][2 * j] = row[j]; X[v][2 * j + 1] = row[j + N]; }
          dgt_fwd(X[v], T[r], tmp);
        }
        for (int j = 0; j < N; ++j) {
          uint64_t r1, i1, r2, i2, r3, i3, r4, i4;
          gmul(&r1, &i1, X[0][2 * j], X[0][2 * j + 1], X[2][2 * j], X[2][2 * j + 1], p);
          gmul(&r2, &i2, X[0][2 * j], X[0][2 * j + 1], X[3][2 * j], X[3][2 * j + 1], p);
          gmul(&r3, &i3, X[1][2 * j], X[1][2 * j + 1], X[2][2 * j], X[2][2 * j + 1], p);
          gmul(&r4, &i4, X[1][2 * j], X[1][2 * j + 1], X[3][2 * j], X[3][2 * j + 1], p);
          X[0][2 * j] = r1; X[0][2 * j + 1] = i1;
          X[2][2 * j] = addmod(r2, r3, p); X[2][2 * j + 1] = addmod(i2, i3, p);
          X[3][2 * j] = r4; X[3][2 * j + 1] = i4;
        }
        const int src[3] = {0, 2, 3};
        for (int o = 0; o < 3; ++o) {
          dgt_inv(X[src[o]], T[r], tmp);
          uint64_t* row = ten + ((size_t)o * nr + r) * nphi;
          for (int j = 0; j < N; ++j) { row[j] = X[src[o]][2 * j]; row[j + N] = X[src[o]][2 * j + 1]; }
        }
      }
      free(tmp);
      for (int v = 0; v < 4; ++v) free(X[v]);
    }
    /* scale each output to Q */
    uint64_t* outs[3] = {c0 + off, c1 + off, c2 + off};
    uint64_t* ub = malloc(8 * (size_t)kl * nphi);
    for (int o = 0; o < 3; ++o) {
      const uint64_t* tq = ten + (size_t)o * nr * nphi;
      oc_complex_scaling(ub, tq, tq + (size_t)k * nphi, nphi, Q, k, B, kl, t);
#pragma omp parallel for schedule(static)
      for (long c = 0; c < nphi; ++c) {
        uint64_t z[64], d[64];
        for (int j = 0; j < kl; ++j) z[j] = ub[(size_t)j * nphi + c];
        mrc_digits(d, z, B, kl, invb);
        for (int i = 0; i < k; ++i) outs[o][(size_t)i * nphi + c] = lifted(d, B, kl, Q[i], lift_b);
      }
    }
    free(ub); free(ten); free(ext);
  }
  free(inv); free(invb);
  for (int r = 0; r < nr; ++r) free_tables(T[r]);
  free(T);
}
