"""Pure-Python big-integer oracle for cuPoly's hot path -- TEST INFRASTRUCTURE ONLY.

Every function restates one piece of cuPoly (pdroalves/cupoly 0.3.5) from its
mathematics; the citation in each docstring is the reference file:line the
behaviour follows.  Nothing here is imported by the product package.

Conventions (cuPoly ``include/cuPoly/settings.h:70-80``,
``src/arithmetic/polynomial.cu:206-217``):
  * a ring element has ``nphi`` coefficients, ``N = nphi // 2``;
  * one residue is a list of N Gaussian integers ``(re, im)`` with
    ``re = a_j mod p`` and ``im = a_{j+N} mod p`` ("folded" encoding);
  * a polynomial over a base is residue-major: ``[nres][N]``.
"""
from __future__ import annotations

import os
import re as _re
from functools import lru_cache

_HERE = os.path.dirname(os.path.abspath(__file__))
_PRIME_HEADER = os.path.join(_HERE, "..", "cupoly_b200", "csrc", "prime_table.h")
_CDT_HEADER = os.path.join(_HERE, "..", "cupoly_b200", "csrc", "cdt_table.h")


# ----------------------------------------------------------------------------
# Parameters
# ----------------------------------------------------------------------------
def _load_prime_table():
    src = open(_PRIME_HEADER).read()
    p = _re.search(r"kPrimes\[kNumPrimes\]\s*=\s*\{([^}]*)\}", src).group(1)
    g = _re.search(r"kPrimitiveRoots\[kNumPrimes\]\s*=\s*\{([^}]*)\}", src).group(1)
    primes = [int(x.strip().rstrip("ULL")) for x in p.split(",") if x.strip()]
    roots = [int(x) for x in g.split(",") if x.strip()]
    return primes, roots


PRIMES, PROOTS = _load_prime_table()
PROOT = dict(zip(PRIMES, PROOTS))


def bases(k: int, kl: int):
    """Q = first k primes, B = next kl primes (cuPoly ``src/cuda/cudaengine.cu:1265-1290``)."""
    return PRIMES[:k], PRIMES[k:k + kl]


_CKKS_HEADER = os.path.join(_HERE, "..", "cupoly_b200", "csrc", "prime_table_ckks.h")


@lru_cache(maxsize=None)
def ckks_bucket(bits: int):
    """The bits-bit CKKS prime bucket (cuPoly ``src/arithmetic/coprimes.cu:9-762``)."""
    src = open(_CKKS_HEADER).read()
    m = _re.search(r"kPrimes%d\[kNumPrimes%d\]\s*=\s*\{([^}]*)\}" % (bits, bits), src)
    return [int(x.strip().rstrip("ULL")) for x in m.group(1).split(",") if x.strip()]


@lru_cache(maxsize=None)
def ckks_roots(bits: int):
    src = open(_CKKS_HEADER).read()
    m = _re.search(r"kRoots%d\[kNumPrimes%d\]\s*=\s*\{([^}]*)\}" % (bits, bits), src)
    return [int(x) for x in m.group(1).split(",") if x.strip()]


for _b in (45, 48, 52, 55):  # primitive roots of the CKKS primes, for the DGT restatement
    PROOT.update(zip(ckks_bucket(_b), ckks_roots(_b)))


def ckks_bases(k: int, kl: int, prec: int):
    """CKKS Q and B (cuPoly ``src/cuda/cudaengine.cu:1192-1232``): Q = the first 63-bit
    prime + k - 1 primes of the prec bucket; B = kl primes of the 45-bit (prec 45) or
    55-bit bucket from index k - 1."""
    qb = ckks_bucket(prec)
    bb = ckks_bucket(45 if prec == 45 else 55)
    return [PRIMES[0]] + qb[:k - 1], bb[k - 1:k - 1 + kl]


def ckks_modulus_raising(xs, Q, B, level):
    """B residues of fast_conv_Q_to_B (``src/cuda/cudaengine.cu:893-925``) for one
    coefficient with residues xs over Q_l = Q[0..level]:
    y_j = sum_i [x_i (Q_l/q_i)^-1]_{q_i} (Q_l/q_i) mod b_j."""
    Ql = prod(Q[:level + 1])
    out = []
    for b in B:
        acc = 0
        for i in range(level + 1):
            Mi = Ql // Q[i]
            acc += (xs[i] * pow(Mi % Q[i], -1, Q[i]) % Q[i]) * Mi
        out.append(acc % b)
    return out


def ckks_modulus_reduction(xs, ys, Q, B, level):
    """Q residues of fast_conv_B_to_Q (``src/cuda/cudaengine.cu:802-845``):
    z_i = (x_i - sum_j [y_j (B/b_j)^-1]_{b_j} (B/b_j)) B^-1 mod q_i, i <= level."""
    Bp = prod(B)
    V = sum((y * pow((Bp // b) % b, -1, b) % b) * (Bp // b) for y, b in zip(ys, B))
    return [(xs[i] - V) * pow(Bp % Q[i], -1, Q[i]) % Q[i] for i in range(level + 1)]


def ckks_rescale(xs, Q, level):
    """ckks_rescale (``src/cuda/cudaengine.cu:851-889``): x_i <- (x_i - x_l) q_l^-1
    mod q_i for i < level; residues from level on unchanged."""
    ql = Q[level]
    return [(xs[i] - xs[level]) * pow(ql, -1, Q[i]) % Q[i] for i in range(level)] + list(xs[level:])


def prod(xs):
    r = 1
    for x in xs:
        r *= x
    return r


# ----------------------------------------------------------------------------
# Gaussian-integer arithmetic mod p (cuPoly ``src/cuda/dgt.cu:527-570``)
# ----------------------------------------------------------------------------
def gi_add(a, b, p):
    return ((a[0] + b[0]) % p, (a[1] + b[1]) % p)


def gi_sub(a, b, p):
    return ((a[0] - b[0]) % p, (a[1] - b[1]) % p)


def gi_mul(a, b, p):
    """(a0 + a1 i)(b0 + b1 i) mod p; cuPoly computes it with Karatsuba (dgt.cu:547-570)."""
    return ((a[0] * b[0] - a[1] * b[1]) % p, (a[0] * b[1] + a[1] * b[0]) % p)


def gi_pow(a, e, p):
    r = (1, 0)
    while e:
        if e & 1:
            r = gi_mul(r, a, p)
        a = gi_mul(a, a, p)
        e >>= 1
    return r


def gi_scale(a, w, p):
    return (a[0] * w % p, a[1] * w % p)


# ----------------------------------------------------------------------------
# Roots
# ----------------------------------------------------------------------------
def omega(p: int, n: int) -> int:
    """Primitive n-th root of unity PROOT^((p-1)/n).

    cuPoly derives every DGT twiddle from the tabulated primitive root:
    stage twiddles from g = PROOT^((p-1)/(2S)) (``dgt.cu:1532-1533``) and the
    inter-pass twiddles from PROOT^((p-1)/N) (``dgt.cu:1920-1932``).
    """
    assert (p - 1) % n == 0
    return pow(PROOT[p], (p - 1) // n, p)


def canonical_xi(p: int, n: int):
    """A Gaussian xi with xi^n = i, chosen canonically.

    Z_p[i] is isomorphic to Z_p x Z_p through a+bi -> (a + b s, a - b s)
    with s = PROOT^((p-1)/4).  With u = PROOT^((p-1)/(4n)) (so u^n = s),
    the pair (u, u^-1) maps back to xi = ((u + u^-1)/2, (u - u^-1)/(2s)).
    The family is consistent: canonical_xi(p, 2n)^2 == canonical_xi(p, n).
    cuPoly instead uses tabulated roots (``NTHROOT``, ``coprimes.cu:868``);
    any xi with xi^n = i gives the same coefficient-domain results.
    """
    assert (p - 1) % (4 * n) == 0
    s = pow(PROOT[p], (p - 1) // 4, p)
    u = pow(PROOT[p], (p - 1) // (4 * n), p)
    ui = pow(u, p - 2, p)
    inv2 = (p + 1) // 2
    re = (u + ui) * inv2 % p
    im = (u - ui) * inv2 % p * pow(s, p - 2, p) % p
    return (re, im)


def brev(x: int, bits: int) -> int:
    r = 0
    for _ in range(bits):
        r = (r << 1) | (x & 1)
        x >>= 1
    return r


def hdgt_split(N: int):
    """(Na, Nb) factorisation of cuPoly's hierarchical DGT (``include/cuPoly/cuda/dgt.h:41-50``)."""
    return {1024: (32, 32), 2048: (64, 32), 4096: (64, 64), 8192: (128, 64),
            16384: (128, 128), 32768: (256, 128)}.get(N)


# ----------------------------------------------------------------------------
# DGT: bit-exact restatement of cuPoly's kernels
# ----------------------------------------------------------------------------
def _gs_dif(x, p, S):
    """In-place S-point Gentleman-Sande DIF (``dgt.cu:681-714, 757-777``).

    Stage s pairs (i, i+m), m = S >> (s+1), and multiplies the difference by
    w_S^(j 2^s) with j = i mod m; w_S = PROOT^((p-1)/S).  Output is in
    bit-reversed order.
    """
    w = omega(p, S)
    logS = S.bit_length() - 1
    for s in range(logS):
        m = S >> (s + 1)
        for cid in range(S // 2):
            j = cid * 2 * m // S
            i = j + (cid % (S // (2 * m))) * 2 * m
            a, b = x[i], x[i + m]
            x[i] = gi_add(a, b, p)
            x[i + m] = gi_scale(gi_sub(a, b, p), pow(w, j << s, p), p)


def _ct_dit_inv(x, p, S):
    """In-place S-point Cooley-Tukey inverse with inverse twiddles, unscaled (``dgt.cu:716-753, 782-805``)."""
    wi = pow(omega(p, S), p - 2, p)
    logS = S.bit_length() - 1
    for s in range(logS - 1, -1, -1):
        m = S >> (s + 1)
        for cid in range(S // 2):
            j = cid * 2 * m // S
            i = j + (cid % (S // (2 * m))) * 2 * m
            a, b = x[i], gi_scale(x[i + m], pow(wi, j << s, p), p)
            x[i] = gi_add(a, b, p)
            x[i + m] = gi_sub(a, b, p)


def dgt_forward_ref(x, p, xi=None):
    """cuPoly's forward DGT of one residue (``dgt.cu:819-908``, dispatch ``:107-205``).

    For N >= 1024 it is the two-pass hierarchical transform with N = Na*Nb:
    pass 1 (``hdgt_tr<Nb>``) twists column b by xi^(t Na + b) and runs an
    Nb-point DIF, writing tmp[b Nb + t]; pass 2 (``hdgt_tr<Na>``) multiplies
    tmp[t Nb + c] by g_N^(t brev_Nb(c)) and runs an Na-point DIF, writing
    out[c Na + t].  For N <= 512 it is one twisted N-point DIF (``dgt<N>``).
    """
    N = len(x)
    xi = canonical_xi(p, N) if xi is None else xi
    split = hdgt_split(N)
    if split is None:
        y = [gi_mul(x[n], gi_pow(xi, n, p), p) for n in range(N)]
        _gs_dif(y, p, N)
        return y
    Na, Nb = split
    gN = omega(p, N)
    lb = Nb.bit_length() - 1
    tmp = [None] * N
    for b in range(Na):
        col = [gi_mul(x[t * Na + b], gi_pow(xi, t * Na + b, p), p) for t in range(Nb)]
        _gs_dif(col, p, Nb)
        for t in range(Nb):
            tmp[t + b * Nb] = col[t]
    out = [None] * N
    for c in range(Nb):
        col = [gi_scale(tmp[t * Nb + c], pow(gN, t * brev(c, lb), p), p) for t in range(Na)]
        _gs_dif(col, p, Na)
        for t in range(Na):
            out[t + c * Na] = col[t]
    return out


def dgt_inverse_ref(X, p, xi=None):
    """cuPoly's inverse DGT of one residue (``dgt.cu:917-1006``; tables ``:1879-1960``).

    Pass 1 (``hidgt<Na>``): contiguous rows c, Na-point CT inverse, times
    g_N^-(brev_Nb(c) t) (Na Nb)^-1.  Pass 2 (``hidgt_tr<Nb>``): columns of
    stride Na, Nb-point CT inverse, times xi^-(t Na + b).  For N <= 512 the
    single-block inverse folds N^-1 into the untwist (``dgt.cu:1654-1662``).
    """
    N = len(X)
    xi = canonical_xi(p, N) if xi is None else xi
    xii = gi_pow(xi, 4 * N - 1, p)  # xi has order 4N
    ninv = pow(N, p - 2, p)
    split = hdgt_split(N)
    if split is None:
        y = list(X)
        _ct_dit_inv(y, p, N)
        return [gi_scale(gi_mul(y[n], gi_pow(xii, n, p), p), ninv, p) for n in range(N)]
    Na, Nb = split
    gNi = pow(omega(p, N), p - 2, p)
    lb = Nb.bit_length() - 1
    tmp = [None] * N
    for c in range(Nb):
        row = list(X[c * Na:(c + 1) * Na])
        _ct_dit_inv(row, p, Na)
        for t in range(Na):
            tmp[c * Na + t] = gi_scale(row[t], pow(gNi, brev(c, lb) * t, p) * ninv % p, p)
    out = [None] * N
    for b in range(Na):
        col = [tmp[t * Na + b] for t in range(Nb)]
        _ct_dit_inv(col, p, Nb)
        for t in range(Nb):
            out[t * Na + b] = gi_mul(col[t], gi_pow(xii, t * Na + b, p), p)
    return out


def dgt_forward_direct(x, p, xi=None):
    """O(N^2) definition: out[pos] = sum_n x[n] xi^n w_N^(n brev(pos)).

    The DGT domain of cuPoly is the twisted DFT of the folded signal stored in
    bit-reversed order, independent of the Na x Nb split.
    """
    N = len(x)
    xi = canonical_xi(p, N) if xi is None else xi
    w = omega(p, N)
    bits = N.bit_length() - 1
    tw = [gi_mul(x[n], gi_pow(xi, n, p), p) for n in range(N)]
    out = []
    for pos in range(N):
        k = brev(pos, bits)
        acc = (0, 0)
        for n in range(N):
            acc = gi_add(acc, gi_scale(tw[n], pow(w, n * k % N, p), p), p)
        out.append(acc)
    return out


# ----------------------------------------------------------------------------
# Folding, polynomial products
# ----------------------------------------------------------------------------
def fold(coeffs, p, N):
    """a_j -> (a_j mod p, a_{j+N} mod p) (``polynomial.cu:206-217``)."""
    c = list(coeffs) + [0] * (2 * N - len(coeffs))
    return [(c[j] % p, c[j + N] % p) for j in range(N)]


def unfold(res):
    N = len(res)
    return [res[j][0] for j in range(N)] + [res[j][1] for j in range(N)]


def negacyclic_mul_schoolbook(a, b, p):
    """c = a*b mod (x^n + 1, p): the definition cuPoly's tests check against NTL
    (``tests/unit_tests/test_bfv_mode.cu:1180-1208``)."""
    n = len(a)
    c = [0] * n
    for i, ai in enumerate(a):
        if ai == 0:
            continue
        for j, bj in enumerate(b):
            k = i + j
            if k < n:
                c[k] += ai * bj
            else:
                c[k - n] -= ai * bj
    return [x % p for x in c]


def polymul_dgt(a, b, p, xi=None):
    """fold -> forward DGT x2 -> pointwise GIMul -> inverse DGT -> unfold."""
    N = len(a) // 2
    A = dgt_forward_ref(fold(a, p, N), p, xi)
    B = dgt_forward_ref(fold(b, p, N), p, xi)
    C = [gi_mul(x, y, p) for x, y in zip(A, B)]
    return unfold(dgt_inverse_ref(C, p, xi))


# ----------------------------------------------------------------------------
# CRT and the exact HPS definitions
# ----------------------------------------------------------------------------
def crt(residues, primes):
    """The unique X in [0, prod(primes)) with X = r_i mod p_i."""
    M = prod(primes)
    x = 0
    for r, p in zip(residues, primes):
        Mi = M // p
        x += r * pow(Mi % p, p - 2, p) % p * Mi
    return x % M


# cuPoly's FPERROR (``include/cuPoly/settings.h:105``) as the exact value of the double 1e-9.
FPERROR_NUM, FPERROR_DEN = (1e-9).as_integer_ratio()


def lift_threshold(S: int) -> int:
    """T = S - floor(S FPERROR): cuPoly's base conversions read X in [T, S) as X - S.

    cuPoly's overflow count v is floor(sum_i y_i / s_i) unless that double lies
    within FPERROR of an integer, where it is rounded instead
    (``src/cuda/cudaengine.cu:513-534, 690-703``); with sum = v + X / S, v rounds
    up exactly when 1 - X / S <= FPERROR, i.e. S - X <= S FPERROR."""
    return S - S * FPERROR_NUM // FPERROR_DEN


def cupoly_lift(X: int, S: int) -> int:
    """The integer cuPoly's base conversion takes for X in [0, S): X, or X - S at or above
    the threshold (small negative values, as the scaled BFV tensor produces)."""
    return X - S if X >= lift_threshold(S) else X


def basis_extension_exact(xs, src, dst):
    """cupoly_lift(X) mod d_j for X = crt(xs, src) in [0, prod(src)), decided exactly.

    cuPoly computes this with a floating-point correction v
    (``src/cuda/cudaengine.cu:483-649, 659-796``); its tests assert X mod d_j on
    random X (``tests/unit_tests/test_bfv_mode.cu:640-730``), where the two agree.
    """
    S = prod(src)
    X = cupoly_lift(crt(xs, src), S)
    return [X % d for d in dst]


def complex_scaling_exact(xq, yb, Q, B, t):
    """round(t X / Q) mod b_j for X = crt(xq ++ yb, Q ++ B) in [0, Q B).

    cuPoly's HPS complex scaling (``src/cuda/cudaengine.cu:382-469``) targets
    this value; t X / Q is never a half-integer because Q is odd.
    """
    Qp = prod(Q)
    X = crt(list(xq) + list(yb), list(Q) + list(B))
    r = (2 * t * X + Qp) // (2 * Qp)
    return [r % b for b in B]


def complex_scaling_tdivq_exact(xq, yb, Q, B, t):
    """``poly_complex_scaling_tDivQ`` (``polynomial.cu:350-404``): Y = round(t X / Q) mod B,
    then its B -> Q conversion with cuPoly's lift (``basis_extension_exact``)."""
    Qp, Bp = prod(Q), prod(B)
    X = crt(list(xq) + list(yb), list(Q) + list(B))
    r = cupoly_lift((2 * t * X + Qp) // (2 * Qp) % Bp, Bp)
    return [r % q for q in Q]


def lift_digits(src):
    """Mixed-radix digits of lift_threshold(prod(src)) - 1 over src (for the C oracle)."""
    T1 = lift_threshold(prod(src)) - 1
    d, rest, base = [], T1, 1
    for s in src:  # X = sum_i d_i prod_{l<i} s_l
        d.append((rest // base) % s)
        base *= s
    return d


def simple_scaling_exact(xq, Q, t):
    """round(t X / Q) mod t for X = crt(xq, Q) (``cudaengine.cu:323-380``; test ``test_bfv_mode.cu:938-983``)."""
    Qp = prod(Q)
    X = crt(xq, Q)
    return (2 * t * X + Qp) // (2 * Qp) % t


# ----------------------------------------------------------------------------
# cuPoly's floating-point HPS path, restated word for word (disagreement counts)
# ----------------------------------------------------------------------------
# cuPoly estimates the CRT overflow and the HPS rounding in double precision.
# These functions reproduce its kernels' arithmetic from IEEE-754 semantics:
# round-to-nearest-even (Python float arithmetic, float(int), float(Fraction)),
# round-down (exact rational, then the next double below when the nearest is
# above), llrint = nearest-even, 64-bit wrap-around for cuPoly's addmod / submod
# macros (include/cuPoly/cuda/dgt.h:74-82).  Where that path is exact they equal
# the *_exact functions above; where it is not, the difference shows.
_U64 = (1 << 64) - 1
FPERROR = 1e-9  # include/cuPoly/settings.h


def _rd(r) -> float:
    """The largest double <= the rational r."""
    from fractions import Fraction
    import math

    f = float(r)
    if Fraction(f) > r:
        f = math.nextafter(f, -math.inf)
    return f


def _fma_rd(a: float, b: float, c: float) -> float:
    from fractions import Fraction

    return _rd(Fraction(a) * Fraction(b) + Fraction(c))


def _drcp_rd(d: float) -> float:
    from fractions import Fraction

    return _rd(1 / Fraction(d))


def _addmod64(a, b, p):
    """cuPoly's addmod on 64-bit words: a + b, minus p when a + b >= p (wrapping)."""
    s = (a + b) & _U64
    return (s - p) & _U64 if s >= p else s


def _submod64(a, b, p):
    """cuPoly's submod on 64-bit words: a - b, or a + (p - b) when a < b (wrapping)."""
    return (a + (p - b)) & _U64 if a < b else (a - b) & _U64


def _v_rule(value: float) -> int:
    """Overflow count from the double sum: the nearest integer when within FPERROR of
    it, else the floor (``src/cuda/cudaengine.cu:532-533, 700-701``)."""
    import math

    r = round(value)
    return r if abs(value - r) <= FPERROR else math.floor(value)


def cupoly_float_ext_q_to_b(xs, Q, B):
    """cuPoly's Q -> B conversion of one coefficient (``cudaengine.cu:483-649``):
    aux_i = x_i [(Q/q_i)^-1]_{q_i}; v from fma_rd(aux_i, rcp_rd(q_i)) summed in double;
    y_j = sum_i aux_i (Q/q_i mod b_j) - v (Q mod b_j) with cuPoly's addmod / submod."""
    Qp = prod(Q)
    aux = [x * pow(Qp // q % q, -1, q) % q for x, q in zip(xs, Q)]
    value = 0.0
    for a, q in zip(aux, Q):
        value = _fma_rd(float(a), _drcp_rd(float(q)), value)
    v = _v_rule(value)
    out = []
    for b in B:
        acc = 0
        for a, q in zip(aux, Q):
            acc = _addmod64(acc, a * (Qp // q % b) % b, b)
        out.append(_submod64(acc, v * (Qp % b) % b, b))
    return out


def cupoly_float_ext_b_to_q(ys, Q, B):
    """cuPoly's B -> Q conversion of one coefficient (``cudaengine.cu:659-796``): as
    the Q -> B one, with v from aux_j / (double) b_j summed in round-to-nearest."""
    Bp = prod(B)
    aux = [y * pow(Bp // b % b, -1, b) % b for y, b in zip(ys, B)]
    value = 0.0
    for a, b in zip(aux, B):
        value += float(a) / float(b)
    v = _v_rule(value)
    out = []
    for q in Q:
        acc = 0
        for a, b in zip(aux, B):
            acc = _addmod64(acc, a * (Bp // b % q) % q, q)
        out.append(_submod64(acc, v * (Bp % q) % q, q))
    return out


def _rr_round(m: int, e: int, prec: int, sticky: bool = False):
    """NTL RR rounding: m 2^e (m >= 0) to ``prec`` mantissa bits, to nearest, ties to
    even; ``sticky`` marks nonzero bits already dropped below m."""
    nb = m.bit_length()
    if nb > prec:
        drop = nb - prec
        kept, rest, half = m >> drop, m & ((1 << drop) - 1), 1 << (drop - 1)
        if rest > half or (rest == half and (sticky or kept & 1)):
            kept += 1
        m, e = kept, e + drop
    return m, e


def _rr_quotient_frac(aux: int, q: int, prec: int = 512):
    """cuPoly's split of aux / q into an integer part and a 128-bit fraction
    (``cudaengine.cu:1479-1486``, ``:1498-1506``): RR::SetPrecision(512); tmp = to_RR(aux)
    / to_RR(q) -- each step rounded to 512 bits as NTL's RR does -- then
    FloorToZZ(tmp) and floor((tmp - floor(tmp)) 2^128).  When aux / q has more than
    384 integer bits, the fraction keeps only the rounded quotient's low bits."""
    ma, ea = _rr_round(aux, 0, prec)
    s = max(prec + 2 + q.bit_length() - ma.bit_length(), 0)
    quo, rem = divmod(ma << s, q)
    m, e = _rr_round(quo, ea - s, prec, rem != 0)
    if e >= 0:
        return m << e, 0
    ip = m >> -e
    frac = m - (ip << -e)  # fractional part = frac 2^e, exact
    return ip, (frac << 128) >> -e


@lru_cache(maxsize=None)
def _cupoly_omega(Q, B, t):
    """omega_int, the 128-bit omega_frac and lambda of ``cudaengine.cu:1463-1492``:
    omega_{l,j} = t [(QB/q_l)^-1]_{q_l} B / q_l split into its integer part mod b_j and
    a 128-bit fraction, both from the 512-bit RR quotient (``_rr_quotient_frac``);
    lambda_j = t [(QB/b_j)^-1]_{b_j} (B/b_j) mod b_j."""
    Qp, Bp = prod(Q), prod(B)
    lam = tuple(t * pow(Bp * Qp // b % b, -1, b) * (Bp // b) % b for b in B)
    om_int, om_frac = {}, {}
    for j, b in enumerate(B):
        for l, q in enumerate(Q):
            aux = t * pow(Qp * Bp // q % q, -1, q) * Bp
            ti, fr = _rr_quotient_frac(aux, q)
            om_int[l, j] = ti % b
            om_frac[l, j] = fr
    return om_int, om_frac, lam


@lru_cache(maxsize=None)
def _cupoly_tomega(Q, t):
    """tomega_int and the 128-bit tomega_frac of ``cudaengine.cu:1494-1509``:
    t [(Q/q_i)^-1]_{q_i} / q_i from the 512-bit RR quotient."""
    Qp = prod(Q)
    return tuple(_rr_quotient_frac(t * pow(Qp // q % q, -1, q), q) for q in Q)


def cupoly_float_complex_scaling(xq, yb, Q, B, t):
    """cuPoly's polynomial_complex_scaling for one coefficient (``cudaengine.cu:382-440``):
    per B prime, sum over Q of x omega_int mod b_j plus the integer part of
    omega_frac x (__umul128hi = floor(omega_frac x / 2^64), 128 bits), the fraction
    parts accumulated in double by fma_rn (exact products: lo 2^-64) and added back by
    llrint, plus x_B lambda_j; cuPoly's addmod throughout (so a B residue can stay
    non-canonical when an integer part reaches b_j)."""
    om_int, om_frac, lam = _cupoly_omega(tuple(Q), tuple(B), t)
    out = []
    for j, b in enumerate(B):
        result, acc = 0, 0.0
        for l, x in enumerate(xq):
            vint = x * om_int[l, j] % b
            c = (om_frac[l, j] * x) >> 64
            hi, lo = c >> 64, c & _U64
            acc = float(lo) * 2.0 ** -64 + acc
            result = _addmod64(result, _addmod64(vint, hi, b), b)
        result = _addmod64(result, round(acc), b)
        result = _addmod64(result, yb[j] * lam[j] % b, b)
        out.append(result)
    return out


def cupoly_float_complex_scaling_tdivq(xq, yb, Q, B, t):
    """``poly_complex_scaling_tDivQ`` on cuPoly's float path: the scaling above, then
    its float B -> Q conversion (``polynomial.cu:350-404``)."""
    return cupoly_float_ext_b_to_q(cupoly_float_complex_scaling(xq, yb, Q, B, t), Q, B)


def cupoly_float_simple_scaling(xq, Q, t, raw=False):
    """cuPoly's simple_scaling for one coefficient, t a power of two (``cudaengine.cu:323-362``,
    tomega from ``:1494-1509``): integer parts and fraction parts of x tomega summed, the
    fraction parts' low words in double and added back by llrint.

    The kernel masks with its constant d_RNST - 1, but nothing ever writes d_RNST
    (declared at ``cudaengine.cu:93``; no cudaMemcpyToSymbol of it in the precompute,
    ``:1337-1673``), so the mask is 2^64 - 1 and the device word is the sum mod 2^64
    (``raw=True``).  Reduced mod t -- as cuPoly's download does for TBase,
    ``polynomial.cu:289`` -- it is the value the kernel intends (the default)."""
    assert t > 0 and t & (t - 1) == 0
    result, acc = 0, 0.0
    for x, (ti, frac) in zip(xq, _cupoly_tomega(tuple(Q), t)):
        vint = (x * ti) & _U64
        c = (frac * x) >> 64
        hi, lo = c >> 64, c & _U64
        acc = acc + float(lo) * 2.0 ** -64
        result = (result + ((vint + hi) & _U64)) & _U64
    word = (result + round(acc)) & _U64
    return word if raw else word & (t - 1)


# ----------------------------------------------------------------------------
# Sampler: Philox4x32-10 and the distributions of the device sampler
# ----------------------------------------------------------------------------
_M = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11, "Parallel random numbers:
    as easy as 1, 2, 3").  Returns four 32-bit words."""
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        hi0, lo0 = p0 >> 32, p0 & _M
        hi1, lo1 = p1 >> 32, p1 & _M
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & _M, lo1, (hi0 ^ c3 ^ k1) & _M, lo0
        k0 = (k0 + 0x9E3779B9) & _M
        k1 = (k1 + 0xBB67AE85) & _M
    return c0, c1, c2, c3


def load_cdt(name):
    """Read one cumulative table (uint64 thresholds) from cdt_table.h."""
    src = open(_CDT_HEADER).read()
    m = _re.search(name + r"\[\]\s*=\s*\{([^}]*)\}", src)
    return [int(x.strip().rstrip("ULL")) for x in m.group(1).split(",") if x.strip()]


# Distribution kinds of the device sampler (values of enum cp_distribution).
DISCRETE_GAUSSIAN, HAMMINGWEIGHT, NARROW, ZO, BINARY, UNIFORM, TERNARY, GAUSSIAN = range(8)
SIGNED_DG = 8  # CKKS engines: DISCRETE_GAUSSIAN without the absolute value (device-internal kind)
UNIFORM_U32 = 9  # cuPoly's BFV UNIFORM (src/cuda/sampler.cu:295-341): one value below 2^32 for all residues
ZO_HALF = 10  # cuPoly's BFV ZO (src/cuda/sampler.cu:236-283): exactly nphi/2 nonzero, each +-1


def zo_half_position(c, nphi, sid, seed):
    """Image of coefficient c under the device's keyed bijection of [0, nphi): a 4-round
    Feistel network with Philox4x32-10 rounds over counters (half, 0x5A000000 + round,
    stream id, ZO_HALF); for odd log2(nphi) it runs on one more bit and walks the cycle
    back into range."""
    k0, k1 = seed & _M, (seed >> 32) & _M
    b = nphi.bit_length() - 1
    hb = (b + 1) >> 1
    m = (1 << hb) - 1
    x = c
    for _ in range(64):
        L, R = x >> hb, x & m
        for r in range(4):
            f = philox4x32_10((R, 0x5A000000 + r, sid, ZO_HALF), (k0, k1))[0] & m
            L, R = R, L ^ f
        x = (L << hb) | R
        if x < nphi:
            return x
    raise RuntimeError("cycle walk limit")


def _cdt_lookup(u63, cdt):
    return sum(1 for t in cdt if u63 >= t)


def sample_small(kind, c, sid, seed):
    """Signed value of coefficient c for the residue-independent kinds.

    Restates the device sampler: Philox4x32-10 with key (seed_lo, seed_hi) and
    counter (c, draw, stream id, kind).  cuPoly's kinds (src/cuda/sampler.cu:
    73-493): NARROW {0,1,2}, BINARY {0,1}, DISCRETE_GAUSSIAN |round(3.2 Z)|;
    ZO is i.i.d. (cuPoly fixes exactly half the coefficients nonzero).
    """
    k0, k1 = seed & _M, (seed >> 32) & _M
    if kind == ZO_HALF:
        raise ValueError("ZO_HALF depends on nphi: use sample_zo_half")
    if kind in (NARROW, TERNARY):
        for d in range(8):
            for w in philox4x32_10((c, d, sid, kind), (k0, k1)):
                if w != 0xFFFFFFFF:
                    x = w % 3
                    return -1 if (kind == TERNARY and x == 2) else x
        raise RuntimeError("rejection limit")
    r = philox4x32_10((c, 0, sid, kind), (k0, k1))
    u63 = ((r[1] & 0x7FFFFFFF) << 32) | r[0]
    if kind == BINARY:
        return r[0] & 1
    if kind == ZO:
        b = r[0] & 3
        return 0 if b < 2 else (1 if b == 2 else -1)
    if kind == DISCRETE_GAUSSIAN:
        return _cdt_lookup(u63, load_cdt("kCdtFolded"))
    if kind == GAUSSIAN:
        m = _cdt_lookup(u63, load_cdt("kCdtSigned"))
        return -m if (r[2] & 1) else m
    if kind == SIGNED_DG:
        m = _cdt_lookup(u63, load_cdt("kCdtFolded"))
        return -m if (r[2] & 1) else m
    raise ValueError(kind)


def sample_uniform_pair(j, r, p, sid, seed):
    """Uniform residues mod p of coefficients j and j + N (Gaussian element j) in residue r:
    draw d = 0, 1, ... gives one candidate of bitlen(p) bits for each coefficient (words 0-1
    for j, words 2-3 for j + N); each coefficient keeps its first candidate below p."""
    k0, k1 = seed & _M, (seed >> 32) & _M
    mask = (1 << p.bit_length()) - 1
    v = [None, None]
    for d in range(16):
        q = philox4x32_10((j, r * 16 + d, sid, UNIFORM), (k0, k1))
        u = (((q[1] << 32) | q[0]) & mask, ((q[3] << 32) | q[2]) & mask)
        for h in (0, 1):
            if v[h] is None and u[h] < p:
                v[h] = u[h]
        if v[0] is not None and v[1] is not None:
            return v
    raise RuntimeError("rejection limit")


def sample_hamming(nphi, sid, seed, h=64):
    """{position: +-1} with exactly min(h, nphi) entries (cuPoly HAMMINGWEIGHT_H = 64, settings.h:43)."""
    k0, k1 = seed & _M, (seed >> 32) & _M
    lg = nphi.bit_length() - 1
    out = {}
    for i in range(min(h, nphi)):
        for d in range(1024):
            q = philox4x32_10((i, d, sid, HAMMINGWEIGHT), (k0, k1))
            pos = (q[0] >> (32 - lg)) if lg else 0
            if pos not in out:
                out[pos] = -1 if (q[1] & 1) else 1
                break
    return out


def sample_zo_half(nphi, sid, seed):
    """cuPoly's ZO with exactly nphi/2 nonzero coefficients: coefficient c is nonzero iff
    its image under the keyed bijection is below nphi/2; its sign is bit 0 of the
    Philox block (c, 1, stream id, ZO_HALF)."""
    k0, k1 = seed & _M, (seed >> 32) & _M
    out = []
    for c in range(nphi):
        if zo_half_position(c, nphi, sid, seed) >= nphi // 2:
            out.append(0)
        else:
            out.append(-1 if philox4x32_10((c, 1, sid, ZO_HALF), (k0, k1))[0] & 1 else 1)
    return out


def sample_poly(kind, primes, nphi, sid, seed, ckks=False):
    """(nres, nphi) coefficient rows the device sampler produces.  On a CKKS engine the
    small kinds are signed, as in cuPoly's CKKS build (``src/cuda/sampler.cu:73-106,
    459-493``): NARROW is uniform {-1, 0, 1} and DISCRETE_GAUSSIAN is nearbyint(3.2 Z)."""
    if ckks:
        kind = {NARROW: TERNARY, DISCRETE_GAUSSIAN: SIGNED_DG}.get(kind, kind)
    rows = []
    if kind == UNIFORM_U32:
        N = nphi // 2
        k0, k1 = seed & _M, (seed >> 32) & _M
        w = [philox4x32_10((j, 0, sid, UNIFORM_U32), (k0, k1)) for j in range(N)]
        row = [q[0] for q in w] + [q[1] for q in w]
        return [list(row) for _ in primes]
    if kind == ZO_HALF:
        vals = sample_zo_half(nphi, sid, seed)
        return [[v % p for v in vals] for p in primes]
    if kind == UNIFORM:
        N = nphi // 2
        rows = []
        for r, p in enumerate(primes):
            pairs = [sample_uniform_pair(j, r, p, sid, seed) for j in range(N)]
            rows.append([v[0] for v in pairs] + [v[1] for v in pairs])
        return rows
    if kind == HAMMINGWEIGHT:
        hw = sample_hamming(nphi, sid, seed)
        vals = [hw.get(c, 0) for c in range(nphi)]
    else:
        vals = [sample_small(kind, c, sid, seed) for c in range(nphi)]
    for p in primes:
        rows.append([v % p for v in vals])
    return rows
