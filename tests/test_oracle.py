"""Pins of the CPU oracle (no GPU): golden fixtures, exact definitions, and the
C restatement against the Python big-integer restatement.

cuPoly ships no golden vectors; its tests are property tests against NTL
(tests/unit_tests/test_bfv_mode.cu).  The same properties are checked here
against Python integers, and the DGT-domain fixtures made with cuPoly's own
root table (tests/golden/ref_nthroot.json) are re-derived.
"""
import json
import os

import numpy as np
import pytest
import sympy

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import fold, gi_rows_to_list, random_poly_int, random_poly_residues, sha, unfold

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_prime_table():
    assert len(O.PRIMES) == 100 and O.PRIMES == sorted(O.PRIMES, reverse=True)
    for p, g in list(zip(O.PRIMES, O.PROOTS))[:12]:
        assert sympy.isprime(p) and p < 2 ** 63 and (p - 1) % (1 << 17) == 0
        for f in sympy.factorint(p - 1):
            assert pow(g, (p - 1) // f, p) != 1
        assert g == sympy.ntheory.primitive_root(p)  # smallest primitive root


def test_prime_table_is_cupolys_bucket():
    """The 100 primes, in order, are cuPoly's COPRIMES_63_BUCKET and the primitive
    roots its PROOTS (src/arithmetic/coprimes.cu:763-866, :26976): SHA-256 of the
    comma-joined decimal lists, taken from that file."""
    import hashlib
    digest = lambda xs: hashlib.sha256(",".join(map(str, xs)).encode()).hexdigest()  # noqa: E731
    assert digest(O.PRIMES) == "ee159669b078b2215faef040edc778ae39fc2f40c4089db139fa03fa251daf36"
    assert digest([O.PROOT[p] for p in O.PRIMES]) == \
        "224baee04d60cb7a9bb6f09cd87d3db8c851c7f025fe42902402b7437d96a926"


@pytest.mark.parametrize("N", [2, 4, 16, 32, 64])
def test_dgt_is_bitreversed_twisted_dft(N):
    p = O.PRIMES[3]
    x = gi_rows_to_list(fold(random_poly_residues(N, [p], 2 * N))[0])
    assert O.dgt_forward_ref(x, p) == O.dgt_forward_direct(x, p)


@pytest.mark.parametrize("N", [1024, 2048, 4096])
def test_hierarchical_roundtrip(N):
    p = O.PRIMES[1]
    x = gi_rows_to_list(fold(random_poly_residues(5, [p], 2 * N))[0])
    assert O.dgt_inverse_ref(O.dgt_forward_ref(x, p), p) == x


@pytest.mark.parametrize("nphi", [32, 128, 256])
def test_polymul_is_negacyclic_product(nphi):
    """cuPoly TestArithmetic.Mul: a*b mod (x^nphi + 1) per prime (test_bfv_mode.cu:1180-1208)."""
    for p in O.PRIMES[:2]:
        a = random_poly_residues(1, [p], nphi)[0].tolist()
        b = random_poly_residues(2, [p], nphi)[0].tolist()
        assert O.polymul_dgt(a, b, p) == O.negacyclic_mul_schoolbook(a, b, p)


def test_canonical_xi_family():
    p = O.PRIMES[0]
    for N in [16, 1024, 32768]:
        xi = O.canonical_xi(p, N)
        assert O.gi_pow(xi, N, p) == (0, 1)
        if N < 32768:
            x2 = O.canonical_xi(p, 2 * N)
            assert O.gi_mul(x2, x2, p) == xi


def test_golden_dgt_python_and_c():
    roots = json.load(open(os.path.join(GOLD, "ref_nthroot.json")))
    for case in json.load(open(os.path.join(GOLD, "dgt_golden.json"))):
        nphi, nres, seed = case["nphi"], case["nres"], case["seed"]
        N = nphi // 2
        primes = O.PRIMES[:nres]
        x = fold(random_poly_residues(seed, primes, nphi))
        xi = [tuple(roots[str(p)][str(N)]) for p in primes]
        y = CO.dgt(x[None], primes, xi=xi)[0]
        assert sha(y) == case["sha256"], case
        assert [[int(a), int(b)] for a, b in y[0, :4].tolist()] == case["head"]
        if nphi <= 256:
            out = np.array([O.dgt_forward_ref(gi_rows_to_list(x[r]), p, xi[r]) for r, p in enumerate(primes)],
                           dtype=np.uint64)
            assert sha(out) == case["sha256"]


def test_golden_hps_c_oracle():
    for case in json.load(open(os.path.join(GOLD, "hps_golden.json"))):
        Q, B = O.bases(case["k"], case["kl"])
        xq = random_poly_residues(case["seed"], Q, case["nphi"])
        yb = random_poly_residues(case["seed"] + 1000, B, case["nphi"])
        assert sha(CO.basis_ext(xq, Q, B)) == case["ext_q_to_b"]
        assert sha(CO.basis_ext(yb, B, Q)) == case["ext_b_to_q"]
        assert sha(CO.complex_scaling(xq, yb, Q, B, case["t"])) == case["complex_scaling"]
        assert sha(CO.simple_scaling(xq, Q, case["t"])) == case["simple_scaling"]


def test_basis_extension_edges():
    """cuPoly's lift, decided exactly: X in [0, Q) reads as X - Q from the threshold
    T = Q - floor(Q FPERROR) on (cuPoly rounds its overflow count up within FPERROR of
    an integer, src/cuda/cudaengine.cu:513-534), as X below it; the C and Python
    restatements agree on both sides of T."""
    for k in (1, 3, 6):
        Q, B = O.bases(k, k + 1)
        Qp = O.prod(Q)
        T = O.lift_threshold(Qp)
        assert Qp - T == Qp * O.FPERROR_NUM // O.FPERROR_DEN
        for X in [0, 1, (Qp - 1) // 2, (Qp + 1) // 2, T - 2, T - 1, T, T + 1, Qp - 2, Qp - 1]:
            want = [(X - Qp if X >= T else X) % b for b in B]
            xs = np.array([[X % q] for q in Q], dtype=np.uint64)
            assert CO.basis_ext(xs, Q, B)[:, 0].tolist() == want
            assert O.basis_extension_exact([X % q for q in Q], Q, B) == want


def test_scaling_rounding_edges():
    """round(t X / Q) next to the half-integer boundary and for t not a power of two."""
    Q, B = O.bases(2, 3)
    Qp, Bp = O.prod(Q), O.prod(B)
    for t in [256, 65537, 3]:
        for X in [0, 1, Qp // (2 * t), Qp // (2 * t) + 1, Qp - 1, Qp * Bp - 1, (Qp * Bp) // 2]:
            xq = np.array([[X % q] for q in Q], dtype=np.uint64)
            yb = np.array([[X % b] for b in B], dtype=np.uint64)
            r = (2 * t * X + Qp) // (2 * Qp)
            assert CO.complex_scaling(xq, yb, Q, B, t)[:, 0].tolist() == [r % b for b in B]
            Xq = X % Qp
            assert int(CO.simple_scaling(xq, Q, t)[0]) == (2 * t * Xq + Qp) // (2 * Qp) % t


def test_c_polymul_matches_schoolbook():
    Q = O.PRIMES[:2]
    a = random_poly_residues(3, Q, 512)
    b = random_poly_residues(4, Q, 512)
    c = CO.polymul(a[None], b[None], Q)[0]
    for r, p in enumerate(Q):
        assert c[r].tolist() == O.negacyclic_mul_schoolbook(a[r].tolist(), b[r].tolist(), p)


def test_c_bfv_mul_matches_bigint_definition():
    """(round(t/Q * tensor) mod B) mod q_i over exact integers (poly_dr2 + poly_complex_scaling_tDivQ)."""
    k, nphi, t = 2, 32, 256
    Q, B = O.bases(k, k + 1)
    Qp, Bp = O.prod(Q), O.prod(B)
    ints = [random_poly_int(40 + i, Qp, nphi) for i in range(4)]
    rows = [np.array([[x % q for x in v] for q in Q], dtype=np.uint64) for v in ints]
    c = CO.bfv_mul(*[r[None] for r in rows], Q, B, t)

    def nmul(u, w):
        out = [0] * nphi
        for i in range(nphi):
            for j in range(nphi):
                if i + j < nphi:
                    out[i + j] += u[i] * w[j]
                else:
                    out[i + j - nphi] -= u[i] * w[j]
        return out

    a0, a1, b0, b1 = ints
    tens = [nmul(a0, b0), [x + y for x, y in zip(nmul(a0, b1), nmul(a1, b0))], nmul(a1, b1)]
    for T, cc in zip(tens, c):
        for j in range(nphi):
            X = T[j] % (Qp * Bp)
            r = O.cupoly_lift((2 * t * X + Qp) // (2 * Qp) % Bp, Bp)  # small negatives stay negative
            assert [r % q for q in Q] == cc[0][:, j].tolist()


def test_philox_known_answers():
    """Random123 known-answer vectors for Philox4x32-10."""
    assert O.philox4x32_10((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert O.philox4x32_10((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF)) == (
        0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert O.philox4x32_10((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == (
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def test_cdt_tables_are_monotone():
    for name in ("kCdtSigned", "kCdtFolded"):
        t = O.load_cdt(name)
        assert len(t) == 19 and all(a < b for a, b in zip(t, t[1:])) and t[-1] < 2 ** 63


def test_sampler_restatement_support():
    primes = O.PRIMES[:2]
    for kind, support in [(O.NARROW, {0, 1, 2}), (O.BINARY, {0, 1}), (O.TERNARY, {-1, 0, 1}), (O.ZO, {-1, 0, 1})]:
        vals = {O.sample_small(kind, c, 0, 42) for c in range(256)}
        assert vals <= support
    hw = O.sample_hamming(128, 0, 42)
    assert len(hw) == 64 and set(hw.values()) <= {-1, 1}
    rows = O.sample_poly(O.UNIFORM, primes, 16, 3, 42)
    assert all(0 <= v < p for row, p in zip(rows, primes) for v in row)


def test_fold_unfold():
    x = np.arange(16, dtype=np.uint64).reshape(2, 8)
    assert (unfold(fold(x)) == x).all()


@pytest.mark.parametrize("k", [1, 2, 4, 5])
def test_cupoly_float_path_equals_exact_on_random_inputs(k):
    """The restatement of cuPoly's double-precision HPS path (overflow count with FPERROR,
    128-bit fractions summed in double, constants from 512-bit RR quotients) gives the
    exact values on random inputs up to k = 5 (the benchmark's BFV size)."""
    import random
    rng = random.Random(k)
    Q, B = O.bases(k, k + 1)
    Qp, Bp = O.prod(Q), O.prod(B)
    for _ in range(150):
        X, Y, Z = rng.randrange(Qp), rng.randrange(Bp), rng.randrange(Qp * Bp)
        xs, ys = [X % q for q in Q], [Y % b for b in B]
        zq, zb = [Z % q for q in Q], [Z % b for b in B]
        assert O.cupoly_float_ext_q_to_b(xs, Q, B) == O.basis_extension_exact(xs, Q, B)
        assert O.cupoly_float_ext_b_to_q(ys, Q, B) == O.basis_extension_exact(ys, B, Q)
        assert O.cupoly_float_complex_scaling(zq, zb, Q, B, 256) == O.complex_scaling_exact(zq, zb, Q, B, 256)
        assert O.cupoly_float_complex_scaling_tdivq(zq, zb, Q, B, 256) == \
            O.complex_scaling_tdivq_exact(zq, zb, Q, B, 256)
        assert O.cupoly_float_simple_scaling(xs, Q, 256) == O.simple_scaling_exact(xs, Q, 256)


def test_cupoly_complex_scaling_is_off_by_one_often_at_k6():
    """At k = 6, kl = 7 (the largest base of cuPoly's own test grid) the 512-bit RR
    quotient behind omega keeps only about 63 fraction bits, so the fraction sum of
    cuPoly's complex scaling lands on the wrong side of the rounding boundary for a
    sizeable share of ordinary coefficients -- always by exactly one (cuPoly's own test
    allows |error| < 2, test_bfv_mode.cu:1092-1095).  Simple scaling and the base
    conversions stay exact there."""
    import random
    rng = random.Random(6)
    Q, B = O.bases(6, 7)
    Qp, Bp = O.prod(Q), O.prod(B)
    wrong = 0
    for _ in range(200):
        Z = rng.randrange(Qp * Bp)
        zq, zb = [Z % q for q in Q], [Z % b for b in B]
        f = O.cupoly_float_complex_scaling(zq, zb, Q, B, 256)
        e = O.complex_scaling_exact(zq, zb, Q, B, 256)
        if f != e:
            wrong += 1
            assert (O.crt(f, B) - O.crt(e, B)) % Bp in (1, Bp - 1)
        xs = [Z % q for q in Q]
        assert O.cupoly_float_ext_q_to_b(xs, Q, B) == O.basis_extension_exact(xs, Q, B)
        assert O.cupoly_float_simple_scaling(xs, Q, 256) == O.simple_scaling_exact(xs, Q, 256)
    assert 10 < wrong < 100


def test_cupoly_complex_scaling_constants_break_beyond_512_bits():
    """cuPoly computes omega = t [(QB/q_l)^-1] B / q_l as a 512-bit RR quotient
    (src/cuda/cudaengine.cu:1463-1490).  Once that quotient needs more than 512 bits
    (k = 10, kl = 11: about 700), its integer part is rounded by about 2^189, so
    omega_int mod b_j is unrelated to the true value and cuPoly's complex scaling is
    wrong on ordinary inputs, not only at edges.  The exact definitions (and the
    device) do not depend on those constants."""
    import random
    rng = random.Random(10)
    Q, B = O.bases(10, 11)
    Qp, Bp = O.prod(Q), O.prod(B)
    wrong = 0
    for _ in range(20):
        Z = rng.randrange(Qp * Bp)
        zq, zb = [Z % q for q in Q], [Z % b for b in B]
        exact = O.complex_scaling_exact(zq, zb, Q, B, 256)
        assert exact == [((2 * 256 * Z + Qp) // (2 * Qp)) % b for b in B]
        wrong += O.cupoly_float_complex_scaling(zq, zb, Q, B, 256) != exact
    assert wrong == 20


def test_cupoly_float_path_is_off_at_its_edges():
    """cuPoly's float path reads X = Q - 1 as X - Q (v rounded up within FPERROR) -- the
    lift the exact definitions follow too -- and rounds t X / Q within 1/Q of a
    half-integer the wrong way about half the time, each time by exactly one; the
    exact definitions used here and on the device are right there."""
    import random
    rng = random.Random(7)
    for k in (1, 3, 5):
        Q, B = O.bases(k, k + 1)
        Qp, Bp = O.prod(Q), O.prod(B)
        xs = [(Qp - 1) % q for q in Q]
        assert O.cupoly_float_ext_q_to_b(xs, Q, B) == [(Qp - 1 - Qp) % b for b in B]
        assert O.basis_extension_exact(xs, Q, B) == [(Qp - 1 - Qp) % b for b in B]
        ti, wrong = pow(256, -1, Qp), 0
        for h in ((Qp - 1) // 2, (Qp + 1) // 2, (Qp - 3) // 2, (Qp + 3) // 2):
            for _ in range(3):
                Z = (h * ti) % Qp + Qp * rng.randrange(Bp)  # 256 Z = h mod Q: next to a half-integer
                zq, zb = [Z % q for q in Q], [Z % b for b in B]
                f = O.cupoly_float_complex_scaling(zq, zb, Q, B, 256)
                ex = O.complex_scaling_exact(zq, zb, Q, B, 256)
                if f != ex:
                    wrong += 1
                    assert all((a - e) % b in (1, b - 1) for a, e, b in zip(f, ex, B))
        assert wrong > 0


@pytest.mark.parametrize("nphi", [4, 8, 32, 64, 128, 2048])
def test_zo_half_restatement_has_exactly_half_nonzero(nphi):
    """cuPoly's ZO (src/cuda/sampler.cu:236-283): exactly nphi/2 coefficients in
    {-1, +1}; the keyed bijection behind it is a permutation of [0, nphi)."""
    for sid in range(3):
        assert sorted(O.zo_half_position(c, nphi, sid, 99) for c in range(nphi)) == list(range(nphi))
        v = O.sample_zo_half(nphi, sid, 99)
        assert set(v) <= {-1, 0, 1} and sum(1 for x in v if x) == nphi // 2


def test_uniform_u32_restatement_is_one_word_on_every_residue():
    """cuPoly's BFV UNIFORM (src/cuda/sampler.cu:295-341): one value below 2^32 per
    coefficient, written to every residue."""
    rows = O.sample_poly(O.UNIFORM_U32, O.PRIMES[:3], 64, 4, 11)
    assert rows[0] == rows[1] == rows[2] and max(rows[0]) < 1 << 32 and len(set(rows[0])) == 64
