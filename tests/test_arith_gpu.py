"""Pointwise arithmetic and cuPoly's TestArithmetic / TestRNS ports on the GPU.

The reference's parameter grid is (logq2, nphi) with k = ceil(logq2 / 63),
kl = k + 1, t = 256 (tests/unit_tests/test_bfv_mode.cu:1492-1508)."""
import math

import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import fold, random_poly_residues, unfold

pytestmark = pytest.mark.gpu

GRID = [(30, 32), (120, 32), (340, 32), (120, 256), (30, 2048), (340, 2048), (170, 4096), (340, 8192)]


def _ref_engine(logq2, nphi):
    from cupoly_b200 import cupoly as cp
    k = math.ceil(logq2 / 63)
    cp.CUDAEngine.init(k, k + 1, nphi, 256)
    ctx = cp.Context()
    cp.Sampler.init(ctx)
    return cp, ctx


def _gi_mul(a, b, p):
    """Exact Gaussian product of folded arrays (numpy object ints)."""
    ar, ai = a[..., 0].astype(object), a[..., 1].astype(object)
    br, bi = b[..., 0].astype(object), b[..., 1].astype(object)
    return np.stack([(ar * br - ai * bi) % p, (ar * bi + ai * br) % p], -1).astype(np.uint64)


def test_pointwise_ops_vs_exact(gpu):
    from cupoly_b200.engine import ADD, MUL, MULMUL, ADDADD, SUB, Engine, from_u64, to_u64
    e = Engine(3, 4, 2048, 256)
    for base in (0, 1, 2):
        primes = e.base_primes(base)
        P = np.array(primes, dtype=object)[:, None]
        xs = [fold(random_poly_residues(10 * base + i, primes, 2048))[None] for i in range(4)]
        a, b, c, d = (from_u64(x) for x in xs)
        A, Bv, Cv, D = (x[0].astype(object) for x in xs)
        out, out2, out3 = e.empty(base), e.empty(base), e.empty(base)

        e.add(out, a, b, base)
        assert np.array_equal(to_u64(out)[0], ((A + Bv) % P[..., None]).astype(np.uint64))
        e.sub(out, a, b, base)
        assert np.array_equal(to_u64(out)[0], ((A - Bv) % P[..., None]).astype(np.uint64))
        e.mul(out, a, b, base)
        ref_mul = np.stack([_gi_mul(xs[0][0, r], xs[1][0, r], p) for r, p in enumerate(primes)])
        assert np.array_equal(to_u64(out)[0], ref_mul)
        e.muladd(out, a, b, c, base)
        assert np.array_equal(to_u64(out)[0], ((ref_mul.astype(object) + Cv) % P[..., None]).astype(np.uint64))
        e.dr2(out, out2, out3, a, b, c, d, base)
        r21 = np.stack([_gi_mul(xs[0][0, r], xs[2][0, r], p) for r, p in enumerate(primes)])
        r22 = np.stack([(_gi_mul(xs[0][0, r], xs[3][0, r], p).astype(object) +
                         _gi_mul(xs[1][0, r], xs[2][0, r], p).astype(object)) % p for r, p in enumerate(primes)])
        r23 = np.stack([_gi_mul(xs[1][0, r], xs[3][0, r], p) for r, p in enumerate(primes)])
        assert np.array_equal(to_u64(out)[0], r21)
        assert np.array_equal(to_u64(out2)[0], r22.astype(np.uint64))
        assert np.array_equal(to_u64(out3)[0], r23)
        e.double_add(out, a, b, out2, c, d, base)
        assert np.array_equal(to_u64(out)[0], ((A + Bv) % P[..., None]).astype(np.uint64))
        assert np.array_equal(to_u64(out2)[0], ((Cv + D) % P[..., None]).astype(np.uint64))
        e.negate(out, a, base)
        assert np.array_equal(to_u64(out)[0], ((-A) % P[..., None]).astype(np.uint64))
        for x in (0, 7, 2 ** 64 - 1):
            e.op_by_int(out, a, base, x, ADD)
            exp = A.copy()
            exp[..., 0] = (exp[..., 0] + x) % P
            assert np.array_equal(to_u64(out)[0], exp.astype(np.uint64))
            e.op_by_int(out, a, base, x, SUB)
            exp = A.copy()
            exp[..., 0] = (exp[..., 0] - x) % P
            assert np.array_equal(to_u64(out)[0], exp.astype(np.uint64))
            e.op_by_int(out, a, base, x, MUL)
            assert np.array_equal(to_u64(out)[0], ((A * x) % P[..., None]).astype(np.uint64))
        e.double_op_by_int(out, a, out2, b, base, 5, 9, MULMUL)
        assert np.array_equal(to_u64(out)[0], ((A * 5) % P[..., None]).astype(np.uint64))
        assert np.array_equal(to_u64(out2)[0], ((Bv * 9) % P[..., None]).astype(np.uint64))
        e.double_op_by_int(out, a, out2, b, base, 5, 9, ADDADD)
        exp = A.copy()
        exp[..., 0] = (exp[..., 0] + 5) % P
        assert np.array_equal(to_u64(out)[0], exp.astype(np.uint64))
        u64 = random_poly_residues(99, primes, 1024)  # (nres, N) multipliers
        bu = from_u64(u64)
        e.mul_u64(out, a, bu, base)
        assert np.array_equal(to_u64(out)[0], ((A * u64.astype(object)[..., None]) % P[..., None]).astype(np.uint64))


@pytest.mark.parametrize("nphi,k", [(2048, 2), (4096, 2), (8192, 5), (16384, 3), (32768, 2), (65536, 1)])
def test_polymul_vs_oracle(gpu, nphi, k):
    """forward DGT x2, pointwise, inverse: the negacyclic product per prime."""
    from cupoly_b200.engine import FORWARD, INVERSE, Engine, from_u64, to_u64
    e = Engine(k, 0, nphi, 256)
    a = random_poly_residues(1, e.Q, nphi)
    b = random_poly_residues(2, e.Q, nphi)
    ta, tb = from_u64(fold(a)[None]), from_u64(fold(b)[None])
    e.dgt(ta, 0, FORWARD)
    e.dgt(tb, 0, FORWARD)
    tc = e.empty(0)
    e.mul(tc, ta, tb, 0)
    e.dgt(tc, 0, INVERSE)
    c = unfold(to_u64(tc))[0]
    assert np.array_equal(c, CO.polymul(a[None], b[None], e.Q)[0])
    if nphi == 2048:
        assert c[0].tolist() == O.negacyclic_mul_schoolbook(a[0].tolist(), b[0].tolist(), e.Q[0])


@pytest.mark.parametrize("logq2,nphi", GRID)
def test_reference_arithmetic(gpu, logq2, nphi):
    """cuPoly TestArithmetic.{Add, Sub, Mul, MulAdd, MulByInt, SetCoeff} and TestRNS.RNS."""
    cp, ctx = _ref_engine(logq2, nphi)
    q = cp.CUDAEngine.RNSProduct
    a, b, c, d, s = cp.poly_t(), cp.poly_t(), cp.poly_t(), cp.poly_t(), cp.poly_t()
    for x in (a, b, c):
        cp.poly_init(ctx, x)
        cp.Sampler.sample(ctx, x, cp.UNIFORM)
    A = [cp.poly_get_coeff(ctx, a, i) for i in range(nphi)]
    Bc = [cp.poly_get_coeff(ctx, b, i) for i in range(nphi)]
    Cc = [cp.poly_get_coeff(ctx, c, i) for i in range(nphi)]
    assert all(0 <= v < q for v in A)
    cp.poly_add(ctx, d, a, b)
    assert [cp.poly_get_coeff(ctx, d, i) for i in range(nphi)] == [(x + y) % q for x, y in zip(A, Bc)]
    cp.poly_sub(ctx, d, a, b)
    assert [cp.poly_get_coeff(ctx, d, i) for i in range(nphi)] == [(x - y) % q for x, y in zip(A, Bc)]
    m = cp.poly_t()
    cp.poly_mul(ctx, m, a, b)
    got = [cp.poly_get_coeff(ctx, m, i) for i in range(nphi)]
    ref = np.array([[v % p for v in A] for p in cp.CUDAEngine.RNSPrimes], dtype=np.uint64)
    refb = np.array([[v % p for v in Bc] for p in cp.CUDAEngine.RNSPrimes], dtype=np.uint64)
    prod_rows = CO.polymul(ref[None], refb[None], cp.CUDAEngine.RNSPrimes)[0]
    exp = [O.crt(prod_rows[:, i].tolist(), cp.CUDAEngine.RNSPrimes) for i in range(nphi)]
    assert got == exp
    ma = cp.poly_t()
    cp.poly_mul_add(ctx, ma, a, b, c)
    assert [cp.poly_get_coeff(ctx, ma, i) for i in range(nphi)] == [(x + y) % q for x, y in zip(exp, Cc)]
    mi = cp.poly_t()
    cp.poly_mul_int(ctx, mi, a, 77)
    assert [cp.poly_get_coeff(ctx, mi, i) for i in range(nphi)] == [x * 77 % q for x in A]
    cp.poly_init(ctx, s)
    cp.poly_set_coeff(ctx, s, 0, 42)
    assert cp.poly_get_coeff(ctx, s, 0) == 42
    ones = cp.poly_t()
    cp.poly_init(ctx, ones)
    for i in range(nphi):
        cp.poly_set_coeff(ctx, ones, i, 1)
    cp.poly_copy_to_device(ctx, ones)
    ones.status = cp.RNSSTATE
    cp.poly_copy_to_host(ctx, ones)
    assert [cp.poly_get_coeff(ctx, ones, i) for i in range(nphi)] == [1] * nphi
    assert cp.poly_get_coeff(ctx, ones, 2 * nphi - 1) == 0
    cp.CUDAEngine.destroy()


@pytest.mark.parametrize("logq2,nphi", [(120, 32), (170, 4096)])
def test_reference_mul_base_b(gpu, logq2, nphi):
    """cuPoly TestArithmetic.MulBaseB: extend both operands to B, multiply in B."""
    cp, ctx = _ref_engine(logq2, nphi)
    e = cp.CUDAEngine.engine
    aq, bq, ab, bb, cb = (cp.poly_t() for _ in range(5))
    for x in (aq, bq):
        cp.poly_init(ctx, x)
        cp.Sampler.sample(ctx, x, cp.UNIFORM_MOD_Q)
    A = [cp.poly_get_coeff(ctx, aq, i) for i in range(nphi)]
    Bc = [cp.poly_get_coeff(ctx, bq, i) for i in range(nphi)]
    cp.poly_basis_extension_Q_to_B(ctx, ab, aq)
    cp.poly_basis_extension_Q_to_B(ctx, bb, bq)
    cp.poly_mul(ctx, cb, ab, bb)
    from cupoly_b200.engine import INVERSE, to_u64
    for poly, vals in ((ab, A), (bb, Bc)):
        t = poly.d_coefs.clone()
        e.dgt(t, 1, INVERSE, stream=ctx.stream)
        got = unfold(to_u64(t))[0]
        assert np.array_equal(got, np.array([[v % p for v in vals] for p in e.B], dtype=np.uint64))
    t = cb.d_coefs.clone()
    e.dgt(t, 1, INVERSE, stream=ctx.stream)
    rows_a = np.array([[v % p for v in A] for p in e.B], dtype=np.uint64)
    rows_b = np.array([[v % p for v in Bc] for p in e.B], dtype=np.uint64)
    assert np.array_equal(unfold(to_u64(t))[0], CO.polymul(rows_a[None], rows_b[None], e.B)[0])
    cp.CUDAEngine.destroy()


def test_engines_coexist(gpu):
    """Several parameter sets at once (cuPoly holds one per process)."""
    from cupoly_b200.engine import FORWARD, Engine, from_u64, to_u64
    engines = [Engine(k, 0, nphi, 256) for k, nphi in [(1, 2048), (4, 8192), (2, 32768)]]
    for e in engines:
        x = fold(random_poly_residues(e.nphi, e.Q, e.nphi))[None]
        t = from_u64(x)
        e.dgt(t, 0, FORWARD)
        assert np.array_equal(to_u64(t), CO.dgt(x, e.Q))


@pytest.mark.parametrize("k,nphi,npolys", [(2, 4096, 3), (5, 8192, 2), (3, 16384, 1), (1, 32, 4), (4, 65536, 1)])
def test_fused_polymul_vs_oracle(gpu, k, nphi, npolys):
    """cp_polymul (out-of-place forward DGTs, inverse forming the products on load)
    against the oracle's negacyclic product per prime; c may alias an input."""
    from cupoly_b200.engine import Engine, QBase, from_u64, to_u64
    from oracle import coracle
    e = Engine(k, 0, nphi, 256)
    a = np.stack([random_poly_residues(7 * i + k, e.Q, nphi) for i in range(npolys)])
    b = np.stack([random_poly_residues(7 * i + k + 100, e.Q, nphi) for i in range(npolys)])
    ref = coracle.polymul(a, b, e.Q)
    da, db = from_u64(fold(a)), from_u64(fold(b))
    c = e.empty(QBase, npolys)
    ws = e.polymul_workspace(QBase, npolys)
    e.polymul(c, da, db, QBase, ws)
    assert np.array_equal(unfold(to_u64(c)), ref)
    e.polymul(da, da, db, QBase, ws)                    # in place over a
    assert np.array_equal(unfold(to_u64(da)), ref)


def _dot_exact(xs, ys, primes):
    """sum_t xs[t] ys[t] per residue, exact (numpy object ints)."""
    acc = None
    for x, y in zip(xs, ys):
        term = np.stack([_gi_mul(x[r], y[r], p) for r, p in enumerate(primes)]).astype(object)
        acc = term if acc is None else acc + term
    return np.stack([acc[r] % p for r, p in enumerate(primes)]).astype(np.uint64)


@pytest.mark.parametrize("n", [1, 2, 5, 64, 65, 130])
def test_dot_vs_exact(gpu, n):
    """cp_dot (cuPoly poly_dot, polynomial.cu:1439-1451) == exact sum of Gaussian products,
    across the 64-term launch boundary; every base of a BFV engine and a CKKS engine."""
    from cupoly_b200.engine import Engine, from_u64, to_u64
    for e, bases in ((Engine(3, 4, 2048, 256), (0, 1, 2)), (Engine.ckks(3, 0, 2048, 52), (0,))):
        for base in bases if n <= 5 else bases[:1]:
            primes = e.base_primes(base)
            xs = [fold(random_poly_residues(1000 + 7 * t + base, primes, 2048)) for t in range(n)]
            ys = [fold(random_poly_residues(5000 + 7 * t + base, primes, 2048)) for t in range(n)]
            out = e.empty(base)
            e.dot(out, [from_u64(x[None]) for x in xs], [from_u64(y[None]) for y in ys], base)
            assert np.array_equal(to_u64(out)[0], _dot_exact(xs, ys, primes))


def test_dot_extreme_operands_and_aliasing(gpu):
    """Every operand at p - 1 + (p - 1) i, so each Karatsuba product (a0 + a1)(b0 + b1) is at
    its maximum (2p - 2)^2, over 64 terms (the widest lazy sum of a launch); an output that
    aliases an operand of the launch; an output that aliases an operand of a later launch is
    refused."""
    from cupoly_b200._lib import CupolyError
    from cupoly_b200.engine import Engine, from_u64, to_u64
    e = Engine(2, 3, 64, 256)
    primes = e.base_primes(0)
    P = np.array(primes, dtype=np.uint64)[:, None]
    x = np.stack([np.full((32, 2), p - 1, dtype=np.uint64) for p in primes])  # (p-1) + (p-1) i
    xs, ys = [x] * 64, [x] * 64
    out = e.empty(0)
    e.dot(out, [from_u64(v[None]) for v in xs], [from_u64(v[None]) for v in ys], 0)
    assert np.array_equal(to_u64(out)[0], _dot_exact(xs, ys, primes))
    assert (to_u64(out)[0] < P[..., None]).all()

    xs = [fold(random_poly_residues(70 + t, primes, 64)) for t in range(70)]
    ys = [fold(random_poly_residues(170 + t, primes, 64)) for t in range(70)]
    exp = _dot_exact(xs[:5], ys[:5], primes)
    da = [from_u64(v[None]) for v in xs]
    db = [from_u64(v[None]) for v in ys]
    e.dot(da[3], da[:5], db[:5], 0)  # c is a[3]: read before written, element by element
    assert np.array_equal(to_u64(da[3])[0], exp)
    da[3] = from_u64(xs[3][None])
    with pytest.raises(CupolyError):
        e.dot(da[66], da, db, 0)
    exp = _dot_exact(xs, ys, primes)
    e.dot(da[2], da, db, 0)  # aliasing the first launch's operands is fine
    assert np.array_equal(to_u64(da[2])[0], exp)


def test_poly_dot_mirror_matches_composition(gpu):
    """poly_dot through the cuPoly mirror equals cuPoly's poly_mul + poly_mul_add composition,
    including an output that is also a later operand (the composition reads the partial sum)."""
    import torch
    from cupoly_b200.engine import to_u64
    cp, ctx = _ref_engine(120, 2048)
    k = 4
    A = [cp.poly_t() for _ in range(k)]
    B = [cp.poly_t() for _ in range(k)]
    for x in A + B:
        cp.poly_init(ctx, x)
        cp.Sampler.sample(ctx, x, cp.UNIFORM_MOD_Q)

    def composed(a, b, c=None):
        c = cp.poly_t() if c is None else c
        cp.poly_mul(ctx, c, a[0], b[0])
        for i in range(1, k):
            cp.poly_mul_add(ctx, c, a[i], b[i], c)
        return c

    def coeffs(x):
        torch.cuda.synchronize()
        return to_u64(x.d_coefs)

    ref = coeffs(composed(A, B))
    got = cp.poly_t()
    cp.poly_dot(ctx, got, A, B, k)
    assert np.array_equal(coeffs(got), ref)
    # c is A[2]: both forms must give cuPoly's bytes
    A2 = [cp.poly_t() for _ in range(k)]
    for i in range(k):
        cp.poly_copy(ctx, A2[i], A[i])
    cp.poly_dot(ctx, A2[2], A2, B, k)
    A3 = [cp.poly_t() for _ in range(k)]
    for i in range(k):
        cp.poly_copy(ctx, A3[i], A[i])
    composed(A3, B, A3[2])
    assert np.array_equal(coeffs(A2[2]), coeffs(A3[2]))
    cp.CUDAEngine.destroy()


def test_dot_batch_vs_dot_and_exact(gpu):
    """cp_dot_batch: per-polynomial operands and shared keys (the relinearization layout: the
    xi_batch decomposition of P polynomials against one set of k key polynomials) equal cp_dot
    per polynomial and the exact sums."""
    import torch

    from cupoly_b200.engine import QBase, UNIFORM, Engine, from_u64, to_u64
    e = Engine(3, 0, 2048, 256)
    k, P = e.k, 5
    x = e.empty(QBase, P)
    e.sample(x, QBase, UNIFORM, 3, 0, npolys=P, to_dgt=True)
    dec = e.empty(QBase, P * k)
    e.xi_batch(dec, x)
    keys = e.empty(QBase, k)
    e.sample(keys, QBase, UNIFORM, 3, 100, npolys=k, to_dgt=False)
    out = e.empty(QBase, P)
    e.dot_batch(out, dec, keys, k, P, QBase, b_shared=True)
    for q in range(P):
        ref = e.empty(QBase)
        e.dot(ref, [dec[q * k + t] for t in range(k)], [keys[t] for t in range(k)], QBase)
        assert torch.equal(out[q], ref[0]), q
    # per-polynomial second operands, against the exact sums; n = 7 terms
    n = 7
    A = [fold(random_poly_residues(900 + i, e.Q, 2048)) for i in range(P * n)]
    B = [fold(random_poly_residues(1900 + i, e.Q, 2048)) for i in range(P * n)]
    da, db = from_u64(np.stack(A)), from_u64(np.stack(B))
    out = e.empty(QBase, P)
    e.dot_batch(out, da, db, n, P, QBase)
    got = to_u64(out)
    for q in range(P):
        assert np.array_equal(got[q], _dot_exact(A[q * n:(q + 1) * n], B[q * n:(q + 1) * n], e.Q)), q
