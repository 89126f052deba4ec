"""CKKS mode on the GPU (cuPoly's CKKS build, tests/unit_tests/test_ckks_mode.cu):
prime selection, the arithmetic tests re-run over CKKS primes (TestArithmetic /
TestRNS, :617-994 with the parameter grid :1236-1250), the DGT and device CRT on
non-63-bit primes, and the CKKS operations (rescale, approximate modulus raising
and reduction, xi / rho) bit-exact against their integer definitions."""
import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import fold, random_poly_residues, unfold

pytestmark = pytest.mark.gpu

# (k, kl, nphi, prec): cuPoly's CKKS grid plus the 52-bit bucket
PARAMS = [(2, 5, 128, 45), (2, 5, 2048, 45), (3, 5, 4096, 45), (5, 5, 8192, 45), (2, 5, 32, 48), (2, 5, 128, 48),
          (2, 5, 2048, 48), (3, 5, 4096, 48), (5, 5, 8192, 48), (2, 5, 128, 55), (2, 5, 2048, 55), (3, 5, 4096, 55),
          (5, 5, 8192, 55), (4, 3, 1024, 52)]


def _eng(k, kl, nphi, prec):
    from cupoly_b200.engine import Engine
    return Engine.ckks(k, kl, nphi, prec)


def _dev(x):
    from cupoly_b200.engine import from_u64
    return from_u64(x)


def _host(t):
    from cupoly_b200.engine import to_u64
    return to_u64(t)


@pytest.mark.parametrize("k,kl,nphi,prec", PARAMS)
def test_ckks_primes_and_arithmetic(gpu, k, kl, nphi, prec):
    from cupoly_b200.engine import FORWARD, INVERSE, QBBase, QBase
    e = _eng(k, kl, nphi, prec)
    Q, B = O.ckks_bases(k, kl, prec)
    assert e.Q == Q and e.B == B
    a = random_poly_residues(k + nphi, e.primes, nphi)
    b = random_poly_residues(kl + nphi, e.primes, nphi, stream=1)
    da, db = _dev(fold(a)[None]), _dev(fold(b)[None])
    e.dgt(da, QBBase, FORWARD)
    e.dgt(db, QBBase, FORWARD)
    c = e.empty(QBBase)
    e.mul(c, da, db, QBBase)          # TestArithmetic.Mul / MulBaseB
    s = e.empty(QBBase)
    e.add(s, da, db, QBBase)          # TestArithmetic.Add
    e.dgt(c, QBBase, INVERSE)
    e.dgt(s, QBBase, INVERSE)
    assert np.array_equal(unfold(_host(c))[0], CO.polymul(a[None], b[None], e.primes)[0])
    ref_add = np.array([(a[r].astype(object) + b[r].astype(object)) % p for r, p in enumerate(e.primes)],
                       dtype=np.uint64)
    assert np.array_equal(unfold(_host(s))[0], ref_add)
    e.dgt(da, QBBase, INVERSE)        # round trip
    assert np.array_equal(unfold(_host(da))[0], a)


def test_ckks_dgt_domain_matches_restatement(gpu):
    from cupoly_b200.engine import FORWARD, QBase
    e = _eng(3, 2, 256, 48)
    x = random_poly_residues(5, e.Q, 256)
    d = _dev(fold(x)[None])
    e.dgt(d, QBase, FORWARD)
    got = _host(d)[0]
    for r, p in enumerate(e.Q):
        X = O.dgt_forward_direct(O.fold(x[r].tolist(), p, 128), p)
        assert [tuple(v) for v in got[r].tolist()] == [tuple(v) for v in X], r


def test_ckks_crt_icrt_generic_primes(gpu):
    import torch

    from cupoly_b200.engine import ints_to_limbs, limbs_to_ints
    e = _eng(4, 3, 512, 45)
    P = O.prod(e.Q)
    from tests.common import random_poly_int
    xs = random_poly_int(9, P, 512)
    xs[0], xs[1] = 0, P - 1
    out = e.empty(0)
    e.crt(out, _dev(ints_to_limbs(xs, 4)[None]), 0)
    got = unfold(_host(out))[0]
    for r, p in enumerate(e.Q):
        assert np.array_equal(got[r], np.array([x % p for x in xs], dtype=np.uint64))
    limbs = torch.empty((1, 512, 4), dtype=torch.int64, device="cuda")
    e.icrt(limbs, out, 0)
    assert limbs_to_ints(_host(limbs[0])) == xs


@pytest.mark.parametrize("k,kl,nphi,prec,level", [(5, 5, 8192, 55, 4), (3, 5, 4096, 48, 1), (4, 3, 1024, 52, 3),
                                                   (2, 5, 128, 45, 1), (6, 4, 2048, 45, 2)])
def test_ckks_rescale(gpu, k, kl, nphi, prec, level):
    from cupoly_b200.engine import FORWARD, INVERSE, QBase
    e = _eng(k, kl, nphi, prec)
    a = random_poly_residues(3 * k, e.Q, nphi)
    b = random_poly_residues(4 * k, e.Q, nphi)
    da, db = _dev(fold(a)[None]), _dev(fold(b)[None])
    e.dgt(da, QBase, FORWARD)
    e.dgt(db, QBase, FORWARD)
    e.ckks_rescale(da, db, level)
    e.dgt(da, QBase, INVERSE)
    e.dgt(db, QBase, INVERSE)
    for x, d in ((a, da), (b, db)):
        got = unfold(_host(d))[0]
        for j in range(0, nphi, max(1, nphi // 64)):
            xs = [int(x[r, j]) for r in range(k)]
            ref = O.ckks_rescale(xs, e.Q, level)
            assert [int(got[r, j]) for r in range(k)] == ref, j
            # exact division: the first `level` residues are floor(A / q_l) for A = CRT over Q_l
            A = O.crt(xs[:level + 1], e.Q[:level + 1])
            assert [A // e.Q[level] % q for q in e.Q[:level]] == ref[:level]


@pytest.mark.parametrize("k,kl,nphi,prec,level", [(5, 5, 8192, 55, 4), (3, 5, 4096, 48, 2), (4, 3, 1024, 52, 1),
                                                   (2, 5, 128, 45, 0), (6, 4, 2048, 45, 3)])
def test_ckks_modulus_raising_and_reduction(gpu, k, kl, nphi, prec, level):
    from cupoly_b200.engine import FORWARD, INVERSE, QBBase, QBase
    e = _eng(k, kl, nphi, prec)
    x = random_poly_residues(11 * k, e.Q, nphi)
    dx = _dev(fold(x)[None])
    e.dgt(dx, QBase, FORWARD)
    out = e.empty(QBBase)
    e.ckks_modulus_raising(out, dx, level)
    e.dgt(out, QBBase, INVERSE)
    got = unfold(_host(out))[0]
    assert np.array_equal(got[:k], x)                         # Q part is the input
    Ql = O.prod(e.Q[:level + 1])
    cols = range(0, nphi, max(1, nphi // 64))
    for j in cols:
        xs = [int(x[r, j]) for r in range(k)]
        ref = O.ckks_modulus_raising(xs, e.Q, e.B, level)
        assert [int(got[k + jb, j]) for jb in range(kl)] == ref, j
        # fast conversion: y_j = X + u Q_l mod b_j with 0 <= u <= level
        X = O.crt(xs[:level + 1], e.Q[:level + 1])
        us = [u for u in range(level + 1) if all((X + u * Ql) % b == y for b, y in zip(e.B, ref))]
        assert len(us) == 1
    # reduction of a QB polynomial
    y = random_poly_residues(13 * k, e.primes, nphi)
    dy = _dev(fold(y)[None])
    e.dgt(dy, QBBase, FORWARD)
    z = e.zeros(QBase)
    e.ckks_modulus_reduction(z, dy, level)
    e.dgt(z, QBase, INVERSE)
    gz = unfold(_host(z))[0]
    for j in cols:
        xs = [int(y[r, j]) for r in range(k)]
        ys = [int(y[k + jb, j]) for jb in range(kl)]
        ref = O.ckks_modulus_reduction(xs, ys, e.Q, e.B, level)
        assert [int(gz[r, j]) for r in range(level + 1)] == ref, j
    assert not gz[level + 1:].any()                           # rows above the level not written


def test_ckks_xi_rho_and_bfv_calls_refused(gpu):
    import ctypes as C

    from cupoly_b200 import _lib
    from cupoly_b200.engine import QBase, _ptr
    e = _eng(3, 4, 512, 55)
    x = random_poly_residues(2, e.Q, 512)
    dx = _dev(fold(x)[None])
    o1, o2 = e.empty(QBase), e.empty(QBase)
    e.ckks_xi(o1, dx)
    e.ckks_rho(o2, dx)
    Bp = O.prod(e.B)
    g1, g2 = unfold(_host(o1))[0], unfold(_host(o2))[0]
    for r, q in enumerate(e.Q):
        binv, bq = pow(Bp % q, -1, q), Bp % q
        assert np.array_equal(g1[r], np.array([int(v) * binv % q for v in x[r]], dtype=np.uint64))
        assert np.array_equal(g2[r], np.array([int(v) * bq % q for v in x[r]], dtype=np.uint64))
    L = _lib.lib()
    ws = e.workspace()
    assert L.cp_bfv_mul(e.handle, *[_ptr(o1)] * 7, _ptr(ws), None) == 3
    assert b"CKKS" in L.cp_last_error()
    assert L.cp_basis_ext_q_to_b(e.handle, _ptr(o1), _ptr(o2), 1, None) == 3
    assert L.cp_engine_ckks_prec(e.handle) == 55
    assert L.cp_ckks_rescale(e.handle, _ptr(o1), None, 0, None) == 1      # level 0
    from cupoly_b200.engine import Engine
    bfv = Engine(2, 0, 64, 256)
    assert L.cp_ckks_xi(bfv.handle, _ptr(o1), _ptr(o2), None) == 3
    assert L.cp_engine_ckks_prec(bfv.handle) == 0
    h = C.c_void_p()
    assert L.cp_ckks_engine_create(C.byref(h), 2, 2, 256, 47, 0) == 1     # unknown bucket


def test_ckks_host_mirror(gpu):
    from cupoly_b200 import cupoly as cp
    cp.CUDAEngine.init_ckks(3, 5, 2048, 48)
    ctx = cp.Context()
    Q = cp.CUDAEngine.RNSProduct
    from tests.common import random_poly_int
    vals = random_poly_int(21, Q, 2048)
    a, b, c = cp.poly_t(), cp.poly_t(), cp.poly_t()
    for i, v in enumerate(vals[:64]):
        cp.poly_set_coeff(ctx, a, i, v)
        cp.poly_set_coeff(ctx, b, i, vals[100 + i])
    cp.poly_mul(ctx, c, a, b)
    ref = O.negacyclic_mul_schoolbook(vals[:64] + [0] * (2048 - 64), vals[100:164] + [0] * (2048 - 64), Q)
    assert [cp.poly_get_coeff(ctx, c, i) for i in range(2048)] == ref
    cp.poly_ckks_rescale(ctx, c, None, 2)
    got = [cp.poly_get_coeff(ctx, c, i) for i in range(2048)]
    # residues 0, 1 of the rescaled polynomial are floor(c / q_2) mod q_0, q_1
    for j in range(0, 2048, 97):
        assert got[j] % Q_mod(cp, 0) == (ref[j] // cp.CUDAEngine.RNSPrimes[2]) % Q_mod(cp, 0)
    cp.CUDAEngine.destroy()


def Q_mod(cp, i):
    return cp.CUDAEngine.RNSPrimes[i]


def test_ckks_sampler_is_signed_like_cupolys_ckks_build(gpu):
    """On a CKKS engine NARROW is uniform {-1, 0, 1} and DISCRETE_GAUSSIAN is signed
    (cuPoly's CKKS build, src/cuda/sampler.cu:73-106, 459-493); bit-exact against the
    oracle's restatement, symmetric in distribution."""
    from cupoly_b200.engine import DISCRETE_GAUSSIAN, NARROW, QBase
    e = _eng(3, 4, 4096, 48)
    for kind in (NARROW, DISCRETE_GAUSSIAN):
        x = e.empty(QBase)
        e.sample(x, QBase, kind, 77, 5, to_dgt=False)
        got = unfold(_host(x))[0]
        ref = np.array(O.sample_poly(kind, e.Q, 4096, 5, 77, ckks=True), dtype=np.uint64)
        assert np.array_equal(got, ref)
        q0 = e.Q[0]
        v = np.where(got[0] > q0 // 2, got[0].astype(object) - q0, got[0].astype(object)).astype(np.int64)
        assert (v < 0).any() and (v > 0).any() and abs(v.mean()) < 0.2
        if kind == NARROW:
            assert set(np.unique(v)) <= {-1, 0, 1}
        else:
            assert np.abs(v).max() <= 19


@pytest.mark.parametrize("prec", [45, 52, 55])
def test_ckks_uniform_sampler_over_narrow_primes(gpu, prec):
    """UNIFORM on a CKKS engine: candidates of bitlen(q_i) bits, so the 45..55-bit primes
    accept as readily as the 63-bit ones (no rejection-limit error); bit-exact against the
    oracle, every residue below its prime, mean near q_i / 2."""
    from cupoly_b200.engine import QBase, UNIFORM
    e = _eng(3, 4, 2048, prec)
    x = e.empty(QBase, 4)
    e.sample(x, QBase, UNIFORM, 91, 11, npolys=4, to_dgt=False)
    e.check()  # raises if any coefficient hit the rejection limit
    got = unfold(_host(x[3:4]))[0]
    ref = np.array(O.sample_poly(UNIFORM, e.Q, 2048, 14, 91, ckks=True), dtype=np.uint64)
    assert np.array_equal(got, ref)
    for r, q in enumerate(e.Q):
        assert int(got[r].max()) < q
        assert abs(float(np.mean(got[r].astype(np.float64))) / q - 0.5) < 0.03


@pytest.mark.parametrize("k,kl,nphi,prec,level", [(3, 4, 4096, 52, 2), (8, 9, 16384, 45, 5), (4, 5, 32768, 55, 3)])
def test_ckks_batched_calls_equal_per_polynomial_calls(gpu, k, kl, nphi, prec, level):
    """Batched modulus raising, reduction and rescale give, polynomial by polynomial, the
    bytes of the one-polynomial calls (DGT domain in and out)."""
    import torch

    from cupoly_b200.engine import QBBase, QBase, UNIFORM
    e = _eng(k, kl, nphi, prec)
    P = 5
    a = e.empty(QBase, P)
    e.sample(a, QBase, UNIFORM, 21, 0, npolys=P, to_dgt=True)
    qb = e.empty(QBBase, P)
    e.sample(qb, QBBase, UNIFORM, 22, 0, npolys=P, to_dgt=True)
    ws = e.ckks_batch_workspace(P)
    raised = e.empty(QBBase, P)
    e.ckks_modulus_raising_batch(raised, a, level, ws)
    reduced = e.zeros(QBase, P)
    e.ckks_modulus_reduction_batch(reduced, qb, level, ws)
    resc = a.clone()
    e.ckks_rescale_batch(resc, level)
    for i in range(P):
        r1 = e.empty(QBBase)
        e.ckks_modulus_raising(r1, a[i:i + 1], level)
        assert torch.equal(r1, raised[i:i + 1]), ("raising", i)
        d1 = e.zeros(QBase)
        e.ckks_modulus_reduction(d1, qb[i:i + 1], level)
        assert torch.equal(d1[:, : level + 1], reduced[i:i + 1, : level + 1]), ("reduction", i)
        s1 = a[i:i + 1].clone()
        e.ckks_rescale(s1, None, level)
        assert torch.equal(s1, resc[i:i + 1]), ("rescale", i)
    e.check()
