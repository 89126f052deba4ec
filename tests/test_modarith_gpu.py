"""The device modular primitives (modarith.cuh) through cp_modarith_eval, against
Python integers: cuPoly's TestDGT.{mod, addmod, submod, mulmod, powmod, GIAdd, GISub,
GIMul} (tests/unit_tests/test_bfv_mode.cu:243-438) as edge grids plus random draws,
over the 63-bit BFV primes (pseudo-Mersenne path) and CKKS bucket primes (generic
Montgomery path)."""
import ctypes as C
import random

import numpy as np
import pytest

from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

ADD, SUB, NEG, MULMOD, SHOUP, RED128, POW, GIMUL, GIMUL3 = range(9)
PRIMES = [O.PRIMES[0], O.PRIMES[57], O.PRIMES[-1], O.ckks_bucket(45)[0], O.ckks_bucket(52)[3],
          O.ckks_bucket(55)[-1]]


def _run(op, p, a, b=None, c=None):
    import torch

    from cupoly_b200 import _lib

    def dev(x):
        return torch.from_numpy(np.array(x, dtype=np.uint64).view(np.int64)).cuda() if x is not None else None

    da, db, dc = dev(a), dev(b), dev(c)
    n = len(a) // 2 if op in (GIMUL, GIMUL3) else len(a)
    out = torch.zeros(len(a), dtype=torch.int64, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    _lib.call("cp_modarith_eval", op, ptr(da), ptr(db), ptr(dc), ptr(out), n, p, None)
    torch.cuda.synchronize()
    return [int(v) for v in out.cpu().numpy().view(np.uint64)]


def _edges(p):
    return [0, 1, 2, 3, p // 2, p // 2 + 1, p - 3, p - 2, p - 1]


@pytest.mark.parametrize("p", PRIMES)
def test_add_sub_neg_mulmod_pow(gpu, p):
    rng = random.Random(p)
    E = _edges(p)
    a = [x for x in E for _ in E] + [rng.randrange(p) for _ in range(4000)]
    b = [y for _ in E for y in E] + [rng.randrange(p) for _ in range(4000)]
    assert _run(ADD, p, a, b) == [(x + y) % p for x, y in zip(a, b)]
    assert _run(SUB, p, a, b) == [(x - y) % p for x, y in zip(a, b)]
    assert _run(NEG, p, a) == [(-x) % p for x in a]
    b64 = b[: len(E) ** 2] + [2 ** 64 - 1, 2 ** 63, p, p + 1] + [rng.getrandbits(64) for _ in range(4000 - 4)]
    assert _run(MULMOD, p, a, b64) == [x * y % p for x, y in zip(a, b64)]
    e = [0, 1, 2, p - 2, p - 1] * (len(a) // 5) + [rng.getrandbits(64) for _ in range(len(a) % 5)]
    assert _run(POW, p, a, e) == [pow(x, y, p) for x, y in zip(a, e)]


@pytest.mark.parametrize("p", PRIMES)
def test_shoup_and_red128(gpu, p):
    rng = random.Random(p + 1)
    a = [0, 1, p - 1, p, 2 * p - 1, 2 ** 63, 2 ** 64 - 1] + [rng.getrandbits(64) for _ in range(4000)]
    w = [rng.choice([0, 1, p - 1]) if i < 7 else rng.randrange(p) for i in range(len(a))]
    ws = [(x << 64) // p for x in w]
    assert _run(SHOUP, p, a, w, ws) == [x * y % p for x, y in zip(a, w)]
    # hi:lo below min(2^127, p 2^64), the largest values included
    bound = min(1 << 127, p << 64)
    vals = [0, 1, bound - 1, bound - p, p * p, (p - 1) * (p - 1)] + [rng.randrange(bound) for _ in range(4000)]
    hi, lo = [v >> 64 for v in vals], [v & (2 ** 64 - 1) for v in vals]
    assert _run(RED128, p, hi, lo) == [v % p for v in vals]


@pytest.mark.parametrize("p", PRIMES)
def test_gaussian_products(gpu, p):
    """GIMul (data x data) and the Karatsuba constant form used by the DGT twist."""
    rng = random.Random(p + 2)
    E = [0, 1, p - 1, p // 2]
    xs = [(x, y) for x in E for y in E] + [(rng.randrange(p), rng.randrange(p)) for _ in range(2000)]
    ys = [(y, x) for x in E for y in E] + [(rng.randrange(p), rng.randrange(p)) for _ in range(2000)]
    a = [v for pr in xs for v in pr]
    b = [v for pr in ys for v in pr]
    want = []
    for (ar, ai), (br, bi) in zip(xs, ys):
        want += [(ar * br - ai * bi) % p, (ar * bi + ai * br) % p]
    assert _run(GIMUL, p, a, b) == want
    c = []
    for br, bi in ys:
        for k in (br, (bi - br) % p, (br + bi) % p):
            c.append((k << 64) // p)
    assert _run(GIMUL3, p, a, b, c) == want
