"""DGT parity on the GPU: bit-exact against the oracle (cuPoly's DGT domain)."""
import json
import os

import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import fold, gi_rows_to_list, random_poly_residues, sha

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _engine(k, nphi, log_radix=0, kl=0):
    from cupoly_b200.engine import Engine
    return Engine(k, kl, nphi, 256, log_radix)


def _fwd(e, x_np, base=0):
    from cupoly_b200.engine import FORWARD, from_u64, to_u64
    x = from_u64(x_np)
    e.dgt(x, base, FORWARD)
    return to_u64(x)


@pytest.mark.parametrize("nphi", [4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536])
@pytest.mark.parametrize("log_radix", [3, 4])
def test_forward_inverse_vs_oracle(gpu, nphi, log_radix):
    from cupoly_b200.engine import INVERSE, from_u64, to_u64
    e = _engine(2, nphi, log_radix)
    x = fold(random_poly_residues(nphi + log_radix, e.Q, nphi))[None]
    y = _fwd(e, x)
    ref = CO.dgt(x, e.Q)
    assert np.array_equal(y, ref)
    t = from_u64(y)
    e.dgt(t, 0, INVERSE)
    assert np.array_equal(to_u64(t), x)


@pytest.mark.parametrize("nphi", [32, 2048])
def test_forward_vs_python_restatement(gpu, nphi):
    e = _engine(1, nphi)
    x = fold(random_poly_residues(3, e.Q, nphi))[None]
    y = _fwd(e, x)
    p = e.Q[0]
    assert [tuple(v) for v in y[0, 0].tolist()] == O.dgt_forward_ref(gi_rows_to_list(x[0, 0]), p)


def test_reference_roots_golden(gpu):
    """With cuPoly's NTHROOT table loaded, the DGT-domain bytes equal the fixtures."""
    roots = json.load(open(os.path.join(GOLD, "ref_nthroot.json")))
    for case in json.load(open(os.path.join(GOLD, "dgt_golden.json"))):
        nphi, nres = case["nphi"], case["nres"]
        e = _engine(nres, nphi, kl=1)
        N = nphi // 2
        xi = [roots[str(p)][str(N)] for p in e.primes[:nres]] + [list(O.canonical_xi(e.primes[-1], N))]
        e.set_nthroot(xi)
        assert e.get_nthroot()[0] == tuple(xi[0])
        x = fold(random_poly_residues(case["seed"], e.Q, nphi))[None]
        assert sha(_fwd(e, x)[0]) == case["sha256"], case


@pytest.mark.parametrize("base", [0, 1, 2])
def test_bases_and_batches(gpu, base):
    """Bases Q, B, QB select the residue offsets; npolys > 1 packs polynomials back to back."""
    e = _engine(3, 4096)
    primes = e.base_primes(base)
    x = np.stack([fold(random_poly_residues(50 + i, primes, 4096)) for i in range(5)])
    y = _fwd(e, x, base)
    assert np.array_equal(y, CO.dgt(x, primes))


def test_set_nthroot_rejects_wrong_root(gpu):
    from cupoly_b200 import CupolyError
    e = _engine(1, 64)
    with pytest.raises(CupolyError):
        e.set_nthroot([(1, 0), (1, 0)])


def test_tbase_is_identity(gpu):
    from cupoly_b200.engine import FORWARD, from_u64, to_u64
    e = _engine(1, 64)
    x = np.arange(64, dtype=np.uint64).reshape(1, 1, 32, 2)
    t = from_u64(x)
    e.dgt(t, 3, FORWARD)
    assert np.array_equal(to_u64(t), x)
