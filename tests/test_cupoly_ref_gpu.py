"""The CUDA path against cuPoly's own outputs (tests/golden/cupoly_ref_golden.json).

The fixture holds what cuPoly 0.3.5's own library computed on a B200 through its
public API (tests/golden/gen_cupoly_golden.py), on the seeded inputs of
tests/common.py.  Here the same inputs go through this library's C ABI with
cuPoly's tabulated roots of i loaded (cp_engine_set_nthroot), and the outputs are
compared word for word:

* DGT-domain bytes of the forward transform (DGTEngine::execute_dgt);
* poly_mul, poly_basis_extension_Q_to_B, poly_simple_scaling_tDivQ,
  poly_complex_scaling_tDivQ, poly_xi_bfv / poly_rho_bfv and the BFV
  multiplication chain, in the coefficient domain.

Where cuPoly's double-precision HPS path rounds the wrong way (its complex
scaling at k = 6 uses 512-bit RR constants with about 63 fraction bits), the
device gives round(t X / Q) exactly; those cases must equal the exact oracle and
differ from cuPoly's words only by one in the scaled value, at the coefficients
the oracle's restatement of cuPoly's path predicts.  When the compiled reference
driver is present (oracle/_ref/cupoly_ref_driver), one more test runs it live on a
fresh seed and compares.
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import cupoly_chain_restated, fold, random_poly_residues, sha, unfold

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "cupoly_ref_driver")


def _doc():
    with open(os.path.join(GOLD, "cupoly_ref_golden.json")) as f:
        return json.load(f)


DOC = _doc() if os.path.exists(os.path.join(GOLD, "cupoly_ref_golden.json")) else {"cases": []}


def _cases(op):
    return [c for c in DOC["cases"] if c["op"] == op]


def _id(c):
    return "nphi%d_k%d_t%d" % (c["nphi"], c["k"], c["t"])


def _inputs(c):
    from tests.golden.gen_cupoly_golden import inputs
    return inputs(c["op"], c["k"], c["kl"], c["nphi"], c["seed"])


def _engine(k, kl, nphi, t):
    from cupoly_b200.engine import Engine
    e = Engine(k, kl, nphi, t)
    roots = json.load(open(os.path.join(GOLD, "ref_nthroot.json")))
    e.set_nthroot([tuple(roots[str(p)][str(nphi // 2)]) for p in e.primes])
    return e


def _to_dgt(e, rows, base):
    from cupoly_b200.engine import FORWARD, from_u64
    d = from_u64(fold(rows)[None])
    e.dgt(d, base, FORWARD)
    return d


def _coeffs(e, d, base):
    from cupoly_b200.engine import INVERSE, to_u64
    x = d.clone()
    e.dgt(x, base, INVERSE)
    return unfold(to_u64(x))


def _same(c, got):
    got = np.ascontiguousarray(got, dtype=np.uint64).reshape(-1)
    assert got.size == c["words"]
    return sha(got) == c["sha256"]


def _only_rounding_differences(got, exact, restated, Q):
    """got (device) == the exact values; cuPoly's words (restated) differ from them by
    exactly one in the scaled value wherever they differ."""
    assert np.array_equal(got, exact)
    Qp = O.prod(Q)
    for j in np.nonzero((restated != exact).any(axis=0))[0]:
        d = O.crt([int(v) for v in restated[:, j]], Q) - O.crt([int(v) for v in exact[:, j]], Q)
        assert d % Qp in (1, Qp - 1)


@pytest.mark.parametrize("c", _cases("dgt"), ids=_id)
def test_dgt_domain_bytes_equal_cupolys(gpu, c):
    from cupoly_b200.engine import to_u64
    k, kl, nphi = c["k"], c["kl"], c["nphi"]
    e = _engine(k, kl, nphi, c["t"])
    d = _to_dgt(e, _inputs(c).reshape(k + kl, nphi), 2)
    assert _same(c, to_u64(d)[0])


@pytest.mark.parametrize("c", _cases("mul"), ids=_id)
def test_poly_mul_equals_cupolys(gpu, c):
    k, nphi = c["k"], c["nphi"]
    e = _engine(k, c["kl"], nphi, c["t"])
    x = _inputs(c).reshape(2, k, nphi)
    a, b = _to_dgt(e, x[0], 0), _to_dgt(e, x[1], 0)
    out = e.empty(0)
    e.mul(out, a, b, 0)
    assert _same(c, _coeffs(e, out, 0)[0])


@pytest.mark.parametrize("c", _cases("ext"), ids=_id)
def test_basis_extension_equals_cupolys(gpu, c):
    k, kl, nphi = c["k"], c["kl"], c["nphi"]
    e = _engine(k, kl, nphi, c["t"])
    a = _to_dgt(e, _inputs(c).reshape(k, nphi), 0)
    out = e.empty(1)
    e.poly_basis_extension_q_to_b(out, a)
    assert _same(c, _coeffs(e, out, 1)[0])


@pytest.mark.parametrize("c", _cases("sscale"), ids=_id)
def test_simple_scaling_equals_cupolys(gpu, c):
    from cupoly_b200.engine import to_u64
    k, nphi, t = c["k"], c["nphi"], c["t"]
    e = _engine(k, c["kl"], nphi, c["t"])
    x = _inputs(c).reshape(k, nphi)
    a = _to_dgt(e, x, 0)
    out = e.empty(3)
    e.poly_simple_scaling_tdivq(out, a)
    got = unfold(to_u64(out))[0, 0]
    # cuPoly's words are its unreduced sums (its d_RNST is never set); reduced mod t
    # they are cuPoly's scaled values, which this library gives exactly.
    cx = [[int(v) for v in x[:, j]] for j in range(nphi)]
    raw = np.array([O.cupoly_float_simple_scaling(v, e.Q, t, raw=True) for v in cx], dtype=np.uint64)
    assert sha(raw) == c["sha256"]
    exact = np.array([O.simple_scaling_exact(v, e.Q, t) for v in cx], dtype=np.uint64)
    assert np.array_equal(got, exact)
    for j in np.nonzero(raw % np.uint64(t) != exact)[0]:
        assert (int(raw[j]) - int(exact[j])) % t in (1, t - 1)


@pytest.mark.parametrize("c", _cases("cscale"), ids=_id)
def test_complex_scaling_equals_cupolys(gpu, c):
    k, kl, nphi, t = c["k"], c["kl"], c["nphi"], c["t"]
    e = _engine(k, kl, nphi, t)
    x = _inputs(c)
    xq, xb = x[:k * nphi].reshape(k, nphi), x[k * nphi:].reshape(kl, nphi)
    aq, ab = _to_dgt(e, xq, 0), _to_dgt(e, xb, 1)
    out = e.empty(0)
    e.poly_complex_scaling_tdivq(out, aq, ab)
    got = _coeffs(e, out, 0)[0]
    if _same(c, got):
        return
    Q, B = e.Q, e.B
    exact = CO.basis_ext(CO.complex_scaling(xq, xb, Q, B, t), B, Q)
    cols = [([int(v) for v in xq[:, j]], [int(v) for v in xb[:, j]]) for j in range(nphi)]
    restated = np.array([O.cupoly_float_complex_scaling_tdivq(a, b, Q, B, t) for a, b in cols], dtype=np.uint64).T
    assert sha(restated) == c["sha256"]
    _only_rounding_differences(got, exact, restated, Q)


@pytest.mark.parametrize("c", _cases("xirho"), ids=_id)
def test_xi_rho_equal_cupolys(gpu, c):
    k, nphi = c["k"], c["nphi"]
    e = _engine(k, c["kl"], nphi, c["t"])
    a = _to_dgt(e, _inputs(c).reshape(k, nphi), 0)
    xi, rho = e.empty(0, k), e.empty(0, k)
    e.xi(xi, a)
    e.rho(rho, a)
    got = np.stack([_coeffs(e, xi, 0), _coeffs(e, rho, 0)])
    assert _same(c, got)


@pytest.mark.parametrize("c", _cases("bfvmul"), ids=_id)
def test_bfv_chain_equals_cupolys(gpu, c):
    k, kl, nphi, t = c["k"], c["kl"], c["nphi"], c["t"]
    e = _engine(k, kl, nphi, t)
    x = _inputs(c).reshape(4, k, nphi)
    ins = [_to_dgt(e, x[i], 0) for i in range(4)]
    outs = [e.empty(0) for _ in range(3)]
    e.bfv_mul(*outs, *ins)
    got = np.stack([_coeffs(e, o, 0)[0] for o in outs])
    if _same(c, got):
        return
    # cuPoly's float complex scaling is off by one on some coefficients (at k = 6 often):
    # the device gives the exact product, and cuPoly's recorded words are its restated chain
    exact = CO.bfv_mul(*[x[i][None] for i in range(4)], e.Q, e.B, t)
    restated = cupoly_chain_restated(x, e.Q, e.B, t)
    assert sha(restated) == c["sha256"]
    for g, ex, r in zip(got, exact, restated):
        _only_rounding_differences(g, ex[0], r, e.Q)


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="cuPoly's sources were not compiled here")
@pytest.mark.parametrize("k,nphi", [(2, 4096), (5, 8192)])
def test_live_cupoly_driver_on_fresh_inputs(gpu, k, nphi):
    """cuPoly's own library, run now on inputs no fixture holds: DGT-domain bytes,
    poly_mul and poly_basis_extension_Q_to_B equal the CUDA path's."""
    kl = k + 1
    from tests.golden.gen_cupoly_golden import inputs
    from cupoly_b200.engine import to_u64
    seed = 9000 + nphi + k
    ops = ["dgt", "mul", "ext"]
    ins = {op: inputs(op, k, kl, nphi, seed + i) for i, op in enumerate(ops)}
    with tempfile.TemporaryDirectory() as d:
        for op in ops:
            ins[op].tofile(os.path.join(d, "in." + op))
        subprocess.run([DRIVER, ",".join(ops), str(k), str(kl), str(nphi), "256", os.path.join(d, "in"),
                        os.path.join(d, "out")], check=True, timeout=300)
        ref = {op: np.fromfile(os.path.join(d, "out." + op), dtype=np.uint64) for op in ops}
    e = _engine(k, kl, nphi, 256)
    dg = _to_dgt(e, ins["dgt"].reshape(k + kl, nphi), 2)
    assert np.array_equal(to_u64(dg)[0].reshape(-1), ref["dgt"][:ref["dgt"].size // 2])
    x = ins["mul"].reshape(2, k, nphi)
    a, b = _to_dgt(e, x[0], 0), _to_dgt(e, x[1], 0)
    out = e.empty(0)
    e.mul(out, a, b, 0)
    assert np.array_equal(_coeffs(e, out, 0)[0].reshape(-1), ref["mul"])
    a = _to_dgt(e, ins["ext"].reshape(k, nphi), 0)
    ob = e.empty(1)
    e.poly_basis_extension_q_to_b(ob, a)
    assert np.array_equal(_coeffs(e, ob, 1)[0].reshape(-1), ref["ext"])


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="cuPoly's sources were not compiled here")
def test_live_cupoly_bfv_chain_on_fresh_inputs(gpu):
    """cuPoly's own BFV multiplication chain, run now on fresh inputs at nphi 8192, k 5, kl 6:
    the batched chain of this library gives the exact product, and cuPoly's words are its
    restated float chain (each difference one of its rounding errors)."""
    from tests.golden.gen_cupoly_golden import inputs
    from cupoly_b200.engine import INVERSE, QBase, from_u64, to_u64
    k, kl, nphi, t = 5, 6, 8192, 256
    x = inputs("bfvmul", k, kl, nphi, 9901)
    with tempfile.TemporaryDirectory() as d:
        x.tofile(os.path.join(d, "in"))
        subprocess.run([DRIVER, "bfvmul", str(k), str(kl), str(nphi), str(t), os.path.join(d, "in"),
                        os.path.join(d, "out")], check=True, timeout=300)
        ref = np.fromfile(os.path.join(d, "out"), dtype=np.uint64).reshape(3, k, nphi)
    e = _engine(k, kl, nphi, t)
    rows = x.reshape(4, k, nphi)
    dev = [_to_dgt(e, rows[i], 0) for i in range(4)]
    c = e.empty(QBase, 3)
    e.bfv_mul_batch(c, *dev, 1, e.bfv_mul_batch_workspace(1))
    e.dgt(c, QBase, INVERSE)
    got = unfold(to_u64(c)).reshape(3, k, nphi)
    exact = CO.bfv_mul(*[rows[i][None] for i in range(4)], e.Q, e.B, t)
    for j in range(3):
        assert np.array_equal(got[j], exact[j][0])
    if not np.array_equal(got, ref):
        restated = cupoly_chain_restated(rows, e.Q, e.B, t)
        assert np.array_equal(restated, ref)
        for j in range(3):
            _only_rounding_differences(got[j], exact[j][0], restated[j], e.Q)
