"""The oracle pinned to cuPoly's own outputs (no GPU needed here).

tests/golden/cupoly_ref_golden.json holds what cuPoly 0.3.5 itself computed:
its library sources, compiled unmodified by oracle/cupoly_ref/Makefile, run
through its public API on a B200 by tests/golden/gen_cupoly_golden.py, on the
seeded inputs of tests/common.py.  Each case is re-derived here from the
oracle and compared word for word (SHA-256 of the output):

* DGT-domain bytes (DGTEngine::execute_dgt, src/cuda/dgt.cu:107-205) against
  the oracle's transform with cuPoly's tabulated roots (ref_nthroot.json);
* poly_mul (src/arithmetic/polynomial.cu:892-914) against the negacyclic
  product;
* poly_basis_extension_Q_to_B, poly_complex_scaling_tDivQ and
  poly_simple_scaling_tDivQ (polynomial.cu:310-450) against the oracle's
  restatement of cuPoly's double-precision HPS path, including its 512-bit
  NTL RR constants -- and each of those against the exact value, with every
  disagreement required to be one of cuPoly's own rounding errors;
* the BFV multiplication chain composed of cuPoly's calls against the same
  composition in the oracle;
* poly_xi_bfv / poly_rho_bfv (polynomial.cu:612-693) against their
  definitions;
* cuPoly's precomputed HPS constants and Barrett factors
  (src/cuda/cudaengine.cu:1463-1510, src/cuda/dgt.cu:1755-1766) against
  Python big integers.
"""
import json
import os

import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import cupoly_chain_restated, fold, sha

GOLD = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLD, "cupoly_ref_golden.json")) as _f:
    DOC = json.load(_f)


def ref_xi(primes, N):
    roots = json.load(open(os.path.join(GOLD, "ref_nthroot.json")))
    return [tuple(roots[str(p)][str(N)]) for p in primes]


def cases(op):
    return [c for c in DOC["cases"] if c["op"] == op]


def _id(c):
    return "nphi%d_k%d_kl%d_t%d" % (c["nphi"], c["k"], c["kl"], c["t"])


def inputs(c):
    """The driver's inputs of case c (same generator as the fixture script)."""
    from tests.golden.gen_cupoly_golden import inputs as gen_inputs
    return gen_inputs(c["op"], c["k"], c["kl"], c["nphi"], c["seed"])


def matches(c, out):
    out = np.ascontiguousarray(out, dtype=np.uint64).reshape(-1)
    assert out.size == c["words"]
    if "full" in c:
        assert out.tolist() == c["full"]
    assert [int(v) for v in out[:6]] == c["head"]
    return sha(out) == c["sha256"]


def cols(rows):
    return [[int(v) for v in rows[:, j]] for j in range(rows.shape[1])]


def test_fixture_covers_the_grid_and_both_benchmark_sizes():
    got = {(c["op"], c["nphi"], c["k"]) for c in DOC["cases"]}
    for nphi, k in [(32, 1), (32, 6), (2048, 6), (4096, 2), (8192, 5), (8192, 6)]:
        for op in ("dgt", "mul", "ext", "cscale", "sscale", "xirho"):
            assert (op, nphi, k) in got
    assert ("bfvmul", 8192, 5) in got and ("bfvmul", 4096, 2) in got


@pytest.mark.parametrize("r", DOC["tables"], ids=_id)
def test_cupoly_tables_equal_the_restatement(r):
    """Q and B are cuPoly's first k and next kl primes; its Barrett MU is
    floor(4^63 / p); omega, lambda and tomega are the 512-bit RR values the
    oracle restates (``_cupoly_omega``, ``_cupoly_tomega``)."""
    k, kl, t = r["k"], r["kl"], r["t"]
    Q, B = O.bases(k, kl)
    assert r["Q"] == Q and r["B"] == B
    assert r["barrett_mu"] == [(4 ** p.bit_length()) // p for p in Q + B]
    om_int, om_frac, lam = O._cupoly_omega(tuple(Q), tuple(B), t)
    assert r["lambda"] == list(lam)
    # cuPoly's layout: index i * k + l for B prime i and Q prime l (cudaengine.cu:1465-1490)
    assert r["omega_int"] == [om_int[l, i] for i in range(kl) for l in range(k)]
    assert r["omega_frac"] == [om_frac[l, i] for i in range(kl) for l in range(k)]
    tom = O._cupoly_tomega(tuple(Q), t)
    assert r["tomega_int"] == [a for a, _ in tom]
    assert r["tomega_frac"] == [b for _, b in tom]


@pytest.mark.parametrize("c", cases("dgt"), ids=_id)
def test_dgt_domain_bytes_equal_cupolys(c):
    k, kl, nphi = c["k"], c["kl"], c["nphi"]
    Q, B = O.bases(k, kl)
    x = inputs(c).reshape(k + kl, nphi)
    got = CO.dgt(fold(x)[None], Q + B, xi=ref_xi(Q + B, nphi // 2))[0]
    assert c["round_trip"]
    assert matches(c, got)


@pytest.mark.parametrize("c", cases("mul"), ids=_id)
def test_poly_mul_equals_cupolys(c):
    k, nphi = c["k"], c["nphi"]
    Q, _ = O.bases(k, c["kl"])
    x = inputs(c).reshape(2, k, nphi)
    assert matches(c, CO.polymul(x[:1], x[1:], Q)[0])


@pytest.mark.parametrize("c", cases("ext"), ids=_id)
def test_basis_extension_equals_cupolys(c):
    k, kl, nphi = c["k"], c["kl"], c["nphi"]
    Q, B = O.bases(k, kl)
    x = inputs(c).reshape(k, nphi)
    flt = np.array([O.cupoly_float_ext_q_to_b(v, Q, B) for v in cols(x)], dtype=np.uint64).T
    assert matches(c, flt)
    # on these random inputs cuPoly's double-precision v is exact
    assert np.array_equal(flt, CO.basis_ext(x, Q, B))


def _disagreements_are_rounding_errors(flt, exact, Q):
    """Where cuPoly's float scaling differs from round(t X / Q), it is off by
    exactly one (the float fraction sum rounded the other way)."""
    Qp = O.prod(Q)
    for j in np.nonzero((flt != exact).any(axis=0))[0]:
        a = O.crt([int(v) for v in flt[:, j]], Q)
        b = O.crt([int(v) for v in exact[:, j]], Q)
        assert (a - b) % Qp in (1, Qp - 1)


@pytest.mark.parametrize("c", cases("cscale"), ids=_id)
def test_complex_scaling_equals_cupolys(c):
    k, kl, nphi, t = c["k"], c["kl"], c["nphi"], c["t"]
    Q, B = O.bases(k, kl)
    x = inputs(c)
    xq, xb = x[:k * nphi].reshape(k, nphi), x[k * nphi:].reshape(kl, nphi)
    cq, cb = cols(xq), cols(xb)
    flt = np.array([O.cupoly_float_complex_scaling_tdivq(a, b, Q, B, t) for a, b in zip(cq, cb)],
                   dtype=np.uint64).T
    assert matches(c, flt)
    exact = np.array([O.complex_scaling_tdivq_exact(a, b, Q, B, t) for a, b in zip(cq, cb)], dtype=np.uint64).T
    _disagreements_are_rounding_errors(flt, exact, Q)


@pytest.mark.parametrize("c", cases("sscale"), ids=_id)
def test_simple_scaling_equals_cupolys(c):
    k, nphi, t = c["k"], c["nphi"], c["t"]
    Q, _ = O.bases(k, c["kl"])
    x = inputs(c).reshape(k, nphi)
    cx = cols(x)
    # cuPoly's device words are not reduced mod t (its d_RNST is never set)
    raw = np.array([O.cupoly_float_simple_scaling(v, Q, t, raw=True) for v in cx], dtype=np.uint64)
    assert matches(c, raw)
    flt = raw & np.uint64(t - 1)
    exact = np.array([O.simple_scaling_exact(v, Q, t) for v in cx], dtype=np.uint64)
    for j in np.nonzero(flt != exact)[0]:
        assert (int(flt[j]) - int(exact[j])) % t in (1, t - 1)


@pytest.mark.parametrize("c", cases("xirho"), ids=_id)
def test_xi_rho_equal_cupolys(c):
    """xi_i(a): residue i of a times (Q/q_i)^-1 mod q_i; rho_i(a): residue i times
    Q/q_i mod q_i; every other residue zero (cudaengine.cu:992-1083)."""
    k, nphi = c["k"], c["nphi"]
    Q, _ = O.bases(k, c["kl"])
    x = inputs(c).reshape(k, nphi)
    Qp = O.prod(Q)
    out = np.zeros((2, k, k, nphi), dtype=np.uint64)
    for i, q in enumerate(Q):
        row = [int(v) for v in x[i]]
        out[0, i, i] = [v * pow(Qp // q % q, -1, q) % q for v in row]
        out[1, i, i] = [v * (Qp // q % q) % q for v in row]
    assert matches(c, out)


@pytest.mark.parametrize("c", cases("bfvmul"), ids=_id)
def test_bfv_chain_equals_cupolys(c):
    """cuPoly's composition (4 x poly_basis_extension_Q_to_B, poly_dr2 over Q and
    over B, 3 x poly_complex_scaling_tDivQ) against the same composition in the
    oracle: float extension, exact tensor, float scaling."""
    k, kl, nphi, t = c["k"], c["kl"], c["nphi"], c["t"]
    Q, B = O.bases(k, kl)
    x = inputs(c).reshape(4, k, nphi)
    outs = cupoly_chain_restated(x, Q, B, t)
    assert matches(c, outs)
    exact = CO.bfv_mul(*[x[i][None] for i in range(4)], Q, B, t)
    for o, e in zip(outs, exact):
        _disagreements_are_rounding_errors(o, e[0], Q)
