"""HPS basis extension, scaling and the BFV multiplication chain on the GPU,
bit-exact against the exact oracle (cuPoly TestRNS ports included)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import fold, random_poly_int, random_poly_residues, sha, unfold

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _dev(x):
    from cupoly_b200.engine import from_u64
    return from_u64(x)


def _host(t):
    from cupoly_b200.engine import to_u64
    return to_u64(t)


@pytest.mark.parametrize("k,kl,nphi", [(1, 2, 32), (2, 3, 2048), (5, 6, 8192), (8, 9, 4096), (16, 17, 32768),
                                        (24, 24, 64), (7, 3, 256)])
def test_basis_extension_exact(gpu, k, kl, nphi):
    from cupoly_b200.engine import Engine
    e = Engine(k, kl, nphi, 256)
    xq = random_poly_residues(k, e.Q, nphi)
    yb = random_poly_residues(k + 1, e.B, nphi)
    out = e.empty(1)
    e.basis_ext_q_to_b(out, _dev(fold(xq)[None]))
    assert np.array_equal(unfold(_host(out))[0], CO.basis_ext(xq, e.Q, e.B))
    outq = e.empty(0)
    e.basis_ext_b_to_q(outq, _dev(fold(yb)[None]))
    assert np.array_equal(unfold(_host(outq))[0], CO.basis_ext(yb, e.B, e.Q))


@pytest.mark.parametrize("k", [3, 7, 10])
def test_basis_extension_edges(gpu, k):
    """cuPoly's lift on both sides of its threshold T = Q - floor(Q FPERROR): X below T
    converts as X, X from T up as X - Q (cuPoly's v rounds up within FPERROR of an
    integer, src/cuda/cudaengine.cu:513-534), in the digit path (k < 7) and the fast
    path with its exact fallback (k >= 7); also B -> Q."""
    from cupoly_b200.engine import Engine
    e = Engine(k, 0, 64, 256)
    for src, dst, fwd in ((e.Q, e.B, True), (e.B, e.Q, False)):
        S = O.prod(src)
        T = O.lift_threshold(S)
        vals = [0, 1, S - 1, (S - 1) // 2, (S + 1) // 2, 12345, T - 1, T, T + 1, T - 2, S - 2]
        vals += [T + (S - T) * i // 26 for i in range(26)] + [T - 1 - (i << 40) for i in range(27)]
        assert len(vals) == e.nphi
        xs = np.array([[v % q for v in vals] for q in src], dtype=np.uint64)
        out = e.empty(1 if fwd else 0)
        (e.basis_ext_q_to_b if fwd else e.basis_ext_b_to_q)(out, _dev(fold(xs)[None]))
        want = [[O.cupoly_lift(v, S) % m for v in vals] for m in dst]
        assert unfold(_host(out))[0].tolist() == want


@pytest.mark.parametrize("k,nphi,t", [(1, 32, 256), (2, 2048, 256), (5, 8192, 256), (3, 4096, 65537),
                                      (16, 32768, 65537), (4, 64, 3)])
def test_complex_and_simple_scaling(gpu, k, nphi, t):
    from cupoly_b200.engine import Engine
    e = Engine(k, 0, nphi, t)
    xq = random_poly_residues(3 * k, e.Q, nphi)
    yb = random_poly_residues(3 * k + 1, e.B, nphi)
    out = e.empty(1)
    e.complex_scaling(out, _dev(fold(xq)[None]), _dev(fold(yb)[None]))
    assert np.array_equal(unfold(_host(out))[0], CO.complex_scaling(xq, yb, e.Q, e.B, t))
    ot = e.empty(3)
    e.simple_scaling(ot, _dev(fold(xq)[None]))
    assert np.array_equal(unfold(_host(ot))[0, 0], CO.simple_scaling(xq, e.Q, t))


def test_golden_hps(gpu):
    from cupoly_b200.engine import Engine
    for case in json.load(open(os.path.join(GOLD, "hps_golden.json"))):
        e = Engine(case["k"], case["kl"], case["nphi"], case["t"])
        xq = random_poly_residues(case["seed"], e.Q, case["nphi"])
        yb = random_poly_residues(case["seed"] + 1000, e.B, case["nphi"])
        out = e.empty(1)
        e.basis_ext_q_to_b(out, _dev(fold(xq)[None]))
        assert sha(unfold(_host(out))[0]) == case["ext_q_to_b"]
        outq = e.empty(0)
        e.basis_ext_b_to_q(outq, _dev(fold(yb)[None]))
        assert sha(unfold(_host(outq))[0]) == case["ext_b_to_q"]
        e.complex_scaling(out, _dev(fold(xq)[None]), _dev(fold(yb)[None]))
        assert sha(unfold(_host(out))[0]) == case["complex_scaling"]
        ot = e.empty(3)
        e.simple_scaling(ot, _dev(fold(xq)[None]))
        assert sha(unfold(_host(ot))[0, 0]) == case["simple_scaling"]


def _bfv_case(k, nphi, t, seed):
    from cupoly_b200.engine import FORWARD, INVERSE, Engine
    e = Engine(k, 0, nphi, t)
    rows = [random_poly_residues(seed + i, e.Q, nphi) for i in range(4)]
    dev = []
    for r in rows:
        d = _dev(fold(r)[None])
        e.dgt(d, 0, FORWARD)
        dev.append(d)
    outs = [e.empty(0) for _ in range(3)]
    e.bfv_mul(*outs, *dev)
    got = []
    for o in outs:
        e.dgt(o, 0, INVERSE)
        got.append(unfold(_host(o))[0])
    ref = CO.bfv_mul(*[r[None] for r in rows], e.Q, e.B, t)
    return got, [r[0] for r in ref], e, dev


@pytest.mark.parametrize("k,nphi,t", [(1, 32, 256), (2, 4096, 256), (5, 8192, 256), (3, 2048, 65537)])
def test_bfv_mul_plain_vs_oracle(gpu, k, nphi, t):
    got, ref, e, dev = _bfv_case(k, nphi, t, 100 + k)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


def test_bfv_mul_keeps_inputs(gpu):
    got, ref, e, dev = _bfv_case(2, 2048, 256, 7)
    got2, _, _, _ = _bfv_case(2, 2048, 256, 7)
    for a, b in zip(got, got2):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("logq2,nphi", [(30, 32), (120, 2048), (250, 8192)])
def test_reference_rns_tests(gpu, logq2, nphi):
    """cuPoly TestRNS.{SimpleBasisExtensionQuadQtoB, SimpleScalingtDivQ,
    ComplexBasisScalingUniform, WorddecompPowersOf} (test_bfv_mode.cu:492-1104)."""
    from cupoly_b200 import cupoly as cp
    from cupoly_b200.engine import INVERSE
    k = math.ceil(logq2 / 63)
    t = 256
    cp.CUDAEngine.init(k, k + 1, nphi, t)
    ctx = cp.Context()
    e = cp.CUDAEngine.engine
    q = cp.CUDAEngine.RNSProduct
    # quadratic input i^2 mod t extended to B
    aq, ab = cp.poly_t(), cp.poly_t()
    cp.poly_init(ctx, aq)
    for i in range(nphi):
        cp.poly_set_coeff(ctx, aq, i, i * i % t)
    cp.poly_basis_extension_Q_to_B(ctx, ab, aq)
    tb = ab.d_coefs.clone()
    e.dgt(tb, 1, INVERSE, stream=ctx.stream)
    assert unfold(_host(tb))[0].tolist() == [[i * i % t % b for i in range(nphi)] for b in e.B]
    # simple scaling vs round(t x / q) mod t
    a, b = cp.poly_t(), cp.poly_t()
    cp.poly_init(ctx, a)
    cp.Sampler.sample(ctx, a, cp.UNIFORM_MOD_Q)
    A = [cp.poly_get_coeff(ctx, a, i) for i in range(nphi)]
    cp.poly_simple_scaling_tDivQ(ctx, b, a)
    assert [cp.poly_get_coeff(ctx, b, i) for i in range(nphi)] == [(2 * t * x + q) // (2 * q) % t for x in A]
    # complex scaling: |b - t c / q| < 2 in the reference; here exact round(t c / q)
    aq2, ab2, out = cp.poly_t(), cp.poly_t(), cp.poly_t()
    cp.poly_init(ctx, aq2)
    cp.Sampler.sample(ctx, aq2, cp.UNIFORM_MOD_Q)
    C = [cp.poly_get_coeff(ctx, aq2, i) for i in range(nphi)]
    cp.poly_basis_extension_Q_to_B(ctx, ab2, aq2)
    cp.poly_complex_scaling_tDivQ(ctx, out, aq2, ab2)
    got = [cp.poly_get_coeff(ctx, out, i) for i in range(nphi)]
    assert got == [(2 * t * c + q) // (2 * q) for c in C]
    assert all(abs(g - t * c / q) < 2 for g, c in zip(got, C))
    # <rho(a), xi(b)> == a * b mod q
    x, y, prod_ = cp.poly_t(), cp.poly_t(), cp.poly_t()
    for p_ in (x, y):
        cp.poly_init(ctx, p_)
        cp.Sampler.sample(ctx, p_, cp.DISCRETE_GAUSSIAN)
    R = [cp.poly_t() for _ in range(k)]
    X = [cp.poly_t() for _ in range(k)]
    cp.poly_rho_bfv(ctx, R, x)
    cp.poly_xi_bfv(ctx, X, y)
    acc = cp.poly_t()
    cp.poly_init(ctx, acc)
    for i in range(k):
        cp.poly_mul_add(ctx, acc, R[i], X[i], acc)
    cp.poly_mul(ctx, prod_, x, y)
    assert [cp.poly_get_coeff(ctx, acc, i) for i in range(nphi)] == \
        [cp.poly_get_coeff(ctx, prod_, i) for i in range(nphi)]
    dot = cp.poly_t()
    cp.poly_dot(ctx, dot, R, X, k)  # the fused form of the loop above
    assert [cp.poly_get_coeff(ctx, dot, i) for i in range(nphi)] == \
        [cp.poly_get_coeff(ctx, prod_, i) for i in range(nphi)]
    cp.CUDAEngine.destroy()


def test_simple_scaling_exact_vs_bigint(gpu):
    from cupoly_b200.engine import Engine
    e = Engine(3, 0, 64, 65537)
    Qp = O.prod(e.Q)
    ints = random_poly_int(5, Qp, 64)
    xq = np.array([[v % q for v in ints] for q in e.Q], dtype=np.uint64)
    ot = e.empty(3)
    e.simple_scaling(ot, _dev(fold(xq)[None]))
    assert unfold(_host(ot))[0, 0].tolist() == [(2 * 65537 * v + Qp) // (2 * Qp) % 65537 for v in ints]


@pytest.mark.parametrize("k,nphi,npairs", [(2, 2048, 3), (5, 8192, 4)])
def test_bfv_mul_batch_vs_plain_and_oracle(gpu, k, nphi, npairs):
    """Batched chain == per-call chain == oracle, pair by pair."""
    import torch
    from cupoly_b200.engine import FORWARD, INVERSE, Engine
    e = Engine(k, 0, nphi, 256)
    rows = [np.stack([random_poly_residues(200 + 10 * i + j, e.Q, nphi) for i in range(npairs)]) for j in range(4)]
    dev = []
    for r in rows:
        d = _dev(fold(r))
        e.dgt(d, 0, FORWARD)
        dev.append(d)
    c = e.empty(0, 3 * npairs)
    e.bfv_mul_batch(c, *dev, npairs, e.bfv_mul_batch_workspace(npairs))
    for i in range(npairs):
        outs = [e.empty(0) for _ in range(3)]
        e.bfv_mul(*outs, *[d[i:i + 1] for d in dev])
        for j in range(3):
            assert torch.equal(outs[j][0], c[j * npairs + i])
    e.dgt(c, 0, INVERSE)
    got = unfold(_host(c))
    ref = CO.bfv_mul(*rows, e.Q, e.B, 256)
    for j in range(3):
        assert np.array_equal(got[j * npairs:(j + 1) * npairs], ref[j])


@pytest.mark.parametrize("k", [2, 5, 6, 7, 10, 12])
def test_scaling_exact_fallback_edges(gpu, k):
    """Coefficients where the FP64 overflow count is not trusted take the exact path:
    t X mod Q near 0, near Q/2 (both sides) and near Q; X small (round(t X / Q) mod B
    near 0, so the B -> Q step falls back too).  Complex scaling and the whole
    scale-and-convert step (fused for |Q| <= 3, two kernels above) against the oracle."""
    from cupoly_b200.engine import FORWARD, INVERSE, Engine
    t = 256
    nphi = 64
    e = Engine(k, 0, nphi, t)
    Qp, Bp = O.prod(e.Q), O.prod(e.B)
    ti = pow(t, -1, Qp)
    xs = [0, 1, 2, 3, Qp - 1, Qp - 2, (Qp - 1) // 2, (Qp + 1) // 2]
    for z in ((Qp - 1) // 2, (Qp + 1) // 2, (Qp - 3) // 2, (Qp + 3) // 2, 1, 2, Qp - 1, Qp - 2):
        xs.append(z * ti % Qp)                      # t X == z (mod Q)
    xs += [Qp * m + r for m in (0, 1, 5) for r in (0, 1)]   # X in [0, QB): small and multiples of Q
    xs += random_poly_int(5, Qp * Bp, nphi - len(xs))
    assert len(xs) == nphi and all(0 <= x < Qp * Bp for x in xs)
    xq = np.array([[x % q for x in xs] for q in e.Q], dtype=np.uint64)
    yb = np.array([[x % b for x in xs] for b in e.B], dtype=np.uint64)
    out = e.empty(1)
    e.complex_scaling(out, _dev(fold(xq)[None]), _dev(fold(yb)[None]))
    cs = CO.complex_scaling(xq, yb, e.Q, e.B, t)
    assert np.array_equal(unfold(_host(out))[0], cs)
    for x, col in zip(xs[:24], cs.T[:24]):       # definition: round(t X / Q) mod b_j
        assert [int(v) for v in col] == [((2 * t * x + Qp) // (2 * Qp)) % b for b in e.B]
    # scale and convert to Q in one call (DGT domain in and out)
    dq, db = _dev(fold(xq)[None]), _dev(fold(yb)[None])
    e.dgt(dq, 0, FORWARD)
    e.dgt(db, 1, FORWARD)
    oq = e.empty(0)
    e.poly_complex_scaling_tdivq(oq, dq, db)
    e.dgt(oq, 0, INVERSE)
    assert np.array_equal(unfold(_host(oq))[0], CO.basis_ext(cs, e.B, e.Q))
    # basis extensions near the boundaries
    o1 = e.empty(1)
    e.basis_ext_q_to_b(o1, _dev(fold(xq)[None]))
    assert np.array_equal(unfold(_host(o1))[0], CO.basis_ext(xq, e.Q, e.B))
    o0 = e.empty(0)
    e.basis_ext_b_to_q(o0, _dev(fold(yb)[None]))
    assert np.array_equal(unfold(_host(o0))[0], CO.basis_ext(yb, e.B, e.Q))


@pytest.mark.parametrize("k,t", [(2, 256), (5, 256), (5, 65536)])
def test_device_matches_cupolys_float_path_where_it_is_exact(gpu, k, t):
    """Against a word-for-word restatement of cuPoly's double-precision HPS kernels
    (oracle/pyoracle.py cupoly_float_*): on random coefficients and at X = Q - 1, Q - 2
    (above the lift threshold) the device's Q -> B, B -> Q, complex and simple scaling
    agree with cuPoly's path everywhere; next to the half-integer rounding boundary,
    the only place cuPoly's path differs from the exact value, the device gives the
    exact one."""
    from cupoly_b200.engine import Engine
    nphi = 512
    e = Engine(k, 0, nphi, t)
    Q, B = list(e.Q), list(e.B)
    Qp, Bp = O.prod(Q), O.prod(B)
    rng = np.random.default_rng(k * 1000 + t)
    Xs = [int(rng.integers(0, 1 << 62)) * (1 << 62) % Qp for _ in range(nphi)]
    Xs[0], Xs[1] = Qp - 1, Qp - 2
    ti = pow(t, -1, Qp)
    Zs = [int(rng.integers(0, 1 << 62)) * (1 << 60) % (Qp * Bp) for _ in range(nphi)]
    for i, h in enumerate(((Qp - 1) // 2, (Qp + 1) // 2, (Qp - 3) // 2, (Qp + 3) // 2)):
        Zs[i] = (h * ti) % Qp + Qp * (i + 1)
    xq = np.array([[X % q for X in Xs] for q in Q], dtype=np.uint64)
    yb = np.array([[X % b for X in Xs] for b in B], dtype=np.uint64)  # X < Q < B: a valid B value too
    zq = np.array([[Z % q for Z in Zs] for q in Q], dtype=np.uint64)
    zb = np.array([[Z % b for Z in Zs] for b in B], dtype=np.uint64)
    ob, oq, oc, ot = e.empty(1), e.empty(0), e.empty(1), e.empty(3)
    e.basis_ext_q_to_b(ob, _dev(fold(xq)[None]))
    e.basis_ext_b_to_q(oq, _dev(fold(yb)[None]))
    e.complex_scaling(oc, _dev(fold(zq)[None]), _dev(fold(zb)[None]))
    e.simple_scaling(ot, _dev(fold(xq)[None]))
    ob, oq, oc = (unfold(_host(x))[0] for x in (ob, oq, oc))
    ot = unfold(_host(ot))[0, 0]
    edge_c = {0, 1, 2, 3}
    diff = {"q_to_b": [], "b_to_q": [], "complex": [], "simple": []}
    for c in range(nphi):
        xs, ys = [int(v) for v in xq[:, c]], [int(v) for v in yb[:, c]]
        zqs, zbs = [int(v) for v in zq[:, c]], [int(v) for v in zb[:, c]]
        if [int(v) for v in ob[:, c]] != O.cupoly_float_ext_q_to_b(xs, Q, B):
            diff["q_to_b"].append(c)
        if [int(v) for v in oq[:, c]] != O.cupoly_float_ext_b_to_q(ys, Q, B):
            diff["b_to_q"].append(c)
        if [int(v) for v in oc[:, c]] != O.cupoly_float_complex_scaling(zqs, zbs, Q, B, t):
            diff["complex"].append(c)
        if t & (t - 1) == 0 and int(ot[c]) != O.cupoly_float_simple_scaling(xs, Q, t):
            diff["simple"].append(c)
    # X = Q - 1 and Q - 2 lie above cuPoly's lift threshold: both read them as X - Q
    assert diff["q_to_b"] == [] and diff["b_to_q"] == []
    assert [int(v) for v in ob[:, 0]] == [(Qp - 1 - Qp) % b for b in B]
    # scaling: disagreements only at the engineered half-integer edges, where the device is exact
    assert set(diff["complex"]) <= edge_c
    for c in diff["complex"]:
        assert [int(v) for v in oc[:, c]] == O.complex_scaling_exact([int(v) for v in zq[:, c]],
                                                                      [int(v) for v in zb[:, c]], Q, B, t)
    assert set(diff["simple"]) <= {0, 1}


def test_xi_rho_batch_equals_per_polynomial_calls(gpu):
    """cp_xi_batch / cp_rho_batch: polynomial p's decomposition equals the one-polynomial call."""
    import torch

    from cupoly_b200.engine import Engine, QBase, UNIFORM
    e = Engine(4, 0, 4096, 256)
    P, k = 6, 4
    a = e.empty(QBase, P)
    e.sample(a, QBase, UNIFORM, 31, 0, npolys=P, to_dgt=True)
    for batch, single in ((e.xi_batch, e.xi), (e.rho_batch, e.rho)):
        out = e.empty(QBase, P * k)
        batch(out, a)
        for p in range(P):
            one = e.empty(QBase, k)
            single(one, a[p:p + 1])
            assert torch.equal(one, out[p * k:(p + 1) * k]), (batch.__name__, p)


@pytest.mark.parametrize("k,nphi,t,npairs,seed", [(10, 16384, 256, 4, 1), (16, 32768, 65537, 2, 2),
                                                  (8, 4096, 65537, 8, 3), (3, 16384, 256, 6, 4),
                                                  (7, 8192, 3, 5, 5)])
def test_bfv_mul_batch_at_the_large_configurations_vs_oracle(gpu, k, nphi, t, npairs, seed):
    """The batched chain at nphi 2^14 with a 10-prime basis (the configuration the targets
    are stated on), at nphi 32768 / k 16 / t 65537, and at other widths and plaintext moduli
    (t = 3: not a power of two), bit-exact against the oracle pair by pair, in the tuned plans
    (split stages included)."""
    from cupoly_b200.engine import FORWARD, INVERSE, Engine
    e = Engine(k, 0, nphi, t)
    rows = [np.stack([random_poly_residues(1000 * seed + 10 * i + j, e.Q, nphi) for i in range(npairs)])
            for j in range(4)]
    dev = []
    for r in rows:
        d = _dev(fold(r))
        e.dgt(d, 0, FORWARD)
        dev.append(d)
    c = e.empty(0, 3 * npairs)
    e.bfv_mul_batch(c, *dev, npairs, e.bfv_mul_batch_workspace(npairs))
    e.dgt(c, 0, INVERSE)
    got = unfold(_host(c))
    ref = CO.bfv_mul(*rows, e.Q, e.B, t)
    for j in range(3):
        assert np.array_equal(got[j * npairs:(j + 1) * npairs], ref[j]), (j, k, nphi)


@pytest.mark.parametrize("k,nphi,t,npairs", [(1, 2048, 256, 3), (5, 8192, 256, 2), (7, 4096, 65537, 2),
                                             (10, 16384, 3, 1)])
def test_bfv_mul_exact_paths_vs_oracle(gpu, k, nphi, t, npairs):
    """Every base conversion and scaling forced onto its exact path: the batched chain (whose
    inverse transforms leave prescaled values for the conversions, undone on that path) and the
    per-call chain still equal the oracle, and so do the plain conversions."""
    import torch
    from cupoly_b200.engine import FORWARD, INVERSE, Engine
    e = Engine(k, 0, nphi, t)
    rows = [np.stack([random_poly_residues(700 + 10 * i + j, e.Q, nphi) for i in range(npairs)]) for j in range(4)]
    dev = []
    for r in rows:
        d = _dev(fold(r))
        e.dgt(d, 0, FORWARD)
        dev.append(d)
    fast = e.empty(0, 3 * npairs)
    e.bfv_mul_batch(fast, *dev, npairs, e.bfv_mul_batch_workspace(npairs))
    e.set_hps_force_exact(True)
    try:
        c = e.empty(0, 3 * npairs)
        e.bfv_mul_batch(c, *dev, npairs, e.bfv_mul_batch_workspace(npairs))
        outs = [e.empty(0) for _ in range(3)]
        e.bfv_mul(*outs, *[d[:1] for d in dev])
        xq = rows[0][0]
        ob = e.empty(1)
        e.basis_ext_q_to_b(ob, _dev(fold(xq)[None]))
        yb = random_poly_residues(701, e.B, nphi)
        oq = e.empty(0)
        e.basis_ext_b_to_q(oq, _dev(fold(yb)[None]))
        cs = e.empty(1)
        e.complex_scaling(cs, _dev(fold(xq)[None]), _dev(fold(yb)[None]))
        torch.cuda.synchronize()
    finally:
        e.set_hps_force_exact(False)
    assert torch.equal(fast, c)
    for j in range(3):
        assert torch.equal(outs[j][0], c[j * npairs])
    e.dgt(c, 0, INVERSE)
    got = unfold(_host(c))
    ref = CO.bfv_mul(*rows, e.Q, e.B, t)
    for j in range(3):
        assert np.array_equal(got[j * npairs:(j + 1) * npairs], ref[j]), (j, k, nphi)
    assert np.array_equal(unfold(_host(ob))[0], CO.basis_ext(xq, e.Q, e.B))
    assert np.array_equal(unfold(_host(oq))[0], CO.basis_ext(yb, e.B, e.Q))
    assert np.array_equal(unfold(_host(cs))[0], CO.complex_scaling(xq, yb, e.Q, e.B, t))
