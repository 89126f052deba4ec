"""Sampler on the GPU: bit-exact against the oracle's Philox restatement,
cuPoly's TestSampler support checks, and statistics over 2^24 samples."""
import math

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.common import unfold

pytestmark = pytest.mark.gpu
KINDS = [O.DISCRETE_GAUSSIAN, O.HAMMINGWEIGHT, O.NARROW, O.ZO, O.BINARY, O.UNIFORM, O.TERNARY, O.GAUSSIAN,
         O.UNIFORM_U32, O.ZO_HALF]


def _sample(e, kind, nphi, sid, seed, npolys=1, base=0):
    from cupoly_b200.engine import to_u64
    out = e.empty(base, npolys)
    e.sample(out, base, kind, seed, sid, npolys=npolys, to_dgt=False)
    e.check()
    return unfold(to_u64(out))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("nphi", [32, 256, 2048])
def test_bitexact_vs_oracle(gpu, kind, nphi):
    from cupoly_b200.engine import Engine
    e = Engine(2, 0, nphi, 256)
    got = _sample(e, kind, nphi, 5, 0x1234_5678_9ABC)
    assert got[0].tolist() == O.sample_poly(kind, e.Q, nphi, 5, 0x1234_5678_9ABC)


def test_batches_use_consecutive_stream_ids(gpu):
    from cupoly_b200.engine import Engine
    e = Engine(1, 0, 64, 256)
    got = _sample(e, O.TERNARY, 64, 10, 7, npolys=3)
    for i in range(3):
        assert got[i].tolist() == O.sample_poly(O.TERNARY, e.Q, 64, 10 + i, 7)


@pytest.mark.parametrize("nphi", [32, 128, 2048, 8192])
def test_reference_sampler_properties(gpu, nphi):
    """cuPoly TestSampler.{Uniform, Narrow, DiscreteGaussian, HammingWeight} (test_bfv_mode.cu:1405-1487)."""
    from cupoly_b200 import cupoly as cp
    cp.CUDAEngine.init(2, 3, nphi, 256)
    ctx = cp.Context()
    cp.Sampler.init(ctx)
    q = cp.CUDAEngine.RNSProduct
    for _ in range(3):
        a = cp.Sampler.sample(ctx, cp.UNIFORM)
        assert all(0 <= cp.poly_get_coeff(ctx, a, i) < q for i in range(nphi))
        a = cp.Sampler.sample(ctx, cp.NARROW)
        assert all(cp.poly_get_coeff(ctx, a, i) in (0, 1, 2) for i in range(nphi))
        a = cp.Sampler.sample(ctx, cp.DISCRETE_GAUSSIAN)
        vals = [cp.poly_get_coeff(ctx, a, i) for i in range(nphi)]
        assert all(v <= cp.GAUSSIAN_STD_DEVIATION * 6 for v in vals) and sum(vals) > 0
        a = cp.Sampler.sample(ctx, cp.HAMMINGWEIGHT)
        assert sum(1 for i in range(nphi) if cp.poly_get_coeff(ctx, a, i) > 0) == min(64, nphi)
    cp.CUDAEngine.destroy()


def test_statistics_2_24(gpu):
    """Support, mean and variance over 2^24 samples (within 5 standard errors)."""
    from cupoly_b200.engine import Engine, to_u64
    e = Engine(16, 17, 32768, 65537)
    npolys = (1 << 24) // 32768
    p = e.Q[0]
    # ternary: {-1, 0, 1} each 1/3: mean 0, variance 2/3
    out = e.empty(0, npolys)
    e.sample(out, 0, O.TERNARY, 99, 0, npolys=npolys, to_dgt=False)
    e.check()
    h = to_u64(out[:, [0, 1, 6, 11]])
    v = h[:, 0].reshape(-1)
    s = np.where(v == np.uint64(p - 1), -1, v.astype(np.int64))
    assert set(np.unique(s).tolist()) == {-1, 0, 1}
    n = s.size
    assert abs(s.mean()) < 5 * math.sqrt(2 / 3 / n)
    assert abs(s.var() - 2 / 3) < 5 * math.sqrt((s.astype(float) ** 4).mean() / n)
    for j, r in enumerate((1, 6, 11)):  # same value on every residue
        vr = h[:, j + 1].reshape(-1)
        assert np.array_equal(np.where(vr == np.uint64(e.Q[r] - 1), -1, vr.astype(np.int64)), s)
    # discrete Gaussian sigma = 3.19, |x| <= 19
    e.sample(out, 0, O.GAUSSIAN, 99, 1, npolys=npolys, to_dgt=False)
    e.check()
    v = to_u64(out[:, 0]).reshape(-1)
    g = np.where(v > np.uint64(p // 2), -((np.uint64(p) - v).astype(np.int64)), v.astype(np.int64))
    assert np.abs(g).max() <= 19
    xs = np.arange(-19, 20)
    rho = np.exp(-xs.astype(float) ** 2 / (2 * 3.19 ** 2))
    var_t = float((xs ** 2 * rho).sum() / rho.sum())
    assert abs(g.mean()) < 5 * math.sqrt(var_t / g.size)
    m4 = float((xs ** 4 * rho).sum() / rho.sum())
    assert abs(g.var() - var_t) < 5 * math.sqrt((m4 - var_t ** 2) / g.size)
    # uniform mod q_i, independent residues: mean (q-1)/2, variance (q^2-1)/12
    e.sample(out, 0, O.UNIFORM, 99, 2, npolys=npolys, to_dgt=False)
    e.check()
    for r in (0, 7):
        q = e.Q[r]
        u = to_u64(out[:, r]).reshape(-1).astype(np.float64) / q
        assert u.max() < 1.0
        assert abs(u.mean() - 0.5) < 5 * math.sqrt(1 / 12 / u.size)
        assert abs(u.var() - 1 / 12) < 5 * math.sqrt(1 / 180 / u.size)


def _chi2_pvalue(counts, probs, min_expected=5.0):
    """Pearson chi-square p-value, tail bins merged until each expects >= min_expected."""
    from scipy.stats import chi2
    n = sum(counts)
    obs, exp = [], []
    acc_o = acc_e = 0.0
    for c, p in zip(counts, probs):
        acc_o += c
        acc_e += p * n
        if acc_e >= min_expected:
            obs.append(acc_o)
            exp.append(acc_e)
            acc_o = acc_e = 0.0
    if acc_e > 0:  # leftover tail joins the last bin
        obs[-1] += acc_o
        exp[-1] += acc_e
    stat = sum((o - e) ** 2 / e for o, e in zip(obs, exp))
    return float(chi2.sf(stat, len(obs) - 1))


def test_chi_square_2_24(gpu):
    """Per-value frequencies over 2^24 samples against the defining distributions
    (Pearson chi-square, p > 1e-4 on the seeded run): ternary's 3 values at 1/3;
    the signed discrete Gaussian's 39 values (sigma 3.19, |x| <= 19) with
    rho(x) = exp(-x^2 / (2 sigma^2)); cuPoly's DISCRETE_GAUSSIAN |nearbyint(3.2 Z)|
    over its 20 magnitudes from the normal distribution; NARROW's 3 values."""
    from scipy.stats import norm
    from cupoly_b200.engine import Engine, to_u64
    e = Engine(1, 0, 32768, 65537)
    npolys = (1 << 24) // 32768
    p = e.Q[0]
    out = e.empty(0, npolys)

    def draw(kind, sid):
        e.sample(out, 0, kind, 2024, sid, npolys=npolys, to_dgt=False)
        e.check()
        v = to_u64(out[:, 0]).reshape(-1)
        return np.where(v > np.uint64(p // 2), -((np.uint64(p) - v).astype(np.int64)), v.astype(np.int64))

    t = draw(O.TERNARY, 0)
    cnt = [int((t == x).sum()) for x in (-1, 0, 1)]
    assert sum(cnt) == t.size
    assert _chi2_pvalue(cnt, [1 / 3] * 3) > 1e-4

    g = draw(O.GAUSSIAN, 1)
    xs = np.arange(-19, 20)
    rho = np.exp(-xs.astype(float) ** 2 / (2 * 3.19 ** 2))
    cnt = [int((g == x).sum()) for x in xs]
    assert sum(cnt) == g.size
    assert _chi2_pvalue(cnt, list(rho / rho.sum())) > 1e-4

    d = draw(O.DISCRETE_GAUSSIAN, 2)
    ms = np.arange(0, 20)
    pm = np.array([norm.cdf(0.5 / 3.2) - norm.cdf(-0.5 / 3.2)] +
                  [2 * (norm.cdf((m + 0.5) / 3.2) - norm.cdf((m - 0.5) / 3.2)) for m in range(1, 20)])
    cnt = [int((d == m).sum()) for m in ms]
    assert sum(cnt) == d.size
    assert _chi2_pvalue(cnt, list(pm / pm.sum())) > 1e-4

    n = draw(O.NARROW, 3)
    cnt = [int((n == x).sum()) for x in (0, 1, 2)]
    assert sum(cnt) == n.size
    assert _chi2_pvalue(cnt, [1 / 3] * 3) > 1e-4


def test_cupoly_uniform_and_zo_semantics(gpu):
    """cuPoly's BFV UNIFORM: one value below 2^32 on every residue, uniform (chi-square
    over 16 bins of the top 4 bits, 2^24 samples); cuPoly's ZO: exactly nphi/2 nonzero
    coefficients per polynomial, signs balanced, every position nonzero about half the
    time across polynomials (chi-square over positions)."""
    from cupoly_b200.engine import UNIFORM_U32, ZO_HALF, Engine, to_u64
    e = Engine(3, 0, 32768, 256)
    npolys = (1 << 24) // 32768
    out = e.empty(0, npolys)
    e.sample(out, 0, UNIFORM_U32, 77, 0, npolys=npolys, to_dgt=False)
    e.check()
    h = to_u64(out)
    u = h[:, 0].reshape(-1)
    assert u.max() < (1 << 32)
    for r in (1, 2):
        assert np.array_equal(h[:, r].reshape(-1), u)
    cnt = np.bincount((u >> np.uint64(28)).astype(np.int64), minlength=16).tolist()
    assert _chi2_pvalue(cnt, [1 / 16] * 16) > 1e-4

    e2 = Engine(2, 0, 2048, 256)
    P = 4096
    z = e2.empty(0, P)
    e2.sample(z, 0, ZO_HALF, 78, 0, npolys=P, to_dgt=False)
    e2.check()
    v = unfold(to_u64(z))[:, 0]  # (P, nphi)
    q = e2.Q[0]
    s = np.where(v == np.uint64(q - 1), -1, v.astype(np.int64))
    assert set(np.unique(s).tolist()) == {-1, 0, 1}
    assert ((s != 0).sum(axis=1) == 1024).all()
    plus, minus = int((s == 1).sum()), int((s == -1).sum())
    assert abs(plus - minus) < 5 * math.sqrt(plus + minus)
    pos = (s != 0).sum(axis=0)  # per position: Binomial(P, 1/2)
    stat = float((((pos - P / 2) ** 2) / (P / 4)).sum())
    from scipy.stats import chi2
    assert chi2.sf(stat, 2048 - 1) > 1e-4


def test_mirror_sampler_keeps_cupolys_meanings(gpu):
    """Sampler.sample(ctx, UNIFORM) and (ctx, ZO) through the cuPoly mirror give cuPoly's
    BFV distributions; UNIFORM_MOD_Q and ZO_IID give the library's independent forms."""
    from cupoly_b200 import cupoly as cp
    nphi = 2048
    cp.CUDAEngine.init(2, 3, nphi, 256)
    ctx = cp.Context()
    cp.Sampler.init(ctx)
    a = cp.Sampler.sample(ctx, cp.UNIFORM)
    assert all(0 <= cp.poly_get_coeff(ctx, a, i) < (1 << 32) for i in range(nphi))
    a = cp.Sampler.sample(ctx, cp.UNIFORM_MOD_Q)
    assert max(cp.poly_get_coeff(ctx, a, i) for i in range(nphi)) >= (1 << 64)
    q = cp.CUDAEngine.RNSProduct
    a = cp.Sampler.sample(ctx, cp.ZO)
    vals = [cp.poly_get_coeff(ctx, a, i) for i in range(nphi)]
    assert all(v in (0, 1, q - 1) for v in vals) and sum(1 for v in vals if v) == nphi // 2
    a = cp.Sampler.sample(ctx, cp.ZO_IID)
    vals = [cp.poly_get_coeff(ctx, a, i) for i in range(nphi)]
    assert all(v in (0, 1, q - 1) for v in vals) and sum(1 for v in vals if v) != nphi // 2
    cp.CUDAEngine.destroy()
