"""Sampler on the GPU: bit-exact against the oracle's Philox restatement,
cuPoly's TestSampler support checks, and statistics over 2^24 samples."""
import math

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.common import unfold

pytestmark = pytest.mark.gpu
KINDS = [O.DISCRETE_GAUSSIAN, O.HAMMINGWEIGHT, O.NARROW, O.ZO, O.BINARY, O.UNIFORM, O.TERNARY, O.GAUSSIAN]


def _sample(e, kind, nphi, sid, seed, npolys=1, base=0):
    from cupoly_b200.engine import to_u64
    out = e.empty(base, npolys)
    e.sample(out, base, kind, seed, sid, npolys=npolys, to_dgt=False)
    e.check()
    return unfold(to_u64(out))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("nphi", [32, 256])
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
