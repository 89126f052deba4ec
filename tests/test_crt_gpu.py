"""Device CRT / ICRT (cuPoly poly_crt / poly_icrt, src/arithmetic/polynomial.cu:190-296)
and the binary residue wire format, bit-exact against Python big integers."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests.common import fold, random_poly_int, random_poly_residues, splitmix64, unfold

pytestmark = pytest.mark.gpu


def _limbs_random(seed, nphi, nlimbs):
    w = splitmix64(seed, 17, nphi * nlimbs).reshape(nphi, nlimbs)
    w[0] = 0                                    # zero
    w[1] = np.uint64(0xFFFFFFFFFFFFFFFF)        # 2^(64 nlimbs) - 1
    return w


@pytest.mark.parametrize("k,nphi,nlimbs,base", [(2, 4096, 1, 0), (5, 8192, 3, 0), (5, 8192, 64, 1), (3, 64, 7, 2),
                                                 (16, 2048, 33, 2), (1, 4, 2, 0)])
def test_crt_matches_big_integers(gpu, k, nphi, nlimbs, base):
    from cupoly_b200.engine import Engine, from_u64, limbs_to_ints, to_u64
    e = Engine(k, 0, nphi, 256)
    limbs = _limbs_random(k * 31 + nlimbs, nphi, nlimbs)
    out = e.empty(base)
    e.crt(out, from_u64(limbs[None]), base)
    got = unfold(to_u64(out))[0]
    xs = limbs_to_ints(limbs)
    for r, p in enumerate(e.base_primes(base)):
        assert np.array_equal(got[r], np.array([x % p for x in xs], dtype=np.uint64)), (r, p)


@pytest.mark.parametrize("k,nphi,base", [(1, 32, 0), (2, 4096, 0), (5, 8192, 0), (6, 1024, 1), (24, 64, 0),
                                          (12, 256, 1)])
def test_icrt_matches_crt(gpu, k, nphi, base):
    from cupoly_b200.engine import Engine, from_u64, limbs_to_ints, to_u64
    e = Engine(k, min(k + 1, 24), nphi, 256)
    primes = e.base_primes(base)
    res = random_poly_residues(7 * k + base, primes, nphi)
    res[:, 0] = 0                                            # X = 0
    res[:, 1] = np.array([p - 1 for p in primes], dtype=np.uint64)  # X = -1 mod P = P - 1
    nl = len(primes) + 1
    import torch
    limbs = torch.empty((1, nphi, nl), dtype=torch.int64, device="cuda")
    e.icrt(limbs, from_u64(fold(res)[None]), base)
    got = limbs_to_ints(to_u64(limbs[0]))
    P = O.prod(primes)
    assert got[0] == 0 and got[1] == P - 1
    for j in range(nphi):
        assert got[j] == O.crt([int(res[r, j]) for r in range(len(primes))], primes), j


def test_icrt_tbase_and_round_trip(gpu):
    import torch

    from cupoly_b200.engine import Engine, TBase, from_u64, ints_to_limbs, limbs_to_ints, to_u64
    nphi, k = 2048, 5
    e = Engine(k, 0, nphi, 65537)
    Q = O.prod(e.Q)
    xs = random_poly_int(3, Q, nphi)
    xs[0], xs[1] = 0, Q - 1
    out = e.empty(0)
    e.crt(out, from_u64(ints_to_limbs(xs, k)[None]), 0)
    limbs = torch.empty((1, nphi, k), dtype=torch.int64, device="cuda")
    e.icrt(limbs, out, 0)
    assert limbs_to_ints(to_u64(limbs[0])) == xs
    t_res = np.array([[x % 65537 for x in xs]], dtype=np.uint64)
    lt = torch.empty((1, nphi, 1), dtype=torch.int64, device="cuda")
    e.icrt(lt, from_u64(fold(t_res)[None]), TBase)
    assert limbs_to_ints(to_u64(lt[0])) == t_res[0].tolist()


def test_crt_icrt_reject_bad_arguments(gpu):
    import ctypes as C

    import torch

    from cupoly_b200 import _lib
    from cupoly_b200.engine import Engine, _ptr
    e = Engine(3, 0, 64, 256)
    L = _lib.lib()
    x = e.empty(0)
    limbs = torch.zeros((1, 64, 2), dtype=torch.int64, device="cuda")
    assert L.cp_crt(e.handle, _ptr(x), _ptr(limbs), 0, 0, 1, None) == 1          # nlimbs 0
    assert L.cp_crt(e.handle, _ptr(x), _ptr(limbs), 65, 0, 1, None) == 1         # nlimbs > 64
    assert L.cp_crt(e.handle, _ptr(x), _ptr(limbs), 2, 3, 1, None) == 1          # T base
    assert L.cp_icrt(e.handle, _ptr(limbs), 2, _ptr(x), 0, 1, None) == 1         # nlimbs < |Q|
    assert L.cp_icrt(e.handle, _ptr(limbs), 3, _ptr(x), 2, 1, None) == 1         # QB base
    assert b"nlimbs" in L.cp_last_error() or b"base" in L.cp_last_error()


def test_wire_round_trip_and_validation(gpu):
    import ctypes as C

    from cupoly_b200 import _lib
    from cupoly_b200.engine import Engine, QBase, from_u64, to_u64
    e = Engine(4, 0, 1024, 256)
    rows = [random_poly_residues(40 + i, e.Q, 1024) for i in range(3)]
    x = from_u64(np.stack([fold(r) for r in rows]))
    data = e.export_residues(x, QBase, 1)
    assert len(data) == e.wire_bytes(QBase, 3) == 64 + 4 * 8 + 3 * 4 * 512 * 16
    y = e.empty(QBase, 3)
    assert e.import_residues(y, data, QBase) == 1
    assert np.array_equal(to_u64(y), to_u64(x))
    L = _lib.lib()

    def rejected(blob, npolys=3, base=QBase):
        dom = C.c_int()
        rc = L.cp_import_residues(e.handle, C.c_void_p(y.data_ptr()), blob, len(blob), base, npolys, C.byref(dom), None)
        return rc == 1

    bad = bytearray(data)
    bad[0] ^= 1
    assert rejected(bytes(bad))                      # magic
    bad = bytearray(data)
    bad[9] ^= 1                                      # nphi 1024 -> 768
    assert rejected(bytes(bad))                      # ring degree
    bad = bytearray(data)
    bad[64] ^= 2
    assert rejected(bytes(bad))                      # primes
    assert rejected(data[:-16])                      # size
    assert rejected(data, npolys=2)                  # count
    bad = bytearray(data)
    body = 64 + 4 * 8
    bad[body:body + 8] = (e.Q[0]).to_bytes(8, "little")
    assert rejected(bytes(bad))                      # residue not reduced
    assert b"reduced" in L.cp_last_error()
    assert np.array_equal(to_u64(y), to_u64(x))      # nothing copied by the refused calls


def test_host_mirror_exports_and_device_crt(gpu):
    from cupoly_b200 import cupoly as cp
    cp.CUDAEngine.init(3, 4, 256, 256)
    ctx = cp.Context()
    Q = cp.CUDAEngine.RNSProduct
    a = cp.poly_t()
    vals = random_poly_int(11, Q, 256)
    for i, v in enumerate(vals):
        cp.poly_set_coeff(ctx, a, i, v)
    cp.poly_set_coeff(ctx, a, 7, -5)                 # negative: Q - 5
    b = cp.poly_t()
    cp.poly_mul(ctx, b, a, a)                        # forces device CRT, DGT, inverse, device ICRT
    ref = O.negacyclic_mul_schoolbook([x % Q for x in [*vals[:7], Q - 5, *vals[8:]]],
                                      [x % Q for x in [*vals[:7], Q - 5, *vals[8:]]], Q)
    assert [cp.poly_get_coeff(ctx, b, i) for i in range(256)] == ref
    s = cp.poly_export_residues(ctx, b)
    c = cp.poly_import_residues(ctx, s, cp.QBase)
    assert cp.poly_are_equal(ctx, b, c)
    d = cp.poly_import(ctx, cp.poly_export(ctx, b))
    assert [cp.poly_get_coeff(ctx, d, i) for i in range(256)] == ref
    f = cp.poly_import_binary(ctx, cp.poly_export_binary(ctx, b))
    assert [cp.poly_get_coeff(ctx, f, i) for i in range(256)] == ref
    cp.CUDAEngine.destroy()


def test_wire_import_checks_large_payloads_on_host_threads(gpu):
    """Payloads over 4 MB are checked on several host threads: a residue at or above its
    prime anywhere (first, middle or last row) is still refused before any copy."""
    import torch

    from cupoly_b200.engine import Engine, QBase, UNIFORM
    e = Engine(5, 0, 8192, 256)
    P = 16
    x = e.empty(QBase, P)
    e.sample(x, QBase, UNIFORM, 3, 0, npolys=P, to_dgt=False)
    data = e.export_residues(x, QBase, 0)
    assert len(data) > 4 << 20
    y = e.empty(QBase, P)
    assert e.import_residues(y, data, QBase) == 0 and torch.equal(x, y)
    body = 64 + 5 * 8
    row = 2 * e.N * 8
    nrows = P * 5
    y.zero_()
    for r in (0, nrows // 2, nrows - 1):
        bad = bytearray(data)
        off = body + r * row + row - 8  # last word of row r
        bad[off:off + 8] = e.Q[r % 5].to_bytes(8, "little")
        with pytest.raises(Exception, match="reduced"):
            e.import_residues(y, bytes(bad), QBase)
    assert int(y.abs().sum()) == 0  # nothing copied by the refused calls
