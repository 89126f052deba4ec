"""cuPoly's polynomial API, re-created over the C ABI.

Mirrors the names, argument meaning and state machine of cuPoly 0.3.5
(include/cuPoly/arithmetic/polynomial.h, cudaengine.h, dgt.h, sampler.h,
context.h) so that code written against cuPoly reads the same:

    CUDAEngine.init(k, k + 1, nphi, t)
    ctx = Context()
    Sampler.init(ctx)
    a, b, c = poly_t(), poly_t(), poly_t()
    Sampler.sample(ctx, a, UNIFORM); Sampler.sample(ctx, b, UNIFORM)
    poly_mul(ctx, c, a, b)
    poly_get_coeff(ctx, c, 0)

Coefficients on the host are Python integers (cuPoly: NTL ZZ).  A poly_t
keeps cuPoly's lazy host/device state machine (polynomial.h:39-66): device
data is in the DGT domain while the status is RNSSTATE or BOTHSTATE.
Errors raise (cuPoly: assert / std::runtime_error / exit(1)).
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np
import torch

from .engine import (ADD, ADDADD, BBase, BINARY, DESTROY_INPUTS, DISCRETE_GAUSSIAN, FORWARD, GAUSSIAN,
                     HAMMINGWEIGHT, INVERSE, MUL, MULMUL, NARROW, QBBase, QBase, SUB, TBase, TERNARY, UNIFORM, ZO,
                     UNIFORM_U32, ZO_HALF, Engine, from_u64, ints_to_limbs, limbs_to_ints, to_u64)

HOSTSTATE, RNSSTATE, BOTHSTATE = 0, 1, 2
# Sampler kinds of this layer beyond cuPoly's: the library's independent forms of
# UNIFORM (uniform mod each q_i) and ZO (i.i.d. -1/0/+1 with 1/4, 1/2, 1/4).
UNIFORM_MOD_Q, ZO_IID = 105, 103
HAMMINGWEIGHT_H = 64
GAUSSIAN_STD_DEVIATION = 3.2
SEED = 42

__all__ = [
    "CUDAEngine", "DGTEngine", "Context", "Sampler", "poly_t", "QBase", "BBase", "QBBase", "TBase", "FORWARD",
    "INVERSE", "ADD", "SUB", "MUL", "MULMUL", "ADDADD", "DISCRETE_GAUSSIAN", "HAMMINGWEIGHT", "NARROW", "ZO",
    "BINARY", "UNIFORM", "TERNARY", "GAUSSIAN", "HOSTSTATE", "RNSSTATE", "BOTHSTATE", "UNIFORM_MOD_Q", "ZO_IID",
]


def _prod(xs):
    r = 1
    for x in xs:
        r *= x
    return r


class CUDAEngine:
    """Process-wide default engine (cuPoly include/cuPoly/cuda/cudaengine.h:59-123)."""

    engine: Optional[Engine] = None
    is_init = False
    N = 0
    t = 0
    RNSPrimes: List[int] = []
    RNSBPrimes: List[int] = []
    RNSProduct = 1
    RNSBProduct = 1
    RNSMpi: List[int] = []
    RNSInvMpi: List[int] = []

    @classmethod
    def init(cls, k: int, kl: int, M: int, t: int, log_radix: int = 0):
        """init(k, kl, M, t): M is the ring degree nphi (cuPoly cudaengine.cu:1691-1731)."""
        if cls.is_init:
            cls.destroy()
        cls.engine = Engine(k, kl if kl > 0 else k + 1, M, t, log_radix)
        cls.N = M >> 1
        cls.t = t
        cls.RNSPrimes = list(cls.engine.Q)
        cls.RNSBPrimes = list(cls.engine.B)
        cls.RNSProduct = _prod(cls.RNSPrimes)
        cls.RNSBProduct = _prod(cls.RNSBPrimes)
        cls.RNSMpi = [cls.RNSProduct // p for p in cls.RNSPrimes]
        cls.RNSInvMpi = [pow(m % p, -1, p) for m, p in zip(cls.RNSMpi, cls.RNSPrimes)]
        cls.is_init = True

    @classmethod
    def init_ckks(cls, k: int, kl: int, M: int, prec: int, log_radix: int = 0):
        """CKKS build's init(k, kl, M, prec): Q = the first 63-bit prime and k - 1
        primes of the prec-bit bucket, B = kl primes (cudaengine.cu:1192-1290)."""
        if cls.is_init:
            cls.destroy()
        cls.engine = Engine.ckks(k, kl if kl > 0 else k + 1, M, prec, log_radix)
        cls.N = M >> 1
        cls.t = prec
        cls.RNSPrimes = list(cls.engine.Q)
        cls.RNSBPrimes = list(cls.engine.B)
        cls.RNSProduct = _prod(cls.RNSPrimes)
        cls.RNSBProduct = _prod(cls.RNSBPrimes)
        cls.RNSMpi = [cls.RNSProduct // p for p in cls.RNSPrimes]
        cls.RNSInvMpi = [pow(m % p, -1, p) for m, p in zip(cls.RNSMpi, cls.RNSPrimes)]
        cls.is_init = True

    @classmethod
    def destroy(cls):
        if cls.engine is not None:
            torch.cuda.synchronize()
            cls.engine.close()
        cls.engine = None
        cls.is_init = False

    @classmethod
    def get_n_residues(cls, base: int) -> int:
        assert cls.is_init
        return cls.engine.n_residues(base)


def _E() -> Engine:
    if not CUDAEngine.is_init:
        raise RuntimeError("CUDAEngine is not initialised")
    return CUDAEngine.engine


class Context:
    """One stream plus scratch (cuPoly include/cuPoly/arithmetic/context.h:34-109).

    By default the context runs on torch's current stream, so tensors handed
    between poly_* calls and ordinary torch code stay ordered; pass
    ``own_stream=True`` for a private stream (then synchronise before touching
    ``d_coefs`` from another stream, as with cuPoly's per-context streams).
    """

    def __init__(self, own_stream: bool = False):
        e = _E()
        self.stream = torch.cuda.Stream() if own_stream else torch.cuda.current_stream()
        with torch.cuda.stream(self.stream):
            self.workspace = e.workspace()
            self.d_aux_coefs = e.empty(QBBase)

    def get_stream(self):
        return self.stream


class poly_t:
    """cuPoly's polynomial struct (polynomial.h:55-66)."""

    def __init__(self):
        self.init = False
        self.coefs: List[int] = []
        self.d_coefs: Optional[torch.Tensor] = None
        self.status = BOTHSTATE
        self.base = QBase


class DGTEngine:
    """cuPoly include/cuPoly/cuda/dgt.h:106-283 (static members)."""

    @staticmethod
    def execute_dgt(data: torch.Tensor, base: int, direction: int, ctx: Context):
        _E().dgt(data, base, direction, npolys=1, stream=ctx.stream)

    @staticmethod
    def execute_add_dgt(c, a, b, base, stream):
        _E().add(c, a, b, base, stream)

    @staticmethod
    def execute_sub_dgt(c, a, b, base, stream):
        _E().sub(c, a, b, base, stream)

    @staticmethod
    def execute_double_add_dgt(c1, a1, b1, c2, a2, b2, base, stream):
        _E().double_add(c1, a1, b1, c2, a2, b2, base, stream)

    @staticmethod
    def execute_dr2_dgt(c21, c22, c23, c01, c02, c11, c12, base, stream):
        _E().dr2(c21, c22, c23, c01, c02, c11, c12, base, stream)

    @staticmethod
    def execute_mul_dgt_gi(c, a, b, base, stream):
        _E().mul(c, a, b, base, stream)

    @staticmethod
    def execute_mul_dgt_u64(c, a, b, base, stream):
        _E().mul_u64(c, a, b, base, stream)

    @staticmethod
    def execute_muladd_dgt(d, a, b, c, base, stream):
        _E().muladd(d, a, b, c, base, stream)


# ---------------------------------------------------------------------------
# state machine (polynomial.cu:45-188)
# ---------------------------------------------------------------------------
def poly_get_residues_size(base: int) -> int:
    return CUDAEngine.N * CUDAEngine.get_n_residues(base) * 16


def poly_init(ctx: Context, a: poly_t, base: int = QBase):
    if a.init:
        return
    e = _E()
    a.base = base
    with torch.cuda.stream(ctx.stream):
        a.d_coefs = e.zeros(base)
    a.coefs = [0] * (2 * CUDAEngine.N)
    a.status = BOTHSTATE
    a.init = True


def poly_free(ctx: Context, a: poly_t):
    if a is None or not a.init:
        return
    ctx.stream.synchronize()
    a.coefs = []
    a.d_coefs = None
    a.init = False


def poly_clear(ctx: Context, a: poly_t):
    poly_init(ctx, a)
    a.coefs = []
    with torch.cuda.stream(ctx.stream):
        a.d_coefs.zero_()
    a.status = BOTHSTATE


def _limbs_of(coefs: List[int], modulus: int, nphi: int):
    """Coefficients (padded to nphi, negatives taken mod `modulus`) as uint64 limbs."""
    c = [x % modulus if x < 0 else x for x in coefs[:nphi]] + [0] * max(0, nphi - len(coefs))
    top = max(c) if c else 0
    nlimbs = max(1, (top.bit_length() + 63) // 64)
    if nlimbs > 64:  # beyond the device limb limit: reduce first (same residues)
        c = [x % modulus for x in c]
        nlimbs = max(1, (max(c).bit_length() + 63) // 64)
    return ints_to_limbs(c, nlimbs)


def poly_crt(ctx: Context, a: poly_t) -> torch.Tensor:
    """Coefficient-domain residues of the host coefficients, computed on the device
    (cuPoly reduces every ZZ coefficient on the host, polynomial.cu:190-221)."""
    assert a.base in (QBase, QBBase)
    e = _E()
    limbs = _limbs_of(a.coefs, _prod(e.base_primes(a.base)), 2 * CUDAEngine.N)
    with torch.cuda.stream(ctx.stream):
        d = from_u64(limbs[None])
        out = e.empty(a.base)
    e.crt(out, d, a.base, stream=ctx.stream)
    return out


def poly_icrt(ctx: Context, a: poly_t, x: torch.Tensor):
    """Coefficients in [0, Q) from coefficient-domain residues, recombined on the
    device (cuPoly: host NTL CRT, polynomial.cu:223-296); base Q or T."""
    if a.base not in (QBase, TBase):
        raise RuntimeError("Unknown base")
    e = _E()
    nl = e.n_residues(a.base)
    with torch.cuda.stream(ctx.stream):
        limbs = torch.empty((1, 2 * CUDAEngine.N, nl), dtype=torch.int64, device="cuda")
    e.icrt(limbs, x, a.base, stream=ctx.stream)
    ctx.stream.synchronize()
    a.coefs = limbs_to_ints(to_u64(limbs[0]))


def poly_copy_to_device(ctx: Context, a: poly_t):
    if a.status in (RNSSTATE, BOTHSTATE):
        return
    e = _E()
    a.d_coefs = poly_crt(ctx, a)
    e.dgt(a.d_coefs, a.base, FORWARD, stream=ctx.stream)
    ctx.stream.synchronize()
    a.status = BOTHSTATE


def poly_copy_to_host(ctx: Context, a: poly_t):
    if a.status in (HOSTSTATE, BOTHSTATE):
        return
    e = _E()
    with torch.cuda.stream(ctx.stream):
        aux = a.d_coefs.clone()
    e.dgt(aux, a.base, INVERSE, stream=ctx.stream)
    poly_icrt(ctx, a, aux)
    a.status = BOTHSTATE


def poly_copy(ctx: Context, b: poly_t, a: poly_t):
    poly_init(ctx, b, a.base)
    if a.status in (RNSSTATE, BOTHSTATE):
        with torch.cuda.stream(ctx.stream):
            b.d_coefs = a.d_coefs.clone()
        b.base = a.base
        b.status = RNSSTATE
    else:
        b.coefs = list(a.coefs)
        b.status = HOSTSTATE


def poly_set_coeff(ctx: Context, a: poly_t, index: int, c: int):
    if not a.init:
        poly_init(ctx, a)
    poly_copy_to_host(ctx, a)
    if c < 0:
        c = CUDAEngine.RNSProduct + c
    if index >= len(a.coefs):
        a.coefs.extend([0] * (index + 1 - len(a.coefs)))
    a.coefs[index] = c
    a.status = HOSTSTATE


def poly_get_coeff(ctx: Context, a: poly_t, index: int) -> int:
    assert a.init
    poly_copy_to_host(ctx, a)
    return a.coefs[index] if index < len(a.coefs) else 0


def poly_get_deg(ctx: Context, a: poly_t) -> int:
    if a.status == RNSSTATE:
        poly_copy_to_host(ctx, a)
    c = a.coefs
    d = len(c) - 1
    while d >= 0 and c[d] == 0:
        d -= 1
    return d


def poly_are_equal(ctx: Context, a: poly_t, b: poly_t) -> bool:
    if poly_get_deg(ctx, a) != poly_get_deg(ctx, b):
        return False
    Q = CUDAEngine.RNSProduct
    return all(poly_get_coeff(ctx, a, i) % Q == poly_get_coeff(ctx, b, i) % Q
               for i in range(poly_get_deg(ctx, a) + 1))


def poly_to_string(ctx: Context, a: poly_t) -> str:
    return "".join("%d, " % poly_get_coeff(ctx, a, i) for i in range(poly_get_deg(ctx, a) + 1))


def poly_export_residues(ctx: Context, a: poly_t) -> str:
    """Coefficient-domain residues as text: for each residue, its nphi values in
    coefficient order, space separated (cuPoly polynomial.cu:1291-1339)."""
    e = _E()
    poly_copy_to_device(ctx, a)
    with torch.cuda.stream(ctx.stream):
        aux = a.d_coefs.clone()
    e.dgt(aux, a.base, INVERSE, stream=ctx.stream)
    ctx.stream.synchronize()
    h = e.unfold(to_u64(aux[0]))
    return " ".join(str(int(v)) for v in h.reshape(-1).astype(np.int64))


def poly_import_residues(ctx: Context, s: str, base: int = QBase) -> poly_t:
    """Inverse of poly_export_residues; returns a new poly_t in RNSSTATE
    (cuPoly polynomial.cu:1341-1383)."""
    e = _E()
    vals = np.array([int(v) for v in s.split()], dtype=np.int64).view(np.uint64)
    nres, nphi = e.n_residues(base), 2 * CUDAEngine.N
    h = np.zeros((nres, nphi), dtype=np.uint64)
    h.reshape(-1)[: vals.size] = vals[: nres * nphi]
    a = poly_t()
    poly_init(ctx, a, base)
    with torch.cuda.stream(ctx.stream):
        a.d_coefs = from_u64(e.fold(h)[None])
    e.dgt(a.d_coefs, base, FORWARD, stream=ctx.stream)
    ctx.stream.synchronize()
    a.status = RNSSTATE
    return a


def poly_export(ctx: Context, p: poly_t) -> str:
    """Coefficients 0..deg as comma-separated integers (cuPoly polynomial.cu:1386-1404)."""
    return ",".join(str(poly_get_coeff(ctx, p, i)) for i in range(poly_get_deg(ctx, p) + 1))


def poly_import(ctx: Context, s: str) -> poly_t:
    """Inverse of poly_export (cuPoly polynomial.cu:1406-1425)."""
    p = poly_t()
    poly_init(ctx, p)
    if s.strip():
        for i, v in enumerate(s.split(",")):
            poly_set_coeff(ctx, p, i, int(v.replace(" ", "")))
    return p


def poly_export_binary(ctx: Context, a: poly_t) -> bytes:
    """Binary wire form (cp_export_residues) of the device data, DGT domain."""
    poly_copy_to_device(ctx, a)
    return _E().export_residues(a.d_coefs, a.base, 1, stream=ctx.stream)


def poly_import_binary(ctx: Context, data: bytes, base: int = QBase) -> poly_t:
    """Inverse of poly_export_binary; coefficient-domain payloads are transformed."""
    e = _E()
    a = poly_t()
    poly_init(ctx, a, base)
    dom = e.import_residues(a.d_coefs, data, base, stream=ctx.stream)
    if dom == 0:
        e.dgt(a.d_coefs, base, FORWARD, stream=ctx.stream)
    ctx.stream.synchronize()
    a.status = RNSSTATE
    return a


# ---------------------------------------------------------------------------
# arithmetic (polynomial.cu:802-1153)
# ---------------------------------------------------------------------------
def _prep(ctx, out: poly_t, base: int, *ins: poly_t):
    for x in ins:
        assert x.init
        poly_copy_to_device(ctx, x)
    poly_init(ctx, out, base)
    if out.d_coefs is None or out.d_coefs.shape[1] != CUDAEngine.get_n_residues(base):
        with torch.cuda.stream(ctx.stream):
            out.d_coefs = _E().zeros(base)


def _done(out: poly_t, base: int):
    out.status = RNSSTATE
    out.base = base


def poly_add(ctx, c, a, b):
    assert a.base == b.base
    _prep(ctx, c, a.base, a, b)
    _E().add(c.d_coefs, a.d_coefs, b.d_coefs, a.base, ctx.stream)
    _done(c, a.base)


def poly_sub(ctx, c, a, b):
    assert a.base == b.base
    _prep(ctx, c, a.base, a, b)
    _E().sub(c.d_coefs, a.d_coefs, b.d_coefs, a.base, ctx.stream)
    _done(c, a.base)


def poly_double_add(ctx, c1, a1, b1, c2, a2, b2):
    assert a1.base == b1.base == a2.base == b2.base
    _prep(ctx, c1, a1.base, a1, b1, a2, b2)
    _prep(ctx, c2, a1.base)
    _E().double_add(c1.d_coefs, a1.d_coefs, b1.d_coefs, c2.d_coefs, a2.d_coefs, b2.d_coefs, a1.base, ctx.stream)
    _done(c1, a1.base)
    _done(c2, a1.base)


def poly_mul(ctx, c, a, b):
    assert a.base == b.base
    _prep(ctx, c, a.base, a, b)
    _E().mul(c.d_coefs, a.d_coefs, b.d_coefs, a.base, ctx.stream)
    _done(c, a.base)


def poly_mul_add(ctx, d, a, b, c):
    assert a.base == b.base == c.base
    _prep(ctx, d, a.base, a, b, c)
    _E().muladd(d.d_coefs, a.d_coefs, b.d_coefs, c.d_coefs, a.base, ctx.stream)
    _done(d, a.base)


def poly_dot(ctx, c, a, b, k):
    """c = sum_{i<k} a[i] b[i] (cuPoly src/arithmetic/polynomial.cu:1439-1451), one fused pass.

    cuPoly composes one poly_mul and k - 1 poly_mul_add calls, so when c is also an
    operand of a later term those calls read the partial sum; that case keeps the
    composition and gives the same bytes.
    """
    if k < 1:
        raise ValueError("poly_dot: k must be at least 1")
    if any(a[i] is c or b[i] is c for i in range(1, k)):
        poly_mul(ctx, c, a[0], b[0])
        for i in range(1, k):
            poly_mul_add(ctx, c, a[i], b[i], c)
        return
    base = a[0].base
    ops = list(a[:k]) + list(b[:k])
    assert all(x.base == base for x in ops)
    _prep(ctx, c, base, *ops)
    _E().dot(c.d_coefs, [x.d_coefs for x in a[:k]], [x.d_coefs for x in b[:k]], base, ctx.stream)
    _done(c, base)


def poly_dr2(ctx, ct21, ct22, ct23, ct01, ct02, ct11, ct12):
    assert ct01.base == ct02.base == ct11.base == ct12.base
    base = ct01.base
    _prep(ctx, ct21, base, ct01, ct02, ct11, ct12)
    _prep(ctx, ct22, base)
    _prep(ctx, ct23, base)
    _E().dr2(ct21.d_coefs, ct22.d_coefs, ct23.d_coefs, ct01.d_coefs, ct02.d_coefs, ct11.d_coefs, ct12.d_coefs,
             base, ctx.stream)
    for x in (ct21, ct22, ct23):
        _done(x, base)


def _op_int(ctx, b, a, x, op):
    _prep(ctx, b, a.base, a)
    _E().op_by_int(b.d_coefs, a.d_coefs, a.base, x, op, ctx.stream)
    _done(b, a.base)


def poly_mul_int(ctx, b, a, x):
    _op_int(ctx, b, a, x, MUL)


def poly_add_int(ctx, b, a, x):
    _op_int(ctx, b, a, x, ADD)


def poly_sub_int(ctx, b, a, x):
    _op_int(ctx, b, a, x, SUB)


def poly_double_mul_int(ctx, b1, a1, b2, a2, x1, x2):
    _prep(ctx, b1, a1.base, a1, a2)
    _prep(ctx, b2, a1.base)
    _E().double_op_by_int(b1.d_coefs, a1.d_coefs, b2.d_coefs, a2.d_coefs, a1.base, x1, x2, MULMUL, ctx.stream)
    _done(b1, a1.base)
    _done(b2, a1.base)


def poly_double_add_int(ctx, b1, a1, b2, a2, x1, x2):
    _prep(ctx, b1, a1.base, a1, a2)
    _prep(ctx, b2, a1.base)
    _E().double_op_by_int(b1.d_coefs, a1.d_coefs, b2.d_coefs, a2.d_coefs, a1.base, x1, x2, ADDADD, ctx.stream)
    _done(b1, a1.base)
    _done(b2, a1.base)


def poly_negate(ctx, a):
    poly_copy_to_device(ctx, a)
    _E().negate(a.d_coefs, a.d_coefs, a.base, ctx.stream)
    a.status = RNSSTATE


# ---------------------------------------------------------------------------
# HPS (polynomial.cu:310-527)
# ---------------------------------------------------------------------------
def poly_simple_scaling_tDivQ(ctx, b, a):
    assert a.base == QBase
    poly_copy_to_device(ctx, a)
    poly_init(ctx, b)
    with torch.cuda.stream(ctx.stream):
        b.d_coefs = _E().zeros(TBase)
    _E().poly_simple_scaling_tdivq(b.d_coefs, a.d_coefs, ctx.stream)
    b.status = RNSSTATE
    b.base = TBase


def poly_complex_scaling_tDivQ(ctx, b_Q, a_Q, a_B):
    """Destroys a_Q and a_B like cuPoly (polynomial.h:346-347)."""
    assert a_Q.base == QBase and a_B.base == BBase
    poly_copy_to_device(ctx, a_Q)
    poly_copy_to_device(ctx, a_B)
    _prep(ctx, b_Q, QBase)
    _E().poly_complex_scaling_tdivq(b_Q.d_coefs, a_Q.d_coefs, a_B.d_coefs, DESTROY_INPUTS, ctx.stream)
    # cuPoly leaves the inputs inverse-transformed but still flagged RNSSTATE
    _done(b_Q, QBase)


def poly_basis_extension_Q_to_B(ctx, a_B, a_Q):
    assert a_Q.base == QBase
    poly_copy_to_device(ctx, a_Q)
    _prep(ctx, a_B, BBase)
    _E().poly_basis_extension_q_to_b(a_B.d_coefs, a_Q.d_coefs, ctx.stream)
    _done(a_B, BBase)


def poly_basis_extension_Q_to_QB(ctx, b, a):
    assert a.base == QBase
    poly_copy_to_device(ctx, a)
    _prep(ctx, b, QBBase)
    _E().poly_basis_extension_q_to_qb(b.d_coefs, a.d_coefs, ctx.stream)
    _done(b, QBBase)


def poly_basis_extension_B_to_Q(ctx, a_Q, a_B):
    assert a_B.base == BBase
    poly_copy_to_device(ctx, a_B)
    _prep(ctx, a_Q, QBase)
    _E().poly_basis_extension_b_to_q(a_Q.d_coefs, a_B.d_coefs, ctx.stream)
    _done(a_Q, QBase)


def _xi_rho(ctx, c: List[poly_t], a: poly_t, rho: bool):
    e = _E()
    poly_copy_to_device(ctx, a)
    with torch.cuda.stream(ctx.stream):
        out = e.empty(QBase, e.k)
    (e.rho if rho else e.xi)(out, a.d_coefs, ctx.stream)
    for i in range(e.k):
        poly_init(ctx, c[i])
        c[i].d_coefs = out[i:i + 1]
        _done(c[i], QBase)


def poly_xi_bfv(ctx, c: List[poly_t], a: poly_t):
    """c[i] has residue i equal to a_i (Q/q_i)^-1 mod q_i (cuPoly polynomial.cu:612-650)."""
    _xi_rho(ctx, c, a, False)


def poly_rho_bfv(ctx, c: List[poly_t], a: poly_t):
    """c[i] has residue i equal to a_i (Q/q_i) mod q_i (cuPoly polynomial.cu:652-693)."""
    _xi_rho(ctx, c, a, True)


# ---------------------------------------------------------------------------
# CKKS mode (polynomial.cu:530-608, 696-800)
# ---------------------------------------------------------------------------
def poly_approx_basis_raising_Q_to_QB(ctx, a, b, level: int):
    """a (QB) <- b (Q) with the B residues of the approximate conversion from Q_level."""
    assert a.init and b.base == QBase
    poly_copy_to_device(ctx, b)
    e = _E()
    a.base = QBBase
    with torch.cuda.stream(ctx.stream):
        a.d_coefs = e.empty(QBBase)
    e.ckks_modulus_raising(a.d_coefs, b.d_coefs, level, stream=ctx.stream)
    a.status = RNSSTATE


def poly_approx_basis_reduction_QB_to_Q(ctx, a, b, level: int):
    """a (Q) residues 0..level <- approximate division of b (QB) by B."""
    assert a.init and a.base == QBase and b.base == QBBase
    poly_copy_to_device(ctx, a)
    poly_copy_to_device(ctx, b)
    _E().ckks_modulus_reduction(a.d_coefs, b.d_coefs, level, stream=ctx.stream)
    a.status = RNSSTATE


def poly_ckks_rescale(ctx, a, b, level: int):
    """Divide a and b by q_level (rounding toward the residue), in place."""
    assert a.init and a.base == QBase
    poly_copy_to_device(ctx, a)
    if b is not None:
        poly_copy_to_device(ctx, b)
    _E().ckks_rescale(a.d_coefs, b.d_coefs if b is not None else None, level, stream=ctx.stream)
    a.status = RNSSTATE
    if b is not None:
        b.status = RNSSTATE


def poly_xi_ckks(ctx, c, a):
    assert a.init and a.base == QBase
    poly_copy_to_device(ctx, a)
    poly_init(ctx, c)
    _E().ckks_xi(c.d_coefs, a.d_coefs, stream=ctx.stream)
    c.status = RNSSTATE


def poly_rho_ckks(ctx, c, a):
    assert a.init and a.base in (QBase, QBBase)
    poly_copy_to_device(ctx, a)
    poly_init(ctx, c)
    _E().ckks_rho(c.d_coefs, a.d_coefs, stream=ctx.stream)
    c.status = RNSSTATE


# ---------------------------------------------------------------------------
# Sampler (sampler.h:53-101)
# ---------------------------------------------------------------------------
class Sampler:
    seed = SEED
    _counter = 0

    @classmethod
    def init(cls, ctx: Context):
        cls._counter = 0

    @classmethod
    def reset(cls, ctx: Context):
        cls._counter = 0

    @classmethod
    def destroy(cls):
        pass

    @staticmethod
    def device_kind(e: Engine, kind: int) -> int:
        """cuPoly's names keep cuPoly's meanings (src/cuda/sampler.cu:236-341): on a BFV
        engine UNIFORM is one value below 2^32 written to every residue and ZO has
        exactly nphi/2 nonzero coefficients.  UNIFORM_MOD_Q and ZO_IID select the
        library's independent forms; cuPoly's CKKS UNIFORM is already per residue."""
        if kind == UNIFORM:
            return UNIFORM if e.ckks_prec else UNIFORM_U32
        if kind == ZO:
            return ZO_HALF
        return {UNIFORM_MOD_Q: UNIFORM, ZO_IID: ZO}.get(kind, kind)

    @classmethod
    def sample(cls, ctx: Context, p: Optional[poly_t] = None, kind: int = UNIFORM):
        """sample(ctx, p, kind) fills p; sample(ctx, kind) returns a new poly_t."""
        if isinstance(p, int):
            p, kind = None, p
        ret = p is None
        if p is None:
            p = poly_t()
        poly_init(ctx, p)
        e = _E()
        sid = cls._counter
        cls._counter += 1
        e.sample(p.d_coefs, p.base, cls.device_kind(e, kind), cls.seed, sid, npolys=1, to_dgt=True,
                 stream=ctx.stream)
        p.status = RNSSTATE
        return p if ret else None
