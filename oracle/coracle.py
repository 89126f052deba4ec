"""ctypes wrapper of the C oracle ``oracle/libcpoly_oracle.so`` -- TEST INFRASTRUCTURE ONLY.

Used by tests/ as the fast full-size checker and by bench.py as the timed CPU
baseline.  Build with ``make -C oracle`` (``build()`` below does it).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import pyoracle

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libcpoly_oracle.so")
_L = None

_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def build():
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["make", "-s", "-C", _HERE], check=True, env=env)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        L.oc_num_threads.restype = C.c_int
        L.oc_set_threads.argtypes = [C.c_int]
        L.oc_dgt.argtypes = [_u64p, C.c_int, C.c_int, C.c_int, _u64p, _u64p, _u64p, C.c_int]
        L.oc_basis_ext.argtypes = [_u64p, _u64p, C.c_long, _u64p, C.c_int, _u64p, C.c_int, _u64p]
        L.oc_complex_scaling.argtypes = [_u64p, _u64p, _u64p, C.c_long, _u64p, C.c_int, _u64p, C.c_int, C.c_uint64]
        L.oc_simple_scaling.argtypes = [_u64p, _u64p, C.c_long, _u64p, C.c_int, C.c_uint64]
        L.oc_polymul.argtypes = [_u64p, _u64p, _u64p, C.c_int, C.c_int, C.c_int, _u64p, _u64p, _u64p]
        L.oc_bfv_mul.argtypes = [_u64p] * 7 + [C.c_int] * 4 + [_u64p, _u64p, _u64p, C.c_uint64, _u64p, _u64p]
        _L = L
    return _L


def _arr(x):
    return np.ascontiguousarray(x, dtype=np.uint64)


def _gens(primes):
    return _arr([pyoracle.PROOT[p] for p in primes])


def _xis(primes, N, xi=None):
    if xi is None:
        xi = [pyoracle.canonical_xi(p, N) for p in primes]
    return _arr([v for pair in xi for v in pair])


def dgt(data: np.ndarray, primes, inverse=False, xi=None) -> np.ndarray:
    """data: (npolys, nres, N, 2) uint64 -> transformed copy (cuPoly's DGT domain)."""
    x = _arr(data).copy()
    npolys, nres, N, _ = x.shape
    lib().oc_dgt(x, npolys, nres, N, _arr(primes), _gens(primes), _xis(primes, N, xi), 1 if inverse else 0)
    return x


def polymul(a: np.ndarray, b: np.ndarray, primes) -> np.ndarray:
    """a, b: (npolys, nres, nphi) coefficient rows -> negacyclic products."""
    a, b = _arr(a), _arr(b)
    npolys, nres, nphi = a.shape
    c = np.empty_like(a)
    lib().oc_polymul(c, a, b, npolys, nres, nphi, _arr(primes), _gens(primes), _xis(primes, nphi // 2))
    return c


def basis_ext(x: np.ndarray, src, dst) -> np.ndarray:
    """x: (nsrc, count) residue rows -> (ndst, count): X mod d with cuPoly's lift
    (pyoracle.basis_extension_exact), decided exactly."""
    x = _arr(x)
    out = np.empty((len(dst), x.shape[1]), dtype=np.uint64)
    lib().oc_basis_ext(out, x, x.shape[1], _arr(src), len(src), _arr(dst), len(dst), _arr(pyoracle.lift_digits(src)))
    return out


def complex_scaling(xq: np.ndarray, yb: np.ndarray, Q, B, t) -> np.ndarray:
    xq, yb = _arr(xq), _arr(yb)
    out = np.empty_like(yb)
    lib().oc_complex_scaling(out, xq, yb, xq.shape[1], _arr(Q), len(Q), _arr(B), len(B), t)
    return out


def simple_scaling(xq: np.ndarray, Q, t) -> np.ndarray:
    xq = _arr(xq)
    out = np.empty(xq.shape[1], dtype=np.uint64)
    lib().oc_simple_scaling(out, xq, xq.shape[1], _arr(Q), len(Q), t)
    return out


def bfv_mul(a0, a1, b0, b1, Q, B, t):
    """Inputs (npairs, k, nphi) coefficient rows mod Q; outputs c0, c1, c2 likewise."""
    a0, a1, b0, b1 = (_arr(v) for v in (a0, a1, b0, b1))
    npairs, k, nphi = a0.shape
    primes = list(Q) + list(B)
    c0, c1, c2 = (np.empty_like(a0) for _ in range(3))
    lib().oc_bfv_mul(c0, c1, c2, a0, a1, b0, b1, npairs, k, len(B), nphi, _arr(primes), _gens(primes),
                     _xis(primes, nphi // 2), t, _arr(pyoracle.lift_digits(Q)), _arr(pyoracle.lift_digits(B)))
    return c0, c1, c2


def set_threads(n: int):
    lib().oc_set_threads(int(n))


def num_threads() -> int:
    return lib().oc_num_threads()
