"""Shared seeded input generator and comparison helpers for the tests.

Residues are i.i.d. uniform in [0, p) from SplitMix64 keyed by
(seed, stream, index), rejection-sampled on 63 bits.  The same generator
feeds the oracle and the device so every case is reproducible from its seed.
"""
from __future__ import annotations

import hashlib

import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, stream: int, n: int) -> np.ndarray:
    """n 64-bit words of SplitMix64 at state seed ^ (stream * golden)."""
    with np.errstate(over="ignore"):
        base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) ^ (np.uint64(stream & 0xFFFFFFFFFFFFFFFF) * _G)
        z = base + _G * (np.arange(1, n + 1, dtype=np.uint64))
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform_mod(seed: int, stream: int, n: int, p: int) -> np.ndarray:
    """n values uniform in [0, p) (rejection on bit_length(p) bits: 63 for the BFV primes)."""
    out = np.empty(0, dtype=np.uint64)
    k = 0
    shift = np.uint64(64 - int(p).bit_length())
    while out.size < n:
        w = splitmix64(seed, stream * 1000003 + k, 2 * n) >> shift
        out = np.concatenate([out, w[w < np.uint64(p)]])
        k += 1
    return out[:n]


def random_poly_residues(seed: int, primes, nphi: int, stream: int = 0) -> np.ndarray:
    """(nres, nphi) uint64: independent uniform residues per prime."""
    return np.stack([uniform_mod(seed, stream * 4096 + r, nphi, p) for r, p in enumerate(primes)])


def random_poly_int(seed: int, Q: int, nphi: int, stream: int = 0):
    """nphi Python integers uniform-ish in [0, Q) (from 64-bit limbs)."""
    limbs = (Q.bit_length() + 63) // 64 + 1
    w = splitmix64(seed, 7919 + stream, nphi * limbs).reshape(nphi, limbs)
    out = []
    for row in w.tolist():
        x = 0
        for v in row:
            x = (x << 64) | v
        out.append(x % Q)
    return out


def fold(rows: np.ndarray) -> np.ndarray:
    """(..., nphi) -> (..., N, 2)."""
    N = rows.shape[-1] // 2
    return np.stack([rows[..., :N], rows[..., N:]], axis=-1)


def unfold(x: np.ndarray) -> np.ndarray:
    return np.concatenate([x[..., 0], x[..., 1]], axis=-1)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()


def gi_rows_to_list(res: np.ndarray):
    """(N, 2) uint64 -> list of (re, im) Python tuples."""
    return [(int(a), int(b)) for a, b in res.tolist()]


def cupoly_chain_restated(x: np.ndarray, Q, B, t: int) -> np.ndarray:
    """cuPoly's BFV multiplication chain (4 x poly_basis_extension_Q_to_B, poly_dr2 over Q and
    over B, 3 x poly_complex_scaling_tDivQ; src/arithmetic/polynomial.cu:350-470, 951-1000)
    restated: its float base extension and float complex scaling (oracle/pyoracle.py) around
    the exact tensor.  x: (4, k, nphi) coefficient rows of a0, a1, b0, b1; returns (3, k, nphi)."""
    from oracle import coracle as CO
    from oracle import pyoracle as O

    k = len(Q)

    def cols(rows):
        return [[int(v) for v in rows[:, j]] for j in range(rows.shape[1])]

    ext = [np.array([O.cupoly_float_ext_q_to_b(v, Q, B) for v in cols(x[i])], dtype=np.uint64).T for i in range(4)]
    qb = [np.concatenate([x[i], ext[i]]) for i in range(4)]
    P = list(Q) + list(B)
    a0, a1, b0, b1 = (CO.polymul(qb[i][None], qb[j][None], P)[0] for i, j in [(0, 2), (0, 3), (1, 2), (1, 3)])
    t1 = np.array([[(int(u) + int(v)) % p for u, v in zip(a1[r], b0[r])] for r, p in enumerate(P)], dtype=np.uint64)
    outs = []
    for ten in (a0, t1, b1):
        tq, tb = cols(ten[:k]), cols(ten[k:])
        outs.append(np.array([O.cupoly_float_complex_scaling_tdivq(a, b, Q, B, t) for a, b in zip(tq, tb)],
                             dtype=np.uint64).T)
    return np.stack(outs)
