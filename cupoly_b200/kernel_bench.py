"""Per-kernel throughput on the current GPU, each against the HBM roofline.

    python -m cupoly_b200.kernel_bench [--only NAME[,NAME...]] [--reps R] [--peak GBS] [--split-mode 0|1]

One JSON line per workload: average milliseconds per launch (CUDA events on the
launching stream, after a warm-up launch), the algorithmic bytes one launch must
move (each input read once, each output written once), the achieved GB/s and its
fraction of the HBM peak (`--peak`, default the copy bandwidth recorded in
MEASURED_PEAKS.json at the repository root when present, else 6650 GB/s).  Every
workload's data exceeds the 126 MB L2, so successive launches stream from HBM.
`--split-mode` sets the split-stage form of every engine (cp_engine_set_split_mode).

Workloads (names for --only):
  dgt_fwd, dgt_inv   forward / inverse DGT, nphi 8192, 3072 residues (512 polynomials over B, in place)
  mul                DGT-domain pointwise product, nphi 8192, k 5, 512 polynomials
  polymul            fused negacyclic product (cp_polymul), nphi 4096, k 2, 2048 polynomials
  basis_ext          exact Q -> B conversion, nphi 8192, k 5 -> 6, 512 polynomials
  complex_scaling    round(t X / Q) mod B, nphi 8192, k 5, kl 6, 384 polynomials
  crt, icrt          coefficient limbs <-> residues, nphi 8192, k 5, 512 polynomials
  sample_ternary, sample_gaussian, sample_uniform
                     2^24 coefficients x 16 residues (nphi 32768, k 16, 512 polynomials)
  dot                key-switching dot product (cp_dot), 16 terms, nphi 32768, k 16; bytes = 32
                     operands read + 1 written
  dot_batch          cp_dot_batch: the xi decomposition of 128 polynomials against 5 shared key
                     polynomials, nphi 8192, k 5; bytes = decompositions + keys read + results written
  mixed_tiles, mixed_graph
                     the benchmark's mixed batch of 1024 negacyclic products (nphi 2048..16384,
                     k 1..8, seeded draw): one persistent launch, or 3 launches per size group
  bfv_chain, bfv_chain_target, bfv_chain_large
                     the batched BFV multiplication chain (cp_bfv_mul_batch) at nphi 8192 / k 5 /
                     128 pairs, nphi 16384 / k 10 / 32 pairs and nphi 32768 / k 16 / t 65537 / 64
                     pairs; bytes = 4 operands read + 3 results written over Q per pair (the
                     algorithmic bytes of one homomorphic multiplication)
"""
from __future__ import annotations

import argparse
import json
import os

import torch

from .engine import (FORWARD, GAUSSIAN, INVERSE, QBase, BBase, TERNARY, UNIFORM, Engine)

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _peak() -> float:
    try:
        with open(os.path.join(_ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


def _time(fn, reps: int) -> float:
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


_SPLIT_MODE = None


def _engine(*args) -> Engine:
    e = Engine(*args)
    if _SPLIT_MODE is not None:
        e.set_split_mode(_SPLIT_MODE)
    return e


def workloads():
    """name -> builder; a builder returns (launch function, algorithmic bytes, description)."""
    W = {}

    def dgt(direction):
        def build():
            e = _engine(5, 6, 8192, 256)
            x = e.empty(BBase, 512)  # 512 x 6 = 3072 residues: the chain's forward DGT over B
            e.sample(x, BBase, UNIFORM, 1, 0, npolys=512, to_dgt=False)
            nres = 512 * 6
            return (lambda: e.dgt(x, BBase, direction), nres * e.N * 16 * 2,
                    "%s DGT, nphi 8192, %d residues" % ("forward" if direction == FORWARD else "inverse", nres), e)
        return build

    W["dgt_fwd"] = dgt(FORWARD)
    W["dgt_inv"] = dgt(INVERSE)

    def mul():
        e = _engine(5, 6, 8192, 256)
        P = 512
        a, b, c = e.empty(QBase, P), e.empty(QBase, P), e.empty(QBase, P)
        e.sample(a, QBase, UNIFORM, 2, 0, npolys=P, to_dgt=False)
        e.sample(b, QBase, UNIFORM, 2, P, npolys=P, to_dgt=False)
        return (lambda: e.mul_batch(c, a, b, QBase, P), 3 * P * 5 * e.N * 16,
                "pointwise Gaussian product, nphi 8192, k 5, %d polys" % P, e)

    W["mul"] = mul

    def polymul():
        e = _engine(2, 3, 4096, 256)
        P = 2048
        a, b, c = e.empty(QBase, P), e.empty(QBase, P), e.empty(QBase, P)
        e.sample(a, QBase, UNIFORM, 3, 0, npolys=P, to_dgt=False)
        e.sample(b, QBase, UNIFORM, 3, P, npolys=P, to_dgt=False)
        ws = e.polymul_workspace(QBase, P)
        return (lambda: e.polymul(c, a, b, QBase, ws, P), 3 * P * 2 * e.N * 16,
                "fused polymul (3 launches), nphi 4096, k 2, %d polys; bytes = a, b read + c written" % P, e)

    W["polymul"] = polymul

    def basis_ext():
        e = _engine(5, 6, 8192, 256)
        P = 512
        x, y = e.empty(QBase, P), e.empty(BBase, P)
        e.sample(x, QBase, UNIFORM, 4, 0, npolys=P, to_dgt=False)
        return (lambda: e.basis_ext_q_to_b(y, x, P), P * (5 + 6) * e.N * 16,
                "exact Q -> B, nphi 8192, k 5 -> 6, %d polys" % P, e)

    W["basis_ext"] = basis_ext

    def complex_scaling():
        e = _engine(5, 6, 8192, 256)
        P = 384
        x, xb, y = e.empty(QBase, P), e.empty(BBase, P), e.empty(BBase, P)
        e.sample(x, QBase, UNIFORM, 5, 0, npolys=P, to_dgt=False)
        e.sample(xb, BBase, UNIFORM, 5, P, npolys=P, to_dgt=False)
        return (lambda: e.complex_scaling(y, x, xb, P), P * (5 + 6 + 6) * e.N * 16,
                "round(t X / Q) mod B, nphi 8192, k 5, kl 6, %d polys" % P, e)

    W["complex_scaling"] = complex_scaling

    def crt(inverse):
        def build():
            e = _engine(5, 6, 8192, 256)
            P = 512
            x = e.empty(QBase, P)
            e.sample(x, QBase, UNIFORM, 6, 0, npolys=P, to_dgt=False)
            limbs = torch.zeros((P, e.nphi, 5), dtype=torch.int64, device="cuda")
            e.icrt(limbs, x, QBase)
            fn = (lambda: e.icrt(limbs, x, QBase)) if inverse else (lambda: e.crt(x, limbs, QBase))
            return (fn, 2 * P * e.nphi * 5 * 8,
                    "%s, nphi 8192, k 5, %d polys, 5-limb coefficients" % ("ICRT" if inverse else "CRT", P), e)
        return build

    W["crt"] = crt(False)
    W["icrt"] = crt(True)

    def sample(kind, name):
        def build():
            e = _engine(16, 17, 32768, 65537)
            P = 512
            x = e.empty(QBase, P)
            return (lambda: e.sample(x, QBase, kind, 7, 0, npolys=P, to_dgt=False), P * 16 * e.N * 16,
                    "%s sampling, 2^24 coefficients x 16 residues (bytes written)" % name, e)
        return build

    def chain(nphi, k, t, P):
        def build():
            e = _engine(k, k + 1, nphi, t)
            ins = [e.empty(QBase, P) for _ in range(4)]
            for v, x in enumerate(ins):
                e.sample(x, QBase, UNIFORM, 8, v * P, npolys=P, to_dgt=True)
            c = e.empty(QBase, 3 * P)
            ws = e.bfv_mul_batch_workspace(P)
            return (lambda: e.bfv_mul_batch(c, *ins, P, ws), P * 7 * k * e.N * 16,
                    "batched BFV multiplication, nphi %d, k %d, kl %d, t %d, %d pairs per call" % (nphi, k, k + 1, t, P), e)
        return build

    def dot():
        e = _engine(16, 17, 32768, 65537)
        nt = 16
        sets = []
        for s in range(2):  # two operand sets alternate: 2 x 138 MB
            ops = e.empty(QBase, 2 * nt)
            e.sample(ops, QBase, UNIFORM, 9, 2 * nt * s, npolys=2 * nt, to_dgt=False)
            sets.append(([ops[i] for i in range(nt)], [ops[nt + i] for i in range(nt)]))
        c = e.empty(QBase)
        it = [0]

        def fn():
            a, b = sets[it[0] & 1]
            it[0] += 1
            e.dot(c, a, b, QBase)

        return (fn, (2 * nt + 1) * 16 * e.N * 16,
                "key-switching dot product (cp_dot), %d terms, nphi 32768, k 16" % nt, e)

    W["dot"] = dot

    def dot_batch():
        e = _engine(5, 6, 8192, 256)
        P, k = 128, 5
        dec, keys, out = e.empty(QBase, P * k), e.empty(QBase, k), e.empty(QBase, P)
        e.sample(dec, QBase, UNIFORM, 10, 0, npolys=P * k, to_dgt=False)
        e.sample(keys, QBase, UNIFORM, 10, P * k, npolys=k, to_dgt=False)
        return (lambda: e.dot_batch(out, dec, keys, k, P, QBase, b_shared=True), (P * k + k + P) * k * e.N * 16,
                "batched key-switching dot (cp_dot_batch), %d decompositions x %d shared keys, nphi 8192, k 5"
                % (P, k), e)

    W["dot_batch"] = dot_batch

    def mixed(mode):
        def build():
            from .batch import MixedPolymul, random_specs
            mp = MixedPolymul(random_specs(1024, 0xC0FFEE), mode=mode)
            for g in mp.groups.values():  # residues below 2^62 are valid for every prime of the table
                g["a"].random_(0, 1 << 62)
                g["b"].random_(0, 1 << 62)
            e = next(iter(mp.groups.values()))["engine"]
            return (mp.run, mp.algorithmic_bytes(),
                    "mixed batch of 1024 polymuls (nphi 2048..16384, k 1..8), %s" %
                    ("one persistent launch (cp_polymul_tiles)" if mode == "tiles"
                     else "3 launches per size group (cp_polymul_list)"), e)
        return build

    W["mixed_tiles"] = mixed("tiles")
    W["mixed_graph"] = mixed("graph")
    W["bfv_chain"] = chain(8192, 5, 256, 128)
    W["bfv_chain_target"] = chain(16384, 10, 256, 32)
    W["bfv_chain_large"] = chain(32768, 16, 65537, 64)
    W["sample_ternary"] = sample(TERNARY, "ternary")
    W["sample_gaussian"] = sample(GAUSSIAN, "Gaussian")
    W["sample_uniform"] = sample(UNIFORM, "uniform mod q_i")
    return W


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--only", default="")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--peak", type=float, default=0.0)
    ap.add_argument("--split-mode", type=int, choices=[0, 1], default=None)
    a = ap.parse_args()
    global _SPLIT_MODE
    _SPLIT_MODE = a.split_mode
    peak = a.peak or _peak()
    W = workloads()
    names = [n for n in a.only.split(",") if n] or list(W)
    for n in names:
        fn, byt, desc, e = W[n]()
        ms = _time(fn, a.reps)
        e.check()
        gbs = byt / ms / 1e6
        print(json.dumps({"kernel": n, "workload": desc, "ms": round(ms, 4), "bytes": byt, "GB_per_s": round(gbs, 1),
                          "peak_GB_per_s": peak, "frac_hbm": round(gbs / peak, 4)}), flush=True)
        del fn, e
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
