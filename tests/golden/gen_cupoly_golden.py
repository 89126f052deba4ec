#!/usr/bin/env python3
"""Golden outputs of cuPoly itself, for tests/golden/cupoly_ref_golden.json.

cuPoly's own library sources are compiled, unmodified, by
``oracle/cupoly_ref/Makefile`` into ``oracle/_ref/cupoly_ref_driver`` (in a
checkout that has them); the driver runs cuPoly's public API on a GPU.  This
script feeds it the tests' seeded inputs (``tests/common.py``) and records,
per case, the SHA-256 of cuPoly's output words and their first values:

    make -C oracle/cupoly_ref
    python tests/golden/gen_cupoly_golden.py OUT_DIR   # needs a GPU

The cases cover cuPoly's gtest grid (``tests/unit_tests/test_bfv_mode.cu:1492-1508``:
k = ceil(log2 q / 63), kl = k + 1, t = 256), the polymul size nphi 4096 / k 2
and the BFV multiplication size nphi 8192 / k 5 / kl 6.  ``tables`` records
cuPoly's precomputed HPS constants and Barrett factors as numbers.
``time`` records cuPoly's own per-call GPU times at those two sizes.
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle import pyoracle as O  # noqa: E402
from tests.common import fold, random_poly_residues, sha  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "cupoly_ref_driver")

# (nphi, k) of cuPoly's gtest grid, then the two benchmark sizes.
GRID = [(32, 1), (32, 2), (32, 3), (32, 6), (128, 1), (128, 2), (256, 2), (2048, 1), (2048, 2), (2048, 6),
        (4096, 3), (8192, 3), (8192, 4), (8192, 6), (4096, 2), (8192, 5)]
OPS = ["dgt", "mul", "ext", "cscale", "sscale", "xirho"]
BFV_SIZES = [(32, 3), (2048, 6), (4096, 2), (8192, 5)]
EXTRA = [("cscale", 2048, 2, 65536), ("sscale", 2048, 2, 65536), ("bfvmul", 2048, 2, 65536)]
FULL_LIMIT = 512  # keep every output word of cases at most this long


def inputs(op, k, kl, nphi, seed):
    """The driver's input words of one case (coefficient-domain rows)."""
    Q, B = O.bases(k, kl)
    if op == "dgt":
        rows = [random_poly_residues(seed, Q + B, nphi)]
    elif op in ("mul",):
        rows = [random_poly_residues(seed, Q, nphi, stream=s) for s in range(2)]
    elif op == "cscale":
        rows = [random_poly_residues(seed, Q, nphi, stream=0), random_poly_residues(seed, B, nphi, stream=1)]
    elif op == "bfvmul":
        rows = [random_poly_residues(seed, Q, nphi, stream=s) for s in range(4)]
    else:
        rows = [random_poly_residues(seed, Q, nphi)]
    return np.concatenate([r.reshape(-1) for r in rows]).astype(np.uint64)


def run_many(ops, k, kl, nphi, t, words_in):
    """One driver process (one cuPoly engine) for several ops; {op: output words}."""
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in"), os.path.join(d, "out")
        for op in ops:
            words_in.get(op, np.zeros(0, dtype=np.uint64)).tofile(fin + "." + op)
        if len(ops) == 1:
            os.replace(fin + "." + ops[0], fin)
        subprocess.run([DRIVER, ",".join(ops), str(k), str(kl), str(nphi), str(t), fin, fout], check=True,
                       timeout=600)
        if ops == ["time"]:
            return {"time": json.load(open(fout))}
        paths = {op: (fout + "." + op if len(ops) > 1 else fout) for op in ops}
        return {op: np.fromfile(path, dtype=np.uint64) for op, path in paths.items()}


def record(op, k, kl, nphi, t, seed, x, out):
    rec = {"op": op, "k": k, "kl": kl, "nphi": nphi, "t": t, "seed": seed}
    if op == "dgt":
        half = out.size // 2
        folded = fold(x.reshape(k + kl, nphi)).reshape(-1)
        rec["round_trip"] = bool(np.array_equal(out[half:], folded))
        out = out[:half]
    rec["words"] = int(out.size)
    rec["sha256"] = sha(out)
    rec["head"] = [int(v) for v in out[:6]]
    if out.size <= FULL_LIMIT:
        rec["full"] = [int(v) for v in out]
    return rec


def tables(k, kl, nphi, t, w):
    w = w.tolist()
    kk = k * kl
    rec = {"k": k, "kl": kl, "nphi": nphi, "t": t}
    rec["Q"], w = w[:k], w[k:]
    rec["B"], w = w[:kl], w[kl:]
    rec["barrett_mu"], w = w[:k + kl], w[k + kl:]
    rec["omega_int"], w = w[:kk], w[kk:]
    fr, w = w[:2 * kk], w[2 * kk:]
    rec["omega_frac"] = [fr[2 * i] | (fr[2 * i + 1] << 64) for i in range(kk)]
    rec["lambda"], w = w[:kl], w[kl:]
    rec["tomega_int"], w = w[:k], w[k:]
    fr = w[:2 * k]
    rec["tomega_frac"] = [fr[2 * i] | (fr[2 * i + 1] << 64) for i in range(k)]
    return rec


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    doc = {"source": "cuPoly 0.3.5 library sources, compiled by oracle/cupoly_ref/Makefile, run on a B200",
           "tables": [], "cases": [], "timing": {}}
    path = os.path.join(out_dir, "cupoly_ref_golden.json")

    def save():
        with open(path, "w") as f:
            json.dump(doc, f, indent=0)

    points = {}  # (nphi, k, t) -> [ops]
    for nphi, k in GRID:
        points.setdefault((nphi, k, 256), []).extend(OPS)
    for nphi, k in BFV_SIZES:
        points.setdefault((nphi, k, 256), []).append("bfvmul")
    for op, nphi, k, t in EXTRA:
        points.setdefault((nphi, k, t), []).append(op)
    seed = 100
    for (nphi, k, t), ops in points.items():
        kl = k + 1
        seeds, ins = {}, {}
        for op in ops:
            seed += 1
            seeds[op] = seed
            ins[op] = inputs(op, k, kl, nphi, seed)
        outs = run_many(["tables"] + ops, k, kl, nphi, t, ins)
        doc["tables"].append(tables(k, kl, nphi, t, outs["tables"]))
        for op in ops:
            doc["cases"].append(record(op, k, kl, nphi, t, seeds[op], ins[op], outs[op]))
            print(op, nphi, k, t, doc["cases"][-1]["sha256"][:16], flush=True)
        save()
    for name, (k, nphi) in {"nphi4096_k2": (2, 4096), "nphi8192_k5_kl6": (5, 8192)}.items():
        doc["timing"][name] = run_many(["time"], k, k + 1, nphi, 200, {})["time"]
        save()
    print("cases", len(doc["cases"]), "timing", doc["timing"])


if __name__ == "__main__":
    main(sys.argv[1])
