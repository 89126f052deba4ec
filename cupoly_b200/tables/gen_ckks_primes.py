#!/usr/bin/env python3
"""Generate ``cupoly_b200/csrc/prime_table_ckks.h``: the RNS primes of CKKS mode.

cuPoly's CKKS mode builds Q from the first 63-bit prime followed by k - 1
primes of a "precision" bucket (45, 48, 52 or 55 bits) and B from the 45-bit
bucket (precision 45) or the 55-bit bucket (precisions 48, 52, 55), starting
at index k - 1 (cuPoly ``src/cuda/cudaengine.cu:1198-1232``; buckets in
``src/arithmetic/coprimes.cu:9-762``).  Results mod q_i are only comparable
with cuPoly's over the same primes, so the lists are read from cuPoly's
source; each prime is re-verified and its smallest primitive root and the
2-adic valuation of p - 1 (which bounds the ring degree) are computed here.

Usage (run once, output committed):
    python cupoly_b200/tables/gen_ckks_primes.py SRC_COPRIMES_CU > cupoly_b200/csrc/prime_table_ckks.h
"""
import re
import sys

import sympy

from gen_primes import smallest_primitive_root


def read(src: str, bits: int):
    m = re.search(r"COPRIMES_%d_BUCKET\[\]\s*=\s*\{([^}]*)\}" % bits, src)
    if not m:
        raise SystemExit("COPRIMES_%d_BUCKET not found" % bits)
    return [int(x) for x in m.group(1).replace("\n", " ").replace("\t", " ").split(",") if x.strip()]


def v2(n: int) -> int:
    return (n & -n).bit_length() - 1


def main():
    src = open(sys.argv[1]).read()
    out = ["// Generated by cupoly_b200/tables/gen_ckks_primes.py -- do not edit.",
           "// CKKS-mode prime buckets (descending), their smallest primitive roots and",
           "// the 2-adic valuation of p - 1 (a ring degree nphi needs 2 nphi | p - 1).",
           "#pragma once", "#include <cstdint>", "namespace cpoly {"]
    for bits in (45, 48, 52, 55):
        ps = read(src, bits)
        assert ps == sorted(ps, reverse=True)
        for p in ps:
            assert sympy.isprime(p) and p.bit_length() == bits
        roots = [smallest_primitive_root(p) for p in ps]
        vals = [v2(p - 1) for p in ps]
        out.append("constexpr int kNumPrimes%d = %d;" % (bits, len(ps)))
        out.append("constexpr uint64_t kPrimes%d[kNumPrimes%d] = {" % (bits, bits))
        for i in range(0, len(ps), 4):
            out.append("  " + ", ".join("%dULL" % p for p in ps[i:i + 4]) + ",")
        out.append("};")
        out.append("constexpr uint32_t kRoots%d[kNumPrimes%d] = {" % (bits, bits))
        for i in range(0, len(roots), 16):
            out.append("  " + ", ".join(str(g) for g in roots[i:i + 16]) + ",")
        out.append("};")
        out.append("constexpr uint8_t kTwoAdic%d[kNumPrimes%d] = {" % (bits, bits))
        for i in range(0, len(vals), 24):
            out.append("  " + ", ".join(str(v) for v in vals[i:i + 24]) + ",")
        out.append("};")
    out.append("}  // namespace cpoly")
    print("\n".join(out))


if __name__ == "__main__":
    main()
