#!/usr/bin/env python3
"""Generate ``cupoly_b200/csrc/prime_table.h``: the 63-bit RNS prime list.

The RNS bases Q and B of cuPoly's BFV mode are drawn, in order, from a fixed
list of 100 primes p < 2^63 with 2^17 | p - 1, sorted in descending order
(cuPoly ``src/arithmetic/coprimes.cu:763-866``; selection in
``src/cuda/cudaengine.cu:1249-1290``).  Results mod q_i are only comparable
with cuPoly's when the same primes are used, so the list itself has to be
the same; everything else about a prime (its smallest primitive root, the
roots of unity, the Gaussian roots of i) is recomputed here or at engine
creation from first principles.

Usage (run once, output committed):
    python cupoly_b200/tables/gen_primes.py SRC_COPRIMES_CU > cupoly_b200/csrc/prime_table.h

``SRC_COPRIMES_CU`` is cuPoly's ``src/arithmetic/coprimes.cu``; only the
integer list ``COPRIMES_63_BUCKET`` is read from it.  Each prime is
re-verified (primality, 2^17 | p-1, descending order) and its smallest
primitive root is computed by factoring p - 1.
"""
import re
import sys

import sympy


def smallest_primitive_root(p: int) -> int:
    """Smallest g in [2, p) that generates (Z/pZ)^*: g^((p-1)/f) != 1 for every prime f | p-1."""
    factors = list(sympy.factorint(p - 1).keys())
    g = 2
    while True:
        if all(pow(g, (p - 1) // f, p) != 1 for f in factors):
            return g
        g += 1


def read_bucket(path: str):
    src = open(path).read()
    m = re.search(r"COPRIMES_63_BUCKET\[\]\s*=\s*\{([^}]*)\}", src)
    if not m:
        raise SystemExit("COPRIMES_63_BUCKET not found")
    return [int(x) for x in m.group(1).replace("\n", " ").replace("\t", " ").split(",") if x.strip()]


def main():
    primes = read_bucket(sys.argv[1])
    assert len(primes) == 100
    assert primes == sorted(primes, reverse=True)
    for p in primes:
        assert sympy.isprime(p) and p < 2**63 and (p - 1) % (1 << 17) == 0
    roots = [smallest_primitive_root(p) for p in primes]
    out = []
    out.append("// Generated by cupoly_b200/tables/gen_primes.py -- do not edit.")
    out.append("// 63-bit NTT-friendly primes (2^17 | p-1), descending, and their smallest")
    out.append("// primitive roots.  The RNS bases are taken from this list in order:")
    out.append("// Q = the first k primes, B = the next kl primes.")
    out.append("#pragma once")
    out.append("#include <cstdint>")
    out.append("namespace cpoly {")
    out.append("constexpr int kNumPrimes = %d;" % len(primes))
    out.append("constexpr uint64_t kPrimes[kNumPrimes] = {")
    for i in range(0, len(primes), 3):
        out.append("  " + ", ".join("%dULL" % p for p in primes[i:i + 3]) + ",")
    out.append("};")
    out.append("constexpr uint32_t kPrimitiveRoots[kNumPrimes] = {")
    for i in range(0, len(roots), 12):
        out.append("  " + ", ".join(str(g) for g in roots[i:i + 12]) + ",")
    out.append("};")
    out.append("}  // namespace cpoly")
    print("\n".join(out))


if __name__ == "__main__":
    main()
