#!/usr/bin/env python3
"""Generate ``cupoly_b200/csrc/cdt_table.h``: cumulative tables for the Gaussian samplers.

Two distributions over magnitudes m = 0..19, each given as 63-bit cumulative
thresholds T_m = floor(2^63 * P(|x| <= m)) for m = 0..18 (m = 19 takes the
rest).  A sample draws u uniform in [0, 2^63) and returns the smallest m
with u < T_m.

* ``kCdtSigned``: the discrete Gaussian D_sigma, sigma = 3.19, truncated to
  |x| <= floor(6 sigma) = 19, rho(x) = exp(-x^2 / (2 sigma^2)); magnitude
  m > 0 carries a uniform sign.
* ``kCdtFolded``: cuPoly's BFV ``DISCRETE_GAUSSIAN`` kind, |nearbyint(3.2 Z)|
  for Z ~ N(0, 1) (cuPoly src/cuda/sampler.cu:459-493, sigma from
  include/cuPoly/settings.h:155), truncated at 6 sigma = 19.2.

Usage: python cupoly_b200/tables/gen_cdt.py > cupoly_b200/csrc/cdt_table.h
"""
import mpmath

mpmath.mp.prec = 256
MAXMAG = 19


def thresholds(pmag):
    total = mpmath.fsum(pmag)
    out, acc = [], mpmath.mpf(0)
    for m in range(MAXMAG):
        acc += pmag[m]
        out.append(int(mpmath.floor(acc / total * mpmath.mpf(2) ** 63)))
    return out


def signed(sigma=mpmath.mpf("3.19")):
    rho = [mpmath.exp(-mpmath.mpf(m * m) / (2 * sigma * sigma)) for m in range(MAXMAG + 1)]
    return [rho[0]] + [2 * r for r in rho[1:]]


def folded(sigma=mpmath.mpf("3.2")):
    def cdf(x):
        return mpmath.ncdf(x / sigma)
    p = [cdf(mpmath.mpf("0.5")) - cdf(mpmath.mpf("-0.5"))]
    for m in range(1, MAXMAG + 1):
        p.append(2 * (cdf(m + mpmath.mpf("0.5")) - cdf(m - mpmath.mpf("0.5"))))
    return p


def main():
    ts, tf = thresholds(signed()), thresholds(folded())
    lines = ["// Generated by cupoly_b200/tables/gen_cdt.py -- do not edit.",
             "#pragma once", "#include <cstdint>", "namespace cpoly {",
             "constexpr int kCdtLen = %d;  // thresholds for magnitudes 0..%d" % (MAXMAG, MAXMAG - 1),
             "constexpr int kCdtMaxMag = %d;" % MAXMAG]
    for name, t in (("kCdtSigned", ts), ("kCdtFolded", tf)):
        lines.append("constexpr uint64_t %s[] = {" % name)
        for i in range(0, len(t), 3):
            lines.append("  " + ", ".join("%dULL" % x for x in t[i:i + 3]) + ",")
        lines.append("};")
    lines.append("}  // namespace cpoly")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
