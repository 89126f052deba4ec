#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/.

Run in a checkout that has cuPoly's sources (the path is an argument; it is
read only here, never at test time):

    python tests/golden/gen_golden.py /path/to/cupoly

Writes:
  ref_nthroot.json -- cuPoly's tabulated Gaussian roots of i, NTHROOT[p][N]
                      (src/arithmetic/coprimes/qis_63.json), for the first 33
                      primes (Q u B of nphi 32768, k 16, kl 17) and every
                      tabulated size N = 16 ... 32768.  With them
                      the DGT-domain bytes can be compared with cuPoly's.
  dgt_golden.json  -- seeded inputs (by seed) and SHA-256 of the forward DGT
                      computed by the Python restatement of cuPoly's
                      hierarchical kernels (oracle/pyoracle.py) with cuPoly's
                      roots; residue 0's first values are kept in clear.
  hps_golden.json  -- SHA-256 of exact basis extension / scaling results
                      (Python big-integer definitions) on seeded inputs.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

import numpy as np  # noqa: E402

from oracle import pyoracle as O  # noqa: E402
from tests.common import fold, gi_rows_to_list, random_poly_residues, sha  # noqa: E402

SIZES = [16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768]
DGT_CASES = [  # (nphi, nres, seed)
    (32, 3, 11), (128, 2, 12), (256, 2, 13), (2048, 2, 14), (4096, 3, 15), (8192, 2, 16),
]
HPS_CASES = [  # (nphi, k, kl, t, seed)
    (32, 1, 2, 256, 21), (64, 2, 3, 256, 22), (128, 3, 4, 65537, 23), (256, 5, 6, 256, 24),
]


def main(ref_root):
    qis = json.load(open(os.path.join(ref_root, "src", "arithmetic", "coprimes", "qis_63.json")))
    roots = {}
    for p in O.PRIMES[:33]:
        tab = qis[str(p)][0]
        roots[str(p)] = {str(N): [tab[str(N)]["re"], tab[str(N)]["imag"]] for N in SIZES}
        for N in SIZES:  # sanity: xi^N == i
            assert O.gi_pow(tuple(roots[str(p)][str(N)]), N, p) == (0, 1)
    json.dump(roots, open(os.path.join(HERE, "ref_nthroot.json"), "w"), indent=1)

    dgt = []
    for nphi, nres, seed in DGT_CASES:
        N = nphi // 2
        primes = O.PRIMES[:nres]
        x = fold(random_poly_residues(seed, primes, nphi))
        out = np.empty_like(x)
        for r, p in enumerate(primes):
            xi = tuple(roots[str(p)][str(N)])
            out[r] = np.array(O.dgt_forward_ref(gi_rows_to_list(x[r]), p, xi), dtype=np.uint64)
        dgt.append({"nphi": nphi, "nres": nres, "seed": seed, "sha256": sha(out),
                    "head": [[int(a), int(b)] for a, b in out[0, :4].tolist()]})
    json.dump(dgt, open(os.path.join(HERE, "dgt_golden.json"), "w"), indent=1)

    hps = []
    for nphi, k, kl, t, seed in HPS_CASES:
        Q, B = O.bases(k, kl)
        xq = random_poly_residues(seed, Q, nphi)
        yb = random_poly_residues(seed + 1000, B, nphi)
        ext = np.array([O.basis_extension_exact(xq[:, c].tolist(), Q, B) for c in range(nphi)], dtype=np.uint64).T
        bq = np.array([O.basis_extension_exact(yb[:, c].tolist(), B, Q) for c in range(nphi)], dtype=np.uint64).T
        cs = np.array([O.complex_scaling_exact(xq[:, c].tolist(), yb[:, c].tolist(), Q, B, t)
                       for c in range(nphi)], dtype=np.uint64).T
        ss = np.array([O.simple_scaling_exact(xq[:, c].tolist(), Q, t) for c in range(nphi)], dtype=np.uint64)
        hps.append({"nphi": nphi, "k": k, "kl": kl, "t": t, "seed": seed, "ext_q_to_b": sha(ext),
                     "ext_b_to_q": sha(bq), "complex_scaling": sha(cs), "simple_scaling": sha(ss)})
    json.dump(hps, open(os.path.join(HERE, "hps_golden.json"), "w"), indent=1)


if __name__ == "__main__":
    main(sys.argv[1])
