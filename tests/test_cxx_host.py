"""The C++ host layer (include/cuPoly/*.h, cupoly_b200/host/, lib/libcupoly.so).

CPU: the in-repo big integer agrees with Python's integers on random operations
(floor division as NTL), the layer builds and exports cuPoly's C++ API, cuPoly's
own demo (demos/src/simple_polyop.cpp, when the reference tree is present) and the
C++ test program compile against it with include-path changes only.
GPU: the C++ test program (cuPoly's TestDGT / TestRNS / TestArithmetic / TestSampler
over cuPoly's (log2 q, nphi) grid, plus CKKS checks) passes.
"""
import os
import random
import subprocess

import pytest

from cupoly_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXX_DIR = os.path.join(ROOT, "tests", "cxx")
# cuPoly's own demo, compiled unmodified against the layer when a cuPoly source
# tree is named by CUPOLY_REF_DIR (the test is skipped otherwise).
REF_DIR = os.environ.get("CUPOLY_REF_DIR", "")
REF_DEMO = os.path.join(REF_DIR, "demos", "src", "simple_polyop.cpp") if REF_DIR else ""

# C++ names (demangled) the layer must export: cuPoly's public API surface.
API = [
    "CUDAEngine::init_bfv(int, int, int, unsigned long)", "CUDAEngine::init_ckks(int, int, int, int)",
    "CUDAEngine::destroy()", "CUDAEngine::get_n_residues(int)", "CUDAEngine::RNSProduct",
    "DGTEngine::execute_dgt(GaussianInteger*, int, int, Context*)",
    "DGTEngine::execute_mul_dgt_gi(GaussianInteger*, GaussianInteger const*, GaussianInteger const*, int, CUstream_st*)",
    "Context::Context()", "Sampler::sample(Context*, polynomial*, int)", "Sampler::sample(Context*, int)",
    "poly_init(Context*, polynomial*, int)", "poly_free(Context*, polynomial*)",
    "poly_add(Context*, polynomial*, polynomial*, polynomial*)",
    "poly_mul(Context*, polynomial*, polynomial*, polynomial*)",
    "poly_dr2(Context*, polynomial*, polynomial*, polynomial*, polynomial*, polynomial*, polynomial*, polynomial*)",
    "poly_basis_extension_Q_to_B(Context*, polynomial*, polynomial*)",
    "poly_complex_scaling_tDivQ(Context*, polynomial*, polynomial*, polynomial*)",
    "poly_simple_scaling_tDivQ(Context*, polynomial*, polynomial*)",
    "poly_xi_bfv(Context*, polynomial*, polynomial*)", "poly_rho_bfv(Context*, polynomial*, polynomial*)",
    "poly_set_coeff(Context*, polynomial*, unsigned int, cupoly::ZZ)", "poly_get_coeff(Context*, polynomial*, int)",
    "poly_export_residues[abi:cxx11](Context*, polynomial*)", "poly_ckks_rescale(Context*, polynomial*, polynomial*, int)",
]


def _compile(src, out, extra=()):
    cmd = ["g++", "-O2", "-Wall"] + B.cxx_flags() + [src, "-o", out] + B.cxx_link_flags() + list(extra)
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


@pytest.fixture(scope="module")
def host_lib():
    B.build()
    assert os.path.exists(B.CXXLIB)
    return B.CXXLIB


def test_zz_matches_python_integers(tmp_path):
    exe = str(tmp_path / "zz_calc")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", B.INCDIR, os.path.join(CXX_DIR, "zz_calc.cpp"),
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rng = random.Random(11)

    def rnd():
        k = rng.choice([0, 1, 2, 63, 64, 65, 127, 128, 129, 200, 500, 1000, 2100])
        x = rng.getrandbits(k) if k else rng.choice([0, 1, 2, 3])
        if k and rng.random() < 0.2:
            x = (1 << k) - rng.choice([0, 1])  # all-ones limbs: Knuth D's correction steps
        return -x if rng.random() < 0.4 else x

    sgn = lambda a: 1 if a >= 0 else -1  # noqa: E731
    ops = {"add": lambda a, b: a + b, "sub": lambda a, b: a - b, "mul": lambda a, b: a * b,
           "div": lambda a, b: a // b, "mod": lambda a, b: a % b,
           "shl": lambda a, b: sgn(a) * (abs(a) << b), "shr": lambda a, b: sgn(a) * (abs(a) >> b),
           "cmp": lambda a, b: (a > b) - (a < b), "bits": lambda a, b: abs(a).bit_length(),
           "limbs": lambda a, b: a}
    lines, want = [], []
    for _ in range(6000):
        op = rng.choice(sorted(ops))
        a, b = rnd(), rnd()
        if op in ("shl", "shr"):
            b = rng.randrange(0, 300)
        if op in ("div", "mod") and b == 0:
            b = 7
        lines.append("%s %d %d" % (op, a, b))
        want.append(str(ops[op](a, b)))
    out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True).stdout.split("\n")
    bad = [(l, o, w) for l, o, w in zip(lines, out, want) if o != w]
    assert not bad, bad[:3]
    assert len(out) >= len(want)


def test_host_layer_exports_cupolys_api(host_lib):
    r = subprocess.run(["nm", "-D", "-C", "--defined-only", host_lib], capture_output=True, text=True)
    assert r.returncode == 0
    missing = [s for s in API if s not in r.stdout]
    assert not missing, missing


def test_cxx_test_program_compiles(host_lib, tmp_path):
    _compile(os.path.join(CXX_DIR, "test_cupoly_host.cpp"), str(tmp_path / "test_cupoly_host"))


@pytest.mark.skipif(not os.path.exists(REF_DEMO), reason="reference tree not present")
def test_reference_demo_compiles_with_include_paths_only(host_lib, tmp_path):
    """cuPoly's demos/src/simple_polyop.cpp, unmodified, against include/cuPoly + the NTL stand-in."""
    _compile(REF_DEMO, str(tmp_path / "simple_polyop"))


@pytest.mark.gpu
def test_cxx_host_layer_suite_on_gpu(gpu, host_lib, tmp_path):
    exe = _compile(os.path.join(CXX_DIR, "test_cupoly_host.cpp"), str(tmp_path / "test_cupoly_host"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    tail = (r.stdout + r.stderr)[-4000:]
    assert r.returncode == 0, tail
    assert " 0 failed" in r.stdout, tail


def _write_cupoly_root_dir(d):
    """A directory laid out like cuPoly's src/arithmetic/coprimes: qis_63.json in its
    format ({p: [{N: {"re", "imag"}}, ...]}) with cuPoly's NTHROOT values from
    tests/golden/ref_nthroot.json."""
    import json
    roots = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_nthroot.json")))
    doc = {p: [{n: {"re": v[0], "imag": v[1]} for n, v in by_n.items()}, {}] for p, by_n in roots.items()}
    with open(os.path.join(d, "qis_63.json"), "w") as f:
        json.dump(doc, f, indent=1)


@pytest.mark.gpu
@pytest.mark.parametrize("k,kl,nphi", [(5, 6, 8192), (16, 17, 32768)])
def test_cxx_layer_loads_cupolys_roots_from_its_coprimes_dir(gpu, host_lib, tmp_path, k, kl, nphi):
    """With CUPOLY_COPRIMES_DIR set, CUDAEngine::init takes cuPoly's NTHROOT and the C++
    layer's DGT-domain bytes are cuPoly's: at nphi 8192 / k 5 / kl 6 they equal the bytes
    cuPoly itself produced on the same input (tests/golden/cupoly_ref_golden.json); at
    nphi 32768 / k 16 / kl 17 (beyond cuPoly's 30-prime limit) they equal the oracle's
    transform with cuPoly's roots.  Without the variable the layer keeps its canonical
    root, says so on stderr, and the bytes equal the oracle's with that root."""
    import json

    import numpy as np

    from oracle import coracle as CO
    from oracle import pyoracle as O
    from tests.common import fold, random_poly_residues, sha
    exe = _compile(os.path.join(CXX_DIR, "dgt_bytes.cpp"), str(tmp_path / "dgt_bytes"))
    Q, B = O.bases(k, kl)
    golden = None
    gpath = os.path.join(ROOT, "tests", "golden", "cupoly_ref_golden.json")
    if os.path.exists(gpath):
        golden = next((c for c in json.load(open(gpath))["cases"]
                       if c["op"] == "dgt" and (c["k"], c["kl"], c["nphi"]) == (k, kl, nphi)), None)
    if golden is not None:
        from tests.golden.gen_cupoly_golden import inputs
        x = inputs("dgt", k, kl, nphi, golden["seed"]).reshape(k + kl, nphi)
    else:
        x = random_poly_residues(77, Q + B, nphi)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    x.astype(np.uint64).tofile(fin)
    rdir = tmp_path / "coprimes"
    rdir.mkdir()
    _write_cupoly_root_dir(str(rdir))
    env = dict(os.environ, CUPOLY_COPRIMES_DIR=str(rdir))
    r = subprocess.run([exe, str(k), str(kl), str(nphi), fin, fout], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(fout, dtype=np.uint64).reshape(k + kl, nphi // 2, 2)
    roots = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_nthroot.json")))
    want = CO.dgt(fold(x)[None], Q + B, xi=[tuple(roots[str(p)][str(nphi // 2)]) for p in Q + B])[0]
    assert np.array_equal(got, want)
    if golden is not None:
        assert sha(got) == golden["sha256"]
    env.pop("CUPOLY_COPRIMES_DIR")
    r = subprocess.run([exe, str(k), str(kl), str(nphi), fin, fout], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "CUPOLY_COPRIMES_DIR" in r.stderr
    got = np.fromfile(fout, dtype=np.uint64).reshape(k + kl, nphi // 2, 2)
    assert np.array_equal(got, CO.dgt(fold(x)[None], Q + B)[0])
