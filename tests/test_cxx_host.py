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
REF_DEMO = "/root/reference/demos/src/simple_polyop.cpp"

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
