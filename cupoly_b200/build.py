"""Build recipe of the in-tree shared libraries.

``cupoly_b200/lib/libcupoly_b200.so``: every ``csrc/*.cu`` file compiled for
sm_100a only and linked with nvcc into one shared object exporting the C ABI of
``include/cupoly_b200.h``.

``cupoly_b200/lib/libcupoly.so``: the C++ host layer (``host/*.cpp``, cuPoly's
``CUDAEngine`` / ``poly_t`` / ``poly_*`` API of ``include/cuPoly/``) compiled
with g++ over that ABI, with the in-repo big integer standing in for NTL's ZZ
(``include/ntl_shim``).  C++ programs written against cuPoly build with
``-I include -I include/ntl_shim -I <cuda>/include -L cupoly_b200/lib -lcupoly
-lcupoly_b200``.

Neither library links against PyTorch.

    python -m cupoly_b200.build          # incremental
    python -m cupoly_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "lib", "obj")
LIBNAME = "libcupoly_b200.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)
HOSTDIR = os.path.join(HERE, "host")
INCDIR = os.path.abspath(os.path.join(HERE, "..", "include"))
CXXLIB = os.path.join(LIBDIR, "libcupoly.so")
PERCALL = os.path.join(LIBDIR, "cupoly_percall")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-I", os.path.join(HERE, "..", "include")]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _deps(src: str):
    """Headers a source depends on (all csrc headers: they are few)."""
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(HERE, "..", "include", "cupoly_b200.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.basename(src).replace(".cu", ".o"))
    if force or _stale(obj, [src] + _deps(src)):
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj


def cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def cxx_flags():
    """Compile flags of a C++ program using the cuPoly host layer."""
    return ["-std=c++17", "-I", INCDIR, "-I", os.path.join(INCDIR, "ntl_shim"), "-I",
            os.path.join(cuda_home(), "include")]


def cxx_link_flags():
    """Link flags of a C++ program using the cuPoly host layer (rpaths to the in-tree libraries)."""
    cudalib = os.path.join(cuda_home(), "lib64")
    return ["-L", LIBDIR, "-Wl,-rpath," + LIBDIR, "-lcupoly", "-lcupoly_b200", "-L", cudalib,
            "-Wl,-rpath," + cudalib, "-lcudart"]


def build_host(force: bool = False) -> str:
    """Compile the C++ host layer into lib/libcupoly.so (needs libcupoly_b200.so)."""
    srcs = sorted(os.path.join(HOSTDIR, f) for f in os.listdir(HOSTDIR) if f.endswith(".cpp"))
    headers = []
    for root, _, files in os.walk(INCDIR):
        headers += [os.path.join(root, f) for f in files if f.endswith(".h")]
    if force or _stale(CXXLIB, srcs + headers + [LIBPATH]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-Wno-unused-parameter"] + cxx_flags() + srcs + \
            ["-o", CXXLIB, "-L", LIBDIR, "-Wl,-rpath,$ORIGIN", "-lcupoly_b200", "-L",
             os.path.join(cuda_home(), "lib64"), "-Wl,-rpath," + os.path.join(cuda_home(), "lib64"), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed for the host layer:\n%s\n%s" % (r.stdout, r.stderr))
    return CXXLIB


def build_percall(force: bool = False) -> str:
    """Compile the per-call timing program of the C++ layer (host/bench/percall.cpp) into
    lib/cupoly_percall; bench.py runs it beside cuPoly's own per-call times."""
    src = os.path.join(HOSTDIR, "bench", "percall.cpp")
    if force or _stale(PERCALL, [src, CXXLIB]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-Wall"] + cxx_flags() + [src, "-o", PERCALL] + cxx_link_flags()
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return PERCALL


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    sources = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), sources))
    if force or _stale(LIBPATH, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIBPATH] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    build_host(force)
    build_percall(force)
    if verbose:
        print(LIBPATH)
        print(CXXLIB)
    return LIBPATH


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force, verbose=True)
    except RuntimeError as exc:
        print(exc, file=sys.stderr)
        sys.exit(1)
