"""The C ABI library loads, exports every declared symbol, and rejects invalid
arguments with status codes (cuPoly: assert / runtime_error / exit) -- no GPU."""
import ctypes as C
import subprocess

import pytest

import cupoly_b200
from cupoly_b200 import _lib


def test_library_loads_and_versions():
    L = cupoly_b200.native_library()
    assert L.cp_version().startswith(b"cupoly_b200")


def test_every_header_symbol_is_exported():
    names = _lib.header_functions()
    assert len(names) >= 30
    L = _lib.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(names) <= exported


def test_no_torch_dependency_in_native_library():
    out = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "torch" not in out and "c10" not in out


@pytest.mark.parametrize("args, fragment", [
    ((0, 1, 4096, 256, 0), "k must be"),
    ((25, 1, 4096, 256, 0), "k must be"),
    ((2, 25, 4096, 256, 0), "kl must be"),
    ((2, 3, 3000, 256, 0), "power of two"),
    ((2, 3, 131072, 256, 0), "power of two"),
    ((2, 3, 4096, 1, 0), "t must be"),
    ((2, 3, 4096, 256, 5), "log_radix"),
    ((2, 3, 2, 256, 0), "nphi must be a power of two in [4, 65536]"),
    ((2, 3, 131072, 256, 0), "nphi must be a power of two"),
    ((2, 3, 3000, 256, 0), "nphi must be a power of two"),
    ((2, 3, 4096, 256, 1), "log_radix"),
])
def test_engine_create_rejects_bad_parameters(args, fragment):
    L = _lib.lib()
    h = C.c_void_p()
    rc = L.cp_engine_create(C.byref(h), *args)
    assert rc == 1 and not h.value
    assert fragment in L.cp_last_error().decode()


def test_null_engine_calls_fail_cleanly():
    L = _lib.lib()
    assert L.cp_dgt(None, None, 0, 0, 1, 0, None) == 1
    assert L.cp_add(None, None, None, None, 0, None) == 1
    assert L.cp_bfv_mul(None, None, None, None, None, None, None, None, None, None) == 1
    assert L.cp_dot(None, None, None, None, 1, 0, None) == 1
    assert L.cp_dot_batch(None, None, None, None, 1, 1, 0, 0, None) == 1
    assert L.cp_engine_set_narrow_plan(None, 2, 10, 96) == 1
    assert L.cp_engine_set_hps_force_exact(None, 1) == 1
    assert L.cp_engine_check_async(None, None, None) == 1
    assert L.cp_engine_get_narrow_plan(None, None, None, None) == 1
    assert L.cp_engine_n_residues(None, 0) == -1
    assert L.cp_workspace_bytes(None) == 0
    assert L.cp_engine_destroy(None) == 0


def test_status_error_raises():
    with pytest.raises(_lib.CupolyError) as ei:
        _lib.call("cp_add", None, None, None, None, 0, None)
    assert ei.value.code == 1


def test_modarith_eval_checks_arguments_before_any_cuda_call():
    L = _lib.lib()
    buf = (C.c_uint64 * 4)()
    p = 9223372036801560577
    assert L.cp_modarith_eval(99, buf, buf, None, buf, 4, p, None) == 1          # unknown op
    assert L.cp_modarith_eval(0, buf, buf, None, buf, 4, p + 1, None) == 1       # even modulus
    assert L.cp_modarith_eval(0, buf, buf, None, buf, 4, 2 ** 63 + 1, None) == 1  # modulus >= 2^63
    assert L.cp_modarith_eval(4, buf, buf, None, buf, 4, p, None) == 1           # SHOUP without companions
    assert "missing operand" in L.cp_last_error().decode()
    assert L.cp_modarith_eval(0, buf, buf, None, buf, 0, p, None) == 0           # nothing to do


def test_engine_create_reports_a_failed_device_allocation():
    """With no usable CUDA device every cudaMalloc fails: engine creation builds its tables on
    the host, reaches the device allocation, frees what it built and returns CP_ERR_OOM with
    the CUDA message and no handle, as often as it is called (the out-of-memory path, driven
    by a real failing allocation rather than a GPU fault)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present: allocations succeed")
    L = _lib.lib()
    for _ in range(3):
        h = C.c_void_p()
        rc = L.cp_engine_create(C.byref(h), 2, 3, 4096, 256, 0)
        assert rc == 4 and not h.value
        assert "cudaMalloc failed for engine tables" in L.cp_last_error().decode()


def test_engine_wrapper_checks_buffers_before_the_abi():
    """Every device pointer the Engine wrapper passes is checked first: a host tensor, a
    non-int64 tensor or a non-tensor is refused without a CUDA call."""
    import torch

    from cupoly_b200.engine import Engine
    e = Engine.__new__(Engine)  # no device needed for the checks below
    e.k, e.kl, e.N, e.device = 5, 6, 4096, 0
    with pytest.raises(ValueError, match="CUDA tensor"):
        e._buf(torch.zeros((1, 5, 4096, 2), dtype=torch.int64), 0, 1, "a")
    with pytest.raises(ValueError, match="CUDA tensor"):
        e._buf(torch.zeros((1, 5, 4096, 2), dtype=torch.int32), 0, 1, "a")
    with pytest.raises(TypeError):
        e._buf([0] * 10, 0, 1, "a")
    with pytest.raises(ValueError, match="CUDA tensor"):
        e._ws(torch.zeros(16, dtype=torch.int64), 128)


def test_per_call_timing_program_is_built_and_checks_its_arguments():
    """build() links cupoly_percall (the C++ layer timed per call, run by bench.py); with bad
    arguments it prints its usage and exits 2 before touching a GPU."""
    import subprocess

    from cupoly_b200 import build as B
    B.build_percall()
    r = subprocess.run([B.PERCALL], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([B.PERCALL, "0", "1", "4096", "10"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "bad arguments" in r.stderr

