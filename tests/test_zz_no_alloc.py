"""cp_bfv_mul_noalloc: the BFV multiplication for callers that cannot allocate
device memory (a runtime that owns all HBM, code that must not take
cudaMalloc's implicit synchronisation, a plugin host with no allocator).

It must give exactly what cp_bfv_mul gives with a caller workspace, call after
call, although every call reuses the same static scratch array inside the
library.  This file sorts last so that a run stopping at the first failure has
run every other test first; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from tests.common import fold, random_poly_residues

pytestmark = pytest.mark.gpu


def _inputs(e, seed):
    from cupoly_b200.engine import FORWARD, from_u64
    dev = []
    for i in range(4):
        d = from_u64(fold(random_poly_residues(seed + i, e.Q, e.nphi))[None])
        e.dgt(d, 0, FORWARD)
        dev.append(d)
    return dev


def _noalloc(e, outs, ins):
    import torch
    from cupoly_b200 import _lib
    ptr = [C.c_void_p(t.data_ptr()) for t in outs + ins]
    return _lib.lib().cp_bfv_mul_noalloc(e.handle, *ptr, C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_matches_workspace_entry_point_on_consecutive_calls(gpu):
    import torch
    from cupoly_b200 import _lib
    from cupoly_b200.engine import Engine
    e = Engine(5, 6, 8192, 256)
    assert _lib.lib().cp_workspace_bytes(e.handle) <= 8 << 20
    for seed in (11, 97):  # two calls in a row, different operands
        ins = _inputs(e, seed)
        ref = [e.empty(0) for _ in range(3)]
        e.bfv_mul(*ref, *ins)  # existing entry point, caller workspace
        got = [e.empty(0).fill_(-1) for _ in range(3)]
        assert _noalloc(e, got, ins) == 0, _lib.lib().cp_last_error()
        torch.cuda.synchronize()
        for g, r in zip(got, ref):
            assert torch.equal(g, r)


def test_noalloc_warm_calls_leave_free_device_memory_unchanged(gpu):
    """After the first call on the device (the warm-up that may load the
    library's device code and its static scratch), calls take no device memory:
    cudaMemGetInfo's free bytes are the same before and after two more calls."""
    import torch
    from cupoly_b200 import _lib
    from cupoly_b200.engine import Engine
    e = Engine(5, 6, 8192, 256)
    ins = _inputs(e, 5)
    got = [e.empty(0) for _ in range(3)]
    assert _noalloc(e, got, ins) == 0, _lib.lib().cp_last_error()  # warm-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert _noalloc(e, got, ins) == 0, _lib.lib().cp_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_parameter_sets_beyond_the_static_scratch(gpu):
    from cupoly_b200 import _lib
    from cupoly_b200.engine import Engine
    e = Engine(10, 11, 16384, 256)
    assert _lib.lib().cp_workspace_bytes(e.handle) > 8 << 20
    outs = [e.empty(0) for _ in range(3)]
    ins = [e.empty(0) for _ in range(4)]
    rc = _noalloc(e, outs, ins)
    assert rc == 3  # CP_ERR_UNSUPPORTED
    assert b"static scratch" in _lib.lib().cp_last_error()
