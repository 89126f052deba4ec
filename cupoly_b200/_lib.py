"""ctypes binding of the C ABI (``include/cupoly_b200.h``).

The in-tree shared library ``cupoly_b200/lib/libcupoly_b200.so`` is the only
compute path: if it is missing or cannot be loaded, importing this module's
``lib()`` raises; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcupoly_b200.so")
HEADER_PATH = os.path.join(_HERE, "..", "include", "cupoly_b200.h")

CP_OK = 0


class CupolyError(RuntimeError):
    """A C ABI call returned a non-zero status."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__("%s failed (status %d): %s" % (fn, code, msg))
        self.code = code


_vp = C.c_void_p
_i = C.c_int
_u64 = C.c_uint64
_u32 = C.c_uint32
_i64 = C.c_int64
_pu64 = C.POINTER(C.c_uint64)

# name -> (restype, argtypes)
SIGNATURES = {
    "cp_version": (C.c_char_p, []),
    "cp_last_error": (C.c_char_p, []),
    "cp_engine_create": (_i, [C.POINTER(_vp), _i, _i, _i, _u64, _i]),
    "cp_ckks_engine_create": (_i, [C.POINTER(_vp), _i, _i, _i, _i, _i]),
    "cp_engine_ckks_prec": (_i, [_vp]),
    "cp_engine_set_plan": (_i, [_vp, _i, _i]),
    "cp_engine_get_plan": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "cp_engine_check_async": (_i, [_vp, _vp, _vp]),
    "cp_engine_set_narrow_plan": (_i, [_vp, _i, _i, C.c_longlong]),
    "cp_engine_get_narrow_plan": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(C.c_longlong)]),
    "cp_engine_set_split_mode": (_i, [_vp, _i]),
    "cp_engine_set_hps_force_exact": (_i, [_vp, _i]),
    "cp_engine_get_split_mode": (_i, [_vp]),
    "cp_ckks_modulus_raising": (_i, [_vp, _vp, _vp, _i, _vp, _vp]),
    "cp_ckks_modulus_reduction": (_i, [_vp, _vp, _vp, _i, _vp, _vp]),
    "cp_ckks_rescale": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cp_ckks_batch_workspace_bytes": (C.c_size_t, [_vp, _i]),
    "cp_ckks_modulus_raising_batch": (_i, [_vp, _vp, _vp, _i, _i, _vp, _vp]),
    "cp_ckks_modulus_reduction_batch": (_i, [_vp, _vp, _vp, _i, _i, _vp, _vp]),
    "cp_ckks_rescale_batch": (_i, [_vp, _vp, _i, _i, _vp]),
    "cp_ckks_xi": (_i, [_vp, _vp, _vp, _vp]),
    "cp_ckks_rho": (_i, [_vp, _vp, _vp, _vp]),
    "cp_engine_destroy": (_i, [_vp]),
    "cp_engine_n_residues": (_i, [_vp, _i]),
    "cp_engine_nphi": (_i, [_vp]),
    "cp_engine_primes": (_i, [_vp, _pu64, _i]),
    "cp_engine_set_nthroot": (_i, [_vp, _pu64]),
    "cp_engine_get_nthroot": (_i, [_vp, _pu64]),
    "cp_workspace_bytes": (C.c_size_t, [_vp]),
    "cp_engine_check": (_i, [_vp, _vp]),
    "cp_dgt": (_i, [_vp, _vp, _i, _i, _i, _i64, _vp]),
    "cp_dgt_list": (_i, [_vp, _vp, _vp, _i, _i, _vp]),
    "cp_mul_list": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "cp_polymul_workspace_bytes": (C.c_size_t, [_vp, _i, _i]),
    "cp_polymul": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "cp_polymul_list": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "cp_polymul_tiles_workspace_bytes": (C.c_size_t, []),
    "cp_polymul_tiles": (_i, [C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                              C.POINTER(_i), _vp, _i, _vp, C.c_size_t, _vp]),
    "cp_add": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "cp_sub": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "cp_double_add": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "cp_mul": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "cp_mul_u64": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "cp_mul_batch": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp]),
    "cp_muladd": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "cp_dot": (_i, [_vp, _vp, C.POINTER(_vp), C.POINTER(_vp), _i, _i, _vp]),
    "cp_dot_batch": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _vp]),
    "cp_dr2": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "cp_negate": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cp_op_by_int": (_i, [_vp, _vp, _vp, _i, _u64, _i, _vp]),
    "cp_double_op_by_int": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _u64, _u64, _i, _vp]),
    "cp_basis_ext_q_to_b": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cp_basis_ext_b_to_q": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cp_complex_scaling": (_i, [_vp, _vp, _vp, _vp, _i, _vp]),
    "cp_simple_scaling": (_i, [_vp, _vp, _vp, _vp]),
    "cp_xi": (_i, [_vp, _vp, _vp, _vp]),
    "cp_rho": (_i, [_vp, _vp, _vp, _vp]),
    "cp_xi_batch": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cp_rho_batch": (_i, [_vp, _vp, _vp, _i, _vp]),
    "cp_poly_basis_extension_q_to_b": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cp_poly_basis_extension_q_to_qb": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cp_poly_basis_extension_b_to_q": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cp_poly_complex_scaling_tdivq": (_i, [_vp, _vp, _vp, _vp, C.c_uint, _vp, _vp]),
    "cp_poly_simple_scaling_tdivq": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "cp_bfv_mul": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cp_bfv_mul_noalloc": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "cp_bfv_mul_batch_workspace_bytes": (C.c_size_t, [_vp, _i]),
    "cp_bfv_mul_batch": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp]),
    "cp_calibrate_int": (_i, [_i, _i, _vp, C.c_longlong, C.POINTER(C.c_float), _vp]),
    "cp_modarith_eval": (_i, [_i, _vp, _vp, _vp, _vp, C.c_longlong, C.c_uint64, _vp]),
    "cp_crt": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp]),
    "cp_icrt": (_i, [_vp, _vp, _i, _vp, _i, _i, _vp]),
    "cp_wire_bytes": (C.c_size_t, [_vp, _i, _i]),
    "cp_export_residues": (_i, [_vp, _vp, C.c_size_t, _vp, _i, _i, _i, _vp]),
    "cp_import_residues": (_i, [_vp, _vp, _vp, C.c_size_t, _i, _i, C.POINTER(_i), _vp]),
    "cp_sample": (_i, [_vp, _vp, _i, _i, _u64, _u32, _i, _i, _vp]),
    "cp_sample_ids": (_i, [_vp, _vp, _i, _i, _u64, _vp, _i, _i, _vp]),
}

_LIB = None


def header_functions(path: str = HEADER_PATH):
    """Names of every function the C header declares."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cp_[a-z0-9_]+)\s*\(", src)))


def lib() -> C.CDLL:
    """Load (once) and return the shared library with typed signatures."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("cupoly_b200 native library not built: %s (run python -m cupoly_b200.build)" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def check(fn: str, code: int) -> int:
    if code != CP_OK:
        msg = lib().cp_last_error().decode(errors="replace")
        raise CupolyError(fn, code, msg)
    return code


def call(fn: str, *args) -> int:
    return check(fn, getattr(lib(), fn)(*args))
