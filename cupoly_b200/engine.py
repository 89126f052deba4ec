"""Engine objects over the C ABI, with device buffers held in torch tensors.

``Engine`` is one (nphi, k, kl, t) parameter set with its own device tables;
any number of engines coexist (cuPoly allows one per process).  Buffers are
int64 tensors of shape ``(npolys, nres, N, 2)`` whose bytes are cuPoly's
GaussianInteger layout (the bit patterns are uint64 residues).  torch is
used only for device memory and streams; every computation is a call into
``libcupoly_b200.so``.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import call

QBase, BBase, QBBase, TBase = 0, 1, 2, 3
FORWARD, INVERSE = 0, 1
ADD, SUB, MUL, MULMUL, ADDADD = 0, 1, 2, 3, 4
(DISCRETE_GAUSSIAN, HAMMINGWEIGHT, NARROW, ZO, BINARY, UNIFORM, TERNARY, GAUSSIAN) = range(8)
UNIFORM_U32, ZO_HALF = 9, 10  # cuPoly's BFV UNIFORM and ZO (enum cp_distribution)
DESTROY_INPUTS = 1


def _ptr(t: Optional[torch.Tensor]):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def to_u64(t: torch.Tensor) -> np.ndarray:
    """Copy a device buffer to a host numpy uint64 array of the same shape."""
    return t.detach().cpu().numpy().view(np.uint64)


def from_u64(a: np.ndarray, device="cuda") -> torch.Tensor:
    """Copy a host uint64 array to a device int64 tensor (same bytes)."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64)).to(device)


def ints_to_limbs(values, nlimbs: int) -> np.ndarray:
    """Non-negative Python ints -> (len, nlimbs) uint64 limbs, least significant first."""
    nbytes = 8 * nlimbs
    buf = b"".join(int(v).to_bytes(nbytes, "little") for v in values)
    return np.frombuffer(buf, dtype=np.uint64).reshape(len(values), nlimbs).copy()


def limbs_to_ints(limbs: np.ndarray) -> List[int]:
    """(n, nlimbs) uint64 limbs -> Python ints."""
    a = np.ascontiguousarray(limbs, dtype=np.uint64)
    raw = a.tobytes()
    w = 8 * a.shape[-1]
    return [int.from_bytes(raw[i * w:(i + 1) * w], "little") for i in range(a.shape[0])]


def int_peaks(iters: int = 256, waves: int = 8, stream=None) -> dict:
    """Measured peak rates (operations/s) of the modular primitives on the current GPU.

    Keys: shoup (constant multiply), mulmod (data x data product), addmod,
    imad32.  Each is timed on one kernel that fills every SM `waves` times.
    """
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    nthreads = props.multi_processor_count * waves * 256
    sink = torch.empty(nthreads, dtype=torch.int64, device="cuda")
    out = {}
    for kind, name in enumerate(("shoup", "mulmod", "addmod", "imad32")):
        ms = C.c_float()
        call("cp_calibrate_int", kind, iters, _ptr(sink), nthreads, C.byref(ms), _stream(stream))  # warm-up
        call("cp_calibrate_int", kind, iters, _ptr(sink), nthreads, C.byref(ms), _stream(stream))
        out[name] = 8.0 * iters * nthreads / (ms.value / 1e3)
    return out


def dgt_op_counts(N: int) -> dict:
    """Algorithmic integer work of one residue-transform of N Gaussian elements.

    Shoup constant multiplies: 2 per non-trivial radix-2 twiddle
    (N/2 log2 N - N + 1 of them) plus 3 per element for the Gaussian twist
    (Karatsuba form); modular adds/subs: 4 per radix-2 butterfly plus 2 per
    element for the twist.
    """
    lg = N.bit_length() - 1
    return {"shoup": 2 * (N // 2 * lg - N + 1) + 3 * N, "addmod": 2 * N * lg + 2 * N}


class Engine:
    """One parameter set: ring degree nphi, |Q| = k, |B| = kl, plaintext modulus t."""

    def __init__(self, k: int, kl: int = 0, nphi: int = 4096, t: int = 256, log_radix: int = 0,
                 ckks_prec: int = 0):
        """BFV engine (63-bit primes, plaintext modulus t), or with ckks_prec in
        {45, 48, 52, 55} a CKKS engine (cuPoly's CKKS build; t unused)."""
        if not torch.cuda.is_available():
            raise RuntimeError("cupoly_b200 needs a CUDA device")
        _lib.lib()
        log_cta, split_mode, narrow = 0, 0, None
        if log_radix == 0:  # use the autotuner's plans for this GPU and size when cached
            from .autotune import cached_narrow_plan, cached_plan, cached_split_mode

            log_radix, log_cta = cached_plan(nphi)
            split_mode = cached_split_mode(nphi)
            if log_radix:  # a tuned entry replaces the library's default small-launch plan
                narrow = cached_narrow_plan(nphi)
        h = C.c_void_p()
        if ckks_prec:
            call("cp_ckks_engine_create", C.byref(h), k, kl, nphi, ckks_prec, log_radix)
            t = 2
        else:
            call("cp_engine_create", C.byref(h), k, kl, nphi, t, log_radix)
        self.ckks_prec = ckks_prec
        if log_cta:
            call("cp_engine_set_plan", h, log_radix, log_cta)
        if split_mode:
            call("cp_engine_set_split_mode", h, split_mode)
        if narrow is not None:
            call("cp_engine_set_narrow_plan", h, narrow[0], narrow[1], narrow[2])
        self.log_radix = log_radix
        self._h = h
        self.k = k
        self.kl = kl if kl > 0 else k + 1
        self.nphi = nphi
        self.N = nphi // 2
        self.t = t
        buf = (C.c_uint64 * (self.k + self.kl))()
        _lib.lib().cp_engine_primes(h, buf, self.k + self.kl)
        self.primes: List[int] = [int(x) for x in buf]
        self.Q = self.primes[: self.k]
        self.B = self.primes[self.k:]
        self._wsbuf: Optional[torch.Tensor] = None
        self.device = torch.cuda.current_device()

    # ---- DGT plan ----
    def set_plan(self, log_radix: int, log_cta: int = 0):
        """Register radix 2^log_radix and in-CTA size 2^log_cta (0: 2^13); rebuilds the tables."""
        call("cp_engine_set_plan", self._h, log_radix, log_cta)
        self.log_radix = log_radix

    def set_split_mode(self, mode: int):
        """0: split stage as its own kernel (HBM pass); 1: inside a thread-block cluster (DSMEM)."""
        call("cp_engine_set_split_mode", self._h, int(mode))

    def set_hps_force_exact(self, on: bool):
        """Diagnostic: every base conversion and scaling takes its exact path (same results)."""
        call("cp_engine_set_hps_force_exact", self._h, 1 if on else 0)

    def get_split_mode(self) -> int:
        return int(_lib.lib().cp_engine_get_split_mode(self._h))

    def set_narrow_plan(self, log_radix: int, log_cta: int, max_units: int):
        """Plan for launches of at most max_units residue transforms (0 removes it); rebuilds the tables."""
        call("cp_engine_set_narrow_plan", self._h, log_radix, log_cta, int(max_units))

    def get_narrow_plan(self):
        r, c, u = C.c_int(), C.c_int(), C.c_longlong()
        call("cp_engine_get_narrow_plan", self._h, C.byref(r), C.byref(c), C.byref(u))
        return {"log_radix": r.value, "log_cta": c.value, "max_units": u.value}

    def get_plan(self):
        r, c, s = C.c_int(), C.c_int(), C.c_int()
        call("cp_engine_get_plan", self._h, C.byref(r), C.byref(c), C.byref(s))
        return {"log_radix": r.value, "log_cta": c.value, "split_bits": s.value}

    # ---- lifecycle ----
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().cp_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def n_residues(self, base: int) -> int:
        return {QBase: self.k, BBase: self.kl, QBBase: self.k + self.kl, TBase: 1}[base]

    def base_primes(self, base: int) -> List[int]:
        return {QBase: self.Q, BBase: self.B, QBBase: self.primes, TBase: [self.t]}[base]

    # ---- argument checks (every device buffer is checked before its pointer crosses the C ABI) ----
    def _buf(self, t, base: int, npolys: int = 1, name: str = "buffer", words: int = 2):
        """Pointer of t after checking that it is a contiguous int64 tensor on this engine's
        device holding at least npolys polynomials over base (`words` 64-bit words per
        element: 2 for Gaussian residues, 1 for cp_mul_u64's multipliers)."""
        if not isinstance(t, torch.Tensor):
            raise TypeError("%s must be a torch tensor" % name)
        if t.dtype != torch.int64 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("%s must be a contiguous int64 CUDA tensor" % name)
        if t.device.index != self.device:
            raise ValueError("%s is on cuda:%s, the engine on cuda:%d" % (name, t.device.index, self.device))
        need = int(npolys) * self.n_residues(base) * self.N * words
        if npolys < 1 or t.numel() < need:
            raise ValueError("%s holds %d words, %d polynomials over base %d need %d"
                             % (name, t.numel(), npolys, base, need))
        return C.c_void_p(t.data_ptr())

    def _bufs(self, base: int, npolys: int = 1, **bufs):
        """_buf of each keyword argument, in order."""
        return [self._buf(t, base, npolys, name) for name, t in bufs.items()]

    def _ws(self, t, nbytes: int, name: str = "workspace"):
        """Pointer of a device workspace after checking it holds nbytes bytes."""
        if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
            raise ValueError("%s must be a contiguous CUDA tensor" % name)
        if t.device.index != self.device:
            raise ValueError("%s is on cuda:%s, the engine on cuda:%d" % (name, t.device.index, self.device))
        if t.numel() * t.element_size() < nbytes:
            raise ValueError("%s holds %d bytes, the call needs %d" % (name, t.numel() * t.element_size(), nbytes))
        return C.c_void_p(t.data_ptr())

    # ---- memory ----
    def empty(self, base: int = QBase, npolys: int = 1) -> torch.Tensor:
        return torch.empty((npolys, self.n_residues(base), self.N, 2), dtype=torch.int64, device="cuda")

    def zeros(self, base: int = QBase, npolys: int = 1) -> torch.Tensor:
        return torch.zeros((npolys, self.n_residues(base), self.N, 2), dtype=torch.int64, device="cuda")

    def workspace(self) -> torch.Tensor:
        if self._wsbuf is None:
            n = _lib.lib().cp_workspace_bytes(self._h)
            self._wsbuf = torch.empty(((n + 15) // 16, 2), dtype=torch.int64, device="cuda")
        return self._wsbuf

    # ---- roots ----
    def set_nthroot(self, xi: Sequence[Sequence[int]]):
        arr = (C.c_uint64 * (2 * len(xi)))(*[int(v) for pair in xi for v in pair])
        call("cp_engine_set_nthroot", self._h, arr)

    def get_nthroot(self):
        n = self.k + self.kl
        arr = (C.c_uint64 * (2 * n))()
        call("cp_engine_get_nthroot", self._h, arr)
        return [(int(arr[2 * i]), int(arr[2 * i + 1])) for i in range(n)]

    def check(self, stream=None):
        call("cp_engine_check", self._h, _stream(stream))

    def check_async(self, flag_host: torch.Tensor, stream=None):
        """Queue a copy of the engine's error flag into flag_host (a pinned int32 tensor) on the stream."""
        call("cp_engine_check_async", self._h, _ptr(flag_host), _stream(stream))

    # ---- DGT ----
    def dgt(self, x: torch.Tensor, base: int, direction: int, npolys: Optional[int] = None, stream=None):
        n = x.shape[0] if npolys is None else npolys
        call("cp_dgt", self._h, self._buf(x, base, n, "x"), base, direction, n, 0, _stream(stream))
        return x

    # ---- pointwise ----
    def add(self, c, a, b, base, stream=None):
        call("cp_add", self._h, *self._bufs(base, c=c, a=a, b=b), base, _stream(stream))

    def sub(self, c, a, b, base, stream=None):
        call("cp_sub", self._h, *self._bufs(base, c=c, a=a, b=b), base, _stream(stream))

    def double_add(self, c1, a1, b1, c2, a2, b2, base, stream=None):
        call("cp_double_add", self._h, *self._bufs(base, c1=c1, a1=a1, b1=b1, c2=c2, a2=a2, b2=b2), base,
             _stream(stream))

    def mul(self, c, a, b, base, stream=None):
        call("cp_mul", self._h, *self._bufs(base, c=c, a=a, b=b), base, _stream(stream))

    def polymul_workspace(self, base: int, npolys: int) -> torch.Tensor:
        n = _lib.lib().cp_polymul_workspace_bytes(self._h, base, npolys)
        return torch.empty(((n + 15) // 16, 2), dtype=torch.int64, device="cuda")

    def polymul(self, c, a, b, base, workspace, npolys=None, stream=None):
        """c = a b mod (x^nphi + 1) per residue, coefficient domain in and out (fused: 3 launches)."""
        n = c.shape[0] if npolys is None else npolys
        ws = self._ws(workspace, _lib.lib().cp_polymul_workspace_bytes(self._h, base, n))
        call("cp_polymul", self._h, *self._bufs(base, n, c=c, a=a, b=b), base, n, ws, _stream(stream))

    def mul_batch(self, c, a, b, base, npolys=None, stream=None):
        n = c.shape[0] if npolys is None else npolys
        call("cp_mul_batch", self._h, *self._bufs(base, n, c=c, a=a, b=b), base, n, _stream(stream))

    def mul_u64(self, c, a, b, base, stream=None):
        call("cp_mul_u64", self._h, *self._bufs(base, c=c, a=a), self._buf(b, base, 1, "b", words=1), base,
             _stream(stream))

    def muladd(self, d, a, b, c, base, stream=None):
        call("cp_muladd", self._h, *self._bufs(base, d=d, a=a, b=b, c=c), base, _stream(stream))

    def dot(self, c, a, b, base, stream=None):
        """c = sum_i a[i] b[i] in the DGT domain, one pass (cuPoly's poly_dot).

        ``a`` and ``b`` are equal-length sequences of residue tensors over ``base``.
        """
        if len(a) != len(b) or not a:
            raise ValueError("dot: a and b must be non-empty and of equal length")
        n = len(a)
        pa = (C.c_void_p * n)(*[self._buf(x, base, 1, "a[%d]" % i) for i, x in enumerate(a)])
        pb = (C.c_void_p * n)(*[self._buf(x, base, 1, "b[%d]" % i) for i, x in enumerate(b)])
        call("cp_dot", self._h, self._buf(c, base, 1, "c"), pa, pb, n, base, _stream(stream))

    def dot_batch(self, c, a, b, n, npolys, base, b_shared=False, stream=None):
        """Polynomial q of c = sum_{t<n} a[q n + t] b[q n + t] (b[t] when b_shared), one launch."""
        pc = self._buf(c, base, npolys, "c")
        pa = self._buf(a, base, n * npolys, "a")
        pb = self._buf(b, base, n if b_shared else n * npolys, "b")
        call("cp_dot_batch", self._h, pc, pa, pb, n, npolys, 1 if b_shared else 0, base, _stream(stream))

    def dr2(self, c21, c22, c23, c01, c02, c11, c12, base, stream=None):
        call("cp_dr2", self._h, *self._bufs(base, c21=c21, c22=c22, c23=c23, c01=c01, c02=c02, c11=c11, c12=c12),
             base, _stream(stream))

    def negate(self, b, a, base, stream=None):
        call("cp_negate", self._h, *self._bufs(base, b=b, a=a), base, _stream(stream))

    def op_by_int(self, b, a, base, x, op, stream=None):
        call("cp_op_by_int", self._h, *self._bufs(base, b=b, a=a), base, int(x), op, _stream(stream))

    def double_op_by_int(self, b1, a1, b2, a2, base, x1, x2, op, stream=None):
        call("cp_double_op_by_int", self._h, *self._bufs(base, b1=b1, a1=a1, b2=b2, a2=a2), base, int(x1), int(x2),
             op, _stream(stream))

    # ---- CKKS (CKKS engines) ----
    @classmethod
    def ckks(cls, k: int, kl: int, nphi: int, prec: int, log_radix: int = 0) -> "Engine":
        return cls(k, kl, nphi, 2, log_radix, ckks_prec=prec)

    def ckks_modulus_raising(self, out_qb, in_q, level: int, stream=None):
        call("cp_ckks_modulus_raising", self._h, self._buf(out_qb, QBBase, 1, "out_qb"), self._buf(in_q, QBase, 1, "in_q"),
             level, _ptr(self.workspace()), _stream(stream))

    def ckks_modulus_reduction(self, out_q, in_qb, level: int, stream=None):
        call("cp_ckks_modulus_reduction", self._h, self._buf(out_q, QBase, 1, "out_q"),
             self._buf(in_qb, QBBase, 1, "in_qb"), level, _ptr(self.workspace()), _stream(stream))

    def ckks_rescale(self, a, b, level: int, stream=None):
        pb = self._buf(b, QBase, 1, "b") if b is not None else _ptr(None)
        call("cp_ckks_rescale", self._h, self._buf(a, QBase, 1, "a"), pb, level, _stream(stream))

    def ckks_batch_workspace(self, npolys: int) -> torch.Tensor:
        n = int(_lib.lib().cp_ckks_batch_workspace_bytes(self._h, npolys))
        return torch.empty(max(1, n // 8), dtype=torch.int64, device="cuda")

    def ckks_modulus_raising_batch(self, out_qb, in_q, level: int, workspace, npolys=None, stream=None):
        n = in_q.shape[0] if npolys is None else npolys
        ws = self._ws(workspace, _lib.lib().cp_ckks_batch_workspace_bytes(self._h, n))
        call("cp_ckks_modulus_raising_batch", self._h, self._buf(out_qb, QBBase, n, "out_qb"),
             self._buf(in_q, QBase, n, "in_q"), level, n, ws, _stream(stream))

    def ckks_modulus_reduction_batch(self, out_q, in_qb, level: int, workspace, npolys=None, stream=None):
        n = in_qb.shape[0] if npolys is None else npolys
        ws = self._ws(workspace, _lib.lib().cp_ckks_batch_workspace_bytes(self._h, n))
        call("cp_ckks_modulus_reduction_batch", self._h, self._buf(out_q, QBase, n, "out_q"),
             self._buf(in_qb, QBBase, n, "in_qb"), level, n, ws, _stream(stream))

    def ckks_rescale_batch(self, x, level: int, npolys=None, stream=None):
        n = x.shape[0] if npolys is None else npolys
        call("cp_ckks_rescale_batch", self._h, self._buf(x, QBase, n, "x"), n, level, _stream(stream))

    def ckks_xi(self, out, a, stream=None):
        call("cp_ckks_xi", self._h, *self._bufs(QBase, out=out, a=a), _stream(stream))

    def ckks_rho(self, out, a, stream=None):
        call("cp_ckks_rho", self._h, *self._bufs(QBase, out=out, a=a), _stream(stream))

    # ---- coefficient I/O (big integers <-> residues, on the device) ----
    def crt(self, out, coefs_limbs: torch.Tensor, base: int = QBase, stream=None):
        """Residues of big-integer coefficients: coefs_limbs is (npolys, nphi, nlimbs) int64 (uint64 limbs)."""
        npolys, nphi, nlimbs = coefs_limbs.shape
        if nphi != self.nphi or coefs_limbs.dtype != torch.int64 or not coefs_limbs.is_contiguous():
            raise ValueError("crt: coefs_limbs must be a contiguous int64 (npolys, nphi, nlimbs) tensor")
        call("cp_crt", self._h, self._buf(out, base, npolys, "out"), _ptr(coefs_limbs), nlimbs, base, npolys,
             _stream(stream))
        return out

    def icrt(self, coefs_limbs: torch.Tensor, x, base: int = QBase, stream=None):
        """Big-integer coefficients in [0, prod of the base) from coefficient-domain residues."""
        npolys, nphi, nlimbs = coefs_limbs.shape
        if nphi != self.nphi or coefs_limbs.dtype != torch.int64 or not coefs_limbs.is_contiguous():
            raise ValueError("icrt: coefs_limbs must be a contiguous int64 (npolys, nphi, nlimbs) tensor")
        call("cp_icrt", self._h, _ptr(coefs_limbs), nlimbs, self._buf(x, base, npolys, "x"), base, npolys,
             _stream(stream))
        return coefs_limbs

    def wire_bytes(self, base: int, npolys: int = 1) -> int:
        return int(_lib.lib().cp_wire_bytes(self._h, base, npolys))

    def export_residues(self, x, base: int, domain: int, stream=None, out: Optional[np.ndarray] = None):
        """Binary wire form of x (npolys, nres, N, 2); domain 0 coefficient, 1 DGT.  Returns
        bytes, or fills and returns `out` (a uint8 array of wire_bytes, e.g. reused or pinned
        host memory, which avoids the allocation and the copy into a bytes object)."""
        n = self.wire_bytes(base, x.shape[0])
        if out is not None:
            if out.dtype != np.uint8 or out.size < n or not out.flags["C_CONTIGUOUS"]:
                raise ValueError("export_residues: out must be a contiguous uint8 array of wire_bytes")
            call("cp_export_residues", self._h, C.c_void_p(out.ctypes.data), out.size,
                 self._buf(x, base, x.shape[0], "x"), base, x.shape[0], domain, _stream(stream))
            return out
        buf = C.create_string_buffer(n)
        call("cp_export_residues", self._h, buf, n, self._buf(x, base, x.shape[0], "x"), base, x.shape[0], domain,
             _stream(stream))
        return buf.raw

    def import_residues(self, x, data, base: int, stream=None) -> int:
        """Fill x (npolys, nres, N, 2) from the wire form (bytes or a uint8 array); returns the
        recorded domain."""
        dom = C.c_int(-1)
        if isinstance(data, np.ndarray):
            src, size = C.c_void_p(np.ascontiguousarray(data).ctypes.data), data.size
        else:
            src, size = data, len(data)
        call("cp_import_residues", self._h, self._buf(x, base, x.shape[0], "x"), src, size, base, x.shape[0],
             C.byref(dom), _stream(stream))
        return dom.value

    # ---- HPS (coefficient domain) ----
    def basis_ext_q_to_b(self, out_b, in_q, npolys=1, stream=None):
        call("cp_basis_ext_q_to_b", self._h, self._buf(out_b, BBase, npolys, "out_b"),
             self._buf(in_q, QBase, npolys, "in_q"), npolys, _stream(stream))

    def basis_ext_b_to_q(self, out_q, in_b, npolys=1, stream=None):
        call("cp_basis_ext_b_to_q", self._h, self._buf(out_q, QBase, npolys, "out_q"),
             self._buf(in_b, BBase, npolys, "in_b"), npolys, _stream(stream))

    def complex_scaling(self, out_b, in_q, in_b, npolys=1, stream=None):
        call("cp_complex_scaling", self._h, self._buf(out_b, BBase, npolys, "out_b"),
             self._buf(in_q, QBase, npolys, "in_q"), self._buf(in_b, BBase, npolys, "in_b"), npolys, _stream(stream))

    def simple_scaling(self, out_t, in_q, stream=None):
        call("cp_simple_scaling", self._h, self._buf(out_t, TBase, 1, "out_t"), self._buf(in_q, QBase, 1, "in_q"),
             _stream(stream))

    def xi(self, out, a, stream=None):
        call("cp_xi", self._h, self._buf(out, QBase, self.k, "out"), self._buf(a, QBase, 1, "a"), _stream(stream))

    def xi_batch(self, out, a, npolys=None, stream=None):
        """out (npolys * k, k, N, 2): the xi decomposition of each of the npolys polynomials of a."""
        n = a.shape[0] if npolys is None else npolys
        call("cp_xi_batch", self._h, self._buf(out, QBase, n * self.k, "out"), self._buf(a, QBase, n, "a"), n,
             _stream(stream))

    def rho_batch(self, out, a, npolys=None, stream=None):
        n = a.shape[0] if npolys is None else npolys
        call("cp_rho_batch", self._h, self._buf(out, QBase, n * self.k, "out"), self._buf(a, QBase, n, "a"), n,
             _stream(stream))

    def rho(self, out, a, stream=None):
        call("cp_rho", self._h, self._buf(out, QBase, self.k, "out"), self._buf(a, QBase, 1, "a"), _stream(stream))

    # ---- composite (DGT domain) ----
    def poly_basis_extension_q_to_b(self, out_b, in_q, stream=None):
        call("cp_poly_basis_extension_q_to_b", self._h, self._buf(out_b, BBase, 1, "out_b"),
             self._buf(in_q, QBase, 1, "in_q"), _ptr(self.workspace()), _stream(stream))

    def poly_basis_extension_q_to_qb(self, out_qb, in_q, stream=None):
        call("cp_poly_basis_extension_q_to_qb", self._h, self._buf(out_qb, QBBase, 1, "out_qb"),
             self._buf(in_q, QBase, 1, "in_q"), _ptr(self.workspace()), _stream(stream))

    def poly_basis_extension_b_to_q(self, out_q, in_b, stream=None):
        call("cp_poly_basis_extension_b_to_q", self._h, self._buf(out_q, QBase, 1, "out_q"),
             self._buf(in_b, BBase, 1, "in_b"), _ptr(self.workspace()), _stream(stream))

    def poly_complex_scaling_tdivq(self, out_q, in_q, in_b, flags=0, stream=None):
        call("cp_poly_complex_scaling_tdivq", self._h, self._buf(out_q, QBase, 1, "out_q"),
             self._buf(in_q, QBase, 1, "in_q"), self._buf(in_b, BBase, 1, "in_b"), flags, _ptr(self.workspace()),
             _stream(stream))

    def poly_simple_scaling_tdivq(self, out_t, in_q, stream=None):
        call("cp_poly_simple_scaling_tdivq", self._h, self._buf(out_t, TBase, 1, "out_t"),
             self._buf(in_q, QBase, 1, "in_q"), _ptr(self.workspace()), _stream(stream))

    def bfv_mul(self, c0, c1, c2, a0, a1, b0, b1, stream=None):
        call("cp_bfv_mul", self._h, *self._bufs(QBase, c0=c0, c1=c1, c2=c2, a0=a0, a1=a1, b0=b0, b1=b1),
             _ptr(self.workspace()), _stream(stream))

    def bfv_mul_batch_workspace(self, npairs: int) -> torch.Tensor:
        n = _lib.lib().cp_bfv_mul_batch_workspace_bytes(self._h, npairs)
        return torch.empty(((n + 15) // 16, 2), dtype=torch.int64, device="cuda")

    def bfv_mul_batch(self, c, a0, a1, b0, b1, npairs, workspace, stream=None):
        """c: (3 * npairs, k, N, 2); inputs (npairs, k, N, 2), all DGT domain."""
        ws = self._ws(workspace, _lib.lib().cp_bfv_mul_batch_workspace_bytes(self._h, npairs))
        call("cp_bfv_mul_batch", self._h, self._buf(c, QBase, 3 * npairs, "c"),
             *self._bufs(QBase, npairs, a0=a0, a1=a1, b0=b0, b1=b1), npairs, ws, _stream(stream))

    # ---- sampler ----
    def sample(self, out, base, kind, seed, stream_id, npolys=None, to_dgt=True, stream=None):
        n = out.shape[0] if npolys is None else npolys
        call("cp_sample", self._h, self._buf(out, base, n, "out"), base, kind, int(seed), int(stream_id), n,
             1 if to_dgt else 0, _stream(stream))

    def sample_ids(self, out, base, kind, seed, stream_ids: torch.Tensor, to_dgt=True, stream=None):
        """Polynomial i of `out` drawn with stream id stream_ids[i] (int32 device tensor)."""
        if stream_ids.dtype != torch.int32 or not stream_ids.is_cuda or not stream_ids.is_contiguous():
            raise ValueError("sample_ids: stream_ids must be a contiguous int32 CUDA tensor")
        n = int(stream_ids.numel())
        call("cp_sample_ids", self._h, self._buf(out, base, n, "out"), base, kind, int(seed), _ptr(stream_ids), n,
             1 if to_dgt else 0, _stream(stream))

    # ---- host helpers (folded layout) ----
    def fold(self, coeffs_per_residue: np.ndarray) -> np.ndarray:
        """(nres, nphi) uint64 coefficient rows -> (nres, N, 2) folded layout."""
        a = np.asarray(coeffs_per_residue, dtype=np.uint64)
        return np.stack([a[:, : self.N], a[:, self.N:]], axis=-1)

    def unfold(self, x: np.ndarray) -> np.ndarray:
        """(..., nres, N, 2) folded -> (..., nres, nphi) coefficient rows."""
        return np.concatenate([x[..., 0], x[..., 1]], axis=-1)
