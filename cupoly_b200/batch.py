"""Batched forms under CUDA graphs.

`MixedPolymul`: many independent negacyclic products c_i = a_i b_i in
Z_q[x]/(x^nphi_i + 1) with per-instance ring size nphi_i and RNS width k_i.
Instances are grouped by ring size; inside a group every residue of every
instance is one entry of a work list (data pointer implied by its position,
prime index = its residue number), and one fused `cp_polymul_list` serves the
whole group whatever the mix of widths: an out-of-place forward DGT per
operand and an inverse DGT that forms the products while loading.  All
groups' launches are captured once in a CUDA graph and replayed (in sequence,
or as one parallel branch per size group).  mode="tiles" runs the whole batch
as ONE persistent launch instead (cp_polymul_tiles): one CTA per SM walks a
device work list of same-size tiles, each residue's forward transforms,
product and inverse done in shared memory in one pass over HBM.

`BFVBatch`: the fused BFV multiplication chain over a fixed batch of pairs,
captured in a CUDA graph.

`PipelinedBFV`, `PipelinedPolymul`: consecutive device-resident batches with two
in flight on two streams; `StreamedBFV`: batches in host memory, copies
overlapped with the chain.
"""
from __future__ import annotations

import ctypes as C
from collections import OrderedDict
from typing import List, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .engine import FORWARD, INVERSE, QBase, Engine, _ptr, _stream, from_u64, to_u64
from ._lib import call


TILE_SIZES = (2048, 4096, 8192, 16384)  # ring sizes of the single-launch form (N = 2^10 .. 2^13)


class MixedPolymul:
    def __init__(self, specs: Sequence[Tuple[int, int]], kmax: int = 8, autotune: bool = False,
                 mode: str = "graph"):
        """specs[i] = (nphi_i, k_i) with 1 <= k_i <= kmax.

        mode "graph": per size group one fused cp_polymul_list (3 launches) with the
        group engine's tuned plan, all captured in one CUDA graph (see capture);
        mode "tiles": the whole batch in ONE persistent launch (cp_polymul_tiles) over
        a device work list of same-size tiles; every size must be in TILE_SIZES."""
        if mode not in ("graph", "tiles"):
            raise ValueError("mode must be 'graph' or 'tiles'")
        self.mode = mode
        self.specs = list(specs)
        self.groups = OrderedDict()  # nphi -> dict
        for i, (nphi, k) in enumerate(self.specs):
            if not 1 <= k <= kmax:
                raise ValueError("k must be in [1, kmax]")
            if mode == "tiles" and nphi not in TILE_SIZES:
                raise ValueError("the single-launch form covers nphi in %s" % (TILE_SIZES,))
            self.groups.setdefault(nphi, {"inst": []})["inst"].append(i)
        self.where = {}  # instance -> (nphi, first residue row)
        for nphi, g in self.groups.items():
            lr = 0
            lc = 0
            if mode == "tiles":  # the tile kernel's plan: radix 8, the whole transform in one CTA
                lr, lc = 3, (nphi // 2).bit_length() - 1
            elif autotune:
                from .autotune import best_plan

                lr, lc = best_plan(nphi)
            g["engine"] = Engine(kmax, 1, nphi, 256, lr)
            if lc:
                g["engine"].set_plan(lr, lc)
            rids, row = [], 0
            for i in g["inst"]:
                k = self.specs[i][1]
                self.where[i] = (nphi, row)
                rids.extend(range(k))
                row += k
            g["rows"] = row
            g["rid"] = torch.tensor(rids, dtype=torch.int32, device="cuda")
            N = nphi // 2
            g["a"] = torch.zeros((row, N, 2), dtype=torch.int64, device="cuda")
            g["b"] = torch.zeros_like(g["a"])
            g["wa"] = torch.empty_like(g["a"])
            g["wb"] = torch.empty_like(g["a"])
            g["c"] = torch.empty_like(g["a"])
        self.graph = None
        if mode == "tiles":
            self._build_tiles()

    def _build_tiles(self):
        """The device work list: each size group's rows cut into tiles of 8192 / N
        rows, largest transforms first (they take longest per tile)."""
        rows = []
        for lg, nphi in reversed(list(enumerate(TILE_SIZES))):
            g = self.groups.get(nphi)
            if g is None:
                continue
            per = 16384 // nphi
            rows += [(lg, r0, min(per, g["rows"] - r0)) for r0 in range(0, g["rows"], per)]
        self.ntiles = len(rows)
        self.tiles = torch.tensor(rows, dtype=torch.int32, device="cuda").reshape(-1, 3)
        L = _lib.lib()
        self.tile_ws = torch.empty(((L.cp_polymul_tiles_workspace_bytes() + 15) // 16, 2), dtype=torch.int64,
                                   device="cuda")
        vp = C.c_void_p
        self._tile_args = [(vp * 4)() for _ in range(5)]
        self._tile_rows = (C.c_int * 4)()
        eng, cc, aa, bb, rr = self._tile_args
        for lg, nphi in enumerate(TILE_SIZES):
            g = self.groups.get(nphi)
            if g is None:
                continue
            eng[lg] = g["engine"].handle
            cc[lg], aa[lg], bb[lg], rr[lg] = (g[x].data_ptr() for x in ("c", "a", "b", "rid"))
            self._tile_rows[lg] = g["rows"]

    # ---- data ----
    def set_inputs(self, i: int, a_rows: np.ndarray, b_rows: np.ndarray):
        """Coefficient rows (k_i, nphi_i), residues mod the first k_i primes."""
        nphi, row = self.where[i]
        k = self.specs[i][1]
        g = self.groups[nphi]
        N = nphi // 2
        for dst, src in ((g["a"], a_rows), (g["b"], b_rows)):
            src = np.asarray(src, dtype=np.uint64)
            dst[row:row + k] = from_u64(np.stack([src[:, :N], src[:, N:]], axis=-1))

    def result(self, i: int) -> np.ndarray:
        nphi, row = self.where[i]
        k = self.specs[i][1]
        x = to_u64(self.groups[nphi]["c"][row:row + k])
        return np.concatenate([x[..., 0], x[..., 1]], axis=-1)

    # ---- execution ----
    def _launch_group(self, g, stream):
        # fused: 2 out-of-place forward DGTs, inverse with products on load
        e, n, rid = g["engine"], g["rows"], g["rid"]
        call("cp_polymul_list", e.handle, _ptr(g["c"]), _ptr(g["a"]), _ptr(g["b"]), _ptr(g["wa"]),
             _ptr(g["wb"]), _ptr(rid), n, _stream(stream))

    def _launch(self, stream=None):
        if self.mode == "tiles":
            eng, cc, aa, bb, rr = self._tile_args
            call("cp_polymul_tiles", eng, cc, aa, bb, rr, self._tile_rows, _ptr(self.tiles), self.ntiles,
                 _ptr(self.tile_ws), self.tile_ws.numel() * 8, _stream(stream))
            return
        for g in self.groups.values():
            self._launch_group(g, stream)

    def _launch_branches(self, stream):
        """Every size group on a stream of its own, forked from and joined back into
        `stream`: in a captured graph the groups become parallel branches, so one
        group's last partial wave of CTAs overlaps the others' launches."""
        if self.mode == "tiles":
            raise ValueError("the single-launch form has no per-group branches")
        if not hasattr(self, "_branch_streams"):
            self._branch_streams = [torch.cuda.Stream() for _ in self.groups]
        for g, bs in zip(self.groups.values(), self._branch_streams):
            bs.wait_stream(stream)
            self._launch_group(g, bs)
        for bs in self._branch_streams:
            stream.wait_stream(bs)

    def run(self):
        """Eager execution (also warms up every kernel before capture)."""
        self._launch()

    def capture(self, branches: bool = False):
        """Capture every group's launches in one CUDA graph: in sequence on one
        stream, or (branches=True) as one parallel branch per size group."""
        self._launch()  # first launches set kernel attributes outside the capture
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(self.graph, stream=s):
                if branches:
                    self._launch_branches(s)
                else:
                    self._launch(stream=s)
        torch.cuda.current_stream().wait_stream(s)
        return self.graph

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def launches_per_run(self) -> int:
        return 1 if self.mode == "tiles" else 3 * len(self.groups)

    def algorithmic_bytes(self) -> int:
        """24 nphi k bytes per product: read a, b and write c (16 B per Gaussian element)."""
        return sum(24 * nphi * k for nphi, k in self.specs)


class BFVBatch:
    """Fused BFV multiplication of a fixed batch of pairs, captured in a CUDA graph."""

    def __init__(self, engine: Engine, npairs: int):
        self.e = engine
        self.P = npairs
        self.ins = [engine.empty(QBase, npairs) for _ in range(4)]
        self.out = engine.empty(QBase, 3 * npairs)
        self.ws = engine.bfv_mul_batch_workspace(npairs)
        self.graph = None

    def _launch(self, stream=None):
        self.e.bfv_mul_batch(self.out, *self.ins, self.P, self.ws, stream=stream)

    def capture(self):
        self._launch()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(self.graph, stream=s):
                self._launch(stream=s)
        torch.cuda.current_stream().wait_stream(s)

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()


def _check_tensor(x: torch.Tensor, shape, what: str):
    """Refuse a tensor the batched kernels would read or write past: they take
    raw pointers and the batch's polynomial count."""
    if tuple(x.shape) != tuple(shape) or x.dtype != torch.int64 or not x.is_contiguous() or not x.is_cuda:
        raise ValueError("%s must be a contiguous int64 CUDA tensor of shape %s, got %s %s%s" %
                         (what, tuple(shape), x.dtype, tuple(x.shape), "" if x.is_contiguous() else " (strided)"))


class PipelinedBFV:
    """BFV multiplication of consecutive device-resident batches, `lanes` of them in flight.

    Batch i runs on stream i mod lanes with that lane's workspace.  Each chain
    launch ends in a partial wave of CTAs; with two batches in flight the other
    batch's launches fill those SMs (on B200, nphi 8192, k 5, 128 pairs: 2.035
    instead of 2.159 ms per batch; neutral at nphi 16384, k 10, 32 pairs, and 5 %
    slower at nphi 32768, k 16, 64 pairs).  Results are those of one cp_bfv_mul_batch
    call per batch.  The outputs of batches in flight at the same time (i and
    i + 1, ..., i + lanes - 1) must be distinct tensors.
    """

    def __init__(self, engine: Engine, npairs: int, lanes: int = 2):
        self.e = engine
        self.P = npairs
        self.lanes = lanes
        self.ws = [engine.bfv_mul_batch_workspace(npairs) for _ in range(lanes)]
        self.streams = [torch.cuda.Stream() for _ in range(lanes)]

    def run(self, batches, outputs, stream=None):
        """batches[i] = (a0, a1, b0, b1): npairs polynomials each, DGT domain, on the
        device; outputs[i] (3 npairs polynomials) receives its result.  The work is
        ordered after what `stream` (default: the current stream) has queued."""
        if len(batches) != len(outputs):
            raise ValueError("PipelinedBFV.run: %d batches but %d outputs" % (len(batches), len(outputs)))
        shape = (self.P, self.e.k, self.e.N, 2)
        for ins, out in zip(batches, outputs):
            if len(ins) != 4:
                raise ValueError("PipelinedBFV.run: a batch is (a0, a1, b0, b1)")
            for x in ins:
                _check_tensor(x, shape, "input")
            _check_tensor(out, (3 * self.P,) + shape[1:], "output")
        cur = stream if stream is not None else torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(cur)
        for i, (ins, out) in enumerate(zip(batches, outputs)):
            j = i % self.lanes
            # The caller's tensors are used on a lane stream: keep the caching
            # allocator from reusing their memory until that stream is done.
            for x in (*ins, out):
                x.record_stream(self.streams[j])
            self.e.bfv_mul_batch(out, *ins, self.P, self.ws[j], stream=self.streams[j])

    def join(self, stream=None):
        """Make `stream` (default: the current stream) wait for every batch issued so far."""
        cur = stream if stream is not None else torch.cuda.current_stream()
        for s in self.streams:
            cur.wait_stream(s)


class PipelinedPolymul:
    """Fused negacyclic products (cp_polymul, coefficient domain in and out) of
    consecutive device-resident batches, `lanes` of them in flight on as many
    streams, each lane with its own workspace (on B200, nphi 4096, k 2, 1024
    products: 305 instead of 339 us per batch).  Results are those of one
    cp_polymul call per batch.  The outputs of batches in flight at the same
    time must be distinct tensors."""

    def __init__(self, engine: Engine, base: int, npolys: int, lanes: int = 2):
        self.e = engine
        self.base = base
        self.P = npolys
        self.lanes = lanes
        self.ws = [engine.polymul_workspace(base, npolys) for _ in range(lanes)]
        self.streams = [torch.cuda.Stream() for _ in range(lanes)]

    def run(self, batches, outputs, stream=None):
        """batches[i] = (a, b), npolys polynomials each; outputs[i] receives a b.

        Every a, b and output must hold exactly npolys contiguous polynomials of
        the base (a short final batch needs its own PipelinedPolymul): the kernels
        read and write npolys polynomials whatever the tensors hold."""
        if len(batches) != len(outputs):
            raise ValueError("PipelinedPolymul.run: %d batches but %d outputs" % (len(batches), len(outputs)))
        shape = (self.P, self.e.n_residues(self.base), self.e.N, 2)
        for (a, b), out in zip(batches, outputs):
            for x, what in ((a, "a"), (b, "b"), (out, "output")):
                _check_tensor(x, shape, what)
        cur = stream if stream is not None else torch.cuda.current_stream()
        for s in self.streams:
            s.wait_stream(cur)
        for i, ((a, b), out) in enumerate(zip(batches, outputs)):
            j = i % self.lanes
            for x in (a, b, out):
                x.record_stream(self.streams[j])
            self.e.polymul(out, a, b, self.base, self.ws[j], self.P, stream=self.streams[j])

    def join(self, stream=None):
        cur = stream if stream is not None else torch.cuda.current_stream()
        for s in self.streams:
            cur.wait_stream(s)


class StreamedBFV:
    """BFV multiplication of a stream of batches that live in host memory.

    Each batch is four pinned host tensors (npairs, k, N, 2) in the DGT domain and
    its result a pinned host tensor (3 npairs, k, N, 2).  Three CUDA streams run
    the host-to-device copy of batch i + 1, the chain on batch i and the
    device-to-host copy of batch i - 1 at the same time over `nbuf` device buffer
    sets, so throughput is bound by the slowest of the three instead of their
    sum.  A copy-in waits only for the chain that last read its input buffers,
    and a chain only for the copy-out that last read its output buffer.
    """

    def __init__(self, engine: Engine, npairs: int, nbuf: int = 3):
        self.e = engine
        self.P = npairs
        self.nbuf = nbuf
        self.bufs = [{"ins": [engine.empty(QBase, npairs) for _ in range(4)],
                      "out": engine.empty(QBase, 3 * npairs)} for _ in range(nbuf)]
        self.ws = engine.bfv_mul_batch_workspace(npairs)
        self.s_in, self.s_comp, self.s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        self.ev_in = [torch.cuda.Event() for _ in range(nbuf)]
        self.ev_comp = [torch.cuda.Event() for _ in range(nbuf)]
        self.ev_out = [torch.cuda.Event() for _ in range(nbuf)]

    def run(self, host_batches, host_outputs):
        """host_batches[i] = [a0, a1, b0, b1] (pinned); host_outputs[i] receives c."""
        for i, (hin, hout) in enumerate(zip(host_batches, host_outputs)):
            b = i % self.nbuf
            buf = self.bufs[b]
            reuse = i >= self.nbuf
            if reuse:  # input buffers of set b were last read by the chain of step i - nbuf
                self.s_in.wait_event(self.ev_comp[b])
            with torch.cuda.stream(self.s_in):
                for d, h in zip(buf["ins"], hin):
                    d.copy_(h, non_blocking=True)
                self.ev_in[b].record(self.s_in)
            self.s_comp.wait_event(self.ev_in[b])
            if reuse:  # output buffer of set b was last read by the copy-out of step i - nbuf
                self.s_comp.wait_event(self.ev_out[b])
            self.e.bfv_mul_batch(buf["out"], *buf["ins"], self.P, self.ws, stream=self.s_comp)
            self.ev_comp[b].record(self.s_comp)
            self.s_out.wait_event(self.ev_comp[b])
            with torch.cuda.stream(self.s_out):
                hout.copy_(buf["out"], non_blocking=True)
                self.ev_out[b].record(self.s_out)

    def join(self, stream):
        """Make `stream` wait for everything issued so far."""
        for s in (self.s_in, self.s_comp, self.s_out):
            stream.wait_stream(s)


def random_specs(n: int, seed: int, sizes=(2048, 4096, 8192, 16384), kmax: int = 8) -> List[Tuple[int, int]]:
    """n (nphi, k) draws: nphi uniform over `sizes`, k uniform in 1..kmax (seeded)."""
    rng = np.random.default_rng(seed)
    return [(int(sizes[rng.integers(len(sizes))]), int(rng.integers(1, kmax + 1))) for _ in range(n)]
