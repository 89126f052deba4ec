"""Serving loop: continuous batching of homomorphic multiplications of mixed sizes.

A request asks for one BFV multiplication (two ciphertexts -> three output
polynomials) at one of several ring sizes.  The server keeps one engine per
size class (its DGT/HPS tables resident in HBM) and a few preallocated batch
*pools* per class.  The host loop

  * admits arrived requests into the filling pool of their class while the
    memory budget allows (each admitted request reserves its operand, result
    and workspace bytes until it completes);
  * launches a pool as one batched call (operands sampled on the device from
    the request's identity, then the fused BFV chain) as soon as it is full or
    its class has fewer than `max_inflight` batches on the GPU -- so requests
    that arrive while others run join the next batch, and batches of different
    classes (and up to `max_inflight` of one class) overlap on separate
    streams;
  * completes requests when their batch's event fires and frees their budget.

The scheduler is host logic with a pluggable executor; `GpuExecutor` runs the
batches through the C ABI, `FakeExecutor` (tests) completes them on a timer.

Failures end requests, never the loop: a request naming no size class is
rejected on arrival; one cancelled before its batch launches leaves the queue or
its pool (its budget returns at once), one cancelled later completes as
cancelled; one that waits in its queue longer than `queue_timeout_s` is
rejected; an executor error at launch, poll or finish (a CUDA or ABI error, a
kernel's error flag) fails that batch's requests, frees their budget and
returns the pool to service.
"""
from __future__ import annotations

import argparse
import collections
import json
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np


@dataclass
class SizeClass:
    nphi: int
    k: int
    kl: int
    t: int
    max_batch: int

    def request_bytes(self) -> int:
        """Device bytes one admitted request holds: 4 operands + 3 results over Q
        and its share of the batch workspace ((7k + 10kl) N per pair)."""
        N = self.nphi // 2
        return (4 * self.k + 3 * self.k + 7 * self.k + 10 * self.kl) * N * 16


def default_classes(max_batches=(256, 128, 64, 32), t=256) -> List[SizeClass]:
    """nphi in {4096, 8192, 16384, 32768} with k = nphi / 2048, kl = k + 1."""
    return [SizeClass(n, n // 2048, n // 2048 + 1, t, b) for n, b in zip((4096, 8192, 16384, 32768), max_batches)]


@dataclass
class Request:
    rid: int
    cls: int
    arrival: float
    admit: float = -1.0
    done: float = -1.0
    slot: int = -1
    pool: int = -1
    status: str = "pending"  # -> done | failed | cancelled | rejected
    error: str = ""
    cancelled: bool = False  # set by the client at any time; honoured before launch, result dropped after

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class Pool:
    cls: int
    index: int
    capacity: int
    reqs: List[Request] = field(default_factory=list)
    busy: bool = False
    handle: object = None


class Scheduler:
    def __init__(self, classes: Sequence[SizeClass], executor, budget_bytes: int, pools_per_class: int = 3,
                 max_inflight: int = 2, queue_timeout_s: Optional[float] = None):
        self.classes = list(classes)
        self.ex = executor
        self.budget = int(budget_bytes)
        self.used = 0
        self.peak_used = 0
        self.max_inflight = max_inflight
        self.queue_timeout = queue_timeout_s
        self.pools: List[List[Pool]] = [[Pool(c, i, cl.max_batch) for i in range(pools_per_class)]
                                        for c, cl in enumerate(self.classes)]
        self.batches = 0
        self.batch_sizes: List[int] = []
        self.failed_batches = 0
        for cl in self.classes:
            if cl.request_bytes() > self.budget:
                raise ValueError("budget smaller than one request of nphi=%d" % cl.nphi)

    def _inflight(self, c: int) -> int:
        return sum(1 for p in self.pools[c] if p.busy)

    def _filling(self, c: int) -> Optional[Pool]:
        """The pool new requests of class c go to: a partly filled idle pool first."""
        idle = [p for p in self.pools[c] if not p.busy]
        for p in idle:
            if p.reqs:
                return p
        return idle[0] if idle else None

    def _end(self, r: Request, status: str, t: float, error: str = "") -> None:
        r.status, r.done, r.error = status, t, error

    def _release(self, pool: Pool, status: str, t: float, error: str = "") -> int:
        """End every request of `pool`, free their budget, return the pool to service."""
        rb = self.classes[pool.cls].request_bytes()
        for r in pool.reqs:
            self._end(r, "cancelled" if (status == "done" and r.cancelled) else status, t, error)
            self.used -= rb
        n = len(pool.reqs)
        pool.reqs, pool.busy, pool.handle = [], False, None
        return n

    def _launch(self, c: int, pool: Pool, t: float) -> int:
        """Launch `pool` after dropping its cancelled requests; returns how many requests ended."""
        ended = 0
        keep = [r for r in pool.reqs if not r.cancelled]
        if len(keep) != len(pool.reqs):
            rb = self.classes[c].request_bytes()
            for r in pool.reqs:
                if r.cancelled:
                    self._end(r, "cancelled", t)
                    self.used -= rb
                    ended += 1
            for i, r in enumerate(keep):
                r.slot = i
            pool.reqs = keep
        if not pool.reqs:
            return ended
        try:
            pool.handle = self.ex.launch(c, pool)
        except Exception as exc:  # noqa: BLE001 -- any executor error fails this batch only
            self.failed_batches += 1
            return ended + self._release(pool, "failed", t, "launch: %s" % exc)
        pool.busy = True
        self.batches += 1
        self.batch_sizes.append(len(pool.reqs))
        return ended

    def run(self, requests: Sequence[Request], clock=time.perf_counter, time_limit_s: float = 600.0):
        """Serve `requests` (arrival times relative to start); returns them, each ended
        with a status (done, failed, cancelled or rejected)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        queues = [collections.deque() for _ in self.classes]
        n, nxt, done = len(reqs), 0, 0
        t0 = clock()
        while done < n:
            now = clock() - t0
            if now > time_limit_s:
                raise TimeoutError("serving loop exceeded %.0f s" % time_limit_s)
            progressed = False
            while nxt < n and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                nxt += 1
                progressed = True
                if not (isinstance(r.cls, int) and 0 <= r.cls < len(self.classes)):
                    self._end(r, "rejected", now, "unknown size class %r" % (r.cls,))
                    done += 1
                else:
                    queues[r.cls].append(r)
            # completions
            for c in range(len(self.classes)):
                for p in self.pools[c]:
                    if not p.busy:
                        continue
                    try:
                        ready = self.ex.poll(p.handle)
                    except Exception as exc:  # noqa: BLE001
                        self.failed_batches += 1
                        done += self._release(p, "failed", clock() - t0, "poll: %s" % exc)
                        progressed = True
                        continue
                    if ready:
                        t_done = clock() - t0
                        try:
                            self.ex.finish(p)
                        except Exception as exc:  # noqa: BLE001
                            self.failed_batches += 1
                            done += self._release(p, "failed", t_done, "finish: %s" % exc)
                        else:
                            done += self._release(p, "done", t_done)
                        progressed = True
            # queue hygiene: cancellations and queue timeouts end requests before admission
            for q in queues:
                if any(r.cancelled or (self.queue_timeout is not None and now - r.arrival > self.queue_timeout)
                       for r in q):
                    kept = collections.deque()
                    for r in q:
                        if r.cancelled:
                            self._end(r, "cancelled", now)
                            done += 1
                        elif self.queue_timeout is not None and now - r.arrival > self.queue_timeout:
                            self._end(r, "rejected", now, "queue timeout")
                            done += 1
                        else:
                            kept.append(r)
                    q.clear()
                    q.extend(kept)
                    progressed = True
            # admission and launch
            for c, cl in enumerate(self.classes):
                q = queues[c]
                while q:
                    pool = self._filling(c)
                    if pool is None:
                        break
                    rb = cl.request_bytes()
                    while q and len(pool.reqs) < pool.capacity and self.used + rb <= self.budget:
                        r = q.popleft()
                        r.admit, r.slot, r.pool = now, len(pool.reqs), pool.index
                        pool.reqs.append(r)
                        self.used += rb
                        progressed = True
                    self.peak_used = max(self.peak_used, self.used)
                    if pool.reqs and (len(pool.reqs) == pool.capacity or self._inflight(c) < self.max_inflight):
                        done += self._launch(c, pool, now)
                        progressed = True
                    else:
                        break
                # a filling pool left partly full launches once an in-flight batch finishes
                pool = self._filling(c)
                if pool is not None and pool.reqs and self._inflight(c) < self.max_inflight:
                    done += self._launch(c, pool, now)
                    progressed = True
            if not progressed:
                busy = any(p.busy for ps in self.pools for p in ps)
                if not busy and nxt < n and all(not q for q in queues):
                    wait = reqs[nxt].arrival - (clock() - t0)
                    if wait > 5e-4:  # sleep, waking 0.3 ms early; spin through the rest (a
                        time.sleep(min(wait - 3e-4, 0.01))  # sleep overshoots by tens of us)
        return reqs

    def stats(self, reqs: Sequence[Request]) -> Dict:
        ok = [r for r in reqs if r.status == "done"]
        lat = np.array([r.latency for r in ok]) * 1e3 if ok else np.zeros(1)
        span = (max(r.done for r in ok) - min(r.arrival for r in ok)) if ok else float("inf")
        counts = collections.Counter(r.status for r in reqs)
        return {"requests": len(reqs), "completed": len(ok), "throughput_req_s": round(len(ok) / span, 1),
                "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "max_ms": round(float(lat.max()), 3), "batches": self.batches,
                "mean_batch": round(float(np.mean(self.batch_sizes)), 2) if self.batch_sizes else 0,
                "failed": counts.get("failed", 0), "cancelled": counts.get("cancelled", 0),
                "rejected": counts.get("rejected", 0), "failed_batches": self.failed_batches,
                "peak_budget_bytes": self.peak_used, "budget_bytes": self.budget}


def poisson_requests(n: int, rate: float, nclasses: int, seed: int) -> List[Request]:
    """Open-loop Poisson arrivals at `rate` req/s; size class uniform; seeded."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    cls = rng.integers(0, nclasses, size=n)
    t = np.cumsum(gaps)
    return [Request(i, int(c), float(a)) for i, (c, a) in enumerate(zip(cls, t))]


class FakeExecutor:
    """Completes a batch `delay(c, size)` seconds after launch (scheduler tests)."""

    def __init__(self, delay, clock=time.perf_counter):
        self.delay = delay
        self.clock = clock
        self.launched = []

    def launch(self, c, pool):
        self.launched.append((c, pool.index, [r.rid for r in pool.reqs]))
        return self.clock() + self.delay(c, len(pool.reqs))

    def poll(self, handle):
        return self.clock() >= handle

    def finish(self, pool):
        pass


class GpuExecutor:
    """Runs batches on the device: operands sampled from each request's identity
    (stream ids 4 rid + v under one seed, uniform mod q_i, DGT domain), then the
    fused BFV chain (`cp_bfv_mul_batch`).  One CUDA stream per pool."""

    def __init__(self, classes: Sequence[SizeClass], pools_per_class: int = 3, seed: int = 0xC0FFEE,
                 keep_results: bool = False):
        import torch

        from .engine import Engine

        self.torch = torch
        self.seed = seed
        self.keep = keep_results
        self.results: Dict[int, "torch.Tensor"] = {}
        self.engines, self.pool_bufs = [], []
        for cl in classes:
            e = Engine(cl.k, cl.kl, cl.nphi, cl.t)
            self.engines.append(e)
            bufs = []
            for _ in range(pools_per_class):
                bufs.append({
                    "ins": [e.empty(0, cl.max_batch) for _ in range(4)],
                    "out": e.empty(0, 3 * cl.max_batch),
                    "ws": e.bfv_mul_batch_workspace(cl.max_batch),
                    "ids_d": torch.empty(4 * cl.max_batch, dtype=torch.int32, device="cuda"),
                    "ids_h": torch.empty(4 * cl.max_batch, dtype=torch.int32).pin_memory(),
                    "stream": torch.cuda.Stream(),
                    "flag_h": torch.zeros(1, dtype=torch.int32).pin_memory(),
                })
            self.pool_bufs.append(bufs)
        torch.cuda.synchronize()
        # A batch of one request (the common case below saturation) replays a CUDA graph of
        # its 12 launches (4 operand samples, the chain), captured once per pool.
        for c, e in enumerate(self.engines):
            for b in self.pool_bufs[c]:
                s = b["stream"]
                with torch.cuda.stream(s):
                    b["ids_d"][:4].zero_()
                    self._enqueue(e, b, 1, s)  # warm-up outside the capture
                s.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=s):
                    self._enqueue(e, b, 1, s)
                b["graph1"] = g
        torch.cuda.synchronize()

    def _enqueue(self, e, b, B, s):
        from .engine import QBase, UNIFORM

        for v in range(4):
            e.sample_ids(b["ins"][v], QBase, UNIFORM, self.seed, b["ids_d"][v * B:(v + 1) * B], stream=s)
        e.bfv_mul_batch(b["out"], *b["ins"], B, b["ws"], stream=s)

    def launch(self, c, pool):
        torch = self.torch
        e, b = self.engines[c], self.pool_bufs[c][pool.index]
        B = len(pool.reqs)
        ids = np.array([[4 * r.rid + v for r in pool.reqs] for v in range(4)], dtype=np.int64).astype(np.uint32)
        b["ids_h"][: 4 * B].copy_(torch.from_numpy(ids.reshape(-1).view(np.int32)))
        s = b["stream"]
        with torch.cuda.stream(s):
            b["ids_d"][: 4 * B].copy_(b["ids_h"][: 4 * B], non_blocking=True)
            if B == 1:
                b["graph1"].replay()
            else:
                self._enqueue(e, b, B, s)
            e.check_async(b["flag_h"], stream=s)  # the error flag follows the batch to the host
            ev = torch.cuda.Event()
            ev.record(s)
        return ev

    def poll(self, ev):
        return ev.query()

    def finish(self, pool):
        # a kernel's error flag (e.g. a sampler rejection limit) fails the batch; the flag was
        # copied behind the batch, so a clear flag needs no device round trip
        b = self.pool_bufs[pool.cls][pool.index]
        if int(b["flag_h"][0]) != 0:
            self.engines[pool.cls].check(b["stream"])  # raises with the message, resets the flag
        if not self.keep:
            return
        b = self.pool_bufs[pool.cls][pool.index]
        B = len(pool.reqs)
        for r in pool.reqs:
            self.results[r.rid] = self.torch.stack([b["out"][j * B + r.slot] for j in range(3)]).clone()

    def run_alone(self, c: int, rid: int):
        """The result of request `rid` computed in a batch of its own."""
        pool = Pool(c, 0, 1, [Request(rid, c, 0.0, slot=0, pool=0)])
        ev = self.launch(c, pool)
        ev.synchronize()
        b = self.pool_bufs[c][0]
        return self.torch.stack([b["out"][j] for j in range(3)]).clone()


def main():
    ap = argparse.ArgumentParser(description="BFV serving loop: open-loop Poisson arrivals of mixed sizes")
    ap.add_argument("--requests", type=int, default=50000)
    ap.add_argument("--rates", default="auto",
                    help="comma-separated req/s, or 'auto': fractions 0.25..1.1 of the measured saturation")
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args()
    classes = default_classes()
    ex = GpuExecutor(classes)
    out = []
    if a.rates == "auto":
        sch = Scheduler(classes, ex, int(a.budget_gb * 2 ** 30))
        sat = sch.stats(sch.run(poisson_requests(a.requests, 1e9, len(classes), a.seed)))["throughput_req_s"]
        print(json.dumps({"saturated_req_s": sat}), flush=True)
        rates = [f * sat for f in (0.25, 0.5, 0.75, 0.9, 1.0, 1.1)]
    else:
        rates = [float(x) for x in a.rates.split(",")]
    for rate in rates:
        sch = Scheduler(classes, ex, int(a.budget_gb * 2 ** 30))
        reqs = sch.run(poisson_requests(a.requests, rate, len(classes), a.seed))
        st = sch.stats(reqs)
        st["rate_req_s"] = rate
        out.append(st)
        print(json.dumps(st), flush=True)
    return out


if __name__ == "__main__":
    main()
