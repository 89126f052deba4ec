"""Serving loop: scheduler logic on the CPU (fake executor) and, on the GPU,
results that are bit-identical alone and in the mix."""
import time

import numpy as np
import pytest

from cupoly_b200.serving import FakeExecutor, Request, Scheduler, SizeClass, default_classes, poisson_requests


def _classes():
    return [SizeClass(4096, 2, 3, 256, 4), SizeClass(8192, 4, 5, 256, 3)]


def test_scheduler_completes_everything_in_order_of_constraints():
    cls = _classes()
    ex = FakeExecutor(lambda c, b: 0.002 + 0.0005 * b)
    sch = Scheduler(cls, ex, budget_bytes=10 ** 12)
    reqs = sch.run(poisson_requests(200, 20000.0, len(cls), seed=3))
    assert all(r.done >= r.admit >= r.arrival for r in reqs)
    assert len({r.rid for r in reqs}) == 200
    for c, pool_idx, rids in ex.launched:
        assert 1 <= len(rids) <= cls[c].max_batch
        assert all(reqs[i].cls == c for i in rids)
    launched = sorted(rid for _, _, rids in ex.launched for rid in rids)
    assert launched == list(range(200))  # every request in exactly one batch
    st = sch.stats(reqs)
    assert st["p99_ms"] >= st["p50_ms"] > 0


def test_requests_join_batches_while_others_run():
    """Continuous batching: a class keeps up to max_inflight batches on the device
    and new arrivals fill the next pool meanwhile."""
    cls = [SizeClass(4096, 2, 3, 256, 8)]
    ex = FakeExecutor(lambda c, b: 0.02)
    sch = Scheduler(cls, ex, budget_bytes=10 ** 12, max_inflight=2)
    reqs = [Request(i, 0, 0.001 * i) for i in range(40)]
    sch.run(reqs)
    sizes = sch.batch_sizes
    assert sizes[0] == 1 and sizes[1] == 1  # idle GPU: launch at once
    assert max(sizes) > 1  # later arrivals batched while two batches run
    assert sum(sizes) == 40


def test_admission_respects_memory_budget():
    cls = _classes()
    budget = 3 * cls[1].request_bytes()
    ex = FakeExecutor(lambda c, b: 0.001)
    sch = Scheduler(cls, ex, budget_bytes=budget)
    reqs = sch.run(poisson_requests(60, 50000.0, len(cls), seed=5))
    assert sch.peak_used <= budget
    assert all(r.done > 0 for r in reqs)
    with pytest.raises(ValueError):
        Scheduler(cls, ex, budget_bytes=cls[0].request_bytes() - 1)


def test_default_classes_follow_k_equals_nphi_over_2048():
    for c in default_classes():
        assert c.k == c.nphi // 2048 and c.kl == c.k + 1 and c.t == 256


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix(gpu):
    import torch

    from cupoly_b200.serving import GpuExecutor

    cls = _classes()
    ex = GpuExecutor(cls, keep_results=True)
    sch = Scheduler(cls, ex, budget_bytes=8 << 30)
    reqs = sch.run(poisson_requests(48, 50000.0, len(cls), seed=9))
    assert max(sch.batch_sizes) > 1  # some requests really shared batches
    for r in reqs:
        alone = ex.run_alone(r.cls, r.rid)
        assert torch.equal(alone, ex.results[r.rid]), r


@pytest.mark.gpu
def test_served_result_matches_oracle(gpu):
    """One request per class: operands re-derived by the oracle's sampler restatement."""
    from cupoly_b200.engine import INVERSE, to_u64
    from cupoly_b200.serving import GpuExecutor
    from oracle import coracle
    from oracle import pyoracle as O
    from tests.common import unfold

    cls = [SizeClass(64, 2, 3, 256, 2), SizeClass(128, 3, 4, 65537, 2)]
    ex = GpuExecutor(cls, keep_results=True, seed=77)
    sch = Scheduler(cls, ex, budget_bytes=1 << 30)
    reqs = sch.run([Request(0, 0, 0.0), Request(1, 1, 0.0), Request(2, 0, 0.0)])
    for r in reqs:
        c = cls[r.cls]
        e = ex.engines[r.cls]
        ops = [np.array(O.sample_poly(O.UNIFORM, e.Q, c.nphi, 4 * r.rid + v, 77), dtype=np.uint64)[None]
               for v in range(4)]
        ref = coracle.bfv_mul(*ops, e.Q, e.B, c.t)
        got = ex.results[r.rid].clone()
        e.dgt(got, 0, INVERSE)
        got = unfold(to_u64(got))
        for j in range(3):
            assert np.array_equal(got[j], ref[j][0])


class _Flaky(FakeExecutor):
    """Fake executor whose launch / poll / finish raise for chosen batches (by launch order)."""

    def __init__(self, delay, fail_launch=(), fail_poll=(), fail_finish=()):
        super().__init__(delay)
        self.fail = {"launch": set(fail_launch), "poll": set(fail_poll), "finish": set(fail_finish)}
        self.count = 0
        self.batch_of = {}

    def launch(self, c, pool):
        i = self.count
        self.count += 1
        if i in self.fail["launch"]:
            raise RuntimeError("injected launch failure (CUDA out of memory)")
        h = super().launch(c, pool)
        self.batch_of[pool.index, c] = i
        return (i, h)

    def poll(self, handle):
        i, h = handle
        if i in self.fail["poll"]:
            raise RuntimeError("injected poll failure")
        return super().poll(h)

    def finish(self, pool):
        if self.batch_of[pool.index, pool.cls] in self.fail["finish"]:
            raise RuntimeError("injected kernel error flag")


def test_executor_failures_fail_only_their_batch():
    """A launch, poll or finish error ends that batch's requests as failed, frees their
    budget and leaves the loop serving everyone else."""
    cls = [SizeClass(4096, 2, 3, 256, 4)]
    ex = _Flaky(lambda c, b: 0.001, fail_launch=[1], fail_poll=[3], fail_finish=[5])
    sch = Scheduler(cls, ex, budget_bytes=10 ** 12, max_inflight=1)
    reqs = sch.run([Request(i, 0, 0.0005 * i) for i in range(80)])
    st = sch.stats(reqs)
    assert st["failed_batches"] == 3 and st["failed"] > 0
    assert st["failed"] + st["completed"] == 80
    assert all(r.status in ("done", "failed") for r in reqs)
    assert all(r.error for r in reqs if r.status == "failed")
    assert sch.used == 0  # every reservation returned
    assert {r.error.split(":")[0] for r in reqs if r.status == "failed"} == {"launch", "poll", "finish"}


def test_malformed_and_cancelled_requests():
    """A request naming no size class is rejected on arrival; one cancelled before its
    batch launches never reaches the executor; one cancelled after launch completes as
    cancelled; the budget is whole again at the end."""
    cls = [SizeClass(4096, 2, 3, 256, 4)]
    reqs = [Request(i, 0, 0.0002 * i) for i in range(30)]
    reqs[3].cls = 9
    reqs[5].cancelled = True
    reqs[6].cancelled = True

    class CancelOnLaunch(FakeExecutor):
        def launch(self, c, pool):
            for r in pool.reqs:
                if r.rid == 20:
                    r.cancelled = True  # the client gives up while its batch runs
            return super().launch(c, pool)

    ex = CancelOnLaunch(lambda c, b: 0.002)
    sch = Scheduler(cls, ex, budget_bytes=10 ** 12)
    out = {r.rid: r for r in sch.run(reqs)}
    assert out[3].status == "rejected" and "size class" in out[3].error
    assert out[5].status == out[6].status == "cancelled"
    launched = {rid for _, _, rids in ex.launched for rid in rids}
    assert 5 not in launched and 6 not in launched and 3 not in launched
    assert 20 in launched and out[20].status == "cancelled"
    assert sum(r.status == "done" for r in out.values()) == 26
    assert sch.used == 0


def test_queue_timeout_rejects_requests_that_wait_too_long():
    cls = [SizeClass(4096, 2, 3, 256, 1)]
    ex = FakeExecutor(lambda c, b: 0.01)
    budget = cls[0].request_bytes()  # one request at a time
    sch = Scheduler(cls, ex, budget_bytes=budget, max_inflight=1, queue_timeout_s=0.025)
    reqs = sch.run([Request(i, 0, 0.0) for i in range(10)])
    st = sch.stats(reqs)
    assert st["rejected"] > 0 and st["completed"] >= 2
    assert all(r.error == "queue timeout" for r in reqs if r.status == "rejected")
    assert sch.peak_used <= budget and sch.used == 0


@pytest.mark.gpu
def test_error_flag_copy_follows_the_batch(gpu):
    """cp_engine_check_async copies the engine's (clear) error flag behind queued work into
    pinned memory; the executor's batches carry it, and a clear flag passes finish()."""
    import torch

    from cupoly_b200.engine import QBase, UNIFORM, Engine
    from cupoly_b200.serving import GpuExecutor

    e = Engine(2, 0, 4096, 256)
    flag = torch.full((1,), 7, dtype=torch.int32).pin_memory()
    x = e.empty(QBase, 4)
    s = torch.cuda.Stream()
    e.sample(x, QBase, UNIFORM, 1, 0, npolys=4, to_dgt=True, stream=s)
    e.check_async(flag, stream=s)
    s.synchronize()
    assert int(flag[0]) == 0
    cls = _classes()
    ex = GpuExecutor(cls)
    sch = Scheduler(cls, ex, budget_bytes=1 << 30)
    reqs = sch.run([Request(i, i % len(cls), 0.0) for i in range(6)])
    assert all(r.status == "done" for r in reqs)
    assert all(int(b["flag_h"][0]) == 0 for bs in ex.pool_bufs for b in bs)
