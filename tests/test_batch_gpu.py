"""Batched forms: mixed-size polymul work lists and graph-captured BFV batches,
bit-exact per instance against the plain per-call path and the oracle."""
import numpy as np
import pytest

from oracle import coracle as CO
from oracle import pyoracle as O
from tests.common import fold, random_poly_residues, unfold

pytestmark = pytest.mark.gpu


def _plain_polymul(nphi, k, a, b):
    from cupoly_b200.engine import FORWARD, INVERSE, Engine, from_u64, to_u64
    e = Engine(k, 0, nphi, 256)
    ta, tb = from_u64(fold(a)[None]), from_u64(fold(b)[None])
    e.dgt(ta, 0, FORWARD)
    e.dgt(tb, 0, FORWARD)
    tc = e.empty(0)
    e.mul(tc, ta, tb, 0)
    e.dgt(tc, 0, INVERSE)
    return unfold(to_u64(tc))[0]


def test_mixed_polymul_matches_plain_and_oracle(gpu):
    from cupoly_b200.batch import MixedPolymul, random_specs
    specs = random_specs(40, seed=3)
    mp = MixedPolymul(specs)
    data = []
    for i, (nphi, k) in enumerate(specs):
        a = random_poly_residues(1000 + i, O.PRIMES[:k], nphi)
        b = random_poly_residues(2000 + i, O.PRIMES[:k], nphi)
        mp.set_inputs(i, a, b)
        data.append((a, b))
    mp.run()
    for i, (nphi, k) in enumerate(specs):
        got = mp.result(i)
        a, b = data[i]
        assert np.array_equal(got, CO.polymul(a[None], b[None], O.PRIMES[:k])[0]), (i, nphi, k)
        if i < 8:
            assert np.array_equal(got, _plain_polymul(nphi, k, a, b))


def test_mixed_polymul_graph_replay_follows_inputs(gpu):
    import torch
    from cupoly_b200.batch import MixedPolymul
    specs = [(2048, 3), (4096, 1), (2048, 8), (16384, 2)]
    mp = MixedPolymul(specs)
    for rnd in range(2):
        for i, (nphi, k) in enumerate(specs):
            mp.set_inputs(i, random_poly_residues(7 * rnd + i, O.PRIMES[:k], nphi),
                          random_poly_residues(50 + 7 * rnd + i, O.PRIMES[:k], nphi))
        mp.replay()
        torch.cuda.synchronize()
        for i, (nphi, k) in enumerate(specs):
            a = random_poly_residues(7 * rnd + i, O.PRIMES[:k], nphi)
            b = random_poly_residues(50 + 7 * rnd + i, O.PRIMES[:k], nphi)
            assert np.array_equal(mp.result(i), CO.polymul(a[None], b[None], O.PRIMES[:k])[0])
    assert mp.launches_per_run() == 9  # one fused cp_polymul_list (3 launches) per size group


def test_bfv_batch_graph_equals_eager(gpu):
    import torch
    from cupoly_b200.batch import BFVBatch
    from cupoly_b200.engine import UNIFORM, Engine
    e = Engine(3, 4, 4096, 256)
    bb = BFVBatch(e, 5)
    for j, x in enumerate(bb.ins):
        e.sample(x, 0, UNIFORM, 9, 100 * j, npolys=5, to_dgt=True)
    eager = e.empty(0, 15)
    e.bfv_mul_batch(eager, *bb.ins, 5, e.bfv_mul_batch_workspace(5))
    bb.replay()
    torch.cuda.synchronize()
    assert torch.equal(bb.out, eager)


def test_autotuner_picks_a_candidate_and_caches(gpu, tmp_path, monkeypatch):
    import json
    monkeypatch.setenv("CUPOLY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    from cupoly_b200 import autotune
    from cupoly_b200.engine import Engine
    cands = autotune.candidates(16384)
    assert (3, 13) in cands and (3, 12) in cands           # radix and stage-split choices
    plan = autotune.best_plan(16384, residues=128, reps=2)
    assert plan in cands
    assert autotune.cached_plan(16384) == plan
    data = json.load(open(tmp_path / "tune.json"))
    ent = next(iter(data.values()))
    assert len(ent["ms_fwd_inv"]) == len(cands) + sum(1 for _, c in cands if c < 13)  # split plans: both forms
    assert ent["split_mode"] in (0, 1)
    e = Engine(2, 0, 16384, 256)                           # picks the cached plan up
    assert (e.get_plan()["log_radix"], e.get_plan()["log_cta"]) == plan


@pytest.mark.parametrize("nphi,plans", [(16384, [(3, 13), (3, 12), (4, 12), (2, 11)]),
                                        (32768, [(3, 13), (4, 13)]), (8192, [(3, 12), (3, 11), (4, 11)])])
def test_every_plan_gives_the_same_transform(gpu, nphi, plans):
    """Radix and stage split change the schedule, never the result: DGT-domain bytes and
    the round trip agree across plans (and with the oracle's restatement)."""
    import numpy as np

    from cupoly_b200.engine import FORWARD, INVERSE, Engine, from_u64, to_u64
    from oracle import coracle
    from tests.common import fold, random_poly_residues
    e = Engine(2, 0, nphi, 256)
    x = random_poly_residues(nphi, e.Q, nphi)
    ref = coracle.dgt(fold(x)[None], e.Q)
    for r, c in plans:
        e.set_plan(r, c)
        d = from_u64(fold(x)[None])
        e.dgt(d, 0, FORWARD)
        assert np.array_equal(to_u64(d), ref), (r, c, e.get_plan())
        e.dgt(d, 0, INVERSE)
        assert np.array_equal(to_u64(d)[0], fold(x)), (r, c)


def test_streamed_bfv_matches_device_batches(gpu):
    """Host-resident batches through StreamedBFV (copies and chain overlapped on three
    streams) give the same bytes as the device-resident batched call."""
    import torch

    from cupoly_b200.batch import StreamedBFV
    from cupoly_b200.engine import Engine, QBase, UNIFORM
    e = Engine(3, 0, 2048, 256)
    P, steps = 8, 5
    host_in, ref = [], []
    ws = e.bfv_mul_batch_workspace(P)
    for s in range(steps):
        ins = []
        for j in range(4):
            x = e.empty(QBase, P)
            e.sample(x, QBase, UNIFORM, 99 + s, 64 * j, npolys=P, to_dgt=True)
            ins.append(x)
        c = e.empty(QBase, 3 * P)
        e.bfv_mul_batch(c, *ins, P, ws)
        ref.append(c.cpu())
        host_in.append([x.cpu().pin_memory() for x in ins])
    outs = [torch.empty_like(r).pin_memory() for r in ref]
    sb = StreamedBFV(e, P)
    sb.run(host_in, outs)
    sb.join(torch.cuda.current_stream())
    torch.cuda.synchronize()
    for o, r in zip(outs, ref):
        assert torch.equal(o, r)


@pytest.mark.parametrize("nphi,plans", [(16384, [(3, 11), (3, 12)]), (32768, [(3, 12), (3, 13)]),
                                        (65536, [(3, 13)])])
def test_cluster_split_stage_gives_the_same_transform(gpu, nphi, plans):
    """The split stage inside a thread-block cluster (chunks exchanged through distributed
    shared memory) gives the bytes of the separate split kernel and of the oracle, forward
    and inverse, for 2- and 4-CTA clusters."""
    from cupoly_b200.engine import FORWARD, INVERSE, Engine, from_u64, to_u64
    from oracle import coracle
    e = Engine(2, 0, nphi, 256)
    x = random_poly_residues(nphi + 1, e.Q, nphi)
    ref = coracle.dgt(fold(x)[None], e.Q)
    for r, c in plans:
        e.set_plan(r, c)
        for mode in (1, 0):
            e.set_split_mode(mode)
            assert e.get_split_mode() == mode and e.get_plan()["split_bits"] > 0
            d = from_u64(fold(x)[None])
            e.dgt(d, 0, FORWARD)
            assert np.array_equal(to_u64(d), ref), (r, c, mode)
            e.dgt(d, 0, INVERSE)
            assert np.array_equal(to_u64(d)[0], fold(x)), (r, c, mode)


def test_cluster_split_stage_in_the_fused_calls(gpu):
    """The batched BFV chain (gather and tensor-product inverse DGTs) and the fused polymul
    (out-of-place forward, product-on-load inverse) give identical bytes in both split
    forms; the plans split 2 bits (nphi 16384, c11) and 1 bit (nphi 32768, c13)."""
    import torch

    from cupoly_b200.engine import QBase, UNIFORM, Engine
    for nphi, k, t, c in ((16384, 3, 256, 11), (32768, 2, 65537, 13)):
        e = Engine(k, 0, nphi, t)
        e.set_plan(3, c)
        P = 2
        ins = []
        for j in range(4):
            x = e.empty(QBase, P)
            e.sample(x, QBase, UNIFORM, 5, 16 * j, npolys=P, to_dgt=True)
            ins.append(x)
        ws = e.bfv_mul_batch_workspace(P)
        pws = e.polymul_workspace(QBase, P)
        out = {}
        for mode in (0, 1):
            e.set_split_mode(mode)
            c3 = e.empty(QBase, 3 * P)
            e.bfv_mul_batch(c3, *ins, P, ws)
            pm = e.empty(QBase, P)
            e.polymul(pm, ins[0], ins[1], QBase, pws, P)
            torch.cuda.synchronize()
            out[mode] = (c3.clone(), pm.clone())
        assert torch.equal(out[0][0], out[1][0]), nphi
        assert torch.equal(out[0][1], out[1][1]), nphi


@pytest.mark.parametrize("nphi,k,t,narrow,main", [(8192, 3, 256, 10, 13), (4096, 2, 256, 9, 13),
                                                  (32768, 2, 65537, 12, 13)])
def test_small_launch_plan_gives_the_same_bytes(gpu, nphi, k, t, narrow, main):
    """With a small-launch plan set, launches at or below its size run with it and larger ones
    with the main plan; the DGT (oracle-checked), the work-list DGT, the fused polymul and the
    batched BFV chain give the bytes of the single-plan engine either way."""
    import ctypes as C

    import torch

    from cupoly_b200._lib import call
    from cupoly_b200.engine import FORWARD, INVERSE, QBase, UNIFORM, Engine, from_u64, to_u64
    from oracle import coracle
    e = Engine(k, 0, nphi, t)
    e.set_plan(3, main)
    e.set_narrow_plan(0, 0, 0)
    assert e.get_narrow_plan()["max_units"] == 0
    x = random_poly_residues(nphi + 5, e.Q, nphi)
    ref = coracle.dgt(fold(x)[None], e.Q)
    P = 3
    ins = []
    for j in range(4):
        v = e.empty(QBase, P)
        e.sample(v, QBase, UNIFORM, 7, 16 * j, npolys=P, to_dgt=True)
        ins.append(v)
    ws, pws = e.bfv_mul_batch_workspace(P), e.polymul_workspace(QBase, P)
    rid = torch.tensor([i % k for i in range(P * k)], dtype=torch.int32, device="cuda")

    def run():
        d = from_u64(fold(x)[None])
        e.dgt(d, 0, FORWARD)
        fwd = to_u64(d).copy()
        e.dgt(d, 0, INVERSE)
        back = to_u64(d)[0].copy()
        c3 = e.empty(QBase, 3 * P)
        e.bfv_mul_batch(c3, *ins, P, ws)
        pm = e.empty(QBase, P)
        e.polymul(pm, ins[0], ins[1], QBase, pws, P)
        lst = ins[2].clone()
        call("cp_dgt_list", e.handle, C.c_void_p(lst.data_ptr()), C.c_void_p(rid.data_ptr()), P * k, INVERSE,
             C.c_void_p(torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        return fwd, back, c3.clone(), pm.clone(), lst

    base = run()
    assert np.array_equal(base[0], ref) and np.array_equal(base[1], fold(x))
    # every launch of run() has at most 4 P k residue transforms: all of them take the
    # small-launch plan with a large limit, none with limit 1 (single-residue launches aside)
    for units in (4 * P * (k + 1), 1):
        e.set_narrow_plan(3, narrow, units)
        got = e.get_narrow_plan()
        assert got["max_units"] == units and got["log_cta"] == min(narrow, (nphi // 2).bit_length() - 1)
        out = run()
        assert np.array_equal(out[0], ref) and np.array_equal(out[1], fold(x)), units
        for a, b in zip(base[2:], out[2:]):
            assert torch.equal(a, b), units
    e.set_narrow_plan(0, 0, 0)


def test_default_and_cached_small_launch_plans(gpu, tmp_path, monkeypatch):
    """Engines start with the library's small-launch plan (radix 4, 2 split bits: up to 96
    residue transforms at nphi 4096 and 8192, up to 16 at nphi 16384, none above) and its
    main plan (2 split bits from nphi 16384 on); a tuned cache entry replaces them,
    including by none."""
    import json
    monkeypatch.setenv("CUPOLY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    from cupoly_b200 import autotune
    from cupoly_b200.engine import Engine
    for nphi, exp, units, main_cta in ((2048, 0, 0, 10), (4096, 9, 96, 11), (8192, 10, 96, 12),
                                       (16384, 11, 16, 11), (32768, 0, 0, 12), (65536, 0, 0, 13)):
        eng = Engine(1, 1, nphi, 65537 if nphi >= 32768 else 256)
        got = eng.get_narrow_plan()
        assert (eng.get_plan()["log_radix"], eng.get_plan()["log_cta"]) == (3, main_cta), nphi
        if exp:
            assert got == {"log_radix": 2, "log_cta": exp, "max_units": units}, nphi
        else:
            assert got["max_units"] == 0, nphi
    wide = autotune.best_plan(8192, residues=128, reps=2)
    narrow = autotune.best_narrow_plan(8192, wide)
    assert narrow[:2] in autotune.candidates(8192) + [tuple(wide)]
    assert narrow[2] in (0,) + autotune.NARROW_UNITS
    assert autotune.cached_narrow_plan(8192) == narrow
    ent = next(iter(json.load(open(tmp_path / "tune.json")).values()))
    assert len(ent["narrow"]["ms_fwd_inv"]) == len(autotune.NARROW_UNITS) * len(
        set(autotune.candidates(8192)) | {tuple(wide)})
    got = Engine(2, 0, 8192, 256).get_narrow_plan()
    if narrow[2]:
        assert (got["log_radix"], got["log_cta"], got["max_units"]) == narrow
    else:
        assert got["max_units"] == 0


def test_pipelined_batches_equal_single_calls(gpu):
    """PipelinedBFV (two batches in flight on two streams) gives each batch the bytes of one
    cp_bfv_mul_batch call on the default stream."""
    import torch

    from cupoly_b200.batch import PipelinedBFV
    from cupoly_b200.engine import QBase, UNIFORM, Engine
    e = Engine(3, 0, 4096, 256)
    P, nb = 8, 5
    batches = []
    for i in range(nb):
        ins = []
        for v in range(4):
            x = e.empty(QBase, P)
            e.sample(x, QBase, UNIFORM, 21 + i, 16 * v, npolys=P, to_dgt=True)
            ins.append(x)
        batches.append(ins)
    outs = [e.empty(QBase, 3 * P) for _ in range(nb)]
    pl = PipelinedBFV(e, P)
    pl.run(batches, outs)
    pl.join()
    ws = e.bfv_mul_batch_workspace(P)
    for ins, out in zip(batches, outs):
        ref = e.empty(QBase, 3 * P)
        e.bfv_mul_batch(ref, *ins, P, ws)
        torch.cuda.synchronize()
        assert torch.equal(ref, out)


def test_pipelined_polymul_equals_single_calls(gpu):
    """PipelinedPolymul gives each batch the bytes of one cp_polymul call."""
    import torch

    from cupoly_b200.batch import PipelinedPolymul
    from cupoly_b200.engine import QBase, UNIFORM, Engine
    e = Engine(2, 0, 4096, 256)
    P, nb = 16, 4
    batches = []
    for i in range(nb):
        a, b = e.empty(QBase, P), e.empty(QBase, P)
        e.sample(a, QBase, UNIFORM, 41 + i, 0, npolys=P, to_dgt=False)
        e.sample(b, QBase, UNIFORM, 41 + i, P, npolys=P, to_dgt=False)
        batches.append((a, b))
    outs = [e.empty(QBase, P) for _ in range(nb)]
    pp = PipelinedPolymul(e, QBase, P)
    pp.run(batches, outs)
    pp.join()
    ws = e.polymul_workspace(QBase, P)
    for (a, b), out in zip(batches, outs):
        ref = e.empty(QBase, P)
        e.polymul(ref, a, b, QBase, ws, P)
        torch.cuda.synchronize()
        assert torch.equal(ref, out)


def test_mixed_polymul_benchmark_draw_all_1024_instances(gpu):
    """The benchmark's mixed batch exactly: random_specs(1024, 0xC0FFEE) (nphi in
    {2048 .. 16384}, k in 1..8), seeded operands per instance; every instance's product
    is bit-exact against the oracle, for the graph in sequence and for the graph with
    one parallel branch per size group."""
    import torch
    from cupoly_b200.batch import MixedPolymul, random_specs
    specs = random_specs(1024, 0xC0FFEE)
    mp = MixedPolymul(specs)
    by_shape = {}
    for i, (nphi, k) in enumerate(specs):
        a = random_poly_residues(30000 + i, O.PRIMES[:k], nphi)
        b = random_poly_residues(40000 + i, O.PRIMES[:k], nphi)
        mp.set_inputs(i, a, b)
        by_shape.setdefault((nphi, k), []).append((i, a, b))
    want = {}
    for (nphi, k), items in by_shape.items():
        c = CO.polymul(np.stack([a for _, a, _ in items]), np.stack([b for _, _, b in items]), O.PRIMES[:k])
        for (i, _, _), ci in zip(items, c):
            want[i] = ci
    for branches in (False, True):
        for g in mp.groups.values():
            g["c"].fill_(-1)
        mp.capture(branches=branches)
        mp.replay()
        torch.cuda.synchronize()
        for i in range(len(specs)):
            assert np.array_equal(mp.result(i), want[i]), (i, specs[i], branches)
    # the single persistent launch over the same draw
    mt = MixedPolymul(specs, mode="tiles")
    assert mt.launches_per_run() == 1
    for i, (nphi, k) in enumerate(specs):
        mt.set_inputs(i, random_poly_residues(30000 + i, O.PRIMES[:k], nphi),
                      random_poly_residues(40000 + i, O.PRIMES[:k], nphi))
    for g in mt.groups.values():
        g["c"].fill_(-1)
    mt.capture()
    mt.replay()
    torch.cuda.synchronize()
    for i in range(len(specs)):
        assert np.array_equal(mt.result(i), want[i]), (i, specs[i], "tiles")


@pytest.mark.parametrize("specs", [[(2048, 1)], [(16384, 3)], [(4096, 2), (2048, 8), (8192, 1), (16384, 5)],
                                   [(2048, 3)] * 5 + [(4096, 3)] * 3])
def test_single_launch_polymul_tiles(gpu, specs):
    """cp_polymul_tiles: partial and full tiles of every size, bit-exact against the
    oracle and against the graph form, with outputs aliasing an input."""
    import torch
    from cupoly_b200.batch import MixedPolymul
    mt = MixedPolymul(specs, mode="tiles")
    data = []
    for i, (nphi, k) in enumerate(specs):
        a = random_poly_residues(500 + i, O.PRIMES[:k], nphi)
        b = random_poly_residues(600 + i, O.PRIMES[:k], nphi)
        mt.set_inputs(i, a, b)
        data.append((a, b))
    mt.run()
    torch.cuda.synchronize()
    for i, (nphi, k) in enumerate(specs):
        a, b = data[i]
        assert np.array_equal(mt.result(i), CO.polymul(a[None], b[None], O.PRIMES[:k])[0]), (i, nphi, k)
    for g in mt.groups.values():  # c aliasing a
        g["c"] = g["a"]
    mt._build_tiles()
    mt.run()
    torch.cuda.synchronize()
    for i, (nphi, k) in enumerate(specs):
        a, b = data[i]
        assert np.array_equal(mt.result(i), CO.polymul(a[None], b[None], O.PRIMES[:k])[0]), (i, nphi, k)


def test_single_launch_polymul_rejects_other_plans(gpu):
    """The tile kernel needs each size's whole-CTA radix-8 plan; an engine with another
    plan is refused before launch."""
    import ctypes as C
    from cupoly_b200 import _lib
    from cupoly_b200.batch import MixedPolymul
    mt = MixedPolymul([(4096, 2)], mode="tiles")
    g = mt.groups[4096]
    g["engine"].set_plan(2, 11)
    eng, cc, aa, bb, rr = mt._tile_args
    rc = _lib.lib().cp_polymul_tiles(eng, cc, aa, bb, rr, mt._tile_rows, C.c_void_p(mt.tiles.data_ptr()),
                                     mt.ntiles, C.c_void_p(mt.tile_ws.data_ptr()), mt.tile_ws.numel() * 8, None)
    assert rc == 1 and b"radix-8 plan" in _lib.lib().cp_last_error()


def test_persistent_plan_in_the_fused_calls(gpu):
    """Plan r3/c13 at nphi 16384 keeps each residue whole in one CTA: one CTA of 1024 threads
    per SM, persistent, walking several units and prefetching the next into L2. Every launch of
    the batched chain and of the fused polymul below has more units than the GPU has SMs, so the
    gather, tensor and product-on-load sources all run with CTAs that walk several units. The
    bytes equal those of the library's default plan (split stage, several CTAs per SM)."""
    import torch

    from cupoly_b200.engine import QBase, UNIFORM, Engine
    nphi, k, t, P, PM = 16384, 4, 256, 16, 48
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert min(3 * P * k, PM * k) > sms  # the smallest transform launches of the two calls
    out = []
    for plan in ((3, 0), (3, 13)):
        e = Engine(k, 0, nphi, t, log_radix=3)
        e.set_narrow_plan(0, 0, 0)
        if plan[1]:
            e.set_plan(*plan)
            assert e.get_plan() == {"log_radix": 3, "log_cta": 13, "split_bits": 0}
        else:
            assert e.get_plan()["split_bits"] > 0
        ins = []
        for j in range(4):
            v = e.empty(QBase, P)
            e.sample(v, QBase, UNIFORM, 21, 16 * j, npolys=P, to_dgt=True)
            ins.append(v)
        c3 = e.empty(QBase, 3 * P)
        e.bfv_mul_batch(c3, *ins, P, e.bfv_mul_batch_workspace(P))
        a, b, c = e.empty(QBase, PM), e.empty(QBase, PM), e.empty(QBase, PM)
        e.sample(a, QBase, UNIFORM, 22, 0, npolys=PM, to_dgt=False)
        e.sample(b, QBase, UNIFORM, 22, PM, npolys=PM, to_dgt=False)
        e.polymul(c, a, b, QBase, e.polymul_workspace(QBase, PM), PM)
        torch.cuda.synchronize()
        out.append((c3.clone(), c.clone()))
        del e
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
