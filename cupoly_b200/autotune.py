"""Autotuner for the DGT plan: register radix and stage split.

The in-CTA transform runs radix-2^r register passes, r in {2, 3, 4}, over the
largest power of two kept whole in one CTA, 2^c (c <= 13); for N = nphi / 2
larger than 2^c the top log2(N) - c (at most 2) bits run in an element-wise
split stage.  Which (r, c) is fastest depends on the GPU and the size (register
pressure, passes, shared memory per CTA and hence CTAs per SM, the extra HBM
pass of the split).  `best_plan(nphi)` times a forward + inverse transform of a
batch for every candidate on the current GPU and caches the winner in a JSON
file keyed by GPU name and nphi (the RNS width only scales the batch, so it
does not change the choice).  Plans with a split stage are timed in both of its
forms (a separate element-wise kernel, or inside a thread-block cluster through
distributed shared memory; cp_engine_set_split_mode); the cluster form is cached
with the plan only when it is more than 2 % faster.  `best_narrow_plan(nphi, wide)`
then picks a second plan for small launches (cp_engine_set_narrow_plan): the
candidate fastest at 16 residue transforms per launch, and the largest launch
size at which it still beats the main plan.  The RNS width k enters the choice
through the launch size: a launch transforms polynomials x k residues, and that
count selects the main or the small-launch plan at run time, so the plan in use is
a function of (nphi, k, batch).  Engines created with log_radix = 0
from Python use the cached plans when they exist and the library default
(radix 8, c = 13, split kernel, no small-launch plan) otherwise.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Tuple

_DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "autotune.json")


def cache_path() -> str:
    return os.environ.get("CUPOLY_B200_TUNE_CACHE", _DEFAULT_CACHE)


def _gpu_name() -> str:
    import torch

    return torch.cuda.get_device_name(torch.cuda.current_device())


def _load() -> Dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _key(nphi: int) -> str:
    return "%s|nphi=%d" % (_gpu_name(), nphi)


def cached_plan(nphi: int) -> Tuple[int, int]:
    """Cached (log_radix, log_cta) for this GPU and nphi, or (0, 0) when none is cached."""
    try:
        ent = _load().get(_key(nphi), {})
        return int(ent.get("log_radix", 0)), int(ent.get("log_cta", 0))
    except Exception:
        return 0, 0


def cached_split_mode(nphi: int) -> int:
    """Cached split-stage form for this GPU and nphi (0 split kernel, 1 cluster); 0 when none."""
    try:
        return int(_load().get(_key(nphi), {}).get("split_mode", 0))
    except Exception:
        return 0


def cached_narrow_plan(nphi: int) -> Tuple[int, int, int]:
    """Cached small-launch plan (log_radix, log_cta, max_units) for this GPU and nphi;
    (0, 0, 0) when none is cached."""
    try:
        ent = _load().get(_key(nphi), {}).get("narrow", {})
        return int(ent.get("log_radix", 0)), int(ent.get("log_cta", 0)), int(ent.get("max_units", 0))
    except Exception:
        return 0, 0, 0


def cached_log_radix(nphi: int) -> int:
    return cached_plan(nphi)[0]


def candidates(nphi: int) -> List[Tuple[int, int]]:
    """(log_radix, log_cta) pairs the library compiles for this size."""
    logn = max(1, (nphi // 2).bit_length() - 1)
    out = []
    for c in (13, 12, 11, 10, 9):
        if c >= logn and c != 13:
            continue  # a cap at or above the size changes nothing: only the default is timed
        lognc = min(logn, c)
        if logn - lognc > 2 or (logn > lognc and lognc < 8):
            continue  # the split stage handles at most 2 bits, of at least 256-element blocks
        for r in (2, 3, 4):
            eff = min(r, lognc)
            while lognc - eff > 10:  # at most 1024 threads per CTA
                eff += 1
            if (eff, c) not in out:
                out.append((eff, c))
    return out


def best_plan(nphi: int, residues: int = 2048, reps: int = 5, save: bool = True) -> Tuple[int, int]:
    """Time every candidate plan at this nphi and return (and cache) the fastest."""
    import torch

    from .engine import FORWARD, INVERSE, UNIFORM, Engine

    key = _key(nphi)
    results = {}
    npolys = max(1, residues // 2)
    for r, c in candidates(nphi):
        e = Engine(2, 1, nphi, 256, r)
        e.set_narrow_plan(0, 0, 0)  # every launch timed with the candidate
        e.set_plan(r, c)
        x = e.empty(0, npolys)
        e.sample(x, 0, UNIFORM, 1, 0, npolys=npolys, to_dgt=False)
        for mode in ((0, 1) if e.get_plan()["split_bits"] > 0 else (0,)):
            e.set_split_mode(mode)
            e.dgt(x, 0, FORWARD)
            e.dgt(x, 0, INVERSE)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                e.dgt(x, 0, FORWARD)
                e.dgt(x, 0, INVERSE)
            b.record()
            torch.cuda.synchronize()
            results[(r, c, mode)] = a.elapsed_time(b) / reps
        del e, x
    # the cluster form must win by more than the run-to-run spread (2 %) to be chosen
    best = min(results, key=lambda k: results[k] * (1.02 if k[2] else 1.0))
    if save:
        data = _load()
        data[key] = {"log_radix": best[0], "log_cta": best[1], "split_mode": best[2],
                     "ms_fwd_inv": {("r%d_c%d_cluster" if k[2] else "r%d_c%d") % k[:2]: round(v, 4)
                                    for k, v in results.items()},
                     "residues": 2 * npolys}
        os.makedirs(os.path.dirname(cache_path()), exist_ok=True)
        with open(cache_path(), "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    return best[:2]


# Launch sizes (residue transforms per launch) at which the small-launch plan is compared
# with the main plan.
NARROW_UNITS = (16, 96, 192, 288, 384, 768, 1536)


def _graph_ms(fn, calls: int = 10, reps: int = 5) -> float:
    """Device milliseconds per fn() call, fn captured `calls` times in a CUDA graph so the
    host's per-launch cost does not hide small launches."""
    import torch

    fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
        for _ in range(calls):
            fn()
    g.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        g.replay()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / (reps * calls)
    del g
    return ms


def best_narrow_plan(nphi: int, wide: Tuple[int, int], save: bool = True) -> Tuple[int, int, int]:
    """Small-launch plan for this nphi: the candidate fastest at the smallest launch size
    (forward + inverse DGT, CUDA-graph timed), used up to the largest size of NARROW_UNITS,
    counted up from the smallest, at which it beats the main plan `wide` by more than 2 %.
    Returns (log_radix, log_cta, max_units); max_units = 0 when the main plan is as fast."""
    from .engine import FORWARD, INVERSE, UNIFORM, Engine

    cands = candidates(nphi)
    if tuple(wide) not in cands:
        cands.append(tuple(wide))
    e = Engine(1, 1, nphi, 256, wide[0] or 3)
    e.set_narrow_plan(0, 0, 0)  # every launch timed with the candidate
    times = {}
    for U in NARROW_UNITS:
        x = e.empty(0, U)
        e.sample(x, 0, UNIFORM, 1, 0, npolys=U, to_dgt=False)
        for r, c in cands:
            e.set_plan(r, c)
            times[(r, c, U)] = _graph_ms(lambda: (e.dgt(x, 0, FORWARD), e.dgt(x, 0, INVERSE)))
        del x
    del e
    u0 = NARROW_UNITS[0]
    narrow = min(cands, key=lambda rc: times[(rc[0], rc[1], u0)])
    max_units = 0
    if narrow != tuple(wide):
        for U in NARROW_UNITS:
            if times[narrow + (U,)] * 1.02 < times[tuple(wide) + (U,)]:
                max_units = U
            else:
                break
    if save:
        data = _load()
        ent = data.setdefault(_key(nphi), {})
        ent["narrow"] = {"log_radix": narrow[0], "log_cta": narrow[1], "max_units": max_units,
                         "ms_fwd_inv": {"r%d_c%d_u%d" % k: round(v, 4) for k, v in times.items()}}
        os.makedirs(os.path.dirname(cache_path()), exist_ok=True)
        with open(cache_path(), "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    return narrow[0], narrow[1], max_units


def best_log_radix(nphi: int, **kw) -> int:
    return best_plan(nphi, **kw)[0]


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="tune the DGT plan for the current GPU")
    ap.add_argument("--nphi", default="2048,4096,8192,16384,32768,65536")
    a = ap.parse_args()
    for n in [int(x) for x in a.nphi.split(",")]:
        wide = best_plan(n)
        print(json.dumps({"nphi": n, "plan": wide, "narrow": best_narrow_plan(n, wide)}), flush=True)
    print(json.dumps(_load(), indent=1))
