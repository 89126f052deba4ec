"""Autotuner for the DGT register radix.

The in-CTA transform runs radix-2^r register passes, r in {2, 3, 4}; the best
r depends on the transform size (registers, passes, shared-memory traffic).
`best_log_radix(nphi)` times forward + inverse transforms of a batch for each
candidate on the current GPU and caches the winner in a JSON file keyed by GPU
name and nphi (the RNS width only scales the batch, so it does not change the
choice).  Engines created with log_radix=0 from Python use the cached choice
when one exists and the library default (radix 8) otherwise.
"""
from __future__ import annotations

import json
import os
from typing import Dict

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


def cached_log_radix(nphi: int) -> int:
    """Cached choice for this GPU and nphi, or 0 when none is cached."""
    try:
        return int(_load().get(_key(nphi), {}).get("log_radix", 0))
    except Exception:
        return 0


def candidates(nphi: int):
    logn = max(1, (nphi // 2).bit_length() - 1)
    lognc = min(logn, 13)
    out = []
    for r in (2, 3, 4):
        eff = min(r, lognc)
        while lognc - eff > 10:  # at most 1024 threads per CTA
            eff += 1
        if eff not in out:
            out.append(eff)
    return out


def best_log_radix(nphi: int, residues: int = 2048, reps: int = 5, save: bool = True) -> int:
    """Time every candidate radix at this nphi and return (and cache) the fastest."""
    import torch

    from .engine import FORWARD, INVERSE, UNIFORM, Engine

    key = _key(nphi)
    results = {}
    npolys = max(1, residues // 2)
    for r in candidates(nphi):
        e = Engine(2, 1, nphi, 256, r)
        x = e.empty(0, npolys)
        e.sample(x, 0, UNIFORM, 1, 0, npolys=npolys, to_dgt=False)
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
        results[r] = a.elapsed_time(b) / reps
        del e, x
    best = min(results, key=results.get)
    if save:
        data = _load()
        data[key] = {"log_radix": best, "ms_fwd_inv": {str(k): round(v, 4) for k, v in results.items()},
                     "residues": 2 * npolys}
        os.makedirs(os.path.dirname(cache_path()), exist_ok=True)
        with open(cache_path(), "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    return best
