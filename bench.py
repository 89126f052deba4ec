#!/usr/bin/env python3
"""Benchmark: BFV homomorphic-multiplication kernel chain on B200.

Workload (one step): a batch of P ciphertext pairs at nphi = 8192, |Q| = 5,
|B| = 6, t = 256 -- basis extension Q -> Q u B of the four input polynomials,
DGT tensor product (3 outputs), HPS t/Q scale-and-round back to Q.  Inputs
and outputs are in the DGT domain (cuPoly's poly_t state RNSSTATE).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line is printed by rank 0.  `value` is whole-job hom-mul/s with the
inputs resident in HBM (batched form, two consecutive batches in flight on two
streams, device-timed, max over ranks);
`e2e` repeats it through the C ABI with pinned host buffers and the
host<->device copies inside the timed region; `plain` is the per-call form
(one cp_bfv_mul per pair); `plain_cxx` times the same per-call sequences as
`cupoly_gpu` through this library's C++ drop-in layer; `polymul` is the
batched DGT polymul/s of the nphi = 4096, k = 2 configuration.  Two reference
legs run on rank 0: `cupoly_gpu` times cuPoly's own kernels per call when its
sources were compiled into oracle/_ref, and `cpu_baseline` the C oracle (the
CPU restatement of the reference path: cuPoly has no CPU implementation of it)
on the host cores.  With --impl reference the C oracle is the timed arm.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NPHI, K_Q, K_B, T_PLAIN = 8192, 5, 6, 256
WORKLOAD = "BFV homomorphic-multiply kernel chain (nphi=8192, k=5, kl=6, t=256)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--pairs", type=int, default=128, help="ciphertext pairs per step (batched form)")
    ap.add_argument("--plain-pairs", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cupoly-gpu", action="store_true", help="skip timing cuPoly's own kernels")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-next", action="store_true", help="skip the CRT / xi-rho / wire / CKKS measurements")
    ap.add_argument("--serving-requests", type=int, default=50000)
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only: no collective on the data path)
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch

        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    """`nvidia-smi -lms 50` logging the GPU's clocks and throttle reasons for the
    duration of a `with` block (the timed region)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self._proc = None

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                           "--format=csv,noheader,nounits", "-lms", "50"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)  # the first sample lands before the timed work starts
        except OSError:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is None:
            return
        time.sleep(0.1)
        self._proc.terminate()
        try:
            out, _ = self._proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self._proc.kill()
            out, _ = self._proc.communicate()
        self.samples = [[x.strip() for x in ln.split(",")] for ln in out.splitlines() if ln.count(",") >= 8]

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and
                          s[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU baseline (the oracle's C restatement of the reference path)
# ---------------------------------------------------------------------------
def cpu_bfv_rate(budget_s: float, pairs_per_call: int = 4):
    import numpy as np

    from oracle import coracle, pyoracle
    from tests.common import random_poly_residues

    Q, B = pyoracle.bases(K_Q, K_B)
    rows = [np.stack([random_poly_residues(31 + 4 * i + j, Q, NPHI) for i in range(pairs_per_call)])
            for j in range(4)]
    coracle.bfv_mul(*[r[:1] for r in rows], Q, B, T_PLAIN)  # warm-up
    done, t0 = 0, time.perf_counter()
    while True:
        coracle.bfv_mul(*rows, Q, B, T_PLAIN)
        done += pairs_per_call
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return done / el, done, el, coracle.num_threads()


def run_reference(args, D: Dist):
    """--impl reference: the CPU restatement timed on the host cores, rank 0 only."""
    if D.rank != 0:
        return
    from oracle import coracle

    coracle.lib()
    cores = coracle.num_threads()
    per_step = 4
    import numpy as np

    from oracle import pyoracle
    from tests.common import random_poly_residues

    Q, B = pyoracle.bases(K_Q, K_B)
    rows = [np.stack([random_poly_residues(31 + 4 * i + j, Q, NPHI) for i in range(per_step)]) for j in range(4)]
    for _ in range(args.warmup):
        coracle.bfv_mul(*rows, Q, B, T_PLAIN)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        coracle.bfv_mul(*rows, Q, B, T_PLAIN)
    el = time.perf_counter() - t0
    v = per_step * args.steps / el
    line = {
        "impl": "reference", "metric": "BFV mul/s", "value": round(v, 3), "unit": "hom-mul/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(el * 1e3 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "pairs_per_step": per_step, "nphi": NPHI, "k": K_Q, "kl": K_B,
                   "t": T_PLAIN},
        "cpu_baseline": {"value": round(v, 3), "unit": "hom-mul/s", "cores": cores, "kind": "port",
                         "sample": "%d pairs per step, C restatement (oracle/cpoly_oracle.c), OpenMP" % per_step},
        "e2e": {"value": round(v, 3), "unit": "hom-mul/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": ("cuPoly runs this path only on the GPU (NTL appears only in its tests), so the oracle's C port "
                 "of the path is the CPU implementation timed; cupoly_gpu holds cuPoly's own kernels per call"),
        "cupoly_gpu": None if args.no_cupoly_gpu else cupoly_gpu_times(),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _timed(fn, reps: int) -> float:
    """Average milliseconds of fn() over reps calls, CUDA events on the current stream."""
    import torch

    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def _dot_row(seed: int, hbm_peak: float):
    """The key-switching inner product sum_i a_i b_i over k = 16 terms at nphi 32768 (one
    relinearization component at the large configuration), fused (cp_dot, one pass) against
    cuPoly's composition (one mul and k - 1 muladd calls), each as 10 calls in a CUDA graph.
    Two operand sets alternate so the 132 MB working set of a call is not served from L2."""
    import torch

    from cupoly_b200.engine import QBase, UNIFORM, Engine

    d = Engine(16, 0, 32768, 65537)
    nt = d.k
    sets = []
    for s in range(2):
        ops = d.empty(QBase, 2 * nt)
        d.sample(ops, QBase, UNIFORM, seed, 60 + s, npolys=2 * nt, to_dgt=False)
        sets.append(([ops[i] for i in range(nt)], [ops[nt + i] for i in range(nt)]))
    acc = [d.empty(QBase), d.empty(QBase)]
    it = [0]

    def fused():
        j = it[0] & 1
        it[0] += 1
        d.dot(acc[j], sets[j][0], sets[j][1], QBase)

    def composed():
        j = it[0] & 1
        it[0] += 1
        a, b = sets[j]
        d.mul(acc[j], a[0], b[0], QBase)
        for i in range(1, nt):
            d.muladd(acc[j], a[i], b[i], acc[j], QBase)

    def graph_of(fn, calls):
        # captured, so the host's per-call cost (16-entry pointer arrays, 16 launches for the
        # composition) does not hide the device time
        fn()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        with torch.cuda.stream(s), torch.cuda.graph(g, stream=s):
            for _ in range(calls):
                fn()
        torch.cuda.synchronize()
        return g

    calls = 10
    gf, gc = graph_of(fused, calls), graph_of(composed, calls)
    ms_f = _timed(gf.replay, 5) / calls
    ref = [x.clone() for x in acc]
    ms_c = _timed(gc.replay, 5) / calls
    assert all(torch.equal(x, y) for x, y in zip(acc, ref)), "fused dot != composition"
    del gf, gc
    poly = d.k * d.N * 16
    byt = (2 * nt + 1) * poly
    d.check()
    row = {"config": "nphi=%d, k=%d, %d terms" % (d.nphi, d.k, nt), "fused_us": round(ms_f * 1e3, 2),
           "composed_us": round(ms_c * 1e3, 2), "speedup": round(ms_c / ms_f, 2),
           "GB_per_s": round(byt / ms_f / 1e6, 1), "frac_hbm": round(byt / ms_f / 1e6 / hbm_peak, 4),
           "bytes_per_call": byt, "composed_bytes_per_call": (3 + 4 * (nt - 1)) * poly}
    del sets, acc, d
    # batched relinearization inner product: the xi decomposition of 128 polynomials (nphi 8192,
    # k 5) against one shared set of k key polynomials, one cp_dot_batch launch
    e = Engine(K_Q, K_B, NPHI, T_PLAIN)
    P, k = 128, e.k
    dec = e.empty(QBase, P * k)
    e.sample(dec, QBase, UNIFORM, seed, 70, npolys=P * k, to_dgt=False)
    keys = e.empty(QBase, k)
    e.sample(keys, QBase, UNIFORM, seed, 71, npolys=k, to_dgt=False)
    out = e.empty(QBase, P)
    gb = graph_of(lambda: e.dot_batch(out, dec, keys, k, P, QBase, b_shared=True), 1)
    ms_b = _timed(gb.replay, 10)
    del gb
    pq = k * e.N * 16
    byt_b = (P * k + k + P) * pq
    e.check()
    row["batch"] = {"config": "nphi=%d, k=%d: %d decompositions x %d shared keys" % (e.nphi, k, P, k),
                    "us_per_call": round(ms_b * 1e3, 2), "us_per_polynomial": round(ms_b * 1e3 / P, 3),
                    "GB_per_s": round(byt_b / ms_b / 1e6, 1), "frac_hbm": round(byt_b / ms_b / 1e6 / hbm_peak, 4)}
    return row


def next_rows(seed: int, hbm_peak: float):
    """Throughput of the calls after the multiplication chain, each with its algorithmic bytes
    (what an ideal kernel reads and writes once) over the measured time:
    device CRT / ICRT (512 polynomials, nphi 8192, k 5: limbs and residues both above L2 size),
    xi and rho (one polynomial per call, as cuPoly's API), the fused key-switching dot product
    (nphi 32768, k 16), the binary wire form (host side,
    128 polynomials), and the CKKS calls (nphi 16384, k 8, kl 9, 52-bit primes, one polynomial
    per call, level k - 1)."""
    import time

    import torch

    from cupoly_b200.engine import FORWARD, QBBase, QBase, UNIFORM, Engine

    out = {}
    e = Engine(K_Q, K_B, NPHI, T_PLAIN)
    n, k, N = e.nphi, e.k, e.N
    P = 512
    x = e.empty(QBase, P)
    e.sample(x, QBase, UNIFORM, seed, 1 << 20, npolys=P, to_dgt=False)
    limbs = torch.zeros((P, n, k), dtype=torch.int64, device="cuda")
    ms_icrt = _timed(lambda: e.icrt(limbs, x, QBase), 5)
    y = e.empty(QBase, P)
    ms_crt = _timed(lambda: e.crt(y, limbs, QBase), 5)
    assert torch.equal(x, y), "CRT(ICRT(x)) != x"
    byt = P * n * k * 8 * 2  # limbs read + residues written (and the reverse)
    out["crt"] = {"config": "nphi=%d, k=%d, %d polys, %d-limb coefficients" % (n, k, P, k),
                  "coeffs_per_s": round(P * n / (ms_crt / 1e3), 1), "GB_per_s": round(byt / ms_crt / 1e6, 1),
                  "frac_hbm": round(byt / ms_crt / 1e6 / hbm_peak, 4)}
    out["icrt"] = {"config": out["crt"]["config"], "coeffs_per_s": round(P * n / (ms_icrt / 1e3), 1),
                   "GB_per_s": round(byt / ms_icrt / 1e6, 1), "frac_hbm": round(byt / ms_icrt / 1e6 / hbm_peak, 4)}
    del limbs, y
    xi = e.empty(QBase, k)
    ms_xi = _timed(lambda: e.xi(xi, x[0:1]), 50)
    ms_rho = _timed(lambda: e.rho(xi, x[0:1]), 50)
    XB = 64
    xib = e.empty(QBase, XB * k)
    ms_xib = _timed(lambda: e.xi_batch(xib, x[:XB]), 10)
    out["xi_rho"] = {"config": "nphi=%d, k=%d, one polynomial -> k polynomials" % (n, k),
                     "xi_us_per_call": round(ms_xi * 1e3, 2), "rho_us_per_call": round(ms_rho * 1e3, 2),
                     "GB_per_s": round((k * N * 16 * (1 + k)) / ms_xi / 1e6, 1),
                     "xi_batch_64_us_per_poly": round(ms_xib * 1e3 / XB, 3),
                     "xi_batch_GB_per_s": round(XB * (k * N * 16 * (1 + k)) / ms_xib / 1e6, 1)}
    del xib
    out["dot"] = _dot_row(seed, hbm_peak)
    W = 128
    blob = torch.empty(e.wire_bytes(QBase, W), dtype=torch.uint8, pin_memory=True).numpy()
    z = e.empty(QBase, W)
    t_exp, t_imp = [], []
    for _ in range(3):  # first round warms the buffers; best of the other two
        t0 = time.perf_counter()
        e.export_residues(x[:W], QBase, 0, out=blob)
        t1 = time.perf_counter()
        e.import_residues(z, blob, QBase)
        t2 = time.perf_counter()
        t_exp.append(t1 - t0)
        t_imp.append(t2 - t1)
    assert torch.equal(z, x[:W])
    out["wire"] = {"config": "%d polys (%d bytes, pinned host buffer)" % (W, blob.size),
                   "export_GB_per_s": round(blob.size / min(t_exp[1:]) / 1e9, 2),
                   "import_GB_per_s": round(blob.size / min(t_imp[1:]) / 1e9, 2),
                   "note": "host wall clock per call: export = header + device-to-host copy; import = header "
                           "and primes checked, every residue checked below its prime on the host, host-to-device copy"}
    del x, xi, z, e
    c = Engine.ckks(8, 9, 16384, 52)
    lvl = 7
    a = c.empty(QBase)
    c.sample(a, QBase, UNIFORM, seed, 3, npolys=1, to_dgt=True)
    qb = c.empty(QBBase)
    r = c.empty(QBase)
    ms_raise = _timed(lambda: c.ckks_modulus_raising(qb, a, lvl), 20)
    ms_red = _timed(lambda: c.ckks_modulus_reduction(r, qb, lvl), 20)
    ms_resc = _timed(lambda: c.ckks_rescale(r, None, lvl), 20)
    PB = 64
    ab = c.empty(QBase, PB)
    c.sample(ab, QBase, UNIFORM, seed, 4, npolys=PB, to_dgt=True)
    qbb, rb, wsb = c.empty(QBBase, PB), c.empty(QBase, PB), c.ckks_batch_workspace(PB)
    mb_raise = _timed(lambda: c.ckks_modulus_raising_batch(qbb, ab, lvl, wsb), 5)
    mb_red = _timed(lambda: c.ckks_modulus_reduction_batch(rb, qbb, lvl, wsb), 5)
    mb_resc = _timed(lambda: c.ckks_rescale_batch(rb, lvl), 5)
    c.check()
    out["ckks"] = {"config": "nphi=16384, k=8, kl=9, prec 52, level 7, DGT domain",
                   "modulus_raising_us": round(ms_raise * 1e3, 1), "modulus_reduction_us": round(ms_red * 1e3, 1),
                   "rescale_us": round(ms_resc * 1e3, 1),
                   "batched_64_us_per_poly": {"modulus_raising": round(mb_raise * 1e3 / PB, 2),
                                              "modulus_reduction": round(mb_red * 1e3 / PB, 2),
                                              "rescale": round(mb_resc * 1e3 / PB, 2)}}
    del a, qb, r, c, ab, qbb, rb, wsb
    torch.cuda.empty_cache()
    return out


# Integer-pipe use of the hot kernels, from ncu captures of the same kernels on a B200
# (sm__pipe_fmaheavy / sm__pipe_alu cycles active and sm__issue_active, % of peak sustained
# active).  Both 64-bit-integer pipes are half rate; the busier one is the integer roofline.
INT_COUNTERS = {
    "source": "ncu capture",
    "kernels": {
        "k_dgt_fwd<12,3,0>": {"workload": "forward DGT, nphi 8192, 3072 residues",
                              "fmaheavy_pct": 69.9, "alu_pct": 51.9, "issue_pct": 54.9, "busier_pipe_frac": 0.699},
        "k_dgt_inv<12,3,0>": {"workload": "inverse DGT, nphi 8192, 3072 residues",
                              "fmaheavy_pct": 74.0, "alu_pct": 54.5, "issue_pct": 58.1, "busier_pipe_frac": 0.740},
        "k_basis_ext_pre<5>": {"workload": "the chain's Q -> B conversion, 512 polynomials",
                               "fmaheavy_pct": 70.5, "alu_pct": 65.1, "issue_pct": 63.5, "busier_pipe_frac": 0.705},
        "k_complex_scaling_pre<5>": {"workload": "the chain's complex scaling, 384 polynomials",
                                     "fmaheavy_pct": 61.2, "alu_pct": 68.0, "issue_pct": 60.8,
                                     "busier_pipe_frac": 0.680},
        "k_basis_ext_pre<6>": {"workload": "the chain's B -> Q conversion, 384 polynomials",
                               "fmaheavy_pct": 67.8, "alu_pct": 64.4, "issue_pct": 62.1, "busier_pipe_frac": 0.678},
        "k_dgt_inv<11,3,0> products on load": {"workload": "fused polymul, nphi 4096, k 2, 2048 products",
                                               "fmaheavy_pct": 74.7, "alu_pct": 58.3, "issue_pct": 60.1,
                                               "busier_pipe_frac": 0.747},
        "k_polymul_tiles": {"workload": "mixed batch of 1024 products, one launch",
                            "fmaheavy_pct": 67.7, "alu_pct": 49.8, "issue_pct": 52.6, "busier_pipe_frac": 0.677},
    },
}

CUPOLY_DRIVER = os.path.join(ROOT, "oracle", "_ref", "cupoly_ref_driver")
PERCALL = os.path.join(ROOT, "cupoly_b200", "lib", "cupoly_percall")


def cupoly_gpu_times():
    """cuPoly's own per-call GPU times on this GPU, when its sources were compiled here
    (oracle/cupoly_ref/Makefile): the polymul at nphi 4096, k 2 (two forward DGTs,
    poly_mul, one inverse DGT per call) and the BFV multiplication chain at nphi 8192,
    k 5, kl 6 (four poly_basis_extension_Q_to_B, poly_dr2 over Q and B, three
    poly_complex_scaling_tDivQ per pair), each timed with CUDA events over 200 calls.
    A reference leg beside the per-call forms; the reference arm's value stays the CPU restatement."""
    if not os.path.exists(CUPOLY_DRIVER):
        return {"unavailable": "cuPoly's sources were not compiled into oracle/_ref"}
    import tempfile

    out = {}
    for name, (k, nphi) in {"polymul_nphi4096_k2": (2, 4096), "bfv_mul_nphi8192_k5_kl6": (5, 8192)}.items():
        with tempfile.TemporaryDirectory() as d:
            f = os.path.join(d, "t.json")
            r = subprocess.run([CUPOLY_DRIVER, "time", str(k), str(k + 1), str(nphi), "200", "-", f],
                               capture_output=True, text=True, timeout=300)
            if r.returncode != 0:
                return {"unavailable": "cuPoly driver failed: " + (r.stderr or r.stdout)[-200:]}
            t = json.load(open(f))
        ms = t["polymul_ms"] if name.startswith("polymul") else t["bfv_mul_ms"]
        out[name] = {"ms_per_call": round(ms, 4), "per_s": round(1e3 / ms, 1)}
    out["source"] = "cuPoly 0.3.5 library (its own kernels), one call per polymul / pair, CUDA events"
    return out


def dropin_percall_times():
    """This library's C++ drop-in layer (libcupoly.so, cuPoly's API) per call, the same two
    call sequences as cupoly_gpu_times on the same sizes, plus the BFV multiplication at
    nphi 16384, k 10, kl 11 (the batched target's size): cupoly_b200/host/bench/percall.cpp,
    CUDA events on the Context's stream over 200 calls."""
    if not os.path.exists(PERCALL):
        return {"unavailable": "cupoly_b200/lib/cupoly_percall was not built"}
    out = {}
    for name, (k, nphi) in {"polymul_nphi4096_k2": (2, 4096), "bfv_mul_nphi8192_k5_kl6": (5, 8192),
                            "bfv_mul_nphi16384_k10_kl11": (10, 16384)}.items():
        r = subprocess.run([PERCALL, str(k), str(k + 1), str(nphi), "200"], capture_output=True, text=True,
                           timeout=300)
        if r.returncode != 0:
            raise RuntimeError("cupoly_percall failed: " + (r.stderr or r.stdout)[-300:])
        t = json.loads(r.stdout.strip().splitlines()[-1])
        ms = t["polymul_ms"] if name.startswith("polymul") else t["bfv_mul_ms"]
        out[name] = {"ms_per_call": round(ms, 4), "per_s": round(1e3 / ms, 1)}
    out["source"] = ("this library's C++ layer (libcupoly.so), one call sequence per product / pair as in "
                     "cupoly_gpu, CUDA events")
    return out


def run_ours(args, D: Dist):
    import torch

    from cupoly_b200.engine import FORWARD, QBase, UNIFORM, Engine

    torch.cuda.set_device(D.local)
    dev_index = D.local
    e = Engine(K_Q, K_B, NPHI, T_PLAIN)
    P = args.pairs
    seed = 0xC0FFEE + 1000003 * D.rank
    ins = []
    for j in range(4):
        x = e.empty(QBase, P)
        e.sample(x, QBase, UNIFORM, seed, 4096 * j, npolys=P, to_dgt=True)
        ins.append(x)
    c = e.empty(QBase, 3 * P)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    # consecutive batches, two in flight on two streams (batch.PipelinedBFV), each writing its
    # own output buffer; every step is one complete cp_bfv_mul_batch of P pairs
    from cupoly_b200.batch import PipelinedBFV
    pipe = PipelinedBFV(e, P, lanes=2)
    outs = [c, e.empty(QBase, 3 * P)]

    def steps(n):
        pipe.run([ins] * n, [outs[i & 1] for i in range(n)], stream)
        pipe.join(stream)

    steps(max(3, args.warmup))
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev_index) as clk:
        D.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        steps(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        D.barrier()
    ms = D.max(ev0.elapsed_time(ev1))
    value = D.world * P * args.steps / (ms / 1e3)
    # inverse DGT (gather) + Q->B + forward DGT(B) + 2 inverse DGTs with the tensor
    # product fused in + complex scaling + B->Q + forward DGT(Q) (nphi <= 16384: one kernel per DGT)
    launches_per_step = 8

    # ---- e2e: host-resident batches through the public API (StreamedBFV: copy-in,
    # chain and copy-out of consecutive batches overlap on three streams); every
    # step's H2D of its inputs and D2H of its result is inside the timed region ----
    from cupoly_b200.batch import StreamedBFV
    hin = [[torch.empty_like(x, device="cpu").pin_memory() for x in ins] for _ in range(2)]
    for hs in hin:
        for h, x in zip(hs, ins):
            h.copy_(x)
    hout = [torch.empty_like(c, device="cpu").pin_memory() for _ in range(2)]
    sb = StreamedBFV(e, P)
    sb.run([hin[0], hin[1]], [hout[0], hout[1]])  # warm-up
    sb.join(stream)
    torch.cuda.synchronize()
    D.barrier()
    ev0.record(stream)
    sb.s_in.wait_stream(stream)
    sb.run([hin[i & 1] for i in range(args.steps)], [hout[i & 1] for i in range(args.steps)])
    sb.join(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = D.max(ev0.elapsed_time(ev1))
    h2d = sum(h.numel() * 8 for h in hin[0])
    d2h = hout[0].numel() * 8
    # the host link alone: one step's copies in, out, and both at once (pinned memory)
    s_a, s_b = torch.cuda.Stream(), torch.cuda.Stream()
    dev_in = sb.bufs[0]["ins"]
    dev_out = sb.bufs[0]["out"]

    def link(copy_in: bool, copy_out: bool, reps: int = 5) -> float:
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s_a.wait_stream(stream)
        s_b.wait_stream(stream)
        for _ in range(reps):
            if copy_in:
                with torch.cuda.stream(s_a):
                    for d, h in zip(dev_in, hin[0]):
                        d.copy_(h, non_blocking=True)
            if copy_out:
                with torch.cuda.stream(s_b):
                    hout[0].copy_(dev_out, non_blocking=True)
        stream.wait_stream(s_a)
        stream.wait_stream(s_b)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    t_in, t_out, t_both = link(True, False), link(False, True), link(True, True)
    pcie = {"h2d_GB_per_s": round(h2d / t_in / 1e6, 1), "d2h_GB_per_s": round(d2h / t_out / 1e6, 1),
            "both_ms_per_step": round(t_both, 3),
            "bound_hom_mul_per_s": round(P / (max(t_both, ms / args.steps) / 1e3), 1),
            "note": "one step's input copies (pinned host -> device) and output copy, alone and at once; "
                    "the bound is the slower of the concurrent copies and the device step"}
    del sb

    # ---- plain per-call form: one cp_bfv_mul per pair ----
    PP = min(args.plain_pairs, P)
    outs = [e.empty(QBase) for _ in range(3)]

    def plain_step():
        for i in range(PP):
            e.bfv_mul(*outs, *[x[i:i + 1] for x in ins])

    plain_step()
    torch.cuda.synchronize()
    ev0.record(stream)
    plain_steps = max(1, args.steps // 4)
    for _ in range(plain_steps):
        plain_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    plain_ms = ev0.elapsed_time(ev1)
    plain_value = PP * plain_steps / (plain_ms / 1e3)

    # ---- dominant kernel: forward DGT over the step's 4P x |B| residues ----
    import json as _json
    peaks = {}
    try:
        peaks = _json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    xb = e.empty(1, 4 * P)
    xb.zero_()
    reps = 20
    e.dgt(xb, 1, FORWARD)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(reps):
        e.dgt(xb, 1, FORWARD)
    ev1.record(stream)
    torch.cuda.synchronize()
    dgt_ms = ev0.elapsed_time(ev1) / reps
    dgt_bytes = 2 * 16 * e.N * 4 * P * K_B  # read + write every Gaussian element once
    achieved = dgt_bytes / (dgt_ms / 1e3) / 1e9
    # integer roofline of the same launch: algorithmic Shoup multiplies and modular
    # adds at the measured peak rates of those primitives on this GPU
    from cupoly_b200.engine import dgt_op_counts, int_peaks
    peaks_int = int_peaks()
    ops = dgt_op_counts(e.N)
    nres_launch = 4 * P * K_B
    t_int = nres_launch * (ops["shoup"] / peaks_int["shoup"] + ops["addmod"] / peaks_int["addmod"])
    int_roof = {"model_ms": round(t_int * 1e3, 4), "measured_ms": round(dgt_ms, 4),
                "frac": round(t_int * 1e3 / dgt_ms, 4),
                "shoup_per_launch": ops["shoup"] * nres_launch, "addmod_per_launch": ops["addmod"] * nres_launch,
                "peak_shoup_per_s": round(peaks_int["shoup"], 1), "peak_addmod_per_s": round(peaks_int["addmod"], 1),
                "peak_mulmod_per_s": round(peaks_int["mulmod"], 1), "peak_imad32_per_s": round(peaks_int["imad32"], 1),
                "note": "frac = (Shoup / peak Shoup + adds / peak add) / measured; peaks measured live by cp_calibrate_int",
                "counters": INT_COUNTERS,
                "frac_counter": INT_COUNTERS["kernels"]["k_dgt_fwd<12,3,0>"]["busier_pipe_frac"]}

    # ---- polymul/s of the nphi = 4096, k = 2 configuration (batched) ----
    e1 = Engine(2, 3, 4096, 256)
    NPm = 1024
    pa, pb, pc = e1.empty(QBase, NPm), e1.empty(QBase, NPm), e1.empty(QBase, NPm)
    e1.sample(pa, QBase, UNIFORM, seed, 1, npolys=NPm, to_dgt=False)
    e1.sample(pb, QBase, UNIFORM, seed, 2 + NPm, npolys=NPm, to_dgt=False)
    from cupoly_b200.engine import INVERSE

    # ---- per-call polymul of the same configuration (one product per call sequence, operands
    # resident as in cuPoly's own timing: each product transforms its two operands in place) ----
    NPp = 64
    qa, qb, qc = pa[:NPp].clone(), pb[:NPp].clone(), e1.empty(QBase)

    def polymul_plain_step():
        for i in range(NPp):
            a_, b_ = qa[i:i + 1], qb[i:i + 1]
            e1.dgt(a_, QBase, FORWARD)
            e1.dgt(b_, QBase, FORWARD)
            e1.mul(qc, a_, b_, QBase)
            e1.dgt(qc, QBase, INVERSE)

    polymul_plain_step()
    torch.cuda.synchronize()
    ev0.record(stream)
    polymul_plain_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    polymul_plain_value = NPp / (ev0.elapsed_time(ev1) / 1e3)

    # ---- batched: coefficient domain in and out, fused cp_polymul (3 launches per batch), two consecutive
    # batches in flight on two streams (batch.PipelinedPolymul), each with its own output
    from cupoly_b200.batch import PipelinedPolymul
    ppm = PipelinedPolymul(e1, QBase, NPm, lanes=2)
    pouts = [pc, e1.empty(QBase, NPm)]
    ppm.run([(pa, pb)] * 2, pouts, stream)
    ppm.join(stream)
    torch.cuda.synchronize()
    ev0.record(stream)
    ppm.run([(pa, pb)] * 6, [pouts[i & 1] for i in range(6)], stream)
    ppm.join(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    polymul_value = NPm * 6 / (ev0.elapsed_time(ev1) / 1e3)
    # the timed outputs must be the bytes of one plain cp_polymul call on the same operands
    pref = e1.empty(QBase, NPm)
    e1.polymul(pref, pa, pb, QBase, e1.polymul_workspace(QBase, NPm), NPm)
    torch.cuda.synchronize()
    if not (torch.equal(pref, pouts[0]) and torch.equal(pref, pouts[1])):
        raise RuntimeError("pipelined polymul outputs differ from a single cp_polymul call")
    del pa, pb, pc, pouts, ppm, qa, qb, qc, pref

    # ---- mixed-size batch: 1024 products, nphi in {2048..16384}, k in 1..8, one CUDA graph ----
    from cupoly_b200.batch import MixedPolymul, random_specs
    mixed_specs = random_specs(1024, seed)
    # two instances (own buffers), their graphs replayed alternately on two streams: two
    # consecutive batches in flight
    m_streams = [torch.cuda.Stream(), torch.cuda.Stream()]

    def mixed_batches(mps_, n):
        for ms_ in m_streams:
            ms_.wait_stream(stream)
        for i in range(n):
            with torch.cuda.stream(m_streams[i & 1]):
                mps_[i & 1].graph.replay()
        for ms_ in m_streams:
            stream.wait_stream(ms_)

    # three forms of the same batch: the per-size-group launches in one graph (in sequence, or
    # one parallel branch per group), and ONE persistent launch over a tile work list
    mixed_forms, mixed_launches = {}, {}
    for form in ("sequence", "branches", "tiles"):
        mps = [MixedPolymul(mixed_specs, mode="tiles" if form == "tiles" else "graph") for _ in range(2)]
        for mp in mps:
            for g in mp.groups.values():  # residues below 2^62 are valid for every prime of the table
                g["a"].random_(0, 1 << 62)
                g["b"].random_(0, 1 << 62)
            mp.capture(branches=form == "branches")
        mixed_batches(mps, 4)
        torch.cuda.synchronize()
        ev0.record(stream)  # 40 batches: the steady state of two in flight, not its ramp
        mixed_batches(mps, 40)
        ev1.record(stream)
        torch.cuda.synchronize()
        mixed_forms[form] = ev0.elapsed_time(ev1) / 40
        mixed_launches[form] = mps[0].launches_per_run()
        mixed_bytes = mps[0].algorithmic_bytes()
        del mps, mp
        torch.cuda.empty_cache()
    best = min(mixed_forms, key=mixed_forms.get)
    mixed_ms = mixed_forms[best]
    mixed = {"config": "1024 products, nphi uniform in {2048, 4096, 8192, 16384}, k uniform in 1..8 (seeded), "
                       "2 batches in flight; fastest of three forms: %s" % best,
             "form": {"sequence": "one CUDA graph, per size group a fused cp_polymul_list (3 launches)",
                      "branches": "the same graph with one parallel branch per size group",
                      "tiles": "one persistent launch (cp_polymul_tiles) over a work list of tiles"}[best],
             "launches_per_batch": mixed_launches[best],
             "polymul_per_s": round(1024 / (mixed_ms / 1e3), 1), "ms_per_batch": round(mixed_ms, 3),
             "ms_per_batch_by_form": {k_: round(v_, 4) for k_, v_ in mixed_forms.items()},
             "launches_by_form": mixed_launches,
             "algorithmic_GB_per_s": round(mixed_bytes / (mixed_ms / 1e3) / 1e9, 1),
             "frac_hbm": round(mixed_bytes / (mixed_ms / 1e3) / 1e9 / hbm_peak, 4),
             "busier_pipe_frac": {"sequence": INT_COUNTERS["kernels"]["k_dgt_inv<11,3,0> products on load"][
                                      "busier_pipe_frac"],
                                  "tiles": INT_COUNTERS["kernels"]["k_polymul_tiles"]["busier_pipe_frac"],
                                  "source": "ncu capture (sequence: the fused polymul's kernels at nphi 4096)"}}
    torch.cuda.empty_cache()

    # ---- target configuration: nphi = 16384 (N = 2^14 coefficients), |Q| = 10, batched vs plain ----
    eT = Engine(10, 11, 16384, T_PLAIN)
    PT, PTp = 32, 4
    insT = []
    for j in range(4):
        x = eT.empty(QBase, PT)
        eT.sample(x, QBase, UNIFORM, seed, 4096 * j, npolys=PT, to_dgt=True)
        insT.append(x)
    cT = eT.empty(QBase, 3 * PT)
    wsT = eT.bfv_mul_batch_workspace(PT)
    eT.bfv_mul_batch(cT, *insT, PT, wsT)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(5):
        eT.bfv_mul_batch(cT, *insT, PT, wsT)
    ev1.record(stream)
    torch.cuda.synchronize()
    tgt_batched = 5 * PT / (ev0.elapsed_time(ev1) / 1e3)
    outsT = [eT.empty(QBase) for _ in range(3)]
    for i in range(PTp):
        eT.bfv_mul(*outsT, *[x[i:i + 1] for x in insT])
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(2):
        for i in range(PTp):
            eT.bfv_mul(*outsT, *[x[i:i + 1] for x in insT])
    ev1.record(stream)
    torch.cuda.synchronize()
    tgt_plain = 2 * PTp / (ev0.elapsed_time(ev1) / 1e3)
    target = {"config": "nphi=16384, k=10, kl=11, t=256", "batched_hom_mul_per_s": round(tgt_batched, 1),
              "pairs_per_call": PT, "plain_hom_mul_per_s": round(tgt_plain, 1),
              "batched_over_plain": round(tgt_batched / tgt_plain, 2)}
    del insT, cT, wsT, outsT, eT
    torch.cuda.empty_cache()

    # ---- large configuration: nphi = 32768, k = 16, kl = 17, t = 65537, 64 pairs + sampling ----
    large = None
    if not args.no_large:
        eL = Engine(16, 17, 32768, 65537)
        PL = 64
        insL = []
        for j in range(4):
            x = eL.empty(QBase, PL)
            eL.sample(x, QBase, UNIFORM, seed, 4096 * j, npolys=PL, to_dgt=True)
            insL.append(x)
        cL = eL.empty(QBase, 3 * PL)
        wsL = eL.bfv_mul_batch_workspace(PL)
        eL.bfv_mul_batch(cL, *insL, PL, wsL)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(3):
            eL.bfv_mul_batch(cL, *insL, PL, wsL)
        ev1.record(stream)
        torch.cuda.synchronize()
        large_ms = ev0.elapsed_time(ev1) / 3
        del insL, cL, wsL
        # fresh noise: 2^24 samples of each distribution (512 polys of nphi 32768), coefficient domain
        from cupoly_b200.engine import GAUSSIAN, TERNARY
        buf = eL.empty(QBase, 512)
        samp = {}
        for name, kind in (("ternary", TERNARY), ("gaussian", GAUSSIAN), ("uniform", UNIFORM)):
            eL.sample(buf, QBase, kind, seed, 0, npolys=512, to_dgt=False)
            torch.cuda.synchronize()
            ev0.record(stream)
            eL.sample(buf, QBase, kind, seed, 7, npolys=512, to_dgt=False)
            ev1.record(stream)
            torch.cuda.synchronize()
            sms = ev0.elapsed_time(ev1)
            samp[name] = {"samples_per_s": round((1 << 24) / (sms / 1e3), 1),
                          "GB_per_s_written": round(buf.numel() * 8 / (sms / 1e3) / 1e9, 1)}
        eL.check()
        large = {"config": "nphi=32768, k=16, kl=17, t=65537, 64 pairs per call", "hom_mul_per_s":
                 round(PL / (large_ms / 1e3), 1), "ms_per_call": round(large_ms, 3),
                 "sampling_2^24": samp}
        del buf, eL
        torch.cuda.empty_cache()

    # ---- the rows after the chain: coefficient I/O, xi / rho, wire format, CKKS ----
    nxt = next_rows(seed, hbm_peak) if (D.rank == 0 and not args.no_next) else None

    # ---- serving loop: open-loop Poisson arrivals, nphi in {4096..32768}, k = nphi/2048 ----
    serving = None
    if not args.no_serving and D.rank == 0:
        from cupoly_b200 import serving as SV
        classes = SV.default_classes()
        ex = SV.GpuExecutor(classes)
        n_req = args.serving_requests
        # saturation: every request offered at once (closed loop)
        sch = SV.Scheduler(classes, ex, 40 << 30)
        sat = sch.stats(sch.run(SV.poisson_requests(n_req, 1e9, len(classes), 1)))["throughput_req_s"]
        sweep = []
        for frac in (0.25, 0.5, 0.75, 0.9, 1.0, 1.1):
            sch = SV.Scheduler(classes, ex, 40 << 30)
            st = sch.stats(sch.run(SV.poisson_requests(n_req, frac * sat, len(classes), 1)))
            sweep.append({"offered_req_s": round(frac * sat, 1), "fraction_of_saturation": frac,
                          "throughput_req_s": st["throughput_req_s"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                          "mean_batch": st["mean_batch"], "peak_budget_bytes": st["peak_budget_bytes"]})
        serving = {"saturated_req_s": sat, "requests_per_rate": n_req, "budget_bytes": 40 << 30, "sweep": sweep,
                   "arrivals": "open-loop Poisson, seeded",
                   "classes": "nphi 4096/8192/16384/32768, k = nphi/2048, kl = k+1, t = 256, uniform mix"}
        del ex, sch
        torch.cuda.empty_cache()

    percall_cxx = dropin_percall_times() if D.rank == 0 else None

    # ---- reference legs, rank 0 only: cuPoly's own kernels per call on this GPU (when its
    # sources were compiled into oracle/_ref) and the CPU restatement of the path on the host
    # cores; the only places this arm executes anything under oracle/ ----
    cupoly_gpu = cupoly_gpu_times() if D.rank == 0 and not args.no_cupoly_gpu else None
    cpu = None
    if D.rank == 0 and not args.no_cpu_baseline:
        rate, done, el, cores = cpu_bfv_rate(10.0)
        cpu = {"value": round(rate, 3), "unit": "hom-mul/s", "cores": cores, "kind": "port",
               "sample": "%d pairs in %.1f s (nphi=8192, k=5) through oracle/cpoly_oracle.c, OpenMP" % (done, el)}
        # the same restatement on one core, on the same seeded inputs (one pair per call)
        from oracle import coracle
        coracle.set_threads(1)
        rate1, done1, el1, _ = cpu_bfv_rate(4.0, pairs_per_call=1)
        coracle.set_threads(cores)
        cpu["single_core"] = {"value": round(rate1, 3), "unit": "hom-mul/s", "cores": 1,
                              "sample": "%d pairs in %.1f s, one thread" % (done1, el1)}

    if D.rank == 0:
        line = {
            "metric": "BFV mul/s", "value": round(value, 2), "unit": "hom-mul/s", "n_gpus": D.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded uniform residues mod q_i (Philox), DGT domain",
            "config": {"workload": WORKLOAD + ", batched form", "pairs_per_step": P, "nphi": NPHI, "k": K_Q,
                       "kl": K_B, "t": T_PLAIN, "parallelism": "replicas x%d" % D.world,
                       "in_flight": "2 consecutive batches on 2 streams (batch.PipelinedBFV)",
                       "l2": "inputs larger than L2 (%.0f MB read per step)" % (4 * P * K_Q * e.N * 16 / 1e6)},
            "e2e": {"value": round(D.world * P * args.steps / (e2e_ms / 1e3), 2), "unit": "hom-mul/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "host_link": pcie},
            "plain": {"value": round(plain_value, 2), "unit": "hom-mul/s",
                      "form": "one cp_bfv_mul call per pair (cuPoly's per-call composition)", "pairs": PP},
            "plain_cxx": percall_cxx,
            "batched_over_plain": round(value / D.world / plain_value, 2),
            "polymul": ({"value": round(polymul_value, 1), "unit": "polymul/s",
                         "config": "nphi=4096, k=2, batch 1024 (fused: 2 forward DGTs, inverse with products on load), 2 batches in flight",
                         "algorithmic_GB_per_s": round(polymul_value * 24 * 4096 * 2 / 1e9, 1),
                         "frac_hbm": round(polymul_value * 24 * 4096 * 2 / 1e9 / hbm_peak, 4),
                         "plain_value": round(polymul_plain_value, 1),
                         "plain_form": "one product per call sequence from Python (2 forward DGTs in place, "
                                       "multiply, inverse DGT; 4 calls)"}
                        if polymul_value else None),
            "mixed_polymul": mixed,
            "target": dict(target, **({"plain_cxx_hom_mul_per_s": percall_cxx["bfv_mul_nphi16384_k10_kl11"]["per_s"],
                                       "batched_over_plain_cxx": round(
                                           target["batched_hom_mul_per_s"] /
                                           percall_cxx["bfv_mul_nphi16384_k10_kl11"]["per_s"], 2)}
                                      if percall_cxx and "bfv_mul_nphi16384_k10_kl11" in percall_cxx else {})),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(achieved / hbm_peak, 4),
                         # dram__bytes_read.sum + dram__bytes_write.sum of this launch (same
                         # kernel, 3072 residues of N = 4096) from one ncu capture; writes read low
                         # because dirty lines are still in L2 when the kernel ends
                         "traffic": 346929920 if (e.N == 4096 and 4 * P * K_B == 3072) else None,
                         "traffic_source": "ncu capture",
                         "kernel": "k_dgt_fwd (forward DGT, %d residues of N=%d per launch, timed alone)" %
                                   (4 * P * K_B, e.N),
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst)" if peaks else "fallback",
                         "int": int_roof},
            "cupoly_gpu": cupoly_gpu,
            "large": large,
            "next_rows": nxt,
            "serving": serving,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches_per_step * args.steps,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    D = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, D)
        else:
            run_ours(args, D)
    finally:
        D.close()


if __name__ == "__main__":
    main()
