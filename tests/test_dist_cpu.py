"""Multi-process plumbing of bench.py on CPU: gloo process group, world size 2.

The hot path shards as independent replicas (no data-path collective); what
the multi-GPU run adds is the process group, the barriers around the timed
region and the max-over-ranks of the device time.  These tests run that
plumbing with the gloo backend on the host.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    D = bench.Dist()
    try:
        v = D.max(10.0 * (rank + 1))
        D.barrier()
        q.put((rank, v, D.pg.get_backend() if D.pg else None))
    finally:
        D.close()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = sorted(q.get(timeout=180) for _ in range(2))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert got == [(0, 20.0, "gloo"), (1, 20.0, "gloo")]
    assert all(p.exitcode == 0 for p in procs)


def test_reference_arm_torchrun_world2():
    """`bench.py --impl reference` under torchrun: rank 0 alone prints one line."""
    from oracle import coracle

    coracle.lib()  # the CPU restatement the reference arm times
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
