"""bench.py host logic on CPU.  Several ranks (replicas, one process per GPU) as two
gloo ranks on 127.0.0.1.  The path has no data-path collective; the ranks
meet only for the slowest rank's time (max over ranks) and a barrier.
Checked here: the max over ranks, the weak-scaling value, per-rank batches
(seed 4 + rank: different structures of the same kind), that the
reference arm runs on rank 0 alone, and the reference arm's JSON line."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        W = bench.__graft_entry__.load_package().workloads
        structs, off, Z, pos, per, latf = bench.workload(W, 8, 4 + rank)
        t = bench.max_over_ranks(1.5 + rank, world, "cpu")
        out.put((rank, t, int(off[-1]), float(np.sum(pos)), int(Z.sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (r0, t0, n0, s0, z0), (r1, t1, n1, s1, z1) = res
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 2.5  # the slowest rank's time on every rank
    assert s0 != s1  # each replica evaluates its own batch


def test_weak_value_and_single_rank_max():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.weak_value(1000, 4, 10, 2.0) == 1000 * 4 * 10 / 2.0
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench

    args = SimpleNamespace(structs=8, steps=1, warmup=0, cpu_sample=4)
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference(args, 1, 2) is None
    assert buf.getvalue() == ""


def test_reference_arm_line_on_cpu():
    """bench.py --impl reference: the reference's algorithm (the oracle source
    built -O3 -march=native -fopenmp on this host) on the host cores prints one
    JSON line with the contract's keys; no GPU involved."""
    import json
    import subprocess

    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--structs", "16",
                        "--steps", "1", "--warmup", "0", "--cpu-sample", "32"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "atom-steps/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["dtype"] == "f64"
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
