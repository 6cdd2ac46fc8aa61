"""The multi-process plumbing of bench.py on CPU: two gloo ranks (what torchrun launches for
--gpus 2) agree on the slowest rank's time, and only rank 0 runs and prints the reference arm."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        got = bench.rank_max(1.5 + rank, world, "cpu")
        w, r, l = bench.dist_setup()
        # reference arm: ranks other than 0 return without work or output
        buf = io.StringIO()
        if r != 0:
            with redirect_stdout(buf):
                bench.run_reference(type("A", (), {"steps": 1, "gpus": world})(), bench.WORKLOADS["dg512"])
        out.put((rank, got, (w, r, l), buf.getvalue()))
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
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [2.5, 2.5]
    assert [r[2] for r in res] == [(2, 0, 0), (2, 1, 1)]
    assert res[1][3] == ""


def test_cpu_baseline_uses_every_usable_core(monkeypatch):
    """A launcher's OMP_NUM_THREADS (torchrun sets 1 for N > 1) does not shrink the CPU
    baseline: the oracle is given every usable core unless a thread count is asked for."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("OMP_NUM_THREADS", "1")
    w = bench.WORKLOADS["dg512"]
    _, threads, sample, _ = bench.cpu_sample(w, 1, n=32)
    assert threads == len(os.sched_getaffinity(0)), sample
    try:
        _, one, _, _ = bench.cpu_sample(w, 1, threads=1, n=32)
        assert one == 1
    finally:  # the OpenMP thread count is process-wide: give later oracle tests every core back
        from oracle.oracle import Oracle
        Oracle("dp").set_threads(len(os.sched_getaffinity(0)))
