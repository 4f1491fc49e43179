"""The N > 1 path of bench.py on CPU: two gloo ranks on 127.0.0.1 run the
same rank plumbing the driver's torchrun launch uses (process group,
barriers, max over ranks, whole-job value, rank-0-only reference arm)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_init()
    try:
        bench.barrier(w)
        mx = bench.reduce_max(w, 1.5 + r)
        # rank r took 2 + r seconds for 10 trees: the job took the slowest
        val = bench.whole_job_value(w, 2.0 + r, 10)

        class A:  # the reference arm returns at once on every rank but 0
            steps, warmup, gpus = 1, 3, w
        if r != 0:
            bench.run_reference(A, w, r)
        bench.barrier(w)
        q.put((r, w, local, mx, val))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    for r, (rr, w, local, mx, val) in enumerate(got):
        assert (rr, w, local) == (r, world, r)
        assert mx == pytest.approx(2.5)
        assert val == pytest.approx(100.0 * 3.0 / (10 * world))


def test_single_rank_is_plain():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(1, 3.25) == 3.25
    assert bench.whole_job_value(1, 2.0, 10) == pytest.approx(20.0)
