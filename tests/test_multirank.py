"""The N>1 plumbing of bench.py on CPU: two gloo ranks.

bench.py --gpus N runs N independent replicas (no collective on the data
path); what crosses ranks is the barrier around the timed region and the
max-over-ranks of the timing.  This checks that reduction and the
weak-scaling aggregate with world_size 2 (gloo, 127.0.0.1), no GPU.
"""
import importlib.util
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        dist.barrier()
        ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        worst = b.max_over_ranks(ms, world)
        mlups = b.aggregate_mlups(256 ** 3, 100, worst, world)
        q.put((rank, worst, mlups))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, worst, mlups in out:
        assert worst == 15.0
        assert mlups == pytest.approx(2 * 256 ** 3 * 100 / 0.015 / 1e6)


def test_single_rank_needs_no_process_group():
    b = _bench()
    assert b.max_over_ranks(3.5, 1) == 3.5
    assert b.aggregate_mlups(1000, 10, 1.0, 1) == pytest.approx(10.0)
