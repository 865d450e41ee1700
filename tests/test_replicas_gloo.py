"""The N-rank timing reduction of bench.py, run as two gloo ranks on CPU."""

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from pymrst_b200.replicas import reduce_timing
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sec, work = reduce_timing(1.0 + rank, 100.0 * (rank + 1), device="cpu")
        q.put((rank, sec, work))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_is_max_time_and_summed_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, sec, work in out:
        assert sec == 2.0 and work == 300.0


def test_single_process_returns_local_values():
    from pymrst_b200.replicas import reduce_timing
    assert reduce_timing(3.0, 7.0) == (3.0, 7.0)
