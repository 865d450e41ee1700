"""Ensemble host logic on CPU: the member split over ranks, and
run_ensemble (ensemble_impl.py:49-67) over two gloo ranks giving the same
result as one process."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pymrst_b200.ensemble import gaussian_samples, run_ensemble, shard_members


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _qoi(theta):
    return np.array([theta.sum(), theta.prod(), float(np.sin(theta[0]))])


def test_shards_are_contiguous_balanced_and_cover_every_member():
    costs = np.array([5, 1, 1, 1, 8, 2, 2, 4, 4, 1], float)
    for world in (1, 2, 3, 4, 10, 12):
        blocks = shard_members(costs, world)
        assert len(blocks) == world
        assert blocks[0][0] == 0 and blocks[-1][1] == costs.size
        for (a, b), (c, d) in zip(blocks, blocks[1:]):
            assert b == c and a <= b
    loads = [costs[a:b].sum() for a, b in shard_members(costs, 2)]
    assert max(loads) <= 0.5 * costs.sum() + costs.max()


def test_single_process_matches_a_loop():
    params = gaussian_samples(np.zeros(3), np.ones(3), 7, np.random.default_rng(1))
    res = run_ensemble(params, _qoi)
    expect = np.column_stack([_qoi(params[:, k]) for k in range(7)])
    np.testing.assert_array_equal(res.qoi, expect)
    assert res.mean.shape == (3,) and res.std.shape == (3,)


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        params = gaussian_samples(np.zeros(3), np.ones(3), 9, np.random.default_rng(2))
        res = run_ensemble(params, _qoi, costs=np.arange(1, 10))
        q.put((rank, res.qoi))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_the_same_result_as_one_process():
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
    params = gaussian_samples(np.zeros(3), np.ones(3), 9, np.random.default_rng(2))
    expect = np.column_stack([_qoi(params[:, k]) for k in range(9)])
    for _, qoi in out:
        np.testing.assert_array_equal(qoi, expect)


def test_autotune_cache_key_and_reuse(tmp_path, monkeypatch):
    """The tuner's cache key buckets the ensemble's shape; a cached entry is
    returned without trials (no GPU needed for either)."""
    import json
    from types import SimpleNamespace
    from pymrst_b200 import ensemble as ens
    monkeypatch.setenv("PMB_TUNE_CACHE", str(tmp_path / "t.json"))
    mem = [(SimpleNamespace(cells=SimpleNamespace(num=3000)), None, None)] * 100
    key = ens.tune_key(mem, 148, True)
    assert key == "ensemble_workers/sm148/graph1/m2^7/c2^12"
    (tmp_path / "t.json").write_text(json.dumps({key: {"workers": 8}}))

    class FakeTorch:
        class cuda:
            @staticmethod
            def current_device():
                return 0

            @staticmethod
            def get_device_properties(i):
                return SimpleNamespace(multi_processor_count=148)
    monkeypatch.setattr(ens, "_torch", lambda: FakeTorch)
    out = ens.tune_workers(mem, None, [None] * 100, [1.0])
    assert out == {"workers": 8, "key": key, "trials": {}}
