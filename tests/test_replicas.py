"""Multi-process paths on the CPU (gloo, world size 2): the replica timing of
bench.py (max over ranks) and the sharding of independent problems across
ranks with only scalar results gathered.  The per-problem work here is the CPU
oracle's log-likelihood, so the test needs no GPU."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from exageostatcpp_b200 import replicas as R


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


SIZES = [120, 40, 200, 64, 150, 90, 33, 170]


def rank_main(rank, world, port, out_dir):
    import datetime
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shards = R.shard_by_cost(SIZES, world)
        mine = {}
        for i in shards[rank]:
            x, y, z = O.load_data(SIZES[i], 100 + i, (1.0, 0.1, 0.5))
            mine[i] = float(O.mle_loglik(x, y, z, (1.0, 0.1, 0.5)))
        allres = R.gather_results(mine, dist)
        t = R.max_over_ranks(1.0 + rank, dist)
        rate = R.replica_rate(10.0, 2.0 + rank, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "res.npy"), np.array([allres[i] for i in range(len(SIZES))]))
            np.save(os.path.join(out_dir, "t.npy"), np.array([t, rate]))
    finally:
        dist.destroy_process_group()


def test_shard_by_cost_balances_and_covers():
    sh = R.shard_by_cost(SIZES, 3)
    assert sorted(i for s in sh for i in s) == list(range(len(SIZES)))
    loads = [sum(SIZES[i] ** 3 for i in s) for s in sh]
    assert max(loads) <= 1.34 * (sum(loads) / 3) + max(x ** 3 for x in SIZES)
    assert R.shard_by_cost(SIZES, 3) == sh  # deterministic on every rank
    assert R.shard_by_cost(SIZES, 1) == [list(range(len(SIZES)))]


def test_single_process_fallbacks():
    assert R.max_over_ranks(3.5) == 3.5
    assert R.gather_results({1: 2.0}) == {1: 2.0}
    assert R.replica_rate(10, 2.0) == 5.0


def test_two_ranks_gloo(tmp_path):
    from oracle import oracle as O
    world = 2
    mp.spawn(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    res = np.load(tmp_path / "res.npy")
    serial = []
    for i, n in enumerate(SIZES):
        x, y, z = O.load_data(n, 100 + i, (1.0, 0.1, 0.5))
        serial.append(float(O.mle_loglik(x, y, z, (1.0, 0.1, 0.5))))
    assert np.array_equal(res, np.array(serial))
    t, rate = np.load(tmp_path / "t.npy")
    assert t == 2.0                      # the slower rank's time
    assert rate == pytest.approx(2 * 10.0 / 3.0)
