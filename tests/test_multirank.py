"""The N > 1 host path on CPU: two gloo ranks agree on the max of their timings and on the
cloud partition; the partition balances the ragged cloud batch."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lydion_b200 import sharding


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [3.0, 5.5][rank]
    m = sharding.max_over_ranks(ms)
    rng = np.random.default_rng(4)
    sides = rng.choice([32, 48, 64, 96, 128, 192, 256], size=(64, 2))
    costs = [int(a * b * 48) for a, b in sides]
    parts = sharding.partition_clouds(costs, world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, m, parts))


def test_two_gloo_ranks_agree():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, p0), (r1, m1, p1) = res
    assert m0 == m1 == 5.5
    assert p0 == p1
    assert sorted(sum(p0, [])) == list(range(64))


def test_partition_is_balanced_and_deterministic():
    rng = np.random.default_rng(7)
    sides = rng.choice([32, 48, 64, 96, 128, 192, 256], size=(512, 2))
    costs = [int(a * b * 48) for a, b in sides]
    for n in (1, 2, 4, 8):
        parts = sharding.partition_clouds(costs, n)
        loads = [sum(costs[q] for q in p) for p in parts]
        assert sorted(sum(parts, [])) == list(range(512))
        assert max(loads) <= sum(costs) / n + max(costs)
        assert parts == sharding.partition_clouds(costs, n)
    with pytest.raises(ValueError):
        sharding.partition_clouds(costs, 0)


def test_weak_scaling_value():
    assert sharding.weak_scaling_throughput(1e6, 4, 2.0) == pytest.approx(2e9)
