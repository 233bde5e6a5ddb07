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


def _slab_worker(rank, world, port, q):
    """Two gloo ranks run the slab driver's communication (TorchComm) on CPU tensors: the column
    sums all-reduce, and each rank receives its neighbour's two boundary rows."""
    import torch
    import torch.distributed as dist
    from lydion_b200 import domain as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    class Fake:
        pass
    r = Fake()
    r.rank, r.n_ranks = rank, world
    r.j0, r.j1, r.hb, r.ht = D.slab_layout(9, world, rank)
    r.sides = lambda: [s for s, h in ((0, r.hb), (1, r.ht)) if h]
    r.neighbour = lambda s: rank - 1 if s == 0 else rank + 1
    r.colsum = torch.arange(5, dtype=torch.float64) * (rank + 1)
    r.send = {s: torch.full((6,), 10.0 * rank + s, dtype=torch.float64) for s in (0, 1)}
    r.recv = {s: torch.zeros(6, dtype=torch.float64) for s in (0, 1)}
    comm = D.TorchComm()
    comm.allreduce([r])
    comm.exchange([r])
    got = {s: r.recv[s][0].item() for s in r.sides()}
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, r.colsum.tolist(), got))


def test_slab_communication_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, c0, g0), (r1, c1, g1) = res
    assert c0 == c1 == [0.0, 3.0, 6.0, 9.0, 12.0]
    # rank 0 (lower slab) receives rank 1's lower boundary rows (its send[0]) into recv[1], and back
    assert g0 == {1: 10.0} and g1 == {0: 1.0}
