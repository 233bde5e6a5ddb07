"""Host-side logic of the multi-GPU mode: independent clouds are the unit of work, so the
step shards across ranks with no data-path collective. Clouds are assigned to ranks by
longest-processing-time bin packing on their cell-bin count, and per-rank device times
are combined by a max over ranks."""
import heapq


def partition_clouds(costs, n_ranks):
    """Greedy LPT assignment of clouds (cost = N_r N_Z N_nu) to ranks -> list of index lists.
    Deterministic: ties break on the lower rank, then on the lower cloud index."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda q: (-costs[q], q))
    heap = [(0, r) for r in range(n_ranks)]
    out = [[] for _ in range(n_ranks)]
    for q in order:
        load, r = heapq.heappop(heap)
        out[r].append(q)
        heapq.heappush(heap, (load + costs[q], r))
    return [sorted(v) for v in out]


def max_over_ranks(value, device=None):
    """Max of a float over all ranks of the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_throughput(units_per_rank, world, ms_max):
    """Whole-job units/s: every rank processed `units_per_rank` units within ms_max."""
    return world * units_per_rank / (ms_max * 1e-3)
