"""The autotuner's search and cache logic, on a fake context whose per-kernel times are a known
function of the launch shape (no GPU)."""
import json

from lydion_b200 import autotune as A


class FakeCtx:
    n_nu, n_r, n_z, precision = 64, 256, 256, 0

    def __init__(self):
        self.t = (16, 0, 0, 0, 0)
        self.timing_on = False
        self.steps = 0
        self.applied = []

    def set_tuning(self, r, c, s, o=0, g=0):
        self.t = (r, c, s, o, g)
        self.applied.append(self.t)

    def synchronize(self):
        pass

    def set_timing(self, on):
        self.timing_on = on

    def timing(self):
        r, c, s, o, g = self.t
        adv = 1.0 + abs(r - 8) * 0.1 + 0.05 * abs(o - 3) + (0.02 if g == 1 else 0.0)
        freq = 2.0 + (0.5 if s == 1 else 0.0) + abs((c or 96) - 64) * 0.01
        return [adv * self.steps, freq * self.steps, 0.1 * self.steps]

    def run(self, n):
        self.steps = n


def test_search_picks_the_fastest_shape():
    ctx = FakeCtx()
    best, table = A.search(ctx, ctx.run, steps=5)
    assert best[:3] == (8, 64, 0) and best[4] == 2
    assert len(table) == len(A.ROWS) * 2 * len(A.STAGING) + len(A.CELLS) * len(A.SOLVERS)
    assert not ctx.timing_on
    ctx = FakeCtx()
    ctx.precision = 1
    best, table = A.search(ctx, ctx.run, steps=5)
    assert best == (8, 64, 0, 3, 2)
    assert len(table) == len(A.ROWS) * len(A.CTAS) * len(A.STAGING) + len(A.CELLS) * len(A.SOLVERS)


def test_cache_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(A, "device_name", lambda device=0: "fake-gpu")
    path = str(tmp_path / "tune.json")
    ctx = FakeCtx()
    assert A.autotune(ctx, ctx.run, steps=3, cache=path) == (8, 64, 0, 3, 2)
    data = json.load(open(path))
    key = A.workload_key(ctx)
    assert key.startswith("fake-gpu|nnu=64|prec=0|clouds=1|")
    assert data[key]["tuning"] == [8, 64, 0, 3, 2]
    # a second call applies the cached shape without timing anything
    ctx2 = FakeCtx()
    assert A.autotune(ctx2, ctx2.run, steps=3, cache=path) == (8, 64, 0, 3, 2)
    assert ctx2.applied == [(8, 64, 0, 3, 2)]


def test_batch_key_depends_on_sizes(monkeypatch):
    monkeypatch.setattr(A, "device_name", lambda device=0: "g")
    a, b = FakeCtx(), FakeCtx()
    a.sizes = [(32, 48), (64, 64)]
    b.sizes = [(32, 48), (64, 96)]
    assert A.workload_key(a) != A.workload_key(b)
    b.sizes = [(64, 64), (32, 48)]
    assert A.workload_key(a) == A.workload_key(b)


def test_reset_runs_before_every_candidate():
    ctx = FakeCtx()
    calls = []
    best, table = A.search(ctx, ctx.run, steps=5, reset=lambda: calls.append(ctx.t))
    assert len(calls) == len(table)


def _writer(path, rank, n):
    from lydion_b200 import autotune as A_
    for k in range(n):
        A_._save(path, {f"rank{rank}|k{k}": {"rank": rank, "k": k}})


def test_concurrent_cache_writes_keep_every_key(tmp_path):
    """Under torchrun every rank tunes its own GPU (its own workload keys) and writes the same
    cache file at once: every key of every writer survives, and no temporary file is left."""
    import multiprocessing as mp
    import os
    path = str(tmp_path / "tuning.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(path, r, 50)) for r in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert [p.exitcode for p in procs] == [0, 0, 0, 0]
    data = json.load(open(path))
    assert sorted(data) == sorted(f"rank{r}|k{k}" for r in range(4) for k in range(50))
    assert all(data[f"rank{r}|k{k}"] == {"rank": r, "k": k} for r in range(4) for k in range(50))
    assert sorted(os.listdir(tmp_path)) == ["tuning.json", "tuning.json.lock"]
