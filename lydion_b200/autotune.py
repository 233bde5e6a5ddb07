"""Launch-shape autotuner for the Lyman-alpha step.

Five knobs of a context are tuned (lyd_set_tuning):
  rows_per_tile    rows of the advection tile each CTA marches through (4..64);
  adv_ctas_per_sm  resident advection CTAs per SM (2..4 with FP32 arithmetic, 2..3 with FP64);
  adv_staging      how the advection stages its rows: per-lane loads (1) or bulk tensor copies
                   of each row's box completed on an mbarrier (2);
  cells_per_block  cells per frequency-kernel block (8..1024, or 0 = automatic);
  solver           frequency tridiagonal solver: 0 = parallel cyclic reduction across the warp,
                   1 = lane-serial elimination.
The advection kernel depends only on rows_per_tile, adv_ctas_per_sm and adv_staging, the
frequency kernel and the reductions only on the other two, so the search is two short sweeps:
rows x CTAs x staging first (advection time), then cells x solver (frequency + reduction time). Every candidate is timed on the device with the
library's per-kernel CUDA events (lyd_set_timing) over a few real steps of the caller's
workload, after one untimed step that applies the new shape.

Tuning advances the context's state by the steps it runs: tune a scratch context built from
the same workload when the state must stay untouched, or pass `reset`, which is called before
every candidate to put the same state back (the advection's tile count against the SMs' CTA
slots, and the active window, make the shapes' times depend on the state they run from). Results are cached as JSON, keyed by
the GPU name and the workload's shape, in $LYDION_TUNE_CACHE or
~/.cache/lydion_b200/tuning.json.
"""
import hashlib
import json
import os
import tempfile

import numpy as np

ROWS = (4, 8, 12, 16, 20, 24, 32, 40, 48)
CTAS = (2, 3, 4)
CELLS = (0, 16, 32, 64, 128, 256, 512)
SOLVERS = (0, 1)
STAGING = (1, 2)        # per-lane loads, bulk tensor copies (the library falls back to the first
                        # where the layout does not allow the second)


def cache_path():
    p = os.environ.get("LYDION_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "lydion_b200", "tuning.json")


def device_name(device=0):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def workload_key(ctx, device=0):
    """GPU name + bins + precision + cloud sizes (hashed for batches)."""
    sizes = getattr(ctx, "sizes", None) or [(ctx.n_r, ctx.n_z)]
    h = hashlib.sha1(np.asarray(sorted(sizes), dtype=np.int64).tobytes()).hexdigest()[:12]
    return f"{device_name(device)}|nnu={ctx.n_nu}|prec={ctx.precision}|clouds={len(sizes)}|sizes={h}|knobs=5"


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(path, entries):
    """Merge `entries` (workload key -> record) into the cache file. Ranks that tune at the same
    time (one process per GPU) may hold different keys: under an exclusive lock on a sidecar
    file each writer re-reads the cache, adds its own keys and replaces the file atomically
    through a temporary file of its own, so no writer drops another's entries and no reader
    ever sees a torn file."""
    import fcntl
    d = os.path.dirname(path) or "."
    os.makedirs(d, exist_ok=True)
    with open(path + ".lock", "a") as lk:
        fcntl.flock(lk, fcntl.LOCK_EX)
        try:
            data = _load(path)
            data.update(entries)
            fd, tmp = tempfile.mkstemp(prefix=os.path.basename(path) + ".", suffix=".tmp", dir=d)
            try:
                with os.fdopen(fd, "w") as f:
                    json.dump(data, f, indent=1, sort_keys=True)
                os.replace(tmp, path)
            except BaseException:
                if os.path.exists(tmp):
                    os.unlink(tmp)
                raise
        finally:
            fcntl.flock(lk, fcntl.LOCK_UN)


def _measure(ctx, run, tuning, steps):
    ctx.set_tuning(*tuning)
    run(1)
    ctx.synchronize()
    ctx.set_timing(True)
    try:
        run(steps)
        ctx.synchronize()
        ms = np.asarray(ctx.timing(), dtype=np.float64) / steps
    finally:
        ctx.set_timing(False)
    return ms


def search(ctx, run, steps=10, rows=ROWS, cells=CELLS, solvers=SOLVERS, ctas=CTAS, staging=STAGING, reset=None):
    """Time every candidate (each after `reset()`, when given); return (best tuning tuple, table
    of (tuning, ms[3]))."""
    table = []
    if getattr(ctx, "precision", 0) == 0:
        ctas = tuple(o for o in ctas if o in (2, 3)) or (0,)   # FP64 arithmetic: 2 or 3 CTAs per SM
    best_rows, best_adv = None, np.inf
    for r in rows:
        for o in ctas:
            for g in staging:
                t = (r, 0, 0, o, g)
                if reset:
                    reset()
                ms = _measure(ctx, run, t, steps)
                table.append((t, ms.tolist()))
                if ms[0] < best_adv:
                    best_rows, best_adv = (r, o, g), ms[0]
    best, best_f = None, np.inf
    for s in solvers:
        for cb in cells:
            t = (best_rows[0], cb, s, best_rows[1], best_rows[2])
            if reset:
                reset()
            ms = _measure(ctx, run, t, steps)
            table.append((t, ms.tolist()))
            if ms[1] + ms[2] < best_f:
                best, best_f = t, ms[1] + ms[2]
    return best, table


def autotune(ctx, run, steps=10, device=0, cache=None, force=False, **grid):
    """Tune `ctx` for the workload `run(n)` (which runs n steps on ctx), apply the best shape,
    and return it. A cached entry for the same GPU and workload shape is applied without
    timing unless `force`."""
    path = cache or cache_path()
    key = workload_key(ctx, device)
    data = _load(path)
    if not force and key in data:
        t = tuple(data[key]["tuning"])
        ctx.set_tuning(*t)
        return t
    best, table = search(ctx, run, steps=steps, **grid)
    ctx.set_tuning(*best)
    _save(path, {key: {"tuning": list(best), "table": [[list(t), ms] for t, ms in table], "steps": steps}})
    return best


def main():
    import argparse
    ap = argparse.ArgumentParser(description="tune the launch shapes of a workload and cache them")
    ap.add_argument("--workload", choices=["c2", "c3"], default="c2")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    from . import workloads as W
    from .m1 import batch_for_clouds, cloud_params, context_for_cloud
    if args.workload == "c2":
        cl = W.config_c2()
        ctx = context_for_cloud(cl)
        p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
        run = lambda n: ctx.static_steps(n, *p, history=False)
        init = {n: ctx.download(n) for n in ("J", "H_r", "H_Z")}
        reset = lambda: [ctx.upload(n, x) for n, x in init.items()]
    else:
        clouds = W.config_c3()
        ctx = batch_for_clouds(clouds)
        pp = cloud_params(clouds)
        run = lambda n: ctx.batch_steps(n, pp, history=False)
        reset = None
    t = autotune(ctx, run, steps=args.steps, force=args.force, reset=reset)
    print(json.dumps({"workload": args.workload, "tuning": list(t), "cache": cache_path()}))
    ctx.close()


if __name__ == "__main__":
    main()
