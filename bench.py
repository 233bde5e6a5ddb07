"""Benchmark of the Lyman-alpha M1 step: cell-bin updates per second on the 256x256 x 64-bin
dusty outflowing cloud (tau0 = 1e8, tau_abs = 1, uniform source r_s = 0.5 R_cl, Hubble
outflow v_max = 200 km/s), one static-cloud driver iteration per step.

The headline value is the FP64 form, the reference's arithmetic. The same line carries the
reduced-precision forms (FP32 flux arithmetic over FP64 storage; FP32 storage) with their
ratio to FP64 and their error against it over 2000 steps, the ragged batch of 512 clouds (48
bins, sides 32..256), the adjoint/forward cost on the 128x128x48 turbulent cloud over 2000
steps with checkpoints every 100 steps, and the 1024x1024x128 field.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One unit of work is one (cell, frequency bin) advanced through one full step: advection of
the active bins, emission/absorption, frequency factors + FP64 tridiagonal solve, flux
correction and the per-step reductions (N_r N_Z N_nu per step regardless of the active
window). With N > 1 (torchrun) every rank advances its own copy of the cloud: the clouds are
independent, so the step has no data-path collective and the scaling is weak.

`--impl reference` times the reference algorithm on the host cores instead: the Julia
reference cannot run on this machine, so its FP64 C restatement under oracle/ stands in.
"""
import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Lyα M1 cell·bin updates/s at 256²×64, mixed vs FP64 GPU; adjoint/forward cost"
UNIT = "cell·bin updates/s"
WORKLOAD = "c2_dusty_outflow_256x256x64_tau1e8"


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0}, "fallback"


def profile_traffic(kernel, precision):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    return profile_figure(kernel, precision, "dram_bytes_per_launch")


def profile_figure(kernel, precision, key):
    """A `key: value` figure of the committed ncu summary of `kernel`, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_c2_{precision}.md")
    if not os.path.exists(path):
        return None
    m = re.search(key + r":\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if len(r) > 5 + q and r[5 + q].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(n_nu, s):
    """Algorithmic HBM bytes per cell-bin of each kernel: the four streams read (J, H_r, H_Z,
    H_voigt) and three written (J, H_r, H_Z) of storage size s, plus the per-cell inputs
    amortised over the bins (advection: 11 doubles -- velocity-gradient terms, u*_r, u*_Z,
    areas, 1/dV, alpha, <1/r>; frequency step: 15 doubles -- alpha, alpha_c, pd, js, T, the
    five gradient terms, dV, the phi normalisation, rCoM/ZCoM, f_r, f_Z)."""
    return {"advect": 7 * s + 11 * 8 / n_nu, "freq": 7 * s + 15 * 8 / n_nu}


def cpu_baseline(cloud, budget_s=15.0, max_steps=40):
    """The FP64 oracle (a C restatement of the reference path, OpenMP on every host core)
    on the same cloud, for a bounded number of steps."""
    from oracle import oracle as O
    st = O.OracleState(cloud)
    st.setup_profiles()
    st.step()  # warm-up (first touch of the scratch arrays)
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        st.step()
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n * cloud.cell_bins / dt, "unit": UNIT, "cores": int(O.lib().orc_num_threads()),
            "kind": "port", "sample": f"{n} full steps of the {cloud.nr}x{cloud.nz}x{cloud.n_nu} cloud, FP64"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    from lydion_b200 import workloads as W
    from oracle import oracle as O
    cloud = W.config_c2()
    st = O.OracleState(cloud)
    st.setup_profiles()
    # one step of the reference arm is one full FP64 step of the whole cloud on the host;
    # the timed count is capped so the run stays within a few minutes of wall clock
    for _ in range(args.warmup):
        st.step()
    t0 = time.perf_counter()
    n = 0
    while n < args.steps and (n == 0 or time.perf_counter() - t0 < 90.0):
        st.step()
        n += 1
    el = time.perf_counter() - t0
    args.steps = n
    v = n * cloud.cell_bins / el
    cores = int(O.lib().orc_num_threads())
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded static cloud set-up)",
            "config": {"workload": WORKLOAD, "cells": [cloud.nr, cloud.nz], "bins": cloud.n_nu, "tau0": 1e8},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} full FP64 steps of the {cloud.nr}x{cloud.nz}x{cloud.n_nu} cloud "
                                       "(C restatement of the Julia reference; Julia is not installed)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _timed(ctx, run, n, stream_of):
    import torch
    stream = stream_of(ctx)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run(n)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def measure_form(cloud, prec, args, barrier, stream_of, local, world, clk=None):
    """One precision form of the C2 step: launch shapes tuned (autotune, cached), W warm-up
    steps, K timed steps between barriers, then per-kernel device times over a separate pass."""
    from lydion_b200 import autotune, sharding
    from lydion_b200.m1 import context_for_cloud
    ctx = context_for_cloud(cloud, precision=prec, device=local)
    p = (cloud.c_tilde, cloud.dt, cloud.z_center, cloud.bc_r_right, cloud.bc_z_bot, cloud.bc_z_top)
    run = lambda n: ctx.static_steps(n, *p, history=False)
    fields = ("J", "H_r", "H_Z")
    init = {n: ctx.download(n) for n in fields}

    def reset(state):   # a saved state (and with it its active window)
        for n, x in state.items():
            ctx.upload(n, x)

    if args.no_tune:
        tuning = ctx.tuning()
    else:
        # Candidates are timed from the state halfway through the timed region: the active window
        # widens over the run, and from the set-up state's narrower window the tuner picked
        # 20-row tiles, which ran the timed steps at 9.44e9 cell-bin/s against 9.56e9 for 16 rows.
        # 30 steps per candidate: neighbouring tile heights differ by ~1 %, less than 10 steps resolve
        run(args.warmup + args.steps // 2)
        mid = {n: ctx.download(n) for n in fields}
        tuning = autotune.autotune(ctx, run, steps=30, device=local, reset=lambda: reset(mid),
                                   cache=os.path.join(tempfile.gettempdir(), "lydion_bench_tuning.json"))
        reset(init)
    run(args.warmup)
    barrier(ctx)
    if clk is not None:
        clk.__enter__()
    barrier(ctx)
    ms = _timed(ctx, run, args.steps, stream_of)
    barrier(ctx)
    clocks = None
    if clk is not None:
        clk.__exit__()
        clocks = clk.summary()
    ms_max = sharding.max_over_ranks(ms, device="cuda")
    value = sharding.weak_scaling_throughput(args.steps * cloud.cell_bins, world, ms_max)
    ctx.set_timing(True)
    kt = min(args.steps, 200)
    run(kt)
    ctx.synchronize()
    kms = ctx.timing() / kt
    ctx.set_timing(False)
    # the active window of the advection over 50 further steps (the work unit counts every bin)
    h = ctx.static_steps(50, *p, history=True)
    active = float(np.mean((h[:, 6] - h[:, 5] + 1) / cloud.n_nu))
    return ctx, {"value": value, "ms_per_step": ms_max / args.steps, "kernel_ms": kms, "tuning": list(tuning),
                 "clocks": clocks, "active_fraction": active}


def form_errors(cloud, local, precs, n_steps=2000):
    """Error of each reduced-precision form against FP64 on the headline cloud: every form runs
    n_steps from the same set-up state. Reported per form: M_F at the last step and over the
    run, the emergent edge-ring spectrum and the final J, each relative to the FP64 quantity's
    maximum, and the spectrum per bin relative to the FP64 bin with a floor of 1e-6 of the
    spectrum's maximum (the wing bins carry the escaping flux)."""
    from lydion_b200._lib import PREC_FP64
    from lydion_b200.m1 import context_for_cloud
    p = (cloud.c_tilde, cloud.dt, cloud.z_center, cloud.bc_r_right, cloud.bc_z_bot, cloud.bc_z_top)
    res = {}
    for prec in (PREC_FP64, *precs.values()):
        ctx = context_for_cloud(cloud, precision=prec, device=local)
        h = ctx.static_steps(n_steps, *p, history=True)
        res[prec] = (h[:, 0].copy(), ctx.edge_spectra()[0].mean(0), ctx.download("J"))
        ctx.close()
    ma, sa, Ja = res[PREC_FP64]
    rel = lambda b, a: float(np.max(np.abs(b - a)) / np.max(np.abs(a)))
    floor = 1e-6 * np.max(np.abs(sa))
    out = {}
    for name, prec in precs.items():
        mb, sb, Jb = res[prec]
        out[name] = {"steps": n_steps, "M_F_last": float(abs(mb[-1] - ma[-1]) / abs(ma[-1])), "M_F_run": rel(mb, ma),
                     "edge_spectrum": rel(sb, sa),
                     "edge_spectrum_per_bin": float(np.max(np.abs(sb - sa) / np.maximum(np.abs(sa), floor))),
                     "J": rel(Jb, Ja), "spec": 1e-5}
    return out


def e2e_form(ctx, cloud, args, barrier, stream_of, world):
    """End to end through the public API with host buffers: per step, J / H_r / H_Z up from
    pinned host memory, one step with its diagnostics record, J / H_r / H_Z back into the same
    pinned arrays. Through lyd_static_step_host, which pipelines the copies and the step over 8
    row chunks; `serial` is the same loop as upload, one step, download calls."""
    import torch
    from lydion_b200 import sharding
    p = (cloud.c_tilde, cloud.dt, cloud.z_center, cloud.bc_r_right, cloud.bc_z_bot, cloud.bc_z_top)
    n = max(3, min(20, args.steps // 50))
    pinned = [torch.empty((cloud.nz, cloud.nr, cloud.n_nu), dtype=torch.float64, pin_memory=True).numpy()
              for _ in range(3)]
    names = ("J", "H_r", "H_Z")
    for a, name in zip(pinned, names):
        a[...] = ctx.download(name)
    barrier(ctx)

    def run_serial(k):
        for _ in range(k):
            for a, name in zip(pinned, names):
                ctx.upload(name, a)
            ctx.static_steps(1, *p, history=True)
            for a, name in zip(pinned, names):
                ctx.download(name, out=a)

    def run(k):
        for _ in range(k):
            ctx.static_step_host(pinned[0], pinned[1], pinned[2], *p, out=pinned, chunks=8)

    ms_serial = sharding.max_over_ranks(_timed(ctx, run_serial, n, stream_of), device="cuda")
    run(1)   # the first call decides the window from the uploaded state
    ms = sharding.max_over_ranks(_timed(ctx, run, n, stream_of), device="cuda")
    nbytes = 3 * cloud.cell_bins * 8
    return {"value": sharding.weak_scaling_throughput(n * cloud.cell_bins, world, ms), "unit": UNIT,
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + 7 * 8, "steps": n,
            "ms_per_step": ms / n, "api": "lyd_static_step_host, 8 row chunks",
            "serial": {"value": sharding.weak_scaling_throughput(n * cloud.cell_bins, world, ms_serial),
                       "ms_per_step": ms_serial / n, "api": "lyd_upload x3, lyd_static_steps(1), lyd_download x3"}}


def dropin_form(cloud, args, stream_of, local):
    """End to end through the drop-in functions with the reference's signatures
    (lydion_b200/lya.py): the static-cloud loop of src/StaticCloudTest.jl:362-392 called
    phase by phase on host numpy arrays, FP64. In copy mode every call moves the state it
    reads and writes (the host arrays are always current); in resident mode the state and the
    inputs stay on the device and only the diagnostics come back. The bytes are those the
    drop-ins moved, counted per step."""
    from lydion_b200 import lya as D
    from lydion_b200.m1 import context_for_cloud
    ctx = context_for_cloud(cloud, device=local)
    hv = ctx.download("Hvoigt")
    state = {n: ctx.download(n) for n in ("J", "H_r", "H_Z")}
    ctx.close()
    # the emission profile over the core bins, normalised per cell (Update_phi_nu!,
    # src/ConstantsAndFunctions.jl:362-393): the static driver's input, made on the host as there
    fq = cloud.freq
    core = slice(fq.kcore_min, fq.kcore_max + 1)
    phi = np.zeros_like(hv)
    phi[..., core] = hv[..., core] / np.sum(hv[..., core] * fq.dnu[core], axis=-1, keepdims=True)
    out = {"workload": WORKLOAD, "precision": "fp64"}
    for mode, n in (("copy_every_call", max(3, min(5, args.steps))), ("resident", max(10, min(50, args.steps)))):
        S = D.generate_lya_arrays_from_saved(cloud.c_tilde, cloud.freq, cloud.geom, cloud.T, hv, phi,
                                             recoil=cloud.recoil)
        for name in ("alpha", "alpha_c", "pd", "js"):
            getattr(S, name)[...] = getattr(cloud, name)
        S.alpha_F[...] = S.alpha[:, :, None] * S.Hvoigt         # src/StaticCloudTest.jl:283-285
        for name, a in state.items():
            getattr(S, name)[...] = a
            getattr(S, name + "_old")[...] = a
        if mode == "resident":
            D.set_resident(S)
        g, ct, dt = cloud.geom, cloud.c_tilde, cloud.dt
        vel = (cloud.u_r_star, cloud.u_Z_star, cloud.dur_dr, cloud.dur_dZ, cloud.duZ_dr, cloud.duZ_dZ,
               cloud.ur_over_r)

        def loop(k):
            for _ in range(k):
                D.advect_lya(ct * dt, S, g, *vel, "Reflect", "Outflow", "Reflect", "Outflow")
                D.lya_emission_absorption_update(S.J, S.J_old, S.H_r, S.H_Z, S.H_r_old, S.H_Z_old, S.js, S.phi_nu,
                                                 S.Hvoigt, S.alpha, S.alpha_c, S.alpha_F, S.pd, S.dru_r, S.dru_Z,
                                                 S.dnu, ct, dt)
                D.frequency_update_J_lya_all_cells(ct * dt, S, cloud.T, *vel[2:], True)
                mf = D.update_f_lya_MF_L_lya(S.f_r, S.f_Z, S.dru_r, S.dru_Z, S.js, g.dV, g.rCoM, g.ZCoM, dt,
                                             cloud.z_center, "Reflect")
                S.M_F, S.M_F_radial_net, S.M_F_radial_out, S.L_lya = mf
                S.f_esc_lya = D.compute_f_esc_lya_cylindrical(S.H_r, S.H_Z, g.A_r, g.A_Z, S.dnu, S.L_lya, "Reflect")
                D.reset_dru(S.dru_r, S.dru_Z)

        loop(1)
        tw = D.twin_of(S)
        u0, d0 = D.transfer_bytes(S)
        ms = _timed(tw.ctx, loop, n, stream_of)
        u1, d1 = D.transfer_bytes(S)
        out[mode] = {"value": n * cloud.cell_bins / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / n, "steps": n,
                     "h2d_bytes_per_step": (u1 - u0) // n, "d2h_bytes_per_step": (d1 - d0) // n}
        D.release(S)
    return out


def batch_form(args, barrier, stream_of, local, world):
    """The ragged batch (512 static clouds x 48 bins, sides 32..256, per-cloud CFL step) in both
    forms: graph-replayed steps of the whole batch (--steps of them, 20 to 500), and the three
    kernels' own share of the step."""
    from lydion_b200 import autotune, sharding
    from lydion_b200 import workloads as W
    from lydion_b200._lib import PREC_FP64, PREC_MIXED
    from lydion_b200.m1 import batch_for_clouds, cloud_params
    clouds = W.config_c3()
    mine = clouds if world == 1 else [clouds[q] for q in sharding.partition_clouds(
        [c.cell_bins for c in clouds], world)[int(os.environ.get("RANK", 0))]]
    pp = cloud_params(mine)
    out = {"workload": "c3_ragged_batch_512_clouds_x48", "clouds": len(clouds),
           "cell_bins": int(sum(c.cell_bins for c in clouds))}
    # timed steps: --steps, at least 20 and at most the 500 of the batch configuration
    steps = max(20, min(500, args.steps))
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        b = batch_for_clouds(mine, precision=prec, device=local)
        run = lambda n: b.batch_steps(n, pp, history=False)
        tuning = autotune.autotune(b, run, steps=2, device=local, rows=(8, 16), cells=(0, 256), solvers=(0,),
                                   cache=os.path.join(tempfile.gettempdir(), "lydion_bench_tuning.json"))
        run(3)
        barrier(b)
        ms = sharding.max_over_ranks(_timed(b, run, steps, stream_of), device="cuda")
        # the three kernels' own device time per step: what is left of the step is launch gaps,
        # all a single persistent kernel could remove
        b.set_timing(True)
        run(2)
        b.synchronize()
        kms = b.timing() / 2
        b.set_timing(False)
        # the same steps as one persistent cooperative launch each (lyd_batch_steps_persistent)
        runp = lambda n: b.batch_steps(n, pp, history=False, persistent=True)
        runp(3)
        barrier(b)
        pms = sharding.max_over_ranks(_timed(b, runp, steps, stream_of), device="cuda")
        # every rank advances its share of the 512 clouds: the whole batch's cell-bins over the
        # slowest rank's time
        out[name] = {"value": steps * out["cell_bins"] / (ms * 1e-3), "ms_per_step": ms / steps, "steps": steps,
                     "tuning": list(tuning),
                     "kernel_ms_per_step": {"advect": float(kms[0]), "freq": float(kms[1]), "reduce": float(kms[2])},
                     "launch_gap_fraction": float(max(0.0, 1.0 - float(np.sum(kms)) / (ms / steps))),
                     "persistent": {"ms_per_step": pms / steps, "graph": b.persistent_graph(),
                                    "over_three_launches": ms / pms}}
        b.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def rhd_form(args, stream_of, local):
    """The RHD-side Lyman-alpha block on the 256 x 256 x 64 grid in FP64: lyd_rhd_lya_prepare
    (11 per-cell host arrays up, opacities, emissivities, H_voigt and phi_nu) and
    lyd_rhd_lya_absorb over per-cell sub-steps of a tenth of each cell's absorption time (the
    sub-steps up, no results back, no commit), on a seeded gas and dust state."""
    from lydion_b200 import workloads as W
    from lydion_b200.m1 import context_for_cloud
    cl = W.config_c2()
    ctx = context_for_cloud(cl, device=local)
    sp, rho_d = W.rhd_gas_state(cl, 20261203)
    prep = lambda k: [ctx.rhd_lya_prepare(sp["T"], sp["nHI"], sp["nH2"], sp["nHII"], sp["nHeI"], sp["ne"], sp["nOHx"],
                                          sp["nCHx"], rho_d, W.DUST_KAPPA_ABS, W.DUST_KAPPA_F, W.DUST_RHO_IGNORE,
                                          z=0.0) for _ in range(k)]
    prep(2)
    n_prep = 10
    prep_ms = _timed(ctx, prep, n_prep, stream_of) / n_prep
    c_tilde = cl.c_tilde
    a, ac, pd = ctx.download("alpha"), ctx.download("alpha_c"), ctx.download("pd")
    dt = 0.1 / (c_tilde * np.maximum(ac + pd * a, 1e-300))
    absorb = lambda k: [ctx.rhd_lya_absorb(dt, c_tilde, results=False) for _ in range(k)]
    absorb(3)
    n_abs = 50
    abs_ms = _timed(ctx, absorb, n_abs, stream_of) / n_abs
    ctx.close()
    n3 = cl.cell_bins
    return {"workload": "rhd_lya_block_256x256x64", "cell_bins": n3,
            "prepare_ms": prep_ms, "absorb_ms": abs_ms,
            "absorb_cell_bins_per_s": n3 / (abs_ms * 1e-3),
            # J_old, H_r_old, H_Z_old, H_voigt read and J, H_r, H_Z written: 56 B per cell-bin in FP64
            "absorb_hbm_gbs": 56.0 * n3 / (abs_ms * 1e-3) / 1e9}


def c5_form(args, stream_of, local):
    """The largest single field (1024 x 1024 cells x 128 bins of a synthetic RHD snapshot: lognormal
    n_H, photoionised bubble, shell outflow, dust): both forms, a few graph-replayed steps each,
    with the per-kernel times and each kernel's algorithmic HBM rate (the working set, 7 x 1.07 GB,
    is far above L2)."""
    from lydion_b200 import workloads as W
    from lydion_b200._lib import PREC_FP64, PREC_MIXED
    from lydion_b200.m1 import context_for_cloud
    cl = W.config_c5()
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    steps = max(3, min(10, args.steps // 300))
    out = {"workload": "c5_rhd_snapshot_1024x1024x128", "cell_bins": int(cl.cell_bins), "steps": steps}
    ab = algorithmic_bytes(cl.n_nu, 8)
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        ctx = context_for_cloud(cl, precision=prec, device=local)
        run = lambda k: ctx.static_steps(k, *p, history=False)
        run(2)
        ctx.synchronize()
        ms = _timed(ctx, run, steps, stream_of)
        ctx.set_timing(True)
        run(steps)
        ctx.synchronize()
        kms = ctx.timing() / steps
        ctx.set_timing(False)
        out[name] = {"value": steps * cl.cell_bins / (ms * 1e-3), "ms_per_step": ms / steps,
                     "kernel_ms_per_step": {"advect": float(kms[0]), "freq": float(kms[1]), "reduce": float(kms[2])},
                     "hbm_gbs": {"advect": ab["advect"] * cl.cell_bins / (kms[0] * 1e-3) / 1e9,
                                 "freq": ab["freq"] * cl.cell_bins / (kms[1] * 1e-3) / 1e9}}
        ctx.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def dd_form(args, stream_of, local, world, rank):
    """The 1024 x 1024 x 128 field split into Z slabs over the ranks (lydion_b200.domain; one
    slab per GPU, halo rows exchanged and reduction columns all-reduced through torch.distributed),
    mixed precision, strong scaling: the whole field's cell-bin updates over the slowest rank's
    device time."""
    import torch
    from lydion_b200 import domain as D
    from lydion_b200 import sharding
    from lydion_b200 import workloads as W
    from lydion_b200._lib import PREC_MIXED
    cl = W.config_c5()
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    steps = max(3, min(10, args.steps // 300))
    r = D.SlabRank(cl, world, rank, precision=PREC_MIXED, device=local)
    drv = D.SlabDriver([r], D.TorchComm() if world > 1 else D.LocalComm())
    drv.find_active()
    for _ in range(2):
        drv.step(*p)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        drv.step(*p)
    e1.record()
    torch.cuda.synchronize()
    ms = sharding.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    r.ctx.close()
    return {"workload": "c5_rhd_snapshot_1024x1024x128_zslabs", "ranks": world, "rows_per_rank": r.j1 - r.j0,
            "steps": steps, "precision": "mixed", "scaling": "strong",
            "value": steps * cl.cell_bins / (ms * 1e-3), "ms_per_step": ms / steps}


def adjoint_form(args, stream_of, local):
    """Adjoint over forward cost on the turbulent cloud (128 x 128 x 48, lognormal n_H, dust,
    v_max = 50 km/s): N forward steps from the graph-replayed step against lyd_adjoint_run of
    the same N steps, every adjoint call starting from the state the timed forward run starts
    from. Three storage modes: automatic (every step's state and advection tape kept from the
    forward sweep when they fit in device memory, so nothing is recomputed), a checkpoint every
    100 steps with one recomputation of each segment, and the binomial (Revolve) schedule with
    62 state snapshots. Each mode's time is the mean of its second and third calls, after the
    call that allocates the workspace."""
    from lydion_b200 import adjoint as A
    from lydion_b200 import workloads as W
    from lydion_b200.m1 import context_for_cloud
    cl = W.config_c4()
    n = 2000      # the adjoint run's specified length, whatever --steps is
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    ctx = context_for_cloud(cl, device=local)
    run = lambda k: ctx.static_steps(k, *p, history=False)
    run(args.warmup)
    ctx.synchronize()
    # every adjoint call starts from the state the timed forward run starts from, so both
    # cover the same n steps (a call leaves the context in its final state)
    fields = ("J", "H_r", "H_Z")
    s0 = [ctx.download(f) for f in fields]

    def restore():
        for f, a in zip(fields, s0):
            ctx.upload(f, a)
        ctx.synchronize()
    fwd = _timed(ctx, run, n, stream_of)
    w64 = np.full(64, 1.0 / 64)
    w_MF, w_bins = A.objective_weights(cl.freq, 1.0, w64)
    out = {"workload": "c4_turbulent_128x128x48", "steps": n, "forward_ms": fwd}
    names = ("forward_sweep", "recompute_with_tapes", "frequency_adjoint", "advection_adjoint")
    for every, label in ((0, "auto"), (100, "every_100"), (-1, "binomial")):
        # one untimed call first: the workspace (grow-only, kept by the context between calls;
        # about 126 GB when every step is kept) is allocated by the first call that needs it.
        # binomial: 61 snapshots besides the initial state, no step advanced more than twice.
        # Then the mean of two timed calls.
        restore()
        ctx.adjoint(n, *p, w_MF=w_MF, w_spec=1e12 * w_bins, checkpoint_every=every, want=("grad_alpha",))
        samples = []
        for _ in range(2):
            restore()
            samples.append(_timed(ctx, lambda k: ctx.adjoint(k, *p, w_MF=w_MF, w_spec=1e12 * w_bins,
                                                             checkpoint_every=every, want=("grad_alpha",)),
                                  n, stream_of))
        adj = float(np.mean(samples))
        out[f"adjoint_ms_{label}"] = adj
        out[f"adjoint_ms_{label}_samples"] = samples
        out[f"ratio_{label}"] = adj / fwd
        restore()
        ctx.set_timing(True)
        ctx.adjoint(n, *p, w_MF=w_MF, w_spec=1e12 * w_bins, checkpoint_every=every, want=("grad_alpha",))
        ctx.set_timing(False)
        ph = ctx.adjoint_timing()
        out[f"phase_ms_{label}"] = {k: float(v) for k, v in zip(names, ph[[0, 1, 3, 4]])}
    out["auto_kept_all_steps"] = out["phase_ms_auto"]["recompute_with_tapes"] == 0.0
    ctx.close()
    return out


def run_gpu(args):
    import torch
    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from lydion_b200 import workloads as W
    from lydion_b200._lib import PREC_FP32, PREC_FP64, PREC_MIXED
    cloud = W.config_c2()

    def barrier(ctx):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ctx.synchronize()

    stream_of = lambda ctx: torch.cuda.ExternalStream(ctx.stream(), device=local)
    # the headline: the FP64 form, the reference's arithmetic
    ctx64, f64 = measure_form(cloud, PREC_FP64, args, barrier, stream_of, local, world, clk=ClockSampler(local))
    e2e = e2e_form(ctx64, cloud, args, barrier, stream_of, world)
    ctx64.close()
    names = ["advect", "freq", "reduce"]
    # the reduced-precision forms: FP32 flux arithmetic over FP64 storage, and FP32 storage
    forms = {}
    for fname, prec in (("mixed", PREC_MIXED), ("fp32_storage", PREC_FP32)):
        if args.only_fp64:
            break
        c, m = measure_form(cloud, prec, args, barrier, stream_of, local, world)
        c.close()
        forms[fname] = {"value": m["value"], "ms_per_step": m["ms_per_step"], "tuning": m["tuning"],
                        "kernel_ms_per_step": {n: float(v) for n, v in zip(names, m["kernel_ms"])},
                        "over_fp64": m["value"] / f64["value"]}
    dropin = None if (args.no_dropin or world > 1) else dropin_form(cloud, args, stream_of, local)
    batch = None if args.no_batch else batch_form(args, barrier, stream_of, local, world)
    adj = None if (args.no_adjoint or world > 1) else adjoint_form(args, stream_of, local)
    c5 = None if (args.no_c5 or world > 1) else c5_form(args, stream_of, local)
    rhd = None if (args.no_rhd or world > 1) else rhd_form(args, stream_of, local)
    err = None if (args.no_error or world > 1 or args.only_fp64) else form_errors(
        cloud, local, {"mixed": PREC_MIXED, "fp32_storage": PREC_FP32})
    dd = dd_form(args, stream_of, local, world, rank) if args.dd_field else None

    # roofline of the dominant kernel of the headline (FP64) form
    kms = f64["kernel_ms"]
    dom = int(np.argmax(kms[:2]))
    ab = algorithmic_bytes(cloud.n_nu, 8)[names[dom]] * cloud.cell_bins
    peaks, src = measured_peaks()
    achieved = ab / (kms[dom] * 1e-3) / 1e9
    variant = "fp64"
    traffic = profile_traffic("k_" + names[dom], variant)
    cpu = cpu_baseline(cloud) if (rank == 0 and world == 1 and not args.no_cpu) else None
    if rank == 0:
        mixed = forms.get("mixed")
        line = {"metric": METRIC, "value": f64["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": f64["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded static cloud set-up, no dataset)",
                "config": {"workload": WORKLOAD, "cells": [cloud.nr, cloud.nz], "bins": cloud.n_nu, "tau0": 1e8,
                           "tau_abs": 1.0, "source_radius": 0.5, "v_max_kms": 200.0, "precision": "fp64",
                           "parallelism": f"{world} independent clouds (one per GPU)" if world > 1 else "single GPU",
                           "l2": "inputs larger than L2: 7 FP64 fields x 33.5 MB resident, 56 B/cell-bin streamed per kernel",
                           "tuning": f64["tuning"]},
                "kernel_ms_per_step": {n: float(v) for n, v in zip(names, kms)},
                "mixed": mixed,
                "mixed_over_fp64": mixed["over_fp64"] if mixed else None,
                "fp32_storage": forms.get("fp32_storage"),
                "form_errors": err,
                "adjoint_over_forward": adj["ratio_every_100"] if adj else None,
                "adjoint_over_forward_mode": "checkpoints every 100 steps, 2000 steps" if adj else None,
                "adjoint_over_forward_keep_all": adj["ratio_auto"] if adj else None,
                "adjoint": adj,
                "largest_field": c5,
                "rhd_lya_block": rhd,
                "largest_field_zslabs": dd,
                "batch": batch,
                "roofline": {"bound": "hbm", "kernel": "k_" + names[dom], "achieved": achieved,
                             "peak": peaks["hbm_gbs"], "peak_source": src, "unit": "GB/s",
                             "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                             "algorithmic_bytes_per_launch": ab, "ms_per_launch": float(kms[dom]),
                             "ncu_fp64_pipe_pct": profile_figure("k_" + names[dom], variant, "fp64_pipe_pct"),
                             "ncu_fma_pipe_pct": profile_figure("k_" + names[dom], variant, "fma_pipe_pct")},
                "active_fraction": f64["active_fraction"],
                "cpu_baseline": cpu,
                "e2e": e2e,
                "e2e_dropin": dropin,
                "gpu_launches": 3 * args.steps,
                "clocks": f64["clocks"]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="lydion", choices=["lydion", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-batch", action="store_true", help="skip the ragged-batch measurement")
    ap.add_argument("--no-dropin", action="store_true", help="skip the end-to-end leg through the drop-in functions")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward measurement")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes instead of the autotuner")
    ap.add_argument("--no-c5", action="store_true", help="skip the 1024x1024x128 field")
    ap.add_argument("--no-rhd", action="store_true", help="skip the RHD-side Lyman-alpha block")
    ap.add_argument("--no-error", action="store_true", help="skip the mixed-against-FP64 error run")
    ap.add_argument("--dd-field", action="store_true",
                    help="also step the 1024x1024x128 field split into Z slabs over the ranks (strong scaling)")
    ap.add_argument("--only-fp64", action="store_true", help="measure the FP64 form only")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
