"""Small, fixed programs to run under a profiler (each ends by itself in seconds):

    python -m lydion_b200.profile_cases adjoint   # turbulent 128x128x48 cloud: 20 steps, then the
                                                  # adjoint of 6 steps (every step kept)
    python -m lydion_b200.profile_cases rhd       # RHD Lya block on the 256x256x64 grid: prepare,
                                                  # then 4 absorption sub-steps of 0.1 t_abs
    python -m lydion_b200.profile_cases step      # the dusty-outflow 256x256x64 cloud, mixed form,
                                                  # 16 rows per advection tile, 4 CTAs/SM: 20 steps
    python -m lydion_b200.profile_cases step64    # the same cloud in FP64, 16 rows per tile,
                                                  # 3 CTAs/SM (the bench's tuned shape): 20 steps
    python -m lydion_b200.profile_cases big64     # a 512x512x128 RHD snapshot in FP64 (33.5M
                                                  # cell-bins, ~2 GB on the device, 15x L2): 6 steps
"""
import sys

import numpy as np


def adjoint_case():
    from . import adjoint as A
    from . import workloads as W
    from .m1 import context_for_cloud
    cl = W.config_c4()
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    ctx = context_for_cloud(cl)
    w_MF, w_bins = A.objective_weights(cl.freq, 1.0, np.full(64, 1.0 / 64))
    ctx.static_steps(20, *p, history=False)
    g = ctx.adjoint(6, *p, w_MF=w_MF, w_spec=1e12 * w_bins, checkpoint_every=0, want=("grad_alpha",))
    ctx.close()
    return float(np.abs(g["grad_alpha"]).max())


def rhd_case():
    from . import workloads as W
    from .m1 import context_for_cloud
    cl = W.config_c2()
    ctx = context_for_cloud(cl)
    sp, rho_d = W.rhd_gas_state(cl, 20261203)
    ctx.rhd_lya_prepare(sp["T"], sp["nHI"], sp["nH2"], sp["nHII"], sp["nHeI"], sp["ne"], sp["nOHx"], sp["nCHx"],
                        rho_d, W.DUST_KAPPA_ABS, W.DUST_KAPPA_F, W.DUST_RHO_IGNORE)
    a, ac, pd = ctx.download("alpha"), ctx.download("alpha_c"), ctx.download("pd")
    dt = 0.1 / (cl.c_tilde * np.maximum(ac + pd * a, 1e-300))
    for _ in range(4):
        ctx.rhd_lya_absorb(dt, cl.c_tilde, results=False)
    ctx.synchronize()
    ctx.close()
    return 0.0


def step_case(fp64=False):
    from . import workloads as W
    from ._lib import PREC_FP64, PREC_MIXED
    from .m1 import context_for_cloud
    cl = W.config_c2()
    ctx = context_for_cloud(cl, precision=PREC_FP64 if fp64 else PREC_MIXED)
    ctx.set_tuning(*((16, 0, 0, 3) if fp64 else (16, 0, 0, 4)))
    h = ctx.static_steps(20, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    ctx.close()
    return float(h[-1, 0])


def big_case():
    from . import workloads as W
    from ._lib import PREC_FP64
    from .m1 import context_for_cloud
    cl = W.rhd_snapshot_cloud(n=512, n_nu=128, name="rhd_snapshot_512x512x128")
    ctx = context_for_cloud(cl, precision=PREC_FP64)
    ctx.set_tuning(20, 0, 0, 3)
    h = ctx.static_steps(6, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    ctx.close()
    return float(h[-1, 0])


if __name__ == "__main__":
    case = sys.argv[1] if len(sys.argv) > 1 else "adjoint"
    print(case, {"adjoint": adjoint_case, "rhd": rhd_case, "step": step_case,
                "step64": lambda: step_case(fp64=True), "big64": big_case}[case]())
