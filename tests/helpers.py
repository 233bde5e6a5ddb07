"""Shared set-up for the parity tests: matched oracle / CUDA states on identical inputs."""
import numpy as np

from lydion_b200 import workloads as W


def random_state(cloud, seed, amp=1e-12, fmax=0.8):
    """A positive J with structure in every direction and an H with |H| < J."""
    rng = np.random.default_rng(seed)
    shape = (cloud.nz, cloud.nr, cloud.n_nu)
    x = np.linspace(-1, 1, cloud.n_nu)
    J = amp * (0.05 + rng.uniform(size=shape)) * np.exp(-4 * x * x)[None, None, :]
    f = fmax * rng.uniform(size=shape)
    th = rng.uniform(0, 2 * np.pi, size=shape)
    return J, J * f * np.cos(th), J * f * np.sin(th)


def matched_pair(oracle_mod, cloud, seed=None, precision=0, device_hvoigt=False, keep_ff=False, j_scale=0.0):
    """An OracleState and an M1Context holding the same inputs (and the same H_voigt /
    phi_nu, taken from the oracle unless device_hvoigt)."""
    from lydion_b200.m1 import context_for_cloud
    st = oracle_mod.OracleState(cloud)
    st.setup_profiles()
    if device_hvoigt:
        ctx = context_for_cloud(cloud, precision=precision, keep_freq_factors=keep_ff, j_scale=j_scale)
    else:
        ctx = context_for_cloud(cloud, precision=precision, hvoigt=st.Hvoigt, phi_nu=st.phi_nu,
                                keep_freq_factors=keep_ff, j_scale=j_scale)
    if seed is not None:
        J, Hr, HZ = random_state(cloud, seed)
        for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            getattr(st, name)[...] = a
            getattr(st, name + "_old")[...] = a
            ctx.upload(name, a)
            ctx.upload(name + "_old", a)
    return st, ctx


def max_rel(a, b, floor=0.0):
    """max |a - b| / max(|b|, floor) over elements whose reference magnitude exceeds floor."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b), floor)
    m = scale > 0
    if not np.any(m):
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)[m] / scale[m]))


def norm_err(a, b):
    """max |a - b| / max |b| (error relative to the field's scale)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / s) if s > 0 else float(np.max(np.abs(a - b)))


CLOUDS = {
    "glf_outflow": lambda: W.small_cloud(nr=12, nz=10, n_nu=16),
    "hll_outflow": lambda: W.small_cloud(nr=11, nz=9, n_nu=16, flux_method=W.FLUX_HLL),
    "glf_zout_48": lambda: W.small_cloud(nr=9, nz=14, n_nu=48, bc_z_bot=W.BC_OUTFLOW, x_max=200.0),
    "hll_point_64": lambda: W.small_cloud(nr=8, nz=8, n_nu=64, rs=0.0, umax_kms=0.0, tau_abs=0.0,
                                          flux_method=W.FLUX_HLL, x_max=600.0),
    "glf_20bins": lambda: W.small_cloud(nr=7, nz=6, n_nu=20, tau0=1e7, x_max=100.0),
}
