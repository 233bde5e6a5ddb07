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


def escaping_flux_per_bin(H_r, H_Z, geom, bc_z_bot):
    """Outward flux per frequency bin through the outer r face, the top face and (when it lets
    flow out) the bottom face: the per-bin sum behind Compute_f_esc_Lya_Cylindrical
    (src/ConstantsAndFunctions.jl:969-993), before the bin widths and 1/L. H arrays are [j, i, k]."""
    esc = np.einsum("j,jk->k", geom.A_r[:, -1], np.maximum(H_r[:, -1, :], 0.0))
    esc += np.einsum("i,ik->k", geom.A_Z[-1, :], np.maximum(H_Z[-1, :, :], 0.0))
    if bc_z_bot == W.BC_OUTFLOW:
        esc += np.einsum("i,ik->k", geom.A_Z[0, :], np.maximum(-H_Z[0, :, :], 0.0))
    return esc


def wing_checks(ctx, st, cloud, floor=1e-6):
    """Per-element errors relative to each element, with a floor of `floor` times the quantity's
    maximum, so faint wing bins are held to the same relative bound as the line centre until
    they fall below the floor: J, the flux fractions H_r/J and H_Z/J, the edge-ring spectrum
    and the per-bin escaping flux of the CUDA state against the oracle's."""
    out = {}
    Jo = st.J
    Jfloor = np.maximum(Jo, floor * Jo.max())
    out["J"] = max_rel(ctx.download("J"), Jo, floor=floor * Jo.max())
    # H changes sign, so near its zeros an error relative to H itself means nothing; it is
    # held relative to the same element's J instead, i.e. as an error of the flux fraction H/J
    for f in ("H_r", "H_Z"):
        out[f] = float(np.max(np.abs(ctx.download(f) - getattr(st, f)) / Jfloor))
    raw_g, raw_o = ctx.edge_spectra()[0], st.edge_spectra()[0]
    out["edge_spectrum"] = max_rel(raw_g, raw_o, floor=floor * np.abs(raw_o).max())
    eg = escaping_flux_per_bin(ctx.download("H_r"), ctx.download("H_Z"), cloud.geom, cloud.bc_z_bot)
    eo = escaping_flux_per_bin(st.H_r, st.H_Z, cloud.geom, cloud.bc_z_bot)
    out["escaping_flux"] = max_rel(eg, eo, floor=floor * np.abs(eo).max())
    return out


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
