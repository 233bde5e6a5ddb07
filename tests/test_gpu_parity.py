"""GPU parity of the CUDA step against the FP64 oracle, through the C ABI.

Tolerances (FP64 path): the kernels follow the reference's operation order, but the GPU
contracts multiply-adds into FMAs and solves the frequency systems by cyclic reduction
instead of dgtsv's pivoted elimination; both solvers are backward stable and agree to the
conditioning of the system (~1e-9 relative at F/dw ~ 4e8, tau0 = 1e8, measured against a
50-digit solve). Element-wise bounds below are relative to the field's maximum.
"""
import numpy as np
import pytest

from helpers import CLOUDS, matched_pair, max_rel, norm_err, random_state, wing_checks
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu

BC_CASES = [("glf_outflow", 1, 1), ("glf_outflow", 0, 0), ("hll_outflow", 1, 0), ("glf_zout_48", 1, 1),
            ("hll_point_64", 0, 1), ("glf_20bins", 1, 1)]


def _set_bcs(cloud, r_right, z_top):
    cloud.bc_r_right = r_right
    cloud.bc_z_top = z_top
    return cloud


@pytest.mark.parametrize("name,bcr,bzt", BC_CASES)
def test_advect_matches_oracle(oracle_mod, name, bcr, bzt):
    cl = _set_bcs(CLOUDS[name](), bcr, bzt)
    st, ctx = matched_pair(oracle_mod, cl, seed=11)
    ctdt = cl.c_tilde * cl.dt
    for _ in range(3):
        km_o = st.advect(ctdt)
        km_g = ctx.find_active_bins()
        assert km_g == km_o
        ctx.advect(ctdt, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    for f in ("J", "H_r", "H_Z"):
        e = norm_err(ctx.download(f), getattr(st, f))
        assert e < 1e-12, (f, e)
    # AdvectLya! leaves J_old = J and H_old = H
    np.testing.assert_array_equal(ctx.download("J_old"), ctx.download("J"))
    np.testing.assert_array_equal(ctx.download("H_Z_old"), ctx.download("H_Z"))


def test_advect_partial_active_window(oracle_mod):
    """Bins outside FindActiveBins' window are passed through untouched."""
    cl = CLOUDS["hll_point_64"]()
    st, ctx = matched_pair(oracle_mod, cl, seed=3)
    J, Hr, HZ = random_state(cl, 3)
    J[..., :6] = 1e-58
    J[..., -6:] = 1e-58
    for name, a in (("J", J), ("H_r", Hr * 0), ("H_Z", HZ * 0)):
        getattr(st, name)[...] = a
        ctx.upload(name, a)
    k = st.advect(cl.c_tilde * cl.dt)
    assert k[0] > 0 and k[1] < cl.n_nu - 1
    ctx.advect(cl.c_tilde * cl.dt, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    assert norm_err(ctx.download("J"), st.J) < 1e-12
    np.testing.assert_array_equal(ctx.download("J")[..., : k[0]], J[..., : k[0]])


@pytest.mark.parametrize("name", ["glf_outflow", "glf_zout_48", "glf_20bins"])
def test_emission_absorption_matches_oracle(oracle_mod, name):
    cl = CLOUDS[name]()
    st, ctx = matched_pair(oracle_mod, cl, seed=5)
    for _ in range(2):
        st.emission_absorption(cl.c_tilde, cl.dt)
        ctx.emission_absorption(cl.c_tilde, cl.dt)
    for f in ("J", "H_r", "H_Z", "J_old", "H_r_old"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-14, f
    for f in ("dru_r", "dru_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-12, f


@pytest.mark.parametrize("name", ["glf_outflow", "hll_point_64", "glf_zout_48", "glf_20bins"])
def test_frequency_update_matches_oracle(oracle_mod, name):
    cl = CLOUDS[name]()
    st, ctx = matched_pair(oracle_mod, cl, seed=7)
    ctdt = cl.c_tilde * cl.dt
    nf, _ = st.frequency_update(ctdt)
    assert nf == 0
    ctx.frequency_update(ctdt)
    for f in ("J", "H_r", "H_Z"):
        e = norm_err(ctx.download(f), getattr(st, f))
        assert e < 1e-9, (f, e)
    assert max_rel(ctx.download("J"), st.J, floor=1e-6 * st.J.max()) < 1e-8


def test_frequency_update_keep_factors(oracle_mod):
    cl = CLOUDS["glf_outflow"]()
    st, ctx = matched_pair(oracle_mod, cl, seed=9, keep_ff=True)
    ctdt = cl.c_tilde * cl.dt
    st.frequency_update(ctdt, True)
    ctx.frequency_update(ctdt, True)
    st.frequency_update(ctdt, False)
    ctx.frequency_update(ctdt, False)
    assert norm_err(ctx.download("J"), st.J) < 1e-9


def test_frequency_update_without_kept_factors_is_an_error(oracle_mod):
    from lydion_b200._lib import LydionError, LYD_ERR_STATE
    cl = CLOUDS["glf_outflow"]()
    _, ctx = matched_pair(oracle_mod, cl, seed=9)
    with pytest.raises(LydionError) as e:
        ctx.frequency_update(cl.c_tilde * cl.dt, False)
    assert e.value.code == LYD_ERR_STATE


@pytest.mark.parametrize("name", ["glf_outflow", "hll_outflow", "glf_zout_48", "hll_point_64"])
def test_static_steps_match_oracle(oracle_mod, name):
    cl = CLOUDS[name]()
    st, ctx = matched_pair(oracle_mod, cl)
    n = 40
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])       # active windows
    np.testing.assert_allclose(d_g[:, 3], d_o[:, 3], rtol=1e-13)   # L
    for col in (0, 1, 2):
        assert max_rel(d_g[5:, col], d_o[5:, col]) < 1e-9, col
    assert max_rel(d_g[10:, 4], d_o[10:, 4], floor=1e-6 * np.abs(d_o[:, 4]).max()) < 1e-8
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-9, f
    np.testing.assert_allclose(ctx.download("f_r"), st.f_r, rtol=1e-8, atol=1e-9 * np.abs(st.f_r).max())
    assert np.all(ctx.download("dru_r") == 0.0)


def test_per_phase_calls_equal_fused_step(oracle_mod):
    cl = CLOUDS["glf_outflow"]()
    _, a = matched_pair(oracle_mod, cl, seed=21)
    _, b = matched_pair(oracle_mod, cl, seed=21)
    ctdt = cl.c_tilde * cl.dt
    for _ in range(3):
        a.advect(ctdt, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
        a.emission_absorption(cl.c_tilde, cl.dt)
        a.frequency_update(ctdt)
        a.reset_dru()
    b.static_steps(3, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    for f in ("J", "H_r", "H_Z"):
        np.testing.assert_array_equal(a.download(f), b.download(f))


def test_update_J_and_H_matches_oracle(oracle_mod):
    cl = CLOUDS["glf_zout_48"]()
    st, ctx = matched_pair(oracle_mod, cl, seed=13)
    ctdt = cl.c_tilde * cl.dt
    st.advect(ctdt)
    st.frequency_update(ctdt)
    ctx.update_J_and_H(cl.dt, cl.c_tilde, True, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    assert norm_err(ctx.download("J"), st.J) < 1e-9


def test_diagnostics_match_oracle(oracle_mod):
    cl = CLOUDS["glf_zout_48"]()
    st, ctx = matched_pair(oracle_mod, cl, seed=17)
    st.emission_absorption(cl.c_tilde, cl.dt)
    ctx.emission_absorption(cl.c_tilde, cl.dt)
    mo = st.force_multiplier(cl.dt)
    mg = ctx.force_multiplier(cl.dt, cl.z_center, cl.bc_z_bot)
    np.testing.assert_allclose(mg, mo, rtol=1e-12)
    np.testing.assert_allclose(ctx.download("f_Z"), st.f_Z, rtol=1e-12, atol=1e-300)
    fo = st.f_esc(mo[3])
    fg = ctx.f_esc(mg[3], cl.bc_z_bot)
    assert fg == pytest.approx(fo, rel=1e-12)
    ro, no, rio, zio = st.edge_spectra()
    rg, ng, rig, zig = ctx.edge_spectra()
    np.testing.assert_array_equal(rig, rio)
    np.testing.assert_array_equal(zig, zio)
    np.testing.assert_allclose(rg, ro, rtol=1e-14, atol=0)   # FMA rounding of the emission update
    np.testing.assert_allclose(ng, no, rtol=1e-13)


def _band_cloud(n_bands=7):
    """A cloud whose 'frequency grid' is n_bands stellar/IR bands (the advection does not read
    the frequencies)."""
    from lydion_b200.grid import FreqGrid
    nu = np.arange(n_bands + 1, dtype=np.float64) + 1.0
    nuC = 0.5 * (nu[1:] + nu[:-1])
    dnu = np.diff(nu)
    fq = FreqGrid(nu, nuC, dnu, 1.0 / dnu, 1.0 / nuC, 0, 0)
    return W.static_cloud(11, 9, n_bands, tau0=1e4, tau_abs=0.5, rs=0.5, umax_kms=100.0, freq=fq,
                          flux_method=W.FLUX_HLL, name="bands")


@pytest.mark.parametrize("kmin,kmax,update_jold", [(0, 6, 0), (2, 4, 1), (0, 6, 1)])
def test_advect_jh_bands_match_oracle(oracle_mod, kmin, kmax, update_jold):
    """AdvectJandH! for 7 stellar/IR bands with HLL, explicit alpha_F, the caller's bin range and
    J_old rule (src/AdvectJandH.jl:2227-2464; PhotoThermoChemistry.jl:3854-3868)."""
    from lydion_b200 import lya
    cl = _band_cloud(7)
    st = oracle_mod.OracleState(cl)
    rng = np.random.default_rng(31)
    J, Hr, HZ = random_state(cl, 8)
    Jold = J * rng.uniform(0.5, 1.5, J.shape)
    aF = rng.uniform(1e-19, 1e-17, J.shape)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ), ("J_old", Jold), ("alpha_F", aF)):
        getattr(st, name)[...] = a
    ctdt = cl.c_tilde * cl.dt
    st.advect_jh(ctdt, kmin, kmax, update_jold)
    Jg, Hrg, HZg, Jog = J.copy(), Hr.copy(), HZ.copy(), Jold.copy()
    lya.advect_J_and_H(ctdt, aF, Jg, Jog, Hrg, HZg, cl.geom, cl.u_r_star, cl.u_Z_star, cl.dur_dr, cl.dur_dZ,
                       cl.duZ_dr, cl.duZ_dZ, cl.ur_over_r, UpdateJold=bool(update_jold), BC_r_right="Outflow",
                       BC_Z_bot="Reflect", BC_Z_top="Outflow", kmin=kmin, kmax=kmax, FluxSolver="HLL")
    for got, ref in ((Jg, st.J), (Hrg, st.H_r), (HZg, st.H_Z)):
        assert norm_err(got, ref) < 1e-12
    np.testing.assert_array_equal(Jg[:, :, :kmin], J[:, :, :kmin])     # bins outside the range pass through
    if update_jold:
        np.testing.assert_array_equal(Jog, Jg)
    else:
        np.testing.assert_array_equal(Jog, Jold)


def test_gravity_force_multiplier_matches_oracle(oracle_mod):
    """The gravity method of Update_f_Lya_MF_L_Lya! (src/ConstantsAndFunctions.jl:691-804)."""
    cl = CLOUDS["glf_outflow"]()
    st, ctx = matched_pair(oracle_mod, cl, seed=23)
    st.emission_absorption(cl.c_tilde, cl.dt)
    ctx.emission_absorption(cl.c_tilde, cl.dt)
    rng = np.random.default_rng(4)
    gr = rng.normal(size=(cl.nz, cl.nr))
    gz = -np.abs(rng.normal(size=(cl.nz, cl.nr)))
    gz[0, :3] = 0.0
    gr[0, :3] = 0.0                    # cells without gravity contribute nothing
    mo = st.force_multiplier_gravity(cl.dt, gr, gz)
    mg = ctx.force_multiplier(cl.dt, cl.z_center, cl.bc_z_bot, f_grav=(gr, gz))
    np.testing.assert_allclose(mg, mo, rtol=1e-12)
    # without gravity the plain method's values
    m4 = ctx.force_multiplier(cl.dt, cl.z_center, cl.bc_z_bot)
    np.testing.assert_allclose(m4, mg[[0, 2, 3, 4]], rtol=1e-14)


def test_device_hvoigt_and_phi_match_oracle(oracle_mod):
    cl = W.small_cloud(nr=6, nz=5, n_nu=64, x_max=600.0)
    cl.T = np.linspace(30.0, 3e4, cl.nr * cl.nz).reshape(cl.nz, cl.nr)
    st, ctx = matched_pair(oracle_mod, cl, device_hvoigt=True)
    hv = ctx.download("Hvoigt")
    assert max_rel(hv, st.Hvoigt, floor=1e-300) < 1e-9
    assert norm_err(hv, st.Hvoigt) < 1e-13


def test_pd_and_cfl_on_device(oracle_mod):
    from lydion_b200.m1 import M1Context
    rng = np.random.default_rng(2)
    n = 500
    nH = 10 ** rng.uniform(-2, 6, n)
    xi = rng.uniform(0, 1, n)
    T = 10 ** rng.uniform(1, 5, n)
    args = (xi * nH, xi * nH, (1 - xi) * nH, 0.08 * nH, 0.1 * rng.uniform(size=n) * nH, T)
    cl = CLOUDS["glf_outflow"]()
    st, ctx = matched_pair(oracle_mod, cl)
    got = ctx.pd_lya(*args, z=3.0)
    L = oracle_mod.lib()
    ref = np.array([L.orc_pd_lya(*(a[q] for a in args), 3.0) for q in range(n)])
    np.testing.assert_allclose(got, ref, rtol=1e-13)
    dt = ctx.cfl_dt(cl.c_tilde, cl.u_r, cl.u_Z, 0.4)
    assert dt == pytest.approx(W.cfl_dt(cl.geom, cl.c_tilde, cl.u_r, cl.u_Z, 0.4), rel=1e-15)


def test_nonfinite_input_is_reported(oracle_mod):
    """An infinite J_old makes the emission update produce a non-finite J, which the kernel
    flags; the flag is reported at the next synchronising call and then cleared."""
    from lydion_b200._lib import LydionError, LYD_ERR_NONFINITE
    cl = CLOUDS["glf_outflow"]()
    _, ctx = matched_pair(oracle_mod, cl, seed=1)
    J = ctx.download("J_old")
    J[2, 3, 5] = np.inf
    ctx.upload("J_old", J)
    ctx.emission_absorption(cl.c_tilde, cl.dt)
    with pytest.raises(LydionError) as e:
        ctx.synchronize()
    assert e.value.code == LYD_ERR_NONFINITE
    J, Hr, HZ = random_state(cl, 2)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ), ("J_old", J)):
        ctx.upload(name, a)
    ctx.emission_absorption(cl.c_tilde, cl.dt)
    ctx.frequency_update(cl.c_tilde * cl.dt)
    ctx.synchronize()


def test_bad_arguments_are_rejected(oracle_mod):
    from lydion_b200._lib import LydionError, LYD_ERR_ARG, LYD_ERR_STATE
    from lydion_b200.m1 import M1Context
    cl = CLOUDS["glf_outflow"]()
    _, ctx = matched_pair(oracle_mod, cl, seed=1)
    with pytest.raises(LydionError) as e:
        ctx.advect(cl.c_tilde * cl.dt, bc_r_left=1)
    assert e.value.code == LYD_ERR_ARG
    with pytest.raises(LydionError):
        ctx.upload("J", np.zeros(7))
    bare = M1Context(cl.n_nu, cl.nr, cl.nz, cl.freq.kcore_min, cl.freq.kcore_max, cl.alpha_floor)
    with pytest.raises(LydionError) as e:
        bare.advect(1.0)
    assert e.value.code == LYD_ERR_STATE
    bare.close()


def test_full_size_c2_steps_match_oracle(oracle_mod):
    """The headline 256x256x64 cloud over 200 fused steps against the oracle: every step's
    active window and M_F; the final J, the flux fractions and the edge-ring spectrum per
    element with a floor of 1e-6 of the maximum (the wing bins); the per-bin escaping flux.
    The escaping flux sums max(H, 0) over the boundary faces: where a boundary cell's H
    changes sign the clipped sum keeps the cancellation error of H, so its bound is looser."""
    cl = W.config_c2()
    st, ctx = matched_pair(oracle_mod, cl)
    n = 200
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    assert max_rel(d_g[1:, 0], d_o[1:, 0]) < 1e-8
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-8, f
    w = wing_checks(ctx, st, cl)
    for q in ("J", "H_r", "H_Z", "edge_spectrum"):
        assert w[q] < 1e-8, (q, w[q])
    assert w["escaping_flux"] < 1e-5, w["escaping_flux"]


def test_c4_turbulent_cloud_200_steps_match_oracle(oracle_mod):
    """The adjoint configuration's turbulent cloud (128 x 128 x 48: lognormal n_H, dust, a
    50 km/s turbulent velocity field) over 200 fused steps against the oracle, with the bounds
    of the headline cloud's test: every step's window and M_F; the final J, the flux fractions
    and the edge-ring spectrum per element with a floor of 1e-6 of the maximum; the per-bin
    escaping flux."""
    cl = W.config_c4()
    st, ctx = matched_pair(oracle_mod, cl)
    n = 200
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    assert max_rel(d_g[1:, 0], d_o[1:, 0]) < 1e-8
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-8, f
    w = wing_checks(ctx, st, cl)
    for q in ("J", "H_r", "H_Z", "edge_spectrum"):
        assert w[q] < 1e-8, (q, w[q])
    assert w["escaping_flux"] < 1e-5, w["escaping_flux"]


def test_c1_point_source_1000_steps_match_oracle(oracle_mod):
    """The plain-FP64 point-source cloud (64 x 64 x 64, tau0 = 1e6, recoil on) over the 1000
    steps it is specified with, against the oracle: the active window of every step, M_F, and
    per element with a floor of 1e-6 of the maximum, the final J, the flux fractions, the
    edge-ring spectrum and the per-bin escaping flux."""
    cl = W.config_c1()
    st, ctx = matched_pair(oracle_mod, cl)
    n = 1000
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    assert max_rel(d_g[1:, 0], d_o[1:, 0]) < 1e-9
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-9, f
    w = wing_checks(ctx, st, cl)
    for q in ("J", "H_r", "H_Z", "edge_spectrum", "escaping_flux"):
        assert w[q] < 1e-8, (q, w[q])


def test_c5_slice_256x256x128_matches_oracle(oracle_mod):
    """A 256 x 256 x 128-bin slice of the largest-field workload (the synthetic RHD snapshot:
    lognormal n_H, photoionised bubble with p_d from pd_Lya on the device, shell outflow, dust)
    over 20 steps against the oracle: windows, M_F, and J, the flux fractions and the edge
    spectrum per element with a floor of 1e-6 of the maximum. After 20 steps no radiation has
    reached the outer faces, so the escaping flux is not compared."""
    from lydion_b200.m1 import context_for_cloud
    cl = W.rhd_snapshot_cloud(n=256, n_nu=128, name="c5_slice_256x256x128")
    ctx = context_for_cloud(cl)          # computes p_d on the device from the species
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    n = 20
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    assert max_rel(d_g[1:, 0], d_o[1:, 0]) < 1e-10
    w = wing_checks(ctx, st, cl)
    for q in ("J", "H_r", "H_Z", "edge_spectrum"):
        assert w[q] < 1e-8, (q, w[q])
    ctx.close()


def test_rhd_snapshot_field_matches_oracle(oracle_mod):
    """The synthetic RHD snapshot (lognormal n_H, photoionised bubble with p_d from pd_Lya,
    shell outflow, dust) at 64 x 64 x 16: a few full steps against the oracle."""
    from lydion_b200.m1 import context_for_cloud
    cl = W.config_c5(16)
    ctx = context_for_cloud(cl)          # computes p_d on the device from the species
    assert np.all(cl.pd >= 0.0) and np.any(cl.pd > 0.0)
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    n = 5
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    # the first step's M_F is ~1e-63 (no flux yet): compare where it is resolved
    assert max_rel(d_g[1:, 0], d_o[1:, 0]) < 1e-9
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-9, f


@pytest.mark.parametrize("n_nu,tol", [(128, 1e-9), (200, 5e-9)])
def test_many_bins_per_lane_match_oracle(oracle_mod, n_nu, tol):
    """4 and 8 bins per lane (N_nu = 128, 200): the two-level cyclic-reduction + PCR solve and the
    plain 8-level PCR over 256 rows. Both the oracle's pivoted elimination and PCR are backward
    stable; their difference follows the systems' conditioning, which grows with the number of
    bins (1.4e-9 of the field maximum at 200 bins and tau0 = 1e7)."""
    cl = W.small_cloud(nr=7, nz=6, n_nu=n_nu, x_max=600.0, tau0=1e7)
    st, ctx = matched_pair(oracle_mod, cl, seed=41)
    n = 12
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    assert max_rel(d_g[:, 0], d_o[:, 0]) < tol
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < tol, f


@pytest.mark.parametrize("bc_z_bot", [W.BC_REFLECT, W.BC_OUTFLOW])
def test_log_stretched_grid_steps_match_oracle(oracle_mod, bc_z_bot):
    """The step on a grid with logarithmic regions (SetupCylindricalGrid with N_r_log and
    N_Z_log_side, src/SpatialGrid.jl:606-915): non-uniform PLM intervals, volumes and areas in
    every kernel, 30 fused steps against the oracle."""
    from lydion_b200 import constants as K
    from lydion_b200 import grid as G
    pc = K.pc
    if bc_z_bot == W.BC_REFLECT:
        geom = G.log_stretched_cylindrical_geometry(1.1 * pc, 0.6 * pc, 1.1 * pc, 0.5 * pc, 10, 6, 9, 5, "Reflect")
    else:
        geom = G.log_stretched_cylindrical_geometry(1.1 * pc, 0.6 * pc, 2.2 * pc, 0.8 * pc, 10, 6, 9, 4, "Outflow")
    cl = W.static_cloud(0, 0, 32, tau0=1e6, tau_abs=0.5, rs=0.5, umax_kms=100.0, bc_z_bot=bc_z_bot,
                        x_max=100.0, geom=geom, name="stretched")
    st, ctx = matched_pair(oracle_mod, cl, seed=19)
    n = 30
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    assert max_rel(d_g[1:, 0], d_o[1:, 0]) < 1e-9
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-9, f
    ctx.close()
