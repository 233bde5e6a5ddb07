"""The drop-in functions with the reference's signatures (lydion_b200/lya.py), through the C
ABI, against the oracle: static-driver iterations of src/StaticCloudTest.jl:357-392 called phase
by phase with exactly the reference's positional arguments, in the default copy mode and with
the state resident on the device; inputs uploaded once per array object unless marked dirty."""
import numpy as np
import pytest

from helpers import norm_err, random_state
from lydion_b200 import lya as D
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _setup(oracle_mod, seed=41):
    cl = W.small_cloud(nr=10, nz=9, n_nu=32)
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    J, Hr, HZ = random_state(cl, seed)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
        getattr(st, name)[...] = a
        getattr(st, name + "_old")[...] = a
    LyaState = D.generate_lya_arrays_from_saved(cl.c_tilde, cl.freq, cl.geom, cl.T, st.Hvoigt, st.phi_nu,
                                                recoil=cl.recoil)
    for name in ("J", "J_old", "H_r", "H_Z", "H_r_old", "H_Z_old", "alpha_F"):
        getattr(LyaState, name)[...] = getattr(st, name)
    for name in ("alpha", "alpha_c", "pd", "js"):
        getattr(LyaState, name)[...] = getattr(cl, name)
    return cl, st, LyaState


def _driver_iteration(cl, LyaState):
    """One iteration of the static-cloud loop (src/StaticCloudTest.jl:362-392), word for word
    apart from the names."""
    g = cl.geom
    c_tilde, dt = cl.c_tilde, cl.dt
    ctdt = c_tilde * dt
    J, J_old, H_r, H_Z = LyaState.J, LyaState.J_old, LyaState.H_r, LyaState.H_Z
    H_r_old, H_Z_old, dru_r, dru_Z = LyaState.H_r_old, LyaState.H_Z_old, LyaState.dru_r, LyaState.dru_Z
    D.advect_lya(ctdt, LyaState, g, cl.u_r_star, cl.u_Z_star, cl.dur_dr, cl.dur_dZ, cl.duZ_dr, cl.duZ_dZ,
                 cl.ur_over_r, "Reflect", "Outflow", "Reflect", "Outflow")
    D.lya_emission_absorption_update(J, J_old, H_r, H_Z, H_r_old, H_Z_old, LyaState.js, LyaState.phi_nu,
                                     LyaState.Hvoigt, LyaState.alpha, LyaState.alpha_c, LyaState.alpha_F, LyaState.pd,
                                     dru_r, dru_Z, LyaState.dnu, c_tilde, dt)
    D.frequency_update_J_lya_all_cells(ctdt, LyaState, cl.T, cl.dur_dr, cl.dur_dZ, cl.duZ_dr, cl.duZ_dZ,
                                       cl.ur_over_r, True)
    mf = D.update_f_lya_MF_L_lya(LyaState.f_r, LyaState.f_Z, dru_r, dru_Z, LyaState.js, g.dV, g.rCoM, g.ZCoM, dt,
                                 cl.z_center, "Reflect")
    LyaState.M_F, LyaState.M_F_radial_net, LyaState.M_F_radial_out, LyaState.L_lya = mf
    LyaState.f_esc_lya = D.compute_f_esc_lya_cylindrical(H_r, H_Z, g.A_r, g.A_Z, LyaState.dnu, LyaState.L_lya,
                                                         "Reflect")
    D.reset_dru(dru_r, dru_Z)
    return mf


def _oracle_iteration(cl, st):
    ctdt = cl.c_tilde * cl.dt
    st.advect(ctdt)
    st.emission_absorption(cl.c_tilde, cl.dt)
    st.frequency_update(ctdt)
    mo = st.force_multiplier(cl.dt)
    fo = st.f_esc(mo[3])
    st.dru_r[...] = 0.0
    st.dru_Z[...] = 0.0
    return mo, fo


def test_reference_signatures_step(oracle_mod):
    cl, st, LyaState = _setup(oracle_mod)
    ctdt = cl.c_tilde * cl.dt
    vel = (cl.u_r_star, cl.u_Z_star, cl.dur_dr, cl.dur_dZ, cl.duZ_dr, cl.duZ_dZ, cl.ur_over_r)
    assert D.find_active_bins(LyaState, cl.geom.dV) == st.find_active_bins()
    # AdvectLya!
    st.advect(ctdt)
    D.advect_lya(ctdt, LyaState, cl.geom, *vel, "Reflect", "Outflow", "Reflect", "Outflow")
    assert norm_err(LyaState.J, st.J) < 1e-12 and norm_err(LyaState.H_r, st.H_r) < 1e-12
    np.testing.assert_array_equal(LyaState.J_old, LyaState.J)
    # LyaEmissionAbsorptionUpdate!
    st.emission_absorption(cl.c_tilde, cl.dt)
    D.lya_emission_absorption_update(LyaState.J, LyaState.J_old, LyaState.H_r, LyaState.H_Z, LyaState.H_r_old,
                                     LyaState.H_Z_old, LyaState.js, LyaState.phi_nu, LyaState.Hvoigt, LyaState.alpha,
                                     LyaState.alpha_c, LyaState.alpha_F, LyaState.pd, LyaState.dru_r, LyaState.dru_Z,
                                     LyaState.dnu, cl.c_tilde, cl.dt)
    assert norm_err(LyaState.J, st.J) < 1e-12 and norm_err(LyaState.dru_Z, st.dru_Z) < 1e-12
    # FrequencyUpdateJLya_AllCells!
    st.frequency_update(ctdt)
    D.frequency_update_J_lya_all_cells(ctdt, LyaState, cl.T, *vel[2:], True)
    assert norm_err(LyaState.J, st.J) < 1e-9
    np.testing.assert_array_equal(LyaState.J_old, LyaState.J)
    # Update_f_Lya_MF_L_Lya! and Compute_f_esc_Lya_Cylindrical
    g = cl.geom
    mo = st.force_multiplier(cl.dt)
    mg = D.update_f_lya_MF_L_lya(LyaState.f_r, LyaState.f_Z, LyaState.dru_r, LyaState.dru_Z, LyaState.js, g.dV,
                                 g.rCoM, g.ZCoM, cl.dt, cl.z_center, "Reflect")
    np.testing.assert_allclose(mg, mo, rtol=1e-11)
    fg = D.compute_f_esc_lya_cylindrical(LyaState.H_r, LyaState.H_Z, g.A_r, g.A_Z, LyaState.dnu, mg[3], "Reflect")
    assert fg == pytest.approx(st.f_esc(mo[3]), rel=1e-8)
    D.reset_dru(LyaState.dru_r, LyaState.dru_Z)
    assert not LyaState.dru_r.any() and not LyaState.dru_Z.any()
    D.release(LyaState)


@pytest.mark.parametrize("resident", [False, True])
def test_static_driver_loop(oracle_mod, resident):
    """Five iterations of the static-cloud loop through the drop-ins, copy mode and resident
    mode, against the oracle: the diagnostics every iteration, the state at the end."""
    cl, st, LyaState = _setup(oracle_mod, seed=43)
    if resident:
        D.set_resident(LyaState)
    for _ in range(5):
        mg = _driver_iteration(cl, LyaState)
        mo, fo = _oracle_iteration(cl, st)
        np.testing.assert_allclose(mg, mo, rtol=1e-9)
        assert LyaState.f_esc_lya == pytest.approx(fo, rel=1e-8)
    if resident:
        D.sync_to_host(LyaState)
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(getattr(LyaState, f), getattr(st, f)) < 1e-9, f
    up, down = D.transfer_bytes(LyaState)
    n3 = LyaState.J.nbytes
    if resident:
        # the state went up once (when resident mode began) and came back once
        assert up < 12 * n3 and down <= 6 * n3 + 4 * LyaState.dru_r.nbytes
    else:
        assert up > 5 * 10 * n3 and down > 5 * 6 * n3
    D.release(LyaState)


def test_inputs_upload_once_unless_marked_dirty(oracle_mod):
    cl, st, LyaState = _setup(oracle_mod, seed=47)
    D.set_resident(LyaState)
    _driver_iteration(cl, LyaState)
    up1 = D.transfer_bytes(LyaState)[0]
    _driver_iteration(cl, LyaState)
    up2 = D.transfer_bytes(LyaState)[0]
    assert up2 == up1          # nothing went up in the second iteration: inputs and state stay on the device
    # an in-place change of an input counts only after mark_dirty
    LyaState.alpha *= 1.5
    D.mark_dirty(LyaState.alpha)
    _driver_iteration(cl, LyaState)
    assert D.transfer_bytes(LyaState)[0] == up2 + LyaState.alpha.nbytes
    D.release(LyaState)


def test_arrays_without_a_twin_are_rejected(oracle_mod):
    cl, st, LyaState = _setup(oracle_mod)
    stray = np.zeros_like(LyaState.dru_r)
    with pytest.raises(ValueError):
        D.reset_dru(stray, LyaState.dru_Z)
    with pytest.raises(ValueError):
        D.update_f_lya_MF_L_lya(LyaState.f_r, LyaState.f_Z, LyaState.dru_r, LyaState.dru_Z, LyaState.js,
                                2.0 * cl.geom.dV, cl.geom.rCoM, cl.geom.ZCoM, cl.dt, cl.z_center, "Reflect")
    D.release(LyaState)


def test_context_free_functions(oracle_mod):
    cl = W.small_cloud(nr=10, nz=9, n_nu=32)
    u_r = np.full((cl.nz, cl.nr), 3.0e6)
    u_Z = np.full((cl.nz, cl.nr), -1.0e6)
    dt = D.get_rhd_cfl_time_step(cl.geom.r, cl.geom.Z, cl.c_tilde, u_r, u_Z, 0.4)
    dr = np.min(np.diff(cl.geom.r))
    dZ = np.min(np.diff(cl.geom.Z))
    u = np.hypot(3.0e6, 1.0e6)
    assert dt == pytest.approx(0.4 * 0.5 * min(dr, dZ) / (cl.c_tilde + u), rel=1e-12)
    p = D.pd_lya(1.0, 1.0, 100.0, 10.0, 0.0, 1e4, 0.0)
    assert isinstance(p, float) and 0.0 <= p < 1.0
    arr = D.pd_lya(np.full(5, 1.0), np.full(5, 1.0), np.full(5, 100.0), np.full(5, 10.0), np.zeros(5),
                   np.full(5, 1e4))
    np.testing.assert_allclose(arr, p, rtol=0, atol=0)
