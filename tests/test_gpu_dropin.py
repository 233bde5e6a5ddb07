"""The drop-in functions with the reference's signatures (lydion_b200/lya.py), through the C
ABI, against the oracle: one static-driver iteration called phase by phase."""
import numpy as np
import pytest

from helpers import max_rel, norm_err, random_state
from lydion_b200 import lya as D
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_reference_signatures_step(oracle_mod):
    cl = W.small_cloud(nr=10, nz=9, n_nu=32)
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    J, Hr, HZ = random_state(cl, 41)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
        getattr(st, name)[...] = a
        getattr(st, name + "_old")[...] = a
    lya = D.generate_lya_arrays_from_saved(cl.c_tilde, cl.freq, cl.geom, cl.T, st.Hvoigt, st.phi_nu,
                                           recoil=cl.recoil)
    for name in ("J", "J_old", "H_r", "H_Z", "H_r_old", "H_Z_old", "alpha_F"):
        getattr(lya, name)[...] = getattr(st, name)
    for name in ("alpha", "alpha_c", "pd", "js"):
        getattr(lya, name)[...] = getattr(cl, name)
    ctdt = cl.c_tilde * cl.dt
    vel = (cl.u_r_star, cl.u_Z_star, cl.dur_dr, cl.dur_dZ, cl.duZ_dr, cl.duZ_dZ, cl.ur_over_r)
    # AdvectLya!
    st.advect(ctdt)
    D.advect_lya(ctdt, lya, cl.geom, *vel, "Reflect", "Outflow", "Reflect", "Outflow")
    assert norm_err(lya.J, st.J) < 1e-12 and norm_err(lya.H_r, st.H_r) < 1e-12
    # LyaEmissionAbsorptionUpdate!
    st.emission_absorption(cl.c_tilde, cl.dt)
    D.lya_emission_absorption_update(lya.J, lya.J_old, lya.H_r, lya.H_Z, lya.H_r_old, lya.H_Z_old, lya.js,
                                     lya.phi_nu, lya.Hvoigt, lya.alpha, lya.alpha_c, lya.alpha_F, lya.pd,
                                     lya.dru_r, lya.dru_Z, lya.dnu, cl.c_tilde, cl.dt, lya=lya, geom=cl.geom)
    assert norm_err(lya.J, st.J) < 1e-12 and norm_err(lya.dru_Z, st.dru_Z) < 1e-12
    # FrequencyUpdateJLya_AllCells!
    st.frequency_update(ctdt)
    D.frequency_update_J_lya_all_cells(ctdt, lya, cl.T, *vel[2:], True, geom=cl.geom)
    assert norm_err(lya.J, st.J) < 1e-9
    np.testing.assert_array_equal(lya.J_old, lya.J)
    # Update_f_Lya_MF_L_Lya! and Compute_f_esc_Lya_Cylindrical
    mo = st.force_multiplier(cl.dt)
    mg = D.update_f_lya_MF_L_lya(lya.f_r, lya.f_Z, lya.dru_r, lya.dru_Z, lya.js, cl.geom.dV, cl.geom.rCoM,
                                 cl.geom.ZCoM, cl.dt, cl.z_center, "Reflect", lya=lya, geom=cl.geom)
    np.testing.assert_allclose(mg, mo, rtol=1e-11)
    fg = D.compute_f_esc_lya_cylindrical(lya.H_r, lya.H_Z, cl.geom.A_r, cl.geom.A_Z, lya.dnu, mg[3], "Reflect",
                                         lya=lya, geom=cl.geom)
    assert fg == pytest.approx(st.f_esc(mo[3]), rel=1e-8)
    assert D.find_active_bins(lya, cl.geom) == st.find_active_bins()
