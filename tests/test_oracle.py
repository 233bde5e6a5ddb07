"""CPU tests of the FP64 oracle: pins against the committed golden fixtures, known answers of
the closure and line-profile functions, and conservation properties of the step."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN
from lydion_b200 import constants as K
from lydion_b200 import grid as G
from lydion_b200 import workloads as W


def test_dgtsv_matches_lapack_fixture(oracle_mod):
    z = np.load(os.path.join(GOLDEN, "dgtsv_cases.npz"))
    n = int(z["n"])
    assert n > 30
    for q in range(n):
        dl, d, du, b = z[f"dl{q}"], z[f"d{q}"], z[f"du{q}"], z[f"b{q}"]
        x_ref, info_ref = z[f"x{q}"], int(z[f"info{q}"])
        x, info = oracle_mod.dgtsv(dl, d, du, b)
        assert info == info_ref, q
        if info == 0:
            # same algorithm, same operation order: agreement to a few ulps
            np.testing.assert_allclose(x, x_ref, rtol=1e-13, atol=0, err_msg=f"case {q}")


def test_dgtsv_single_row(oracle_mod):
    x, info = oracle_mod.dgtsv(np.zeros(0), [4.0], np.zeros(0), [2.0])
    assert info == 0 and x[0] == 0.5
    _, info = oracle_mod.dgtsv(np.zeros(0), [0.0], np.zeros(0), [2.0])
    assert info == 1


def test_voigt_tables_match_fixture(oracle_mod):
    z = np.load(os.path.join(GOLDEN, "voigt_samples.npz"))
    t = oracle_mod.voigt_tables()
    np.testing.assert_array_equal(t["erf"][z["idx"]], z["erf"])
    np.testing.assert_array_equal(t["dawson"][z["idx"]], z["dawson"])
    # node coordinates of CreateLUT: x_i = xmin + i*dx
    x = t["xmin"] + z["idx"] * (1 / t["inv_dx"])
    np.testing.assert_allclose(x, z["x"], rtol=0, atol=1e-12)


def test_closure_known_answers(oracle_mod):
    L = oracle_mod.lib()
    assert L.orc_chi_L84(0.0) == pytest.approx(1 / 3, abs=1e-16)
    assert L.orc_chi_L84(1.0) == pytest.approx(1.0, abs=1e-16)
    # isotropic limit
    D = oracle_mod.vec_fn("orc_D_edd", 0.0, 0.0, 1.0)
    np.testing.assert_allclose(D, [1 / 3, 1 / 3, 0.0])
    # free streaming along r: D_rr -> 1
    D = oracle_mod.vec_fn("orc_D_edd", 1.0 - 1e-12, 0.0, 1.0)
    assert D[0] == pytest.approx(1.0, abs=1e-6) and abs(D[1]) < 1e-6
    # trace of the r-Z block plus phi-phi part is one for the f,n form
    for f in [0.0, 0.2, 0.7, 1.0]:
        for th in np.linspace(0, 2 * np.pi, 7):
            D = oracle_mod.vec_fn("orc_D_edd_from_f_n", f, np.cos(th), np.sin(th))
            chi = L.orc_chi_L84(min(max(f, 1e-10), 1 - 1e-10)) if f > 1e-10 else 1 / 3
            assert D[0] + D[1] == pytest.approx((1 - chi) * 0.5 * 2 + (3 * chi - 1) * 0.5 if f > 1e-10 else 2 / 3)
    # HLL eigenvalues at vanishing flux are +-1/sqrt(3)
    e = oracle_mod.vec_fn("orc_hll_eigenvalues", 0.0, 1.0, n=2)
    np.testing.assert_allclose(e, [-1 / np.sqrt(3), 1 / np.sqrt(3)], rtol=1e-6)
    e = oracle_mod.vec_fn("orc_hll_eigenvalues", 1.0, 1.0, n=2)
    assert e[1] == pytest.approx(1.0, abs=1e-4)
    assert L.orc_minmod(1.0, -2.0) == 0.0 and L.orc_minmod(1.0, 2.0) == 1.0 and L.orc_minmod(-3.0, -2.0) == -2.0


def test_thermal_constants(oracle_mod):
    L = oracle_mod.lib()
    for T in [10.0, 1e2, 1e4]:
        assert L.orc_compute_dnuD(T) == K.compute_dnuD(T)
        assert L.orc_compute_a(T) == K.compute_a(T)
        assert L.orc_compute_sigma0(T) == pytest.approx(K.compute_sigma0(T), rel=1e-15)
    # a ~ 4.7e-4 at 1e4 K and sigma0 ~ 5.9e-14 cm^2 (src/ConstantsAndFunctions.jl:222-223)
    assert 4.5e-4 < K.compute_a(1e4) < 4.9e-4
    assert 5.5e-14 < K.compute_sigma0(1e4) < 6.2e-14


def test_voigt_profile_normalisation(oracle_mod):
    """Bin-averaged H times bin width sums to sqrt(pi) dnuD over a wide grid."""
    cl = W.small_cloud(nr=4, nz=4, n_nu=64, x_max=600.0, tau0=1e4)
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    dnuD = K.compute_dnuD(1e4)
    s = np.sum(st.Hvoigt[0, 0] * cl.freq.dnu)
    assert s == pytest.approx(np.sqrt(np.pi) * dnuD, rel=2e-3)
    # phi_nu is normalised over the core bins and zero outside
    fq = cl.freq
    phi = st.phi_nu[0, 0]
    assert np.sum(phi[fq.kcore_min:fq.kcore_max + 1] * fq.dnu[fq.kcore_min:fq.kcore_max + 1]) == pytest.approx(1.0, rel=1e-13)
    assert np.all(phi[:fq.kcore_min] == 0) and np.all(phi[fq.kcore_max + 1:] == 0)


def test_voigt_tophat_small_bin_uses_H(oracle_mod):
    lut = oracle_mod.OracleLUT()
    L = oracle_mod.lib()
    a = K.compute_a(1e4)
    for x in [0.0, 0.3, 2.0, 7.5]:
        th = L.orc_voigt_tophat(lut.ref, x, x + 5e-6, x - 4e-6, a)
        assert th == L.orc_voigt_H(lut.ref, x, a)


def test_pd_lya_range(oracle_mod):
    L = oracle_mod.lib()
    vals = [L.orc_pd_lya(nh, nh, 1e-4 * nh, 0.1 * nh, 0.0, T, 0.0) for nh in [1e-2, 1e2, 1e6] for T in [1e2, 1e4, 1e5]]
    assert all(0.0 <= v <= 1.0 for v in vals)
    # more ions -> more 2s-2p mixing -> larger destruction probability
    assert L.orc_pd_lya(1e6, 1e6, 1.0, 0.0, 0.0, 1e4, 0.0) > L.orc_pd_lya(1.0, 1.0, 1.0, 0.0, 0.0, 1e4, 0.0)
    # the H2 line-absorption term (src/LymanAlphaDestruction.jl:85-91) needs H I present
    assert L.orc_pd_lya(0.0, 0.0, 1.0, 0.0, 1.0, 3e3, 0.0) > 1e-4
    assert L.orc_pd_lya(0.0, 0.0, 0.0, 0.0, 1.0, 3e3, 0.0) < 1e-10


def test_geometry_uniform_grid():
    g = G.uniform_cylindrical_geometry(3.0, 2.0, 6, 4)
    assert g.dV.shape == (4, 6) and g.A_r.shape == (4, 7) and g.A_Z.shape == (5, 6)
    assert g.dV.sum() == pytest.approx(np.pi * 9.0 * 2.0, rel=1e-14)
    assert np.all(g.A_r[:, 0] == 0.0)
    assert g.dZ_L == pytest.approx(np.full(4, 0.25)) and g.dZ_R == pytest.approx(np.full(4, 0.25))
    # the inner Z ghost centroid mirrors ZCoM[1] about Z = 0
    assert g.dZ_b[0] == pytest.approx(0.25) and g.dZ_b[3] == pytest.approx(2.0)
    with pytest.raises(ValueError):
        G.uniform_cylindrical_geometry(1.0, 1.0, 2, 5)


@pytest.mark.parametrize("bc", ["Reflect", "Outflow"])
def test_log_stretched_grid_intervals(bc):
    """SetupCylindricalGrid with logarithmic regions (src/SpatialGrid.jl:606-830): the uniform
    part is the LinRange of its cells, the logarithmic part's widths start at the uniform width
    and grow by one ratio q, q is the root of L - d (q^n - 1)/(q - 1), and the grid ends at
    rmax / Zmax; with an outflowing bottom the lower Z region mirrors the upper one."""
    pc = K.pc
    rmax, rmax_lin, N_r_lin, N_r_log = 1.1 * pc, 0.6 * pc, 8, 6
    Zmax, LZ, N_Z_lin, N_Z_log = (1.1 * pc, 0.5 * pc, 8, 5) if bc == "Reflect" else (2.2 * pc, 0.8 * pc, 8, 5)
    r, Z = G.log_stretched_interfaces(rmax, rmax_lin, Zmax, LZ, N_r_lin, N_r_log, N_Z_lin, N_Z_log, bc)
    assert r.size - 1 == N_r_lin + N_r_log
    assert Z.size - 1 == N_Z_lin + (2 if bc == "Outflow" else 1) * N_Z_log
    assert r[0] == 0.0 and Z[0] == 0.0 and r[-1] == rmax and Z[-1] == Zmax
    np.testing.assert_array_equal(r[:N_r_lin + 1], G.julia_linrange(0.0, rmax_lin, N_r_lin + 1))
    d = r[1] - r[0]
    q = G.geometric_ratio(rmax - rmax_lin, d, N_r_log)
    assert abs((rmax - rmax_lin) - d * (q ** N_r_log - 1) / (q - 1)) <= 1e-12 * rmax
    w = np.diff(r)[N_r_lin:]
    np.testing.assert_allclose(w, d * q ** np.arange(N_r_log), rtol=1e-10)
    wz = np.diff(Z)
    if bc == "Outflow":
        np.testing.assert_allclose(wz[:N_Z_log], wz[::-1][:N_Z_log], rtol=1e-10)
        dz = wz[N_Z_log]
        qz = G.geometric_ratio(0.5 * (Zmax - LZ), dz, N_Z_log)
        np.testing.assert_allclose(wz[N_Z_log + N_Z_lin:], dz * qz ** np.arange(N_Z_log), rtol=1e-10)
        np.testing.assert_allclose(Z[N_Z_log:N_Z_log + N_Z_lin + 1],
                                   G.julia_linrange(0.5 * (Zmax - LZ), 0.5 * (Zmax + LZ), N_Z_lin + 1), rtol=1e-15)
    else:
        dz = wz[0]
        qz = G.geometric_ratio(Zmax - LZ, dz, N_Z_log)
        np.testing.assert_allclose(wz[N_Z_lin:], dz * qz ** np.arange(N_Z_log), rtol=1e-10)
    # the PLM intervals of the stretched grid: L = r_{i+1/2} - rCoM_i, R = rCoM_{i+1} - r_{i+1/2}
    g = G.log_stretched_cylindrical_geometry(rmax, rmax_lin, Zmax, LZ, N_r_lin, N_r_log, N_Z_lin, N_Z_log, bc)
    np.testing.assert_allclose(g.dr_L, r[1:] - g.rCoM, rtol=1e-14)
    np.testing.assert_allclose(g.dr_R[:-1], g.rCoM[1:] - r[1:-1], rtol=1e-14)
    np.testing.assert_allclose(g.inv_dr_ip1_i[:-1], 1.0 / np.diff(g.rCoM), rtol=1e-14)
    assert g.dV.sum() == pytest.approx(np.pi * rmax ** 2 * Zmax, rel=1e-13)


def test_log_stretched_grid_edge_cases():
    pc = K.pc
    # a "logarithmic" region that n uniform cells already span stays uniform
    r, Z = G.log_stretched_interfaces(1.0 * pc, 0.5 * pc, 1.0 * pc, 0.5 * pc, 5, 5, 5, 5, "Reflect")
    np.testing.assert_allclose(np.diff(r), 0.1 * pc, rtol=1e-12)
    # a region too short for its cells at the uniform width is rejected
    with pytest.raises(ValueError):
        G.log_stretched_interfaces(1.0 * pc, 0.8 * pc, 1.0 * pc, 0.5 * pc, 4, 5, 5, 5, "Reflect")
    with pytest.raises(ValueError):
        G.log_stretched_interfaces(1.0 * pc, 0.5 * pc, 1.0 * pc, 1.5 * pc, 5, 5, 5, 5, "Reflect")
    # one logarithmic cell or none: the whole axis is uniform
    r, Z = G.log_stretched_interfaces(1.0 * pc, 0.5 * pc, 1.0 * pc, 0.5 * pc, 6, 1, 6, 0, "Reflect")
    np.testing.assert_array_equal(r, G.julia_linrange(0.0, 1.0 * pc, 7))


def test_frequency_grids():
    fq = G.symmetric_frequency_grid(64)
    assert fq.n_nu == 64
    x = (fq.nu - K.nu_lya) / K.compute_dnuD(1e4)
    assert x[0] == pytest.approx(-600.0) and x[-1] == pytest.approx(600.0)
    np.testing.assert_allclose(fq.dnu, fq.dnu[::-1], rtol=1e-9)
    assert 0 < fq.kcore_min < 32 <= fq.kcore_max < 63
    ref = G.reference_frequency_grid()
    assert ref.n_nu == 194  # default grid of GenerateLyaArrays with Tmin = 30 K, q = 1.1


def test_find_active_bins_empty_field_is_core(oracle_mod):
    cl = W.small_cloud()
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    assert st.find_active_bins() == (cl.freq.kcore_min, cl.freq.kcore_max)


def _closed_box(oracle_mod, steps, **kw):
    cl = W.small_cloud(nr=10, nz=9, n_nu=16, umax_kms=0.0, tau_abs=0.0, **kw)
    cl.bc_r_right = W.BC_REFLECT
    cl.bc_z_top = W.BC_REFLECT
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    rng = np.random.default_rng(1)
    J = 1e-12 * (1 + rng.uniform(size=st.J.shape))
    st.J[...] = J; st.J_old[...] = J
    st.H_r[...] = 0.3 * J * rng.uniform(-1, 1, J.shape); st.H_Z[...] = 0.3 * J * rng.uniform(-1, 1, J.shape)
    st.H_r[:, 0, :] = 0.0
    return cl, st


def test_advection_conserves_energy_in_closed_box(oracle_mod):
    cl, st = _closed_box(oracle_mod, 1)
    dV = cl.geom.dV[:, :, None]
    e0 = np.sum(st.J * dV)
    for _ in range(5):
        st.advect(0.3 * cl.c_tilde * cl.dt)
    assert np.sum(st.J * dV) == pytest.approx(e0, rel=1e-12)


def test_frequency_step_conserves_photons(oracle_mod):
    cl, st = _closed_box(oracle_mod, 1)
    dnu = cl.freq.dnu
    n0 = np.sum(st.J[..., 1:-1] * dnu[1:-1], axis=-1)
    nf, _ = st.frequency_update(cl.c_tilde * cl.dt)
    assert nf == 0
    n1 = np.sum(st.J[..., 1:-1] * dnu[1:-1], axis=-1)
    # edge bins are outside the system, so only leakage into bins 0 and N-1 changes the sum
    np.testing.assert_allclose(n1, n0, rtol=1e-6)


def test_static_run_is_finite_and_emits(oracle_mod):
    cl = W.small_cloud()
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    d = st.run(60)
    assert np.all(np.isfinite(d)) and np.all(np.isfinite(st.J))
    assert d[-1, 0] > d[5, 0] > 0  # force multiplier builds up
    assert d[-1, 3] == pytest.approx(d[0, 3])  # luminosity is constant
    raw, norm, ri, zi = st.edge_spectra()
    assert raw.shape[0] == (cl.nz - 2) + 2 * (cl.nr - 3)
    assert np.all(ri[: cl.nz - 2] == cl.nr - 2)


def test_gravity_force_multiplier_antiparallel(oracle_mod):
    """With gravity exactly opposite to the radiation force in every cell, M_F_antigravity
    equals M_F; with no gravity it is zero (src/ConstantsAndFunctions.jl:737-750)."""
    from lydion_b200 import workloads as W
    cl = W.small_cloud(nr=8, nz=7, n_nu=16)
    st = oracle_mod.OracleState(cl)
    st.setup_profiles()
    rng = np.random.default_rng(0)
    st.dru_r[...] = rng.normal(size=st.dru_r.shape)
    st.dru_Z[...] = rng.normal(size=st.dru_Z.shape)
    out = st.force_multiplier_gravity(cl.dt, -st.dru_r, -st.dru_Z)
    st.dru_r[...] = st.f_r * cl.dt
    st.dru_Z[...] = st.f_Z * cl.dt
    plain = st.force_multiplier(cl.dt)
    assert out[1] == pytest.approx(out[0], rel=1e-13)
    np.testing.assert_allclose(out[[0, 2, 3, 4]], plain, rtol=1e-13)
    st.dru_r[...] = st.f_r * cl.dt
    st.dru_Z[...] = st.f_Z * cl.dt
    z = np.zeros_like(st.dru_r)
    assert st.force_multiplier_gravity(cl.dt, z, z)[1] == 0.0


def test_rhd_lya_oracle_pins():
    """Pinned points of the RHD-side Lyman-alpha block's oracle: the Storey & Hummer (1995)
    table nodes (src/LymanAlphaEmission.jl:36-65), the flat extrapolation, linear interpolation
    between nodes in log space, and the Case B recombination rate at 1e4 K (2.59e-13 cm^3 s^-1,
    the value of the fit in src/PhotoChemistryAndCooling/GasChemistryRates.jl:176-181)."""
    from oracle import oracle as O
    L = O.lib()
    assert L.orc_prob_lya_sh95(1e4, 1e2, 1) == 0.68808416
    assert L.orc_prob_lya_sh95(1e4, 1e2, 0) == 0.40023971
    assert L.orc_prob_lya_sh95(3e4, 1e14, 1) == 0.96391965
    assert L.orc_prob_lya_sh95(1e6, 1e20, 1) == 0.96391965          # clamped to the grid's corner
    assert L.orc_prob_lya_sh95(1.0, 1.0, 0) == 0.58042473
    mid = L.orc_prob_lya_sh95(1e4, 10 ** 2.5, 1)
    assert abs(mid - 0.5 * (0.68808416 + 0.76220739)) < 1e-15
    assert abs(L.orc_krec_hii(1e4, 1) - 2.59e-13) < 1e-3 * 2.59e-13
    assert L.orc_krec_hii(1e4, 0) > L.orc_krec_hii(1e4, 1)           # Case A exceeds Case B
    E = 6.626069573e-27 * 2.466068e15 / (4 * np.pi)
    js = L.orc_js_rec_lya(1e4, 2.0, 3.0, 1)
    assert abs(js - L.orc_prob_lya_sh95(1e4, 3.0, 1) * L.orc_krec_hii(1e4, 1) * 2.0 * 3.0 * E) < 1e-12 * js
    # collisional excitation is negligible in cold gas and rises steeply with T
    assert L.orc_js_coll_lya(1e3, 1.0, 1.0) < 1e-40 < L.orc_js_coll_lya(1e4, 1.0, 1.0)


def _dual_problem(oracle_mod, flux=0):
    from helpers import random_state
    cl = W.small_cloud(nr=8, nz=7, n_nu=16, flux_method=flux)
    state = random_state(cl, 5)
    rng = np.random.default_rng(11)
    seeds = {"alpha": rng.normal(size=cl.alpha.shape) * cl.alpha,
             "alpha_c": rng.normal(size=cl.alpha_c.shape) * cl.alpha_c,
             "T": rng.normal(size=cl.T.shape) * cl.T,
             "u_r_star": rng.normal(size=cl.u_r_star.shape) * cl.u_r_star,
             "J0": rng.normal(size=state[0].shape) * state[0]}
    w = np.random.default_rng(1).uniform(0.5, 1.5, cl.n_nu)
    return cl, state, seeds, w


def _plain_objective(oracle_mod, cl, state, n, w, ss, shift):
    import copy
    c = copy.deepcopy(cl)
    st0 = list(state)
    for k, d in shift.items():
        if k == "J0":
            st0[0] = state[0] + d
        else:
            setattr(c, k, getattr(cl, k) + d)
    st = oracle_mod.OracleState(c)
    for name, a in zip(("J", "H_r", "H_Z"), st0):
        getattr(st, name)[...] = a
        getattr(st, name + "_old")[...] = a
    st.setup_profiles()
    h = st.run(n)
    return h[-1, 0] + ss * float(np.dot(w, st.edge_spectra()[0].mean(0)))


@pytest.mark.parametrize("flux", [0, 1])
@pytest.mark.parametrize("field,h", [("alpha", 1e-4), ("alpha_c", 1e-4), ("T", 1e-4), ("J0", 1e-5)])
def test_dual_oracle_tangent_matches_central_differences(oracle_mod, flux, field, h):
    """The dual-number build of the oracle (forward-mode derivatives) against central
    differences of the plain oracle along the same direction, over 4 static steps: alpha,
    alpha_c, T (through H_voigt, phi_nu and alpha_F too) and the initial J. The step h is the
    one the difference resolves best: rounding in the stiff frequency solve dominates below it
    (1e-6 gives differences noisy at 1e-4 relative), the objective's kinks above it."""
    cl, state, seeds, w = _dual_problem(oracle_mod, flux)
    sd = {field: seeds[field]}
    ss, n = 1e12, 4
    st = oracle_mod.OracleState(cl)
    for name, a in zip(("J", "H_r", "H_Z"), state):
        getattr(st, name)[...] = a
        getattr(st, name + "_old")[...] = a
    st.setup_profiles()
    obj, tan, mf, dmf = oracle_mod.objective_tangent(st, n, 1.0, ss * w, sd)
    assert obj == pytest.approx(_plain_objective(oracle_mod, cl, state, n, w, ss, {}), rel=1e-13)
    fd = (_plain_objective(oracle_mod, cl, state, n, w, ss, {k: h * v for k, v in sd.items()}) -
          _plain_objective(oracle_mod, cl, state, n, w, ss, {k: -h * v for k, v in sd.items()})) / (2 * h)
    assert tan == pytest.approx(fd, rel=2e-6)
