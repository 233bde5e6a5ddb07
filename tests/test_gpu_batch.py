"""GPU parity of the batched step: many ragged clouds in one context, each with its own time
step and boundaries, against the FP64 oracle run cloud by cloud, and against independent
single-cloud contexts (bitwise, at equal work-list shapes)."""
import numpy as np
import pytest

from helpers import max_rel, norm_err, random_state
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu

N_NU = 24


def _clouds():
    cl = W.batch_clouds(n_clouds=6, n_nu=N_NU, sides=(7, 9, 12, 16, 21), seed=5, x_max=100.0,
                        tau0_range=(1e4, 1e7), T_range=(3e2, 1e4))
    cl[1].bc_z_bot = W.BC_OUTFLOW
    cl[2].bc_r_right = W.BC_REFLECT
    cl[4].bc_z_top = W.BC_REFLECT
    return cl


def _batch(oracle_mod, clouds, seed=3, tuning=None):
    """A batch context and one oracle state per cloud on identical inputs (the oracle's
    H_voigt and phi_nu are uploaded into the batch)."""
    from lydion_b200.m1 import batch_for_clouds
    b = batch_for_clouds(clouds)
    if tuning:
        b.set_tuning(*tuning)
    states = []
    for q, c in enumerate(clouds):
        st = oracle_mod.OracleState(c)
        st.setup_profiles()
        b.upload_cloud(q, "Hvoigt", st.Hvoigt)
        b.upload_cloud(q, "phi_nu", st.phi_nu)
        J, Hr, HZ = random_state(c, seed + q)
        for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            getattr(st, name)[...] = a
            getattr(st, name + "_old")[...] = a
            b.upload_cloud(q, name, a)
            b.upload_cloud(q, name + "_old", a)
        states.append(st)
    return b, states


def test_batch_steps_match_oracle_per_cloud(oracle_mod):
    from lydion_b200.m1 import cloud_params
    clouds = _clouds()
    b, states = _batch(oracle_mod, clouds)
    assert b.cell_bins == sum(c.cell_bins for c in clouds)
    n = 25
    hist = b.batch_steps(n, cloud_params(clouds))
    assert hist.shape == (n, len(clouds), 7)
    for q, (c, st) in enumerate(zip(clouds, states)):
        d_o = st.run(n)
        d_g = hist[:, q, :]
        np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
        np.testing.assert_allclose(d_g[:, 3], d_o[:, 3], rtol=1e-13)
        for col in (0, 1, 2):
            assert max_rel(d_g[5:, col], d_o[5:, col], floor=1e-9 * np.abs(d_o[:, col]).max()) < 1e-9, (q, col)
        for f in ("J", "H_r", "H_Z"):
            assert norm_err(b.download_cloud(q, f), getattr(st, f)) < 1e-9, (q, f)
        raw, norm, ri, zi = b.edge_spectra(q)
        o_raw, o_norm, o_ri, o_zi = st.edge_spectra()
        np.testing.assert_array_equal(ri, o_ri)
        np.testing.assert_array_equal(zi, o_zi)
        assert norm_err(raw, o_raw) < 1e-9


def test_batch_equals_independent_contexts_bitwise(oracle_mod):
    """With the same cells per block, a cloud advances identically inside a batch and alone."""
    from lydion_b200.m1 import cloud_params, context_for_cloud
    clouds = _clouds()
    b, states = _batch(oracle_mod, clouds, seed=9, tuning=(8, 16, 0))
    n = 6
    hist = b.batch_steps(n, cloud_params(clouds))
    for q, (c, st) in enumerate(zip(clouds, states)):
        ctx = context_for_cloud(c, hvoigt=st.Hvoigt, phi_nu=st.phi_nu)
        ctx.set_tuning(8, 16, 0)
        for name in ("J", "H_r", "H_Z"):
            ctx.upload(name, getattr(st, name))
            ctx.upload(name + "_old", getattr(st, name))
        d = ctx.static_steps(n, c.c_tilde, c.dt, c.z_center, c.bc_r_right, c.bc_z_bot, c.bc_z_top)
        np.testing.assert_array_equal(d, hist[:, q, :])
        for f in ("J", "H_r", "H_Z"):
            np.testing.assert_array_equal(ctx.download(f), b.download_cloud(q, f))
        ctx.close()


@pytest.mark.parametrize("tuning", [(4, 8, 0), (64, 1024, 0), (16, 0, 1), (32, 24, 1)])
def test_tuning_variants(oracle_mod, tuning):
    """Tile rows and cells per block change only the work split: J, H are bitwise equal to the
    default shape; the lane-serial solver agrees with the oracle to the PCR tolerance."""
    from lydion_b200.m1 import cloud_params
    clouds = _clouds()
    ref, states = _batch(oracle_mod, clouds, seed=4)
    b, _ = _batch(oracle_mod, clouds, seed=4, tuning=tuning)
    assert b.tuning()[0] == tuning[0]
    n = 8
    h_ref = ref.batch_steps(n, cloud_params(clouds))
    h_b = b.batch_steps(n, cloud_params(clouds))
    np.testing.assert_array_equal(h_b[:, :, 5:7], h_ref[:, :, 5:7])
    for q, st in enumerate(states):
        st.run(n)
        for f in ("J", "H_r", "H_Z"):
            got = b.download_cloud(q, f)
            if tuning[2] == 0:
                np.testing.assert_array_equal(got, ref.download_cloud(q, f))
            assert norm_err(got, getattr(st, f)) < 1e-9, (q, f)


def test_batch_phase_calls_and_window_per_cloud(oracle_mod):
    """The per-phase entry points on a batch apply to every cloud; FindActiveBins reports one
    window per cloud."""
    clouds = _clouds()
    b, states = _batch(oracle_mod, clouds, seed=12)
    c0 = clouds[0]
    ctdt = c0.c_tilde * c0.dt
    kmin, kmax = b.find_active_bins()
    for q, st in enumerate(states):
        k_o = st.find_active_bins()
        assert (kmin[q], kmax[q]) == k_o
    for st, c in zip(states, clouds):
        c.bc_r_right, c.bc_z_bot, c.bc_z_top = W.BC_OUTFLOW, W.BC_REFLECT, W.BC_OUTFLOW
    b.advect(ctdt, W.BC_OUTFLOW, W.BC_REFLECT, W.BC_OUTFLOW)
    b.frequency_update(ctdt)
    for q, (st, c) in enumerate(zip(states, clouds)):
        st.advect(ctdt)
        st.frequency_update(ctdt)
        assert norm_err(b.download_cloud(q, "J"), st.J) < 1e-9, q


def test_batch_rejects_single_cloud_calls():
    from lydion_b200._lib import LydionError
    from lydion_b200.m1 import batch_for_clouds
    clouds = _clouds()[:2]
    b = batch_for_clouds(clouds)
    with pytest.raises(LydionError):
        b.f_esc(1.0)
    with pytest.raises(LydionError):
        b.force_multiplier(1.0, 0.0)
    with pytest.raises(LydionError):
        b.set_tuning(2, 0, 0)
    with pytest.raises(LydionError):
        b.set_tuning(16, 0, 7)


def test_autotune_applies_a_valid_shape(tmp_path):
    from lydion_b200 import autotune as A
    from lydion_b200.m1 import batch_for_clouds, cloud_params
    clouds = _clouds()
    b = batch_for_clouds(clouds)
    pp = cloud_params(clouds)
    t = A.autotune(b, lambda n: b.batch_steps(n, pp, history=False), steps=2, cache=str(tmp_path / "t.json"),
                   rows=(4, 16), cells=(0, 32), solvers=(0, 1))
    got = b.tuning()
    assert got[0] == t[0] and got[2] == t[2] and got[3] == (t[3] if t[3] else 3)
    assert t[1] == 0 and got[1] < 0 or got[1] == t[1]
    h = b.batch_steps(2, pp)
    assert np.isfinite(h).all()


def test_ragged_batch_distribution_matches_oracle(oracle_mod):
    """The first 32 clouds of the 512-cloud ragged batch (its own generator and seed: sides
    32..256 drawn independently in r and Z, tau0 1e4..1e8, T 1e2..1e4 K, dust, outflows up to
    100 km/s; 48 bins; 20.3M cell-bins), 20 steps in one batch context, against the oracle
    cloud by cloud: windows exact, L to 1e-13, the force multipliers floored to 1e-9, J and H
    to 1e-9 of their maxima. The net radial multiplier is a signed sum that crosses zero in
    some clouds (cloud 20: from -1.8e-3 to +1.5e-3 between two steps, against outward and
    inward parts of 1.3 each), so it is held to 1e-9 of the same step's M_F, the sum of the
    magnitudes of its terms."""
    from lydion_b200.m1 import cloud_params
    clouds = W.batch_clouds(n_clouds=32)
    b, states = _batch(oracle_mod, clouds, seed=17)
    n = 20
    hist = b.batch_steps(n, cloud_params(clouds))
    for q, (c, st) in enumerate(zip(clouds, states)):
        d_o = st.run(n)
        d_g = hist[:, q, :]
        np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7], err_msg=str(q))
        np.testing.assert_allclose(d_g[:, 3], d_o[:, 3], rtol=1e-13, err_msg=str(q))
        for col in (0, 2):
            assert max_rel(d_g[5:, col], d_o[5:, col], floor=1e-9 * np.abs(d_o[:, col]).max()) < 1e-9, (q, col)
        assert np.all(np.abs(d_g[:, 1] - d_o[:, 1]) <= 1e-9 * d_o[:, 0]), (q, d_g[:, 1] - d_o[:, 1])
        for f in ("J", "H_r", "H_Z"):
            assert norm_err(b.download_cloud(q, f), getattr(st, f)) < 1e-9, (q, f)
    b.close()
