"""The persistent step (lyd_batch_steps_persistent): each step as one cooperative launch whose
CTAs walk the advection tiles, the frequency-kernel cells and the reduction blocks with bounded
grid barriers between the phases. Same work items and summation orders as the three-launch
step, so the results must be bit-for-bit those of lyd_batch_steps; a barrier that runs out of
polls reports LYD_ERR_TIMEOUT and leaves the context usable."""
import numpy as np
import pytest

from helpers import random_state
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _clouds(n_nu):
    cl = W.batch_clouds(n_clouds=5, n_nu=n_nu, sides=(7, 9, 12, 16, 21), seed=11, x_max=100.0,
                        tau0_range=(1e4, 1e7), T_range=(3e2, 1e4))
    cl[1].bc_z_bot = W.BC_OUTFLOW
    cl[3].bc_r_right = W.BC_REFLECT
    return cl


def _batch(clouds, precision, seed=7, tuning=None):
    from lydion_b200.m1 import batch_for_clouds
    b = batch_for_clouds(clouds, precision=precision)
    if tuning:
        b.set_tuning(*tuning)
    for q, c in enumerate(clouds):
        J, Hr, HZ = random_state(c, seed + q)
        for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            b.upload_cloud(q, name, a)
            b.upload_cloud(q, name + "_old", a)
    return b


def _same(b1, b2, n_clouds):
    for q in range(n_clouds):
        for f in ("J", "H_r", "H_Z"):
            np.testing.assert_array_equal(b1.download_cloud(q, f), b2.download_cloud(q, f), err_msg=f"{q} {f}")


@pytest.mark.parametrize("n_nu", [24, 64, 128, 256])
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_persistent_equals_three_launch_step_bitwise(n_nu, precision):
    from lydion_b200.m1 import cloud_params
    clouds = _clouds(n_nu)
    ref = _batch(clouds, precision)
    per = _batch(clouds, precision)
    n = 6
    h_ref = ref.batch_steps(n, cloud_params(clouds))
    h_per = per.batch_steps(n, cloud_params(clouds), persistent=True)
    np.testing.assert_array_equal(h_per, h_ref)
    _same(ref, per, len(clouds))
    assert per.persistent_graph() in (1, -1)
    # later calls continue from the same state as the three-launch path's
    h_ref = ref.batch_steps(3, cloud_params(clouds))
    h_per = per.batch_steps(3, cloud_params(clouds), persistent=True)
    np.testing.assert_array_equal(h_per, h_ref)
    _same(ref, per, len(clouds))
    ref.close()
    per.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_persistent_hll_flux_bitwise(precision):
    """The HLL flux (wave speeds from the closure's eigenvalues) through the persistent step."""
    from lydion_b200.m1 import cloud_params
    clouds = _clouds(64)
    for c in clouds:
        c.flux_method = W.FLUX_HLL
    ref = _batch(clouds, precision, seed=23)
    per = _batch(clouds, precision, seed=23)
    h_ref = ref.batch_steps(5, cloud_params(clouds))
    h_per = per.batch_steps(5, cloud_params(clouds), persistent=True)
    np.testing.assert_array_equal(h_per, h_ref)
    _same(ref, per, len(clouds))
    ref.close()
    per.close()


def test_persistent_more_work_than_ctas():
    """A 128 x 160 cloud cut into 4-row tiles and 8-cell blocks: more tiles, items and
    reduction blocks than resident CTAs, so every CTA loops over several of each."""
    from lydion_b200.m1 import cloud_params
    clouds = [W.static_cloud(nr=128, nz=160, n_nu=64, tau0=1e6, T0=1e4, umax_kms=100.0, rs=0.5, x_max=100.0)] + _clouds(64)[:2]
    ref = _batch(clouds, 0, tuning=(4, 8, 0))
    per = _batch(clouds, 0, tuning=(4, 8, 0))
    n = 4
    h_ref = ref.batch_steps(n, cloud_params(clouds))
    h_per = per.batch_steps(n, cloud_params(clouds), persistent=True)
    np.testing.assert_array_equal(h_per, h_ref)
    _same(ref, per, len(clouds))
    # the timed form (events around each launch) runs the same launches
    per.set_timing(True)
    ref.batch_steps(2, cloud_params(clouds))
    h_per = per.batch_steps(2, cloud_params(clouds), persistent=True)
    per.set_timing(False)
    _same(ref, per, len(clouds))
    ref.close()
    per.close()


def test_barrier_that_runs_out_reports_timeout_and_context_stays_usable():
    from lydion_b200 import _lib
    from lydion_b200.m1 import cloud_params
    clouds = _clouds(32)
    b = _batch(clouds, 0)
    with pytest.raises(_lib.LydionError) as e:
        # one poll: every CTA that has to wait at a barrier gives up
        b.batch_steps(2, cloud_params(clouds), persistent=True, barrier_polls=1)
    assert e.value.code == _lib.LYD_ERR_TIMEOUT
    # the counters of the reduction are reset: fresh state, then both paths agree again
    for q, c in enumerate(clouds):
        J, Hr, HZ = random_state(c, 7 + q)
        for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            b.upload_cloud(q, name, a)
            b.upload_cloud(q, name + "_old", a)
    ref = _batch(clouds, 0)
    h_ref = ref.batch_steps(3, cloud_params(clouds))
    h_b = b.batch_steps(3, cloud_params(clouds), persistent=True)
    np.testing.assert_array_equal(h_b, h_ref)
    _same(ref, b, len(clouds))
    # and the three-launch path on the same context too
    np.testing.assert_array_equal(b.batch_steps(1, cloud_params(clouds)), ref.batch_steps(1, cloud_params(clouds)))
    with pytest.raises(_lib.LydionError):
        b.batch_steps(1, cloud_params(clouds), persistent=True, barrier_polls=0)
    ref.close()
    b.close()
