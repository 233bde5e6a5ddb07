"""The step on host state (lyd_static_step_host): J, H_r, H_Z up, one step, J, H_r, H_Z down,
pipelined over row chunks, with the active window of the previous step checked against that of
the uploaded J. Its results must be bit for bit those of the device-resident step
(lyd_static_steps) on the same state, whatever the chunking, and when the caller changed J in
between (the window check's redo) too."""
import numpy as np
import pytest

from helpers import random_state
from lydion_b200 import _lib
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pair(cl, precision=0, seed=5, rows=8):
    from lydion_b200.m1 import context_for_cloud
    J, Hr, HZ = random_state(cl, seed)
    ctxs = []
    for _ in range(2):
        ctx = context_for_cloud(cl, precision=precision)
        ctx.set_tuning(rows, 0, 0)
        for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            ctx.upload(name, a)
            ctx.upload(name + "_old", a)
        ctxs.append(ctx)
    return ctxs[0], ctxs[1], (J.copy(), Hr.copy(), HZ.copy())


def _params(cl):
    return (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)


@pytest.mark.parametrize("flux", [W.FLUX_GLF, W.FLUX_HLL])
@pytest.mark.parametrize("chunks", [1, 3, 8, 16])
def test_host_step_equals_device_step_bitwise(flux, chunks):
    cl = W.static_cloud(nr=24, nz=96, n_nu=32, tau0=1e6, T0=1e4, umax_kms=100.0, rs=0.5, tau_abs=0.5,
                        flux_method=flux)
    dev, host, (J, Hr, HZ) = _pair(cl)
    p = _params(cl)
    for step in range(4):
        rec_d = dev.static_steps(1, *p)[0]
        J, Hr, HZ, rec_h = host.static_step_host(J, Hr, HZ, *p, out=(J, Hr, HZ), chunks=chunks)   # in place
        np.testing.assert_array_equal(rec_h, rec_d, err_msg=f"step {step}")
        np.testing.assert_array_equal(J, dev.download("J"), err_msg=f"step {step}")
        np.testing.assert_array_equal(Hr, dev.download("H_r"))
        np.testing.assert_array_equal(HZ, dev.download("H_Z"))
    # the device state of the host-step context is the new state too
    np.testing.assert_array_equal(host.download("J"), J)
    dev.close()
    host.close()


@pytest.mark.parametrize("chunks", [2, 3, 6])
def test_host_step_ragged_last_tile_row_bitwise(chunks):
    """41 rows in tiles of 8: the last tile row holds one row, so the last chunk's upload (which
    starts two rows into it) is empty and the chunk before brings every remaining row."""
    cl = W.static_cloud(nr=20, nz=41, n_nu=32, tau0=1e6, T0=1e4, umax_kms=100.0, rs=0.5, tau_abs=0.5)
    dev, host, (J, Hr, HZ) = _pair(cl)
    p = _params(cl)
    for step in range(3):
        rec_d = dev.static_steps(1, *p)[0]
        J, Hr, HZ, rec_h = host.static_step_host(J, Hr, HZ, *p, out=(J, Hr, HZ), chunks=chunks)
        np.testing.assert_array_equal(rec_h, rec_d, err_msg=f"step {step}")
        np.testing.assert_array_equal(J, dev.download("J"), err_msg=f"step {step}")
        np.testing.assert_array_equal(Hr, dev.download("H_r"))
        np.testing.assert_array_equal(HZ, dev.download("H_Z"))
    dev.close()
    host.close()


@pytest.mark.parametrize("bc_left", [W.BC_REFLECT, W.BC_OUTFLOW])
def test_host_step_cartesian_bitwise(bc_left):
    """A Cartesian grid (the first X interface reflecting or letting flow out), 6 chunks."""
    cl = W.cartesian_cloud(nx=24, ny=64, n_nu=32, bc_left=bc_left)
    dev, host, (J, Hr, HZ) = _pair(cl, seed=13)
    p = _params(cl)
    for _ in range(3):
        rec_d = dev.static_steps(1, *p)[0]
        J, Hr, HZ, rec_h = host.static_step_host(J, Hr, HZ, *p, out=(J, Hr, HZ), chunks=6)
        np.testing.assert_array_equal(rec_h, rec_d)
        np.testing.assert_array_equal(J, dev.download("J"))
        np.testing.assert_array_equal(Hr, dev.download("H_r"))
    dev.close()
    host.close()


def test_host_step_full_size_separate_outputs():
    """The 256 x 256 x 64 cloud, separate output arrays (the inputs stay as they were)."""
    cl = W.config_c2()
    dev, host, (J, Hr, HZ) = _pair(cl, 0, rows=20)
    p = _params(cl)
    J0 = J.copy()
    rec_d = dev.static_steps(1, *p)[0]
    Jn, Hrn, HZn, rec_h = host.static_step_host(J, Hr, HZ, *p, chunks=8)
    np.testing.assert_array_equal(J, J0)
    np.testing.assert_array_equal(rec_h, rec_d)
    np.testing.assert_array_equal(Jn, dev.download("J"))
    np.testing.assert_array_equal(HZn, dev.download("H_Z"))
    rec_d = dev.static_steps(1, *p)[0]
    Jn, Hrn, HZn, rec_h = host.static_step_host(Jn, Hrn, HZn, *p, out=(J, Hr, HZ), chunks=8)
    np.testing.assert_array_equal(rec_h, rec_d)
    np.testing.assert_array_equal(Jn, dev.download("J"))
    dev.close()
    host.close()


def test_changed_state_takes_its_own_window():
    """The caller changes J between steps so that its window differs from the one the previous
    step decided: the step must use the uploaded J's window (the check's redo), as the device
    step does on the same uploaded state."""
    cl = W.static_cloud(nr=24, nz=96, n_nu=32, tau0=1e6, T0=1e4, umax_kms=100.0, rs=0.5, tau_abs=0.5)
    dev, host, (J, Hr, HZ) = _pair(cl, 0, seed=9)
    p = _params(cl)
    for _ in range(2):
        dev.static_steps(1, *p)
        J, Hr, HZ, _ = host.static_step_host(J, Hr, HZ, *p, out=(J, Hr, HZ), chunks=4)
    kmin0, kmax0 = dev.find_active_bins()
    # empty the outer wings (every bin is active in this state): the window must shrink
    for a in (J, Hr, HZ):
        a[..., :6] = 0.0
        a[..., -6:] = 0.0
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
        dev.upload(name, a)
        dev.upload(name + "_old", a)
    rec_d = dev.static_steps(1, *p)[0]
    assert rec_d[5] > kmin0 and rec_d[6] < kmax0, (rec_d[5:], kmin0, kmax0)
    J, Hr, HZ, rec_h = host.static_step_host(J, Hr, HZ, *p, out=(J, Hr, HZ), chunks=4)
    np.testing.assert_array_equal(rec_h, rec_d)
    np.testing.assert_array_equal(J, dev.download("J"))
    np.testing.assert_array_equal(Hr, dev.download("H_r"))
    dev.close()
    host.close()


def test_host_step_rejects_what_it_does_not_cover():
    from lydion_b200.m1 import batch_for_clouds, context_for_cloud
    cl = W.small_cloud(nr=12, nz=10, n_nu=16)
    J, Hr, HZ = random_state(cl, 3)
    p = _params(cl)
    for prec in (_lib.PREC_MIXED, _lib.PREC_FP32):
        ctx = context_for_cloud(cl, precision=prec)
        with pytest.raises(_lib.LydionError):
            ctx.static_step_host(J, Hr, HZ, *p)
        ctx.close()
    ctx = context_for_cloud(cl)
    for bad in (0, 17):
        with pytest.raises(_lib.LydionError):
            ctx.static_step_host(J, Hr, HZ, *p, chunks=bad)
    ctx.close()
    b = batch_for_clouds([cl, W.small_cloud(nr=12, nz=10, n_nu=16)])
    with pytest.raises(_lib.LydionError):
        b.static_step_host(J, Hr, HZ, *p)
    b.close()
