"""Save points on the device: a run restarted from its Lyman-alpha checkpoint continues
bit for bit, and the static-run record holds the step records and edge-ring spectra of the
save points with the reference's dataset names and shapes."""
import numpy as np
import pytest

from helpers import matched_pair
from lydion_b200 import snapshots as S
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_checkpoint_restart_continues_bit_for_bit(oracle_mod, tmp_path):
    cl = W.small_cloud()
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    _, a = matched_pair(oracle_mod, cl, seed=3)
    a.static_steps(10, *p, history=False)
    path = tmp_path / "ck.npz"
    S.save_checkpoint(a, path, t_current=10 * cl.dt, dt=cl.dt, step=10)
    ha = a.static_steps(10, *p)
    _, b = matched_pair(oracle_mod, cl)            # the same inputs (H_voigt, phi_nu) as `a`
    t, dt, step = S.load_checkpoint(b, path)
    assert (t, dt, step) == (10 * cl.dt, cl.dt, 10)
    hb = b.static_steps(10, *p)
    np.testing.assert_array_equal(hb, ha)
    for f in ("J", "H_r", "H_Z"):
        np.testing.assert_array_equal(b.download(f), a.download(f))
    a.close(); b.close()


def test_static_run_record(oracle_mod, tmp_path):
    cl = W.small_cloud()
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    _, ctx = matched_pair(oracle_mod, cl, seed=3)
    rec = S.StaticRunRecord(cl, 3)
    for s in range(3):
        h = ctx.static_steps(5, *p)
        rec.save(ctx, s, (s + 1) * 5 * cl.dt, h[-1])
    rec.write(tmp_path / "run.npz")
    f = np.load(tmp_path / "run.npz")
    raw, norm, ri, zi = ctx.edge_spectra()
    n_edge = (cl.nz - 2) + 2 * (cl.nr - 3)
    assert f["J_Lya_EdgeSpectra"].shape == (3, cl.n_nu, n_edge)
    np.testing.assert_array_equal(f["J_Lya_EdgeSpectra"][2], raw.T)
    np.testing.assert_array_equal(f["J_Lya_EdgeSpectra_Norm"][2], norm.T)
    np.testing.assert_array_equal(f["J_Lya_Edge_rIndex"], ri + 1)
    assert f["M_F_History"][2] == h[-1, 0] and f["f_esc_Lya_History"][2] == h[-1, 4]
    np.testing.assert_allclose(f["Times"], [5 * cl.dt, 10 * cl.dt, 15 * cl.dt])
    ctx.close()
