"""One field split into Z slabs (lyd_dd_*), its ranks emulated in one process on one GPU
(LocalComm: the same all-reduce and halo exchange, done with device copies), against the
undecomposed field: the same active window every step, the same owned J and H bit for bit, and
the diagnostics to the rounding of a different summation order."""
import numpy as np
import pytest

from helpers import random_state
from lydion_b200 import domain as D
from lydion_b200 import workloads as W
from lydion_b200._lib import PREC_FP32, PREC_FP64, PREC_MIXED

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_ranks,precision,bzb", [(2, PREC_FP64, W.BC_REFLECT), (3, PREC_FP64, W.BC_OUTFLOW),
                                                   (4, PREC_MIXED, W.BC_REFLECT), (3, PREC_FP32, W.BC_REFLECT)])
def test_slabs_match_the_whole_field(n_ranks, precision, bzb):
    from lydion_b200.m1 import context_for_cloud
    cl = W.small_cloud(nr=12, nz=15, n_nu=16, bc_z_bot=bzb)
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    J, Hr, HZ = random_state(cl, 4)
    whole = context_for_cloud(cl, precision=precision)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
        whole.upload(name, a)
        whole.upload(name + "_old", a)
    n = 25
    h = whole.static_steps(n, *p)
    ranks = [D.SlabRank(cl, n_ranks, r, precision=precision) for r in range(n_ranks)]
    for r in ranks:
        r.upload_state(J, Hr, HZ)
    recs = D.SlabDriver(ranks, D.LocalComm()).run(n, *p)
    np.testing.assert_array_equal(recs[:, 5:7], h[:, 5:7])                  # windows
    np.testing.assert_allclose(recs[:, 3], h[:, 3], rtol=1e-13)             # L
    for col in (0, 1, 2, 4):
        np.testing.assert_allclose(recs[:, col], h[:, col], rtol=1e-12, atol=1e-14 * np.abs(h[:, col]).max())
    for f in ("J", "H_r", "H_Z"):
        got = np.concatenate([r.owned(f) for r in ranks], axis=0)
        np.testing.assert_array_equal(got, whole.download(f), err_msg=f)
    whole.close()
    for r in ranks:
        r.ctx.close()


def test_slab_partition():
    assert D.slab_partition(15, 4) == [(0, 4), (4, 8), (8, 12), (12, 15)]
    assert D.slab_layout(15, 4, 0) == (0, 4, 0, 2)
    assert D.slab_layout(15, 4, 3) == (12, 15, 2, 0)
    with pytest.raises(ValueError):
        D.slab_partition(7, 4)
