"""The reduced-precision variants against the FP64 step on identical inputs.

LYD_PREC_MIXED keeps the state in FP64 and computes only the advection's reconstruction,
closure, fluxes and limiters in FP32 (the update is accumulated in FP64); LYD_PREC_FP32 also
stores the state in FP32. Errors are stated relative to each quantity's maximum (M_F and the
emergent edge-ring spectrum are the results the mixed form is specified on: <= 1e-5)."""
import numpy as np
import pytest

from helpers import CLOUDS, norm_err, random_state
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pair(cloud, precision, seed=7):
    from lydion_b200.m1 import context_for_cloud
    a = context_for_cloud(cloud)
    b = context_for_cloud(cloud, precision=precision)
    J, Hr, HZ = random_state(cloud, seed)
    for ctx in (a, b):
        for name, x in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            ctx.upload(name, x)
    return a, b


def _run(ctx, cl, n):
    return ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)


@pytest.mark.parametrize("name", ["glf_outflow", "hll_outflow", "glf_zout_48", "hll_point_64"])
def test_mixed_matches_fp64(name):
    from lydion_b200._lib import PREC_MIXED
    cl = CLOUDS[name]()
    a, b = _pair(cl, PREC_MIXED)
    n = 60
    ha, hb = _run(a, cl, n), _run(b, cl, n)
    assert float(np.max(np.abs(hb[:, 0] - ha[:, 0]))) <= 1e-5 * float(np.max(np.abs(ha[:, 0])))
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(b.download(f), a.download(f)) < 2e-5, f
    sa, sb = a.edge_spectra()[0].mean(0), b.edge_spectra()[0].mean(0)
    assert norm_err(sb, sa) < 1e-5


def test_fp32_storage_variant_is_close():
    from lydion_b200._lib import PREC_FP32
    cl = CLOUDS["glf_outflow"]()
    a, b = _pair(cl, PREC_FP32)
    n = 60
    ha, hb = _run(a, cl, n), _run(b, cl, n)
    assert float(np.max(np.abs(hb[:, 0] - ha[:, 0]))) <= 1e-4 * float(np.max(np.abs(ha[:, 0])))
    assert norm_err(b.download("J"), a.download("J")) < 1e-4


def test_mixed_batch_matches_fp64_batch():
    from lydion_b200._lib import PREC_MIXED
    from lydion_b200.m1 import batch_for_clouds, cloud_params
    clouds = W.batch_clouds(n_clouds=4, n_nu=24, sides=(7, 9, 12, 16), seed=3, x_max=100.0,
                            tau0_range=(1e4, 1e7), T_range=(3e2, 1e4))
    a = batch_for_clouds(clouds)
    b = batch_for_clouds(clouds, precision=PREC_MIXED)
    pp = cloud_params(clouds)
    ha, hb = a.batch_steps(40, pp), b.batch_steps(40, pp)
    for q in range(len(clouds)):
        assert float(np.max(np.abs(hb[:, q, 0] - ha[:, q, 0]))) <= 1e-5 * float(np.max(np.abs(ha[:, q, 0]))), q
        assert norm_err(b.download_cloud(q, "J"), a.download_cloud(q, "J")) < 2e-5, q


@pytest.mark.parametrize("prec_name,tol", [("PREC_MIXED", 1e-5), ("PREC_FP32", 1e-4)])
def test_reduced_precision_on_rhd_snapshot(prec_name, tol):
    """The synthetic RHD snapshot (photoionised bubble in neutral 100 K gas, 128 bins) carries
    fluxes whose squares fall below FP32's normal range in the far wings: the FP32 arithmetic
    must stay finite there and keep M_F within its tolerance of the FP64 step."""
    from lydion_b200 import _lib
    from lydion_b200.m1 import context_for_cloud
    cl = W.rhd_snapshot_cloud(n=128, n_nu=128)
    a = context_for_cloud(cl)
    b = context_for_cloud(cl, precision=getattr(_lib, prec_name))
    n = 200
    ha, hb = _run(a, cl, n), _run(b, cl, n)
    assert np.isfinite(hb).all()
    for f in ("J", "H_r", "H_Z"):
        assert np.isfinite(b.download(f)).all(), f
    assert float(np.max(np.abs(hb[:, 0] - ha[:, 0]))) <= tol * float(np.max(np.abs(ha[:, 0])))
