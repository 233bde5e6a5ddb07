"""The advection's two ways of staging rows into shared memory: per-lane loads, and bulk tensor
copies (TMA) of each row's 32-bin x 12-column box completed on an mbarrier, with the ghost cells
of the four boundaries patched as the rows are converted. Both feed the same arithmetic, so a
context run with either must give bit-for-bit the same state and diagnostics, on every boundary
rule, both fluxes, every precision form, batches and the Cartesian geometry; the bulk-copy run is
also held against the oracle."""
import numpy as np
import pytest

from helpers import CLOUDS, matched_pair, norm_err
from lydion_b200 import workloads as W
from lydion_b200._lib import PREC_FP32, PREC_FP64, PREC_MIXED, STAGING_LANES, STAGING_TMA

pytestmark = pytest.mark.gpu

FIELDS = ("J", "H_r", "H_Z")


def _pair(oracle_mod, cl, precision=PREC_FP64, seed=11):
    st, a = matched_pair(oracle_mod, cl, seed=seed, precision=precision)
    _, b = matched_pair(oracle_mod, cl, seed=seed, precision=precision)
    a.set_tuning(8, 0, 0, 0, STAGING_LANES)
    b.set_tuning(8, 0, 0, 0, STAGING_TMA)
    return st, a, b


def _row_bytes_ok(cl, precision):
    return (cl.n_nu * (4 if precision == PREC_FP32 else 8)) % 16 == 0


def _steps(ctx, cl, n):
    return ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)


CASES = [("glf_outflow", 1, 1), ("glf_outflow", 0, 0), ("hll_outflow", 1, 0), ("glf_zout_48", 1, 1),
         ("hll_point_64", 0, 1), ("glf_20bins", 1, 1)]


@pytest.mark.parametrize("name,bcr,bzt", CASES)
def test_bulk_copy_staging_equals_lane_loads(oracle_mod, name, bcr, bzt):
    cl = CLOUDS[name]()
    cl.bc_r_right, cl.bc_z_top = bcr, bzt
    st, a, b = _pair(oracle_mod, cl)
    assert a.tuning()[4] == STAGING_LANES
    assert b.tuning()[4] == (STAGING_TMA if _row_bytes_ok(cl, PREC_FP64) else STAGING_LANES)
    n = 12
    ha, hb = _steps(a, cl, n), _steps(b, cl, n)
    np.testing.assert_array_equal(ha, hb)
    for f in FIELDS:
        np.testing.assert_array_equal(a.download(f), b.download(f))
    d_o = st.run(n)
    np.testing.assert_array_equal(hb[:, 5:7], d_o[:, 5:7])
    for f in FIELDS:
        assert norm_err(b.download(f), getattr(st, f)) < 1e-9, f
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP32])
def test_bulk_copy_staging_reduced_precision(oracle_mod, precision):
    cl = W.small_cloud(nr=21, nz=19, n_nu=64, x_max=600.0, bc_z_bot=W.BC_OUTFLOW)
    _, a, b = _pair(oracle_mod, cl, precision=precision)
    assert b.tuning()[4] == STAGING_TMA
    _steps(a, cl, 15)
    _steps(b, cl, 15)
    for f in FIELDS:
        np.testing.assert_array_equal(a.download(f), b.download(f))
    a.close()
    b.close()


@pytest.mark.parametrize("bc_left", [W.BC_OUTFLOW, W.BC_REFLECT])
def test_bulk_copy_staging_cartesian(oracle_mod, bc_left):
    cl = W.cartesian_cloud(nx=19, ny=13, n_nu=32, bc_left=bc_left, flux_method=W.FLUX_HLL)
    st, a, b = _pair(oracle_mod, cl, seed=5)
    n = 10
    np.testing.assert_array_equal(_steps(a, cl, n), _steps(b, cl, n))
    for f in FIELDS:
        np.testing.assert_array_equal(a.download(f), b.download(f))
    st.run(n)
    assert norm_err(b.download("J"), st.J) < 1e-9
    a.close()
    b.close()


def test_bulk_copy_staging_tile_heights(oracle_mod):
    """Tiles of 4 rows (the copy of row j0 + 2 is the last one a tile issues) up to 64 rows
    (taller than the cloud), on a cloud whose height is not a multiple of the tile's."""
    cl = W.small_cloud(nr=26, nz=23, n_nu=48, x_max=200.0)
    _, a, _b = _pair(oracle_mod, cl)
    _b.close()
    _steps(a, cl, 6)
    ref = {f: a.download(f) for f in FIELDS}
    a.close()
    for rows in (4, 5, 16, 64):
        _, b = matched_pair(oracle_mod, cl, seed=11)
        b.set_tuning(rows, 0, 0, 0, STAGING_TMA)
        _steps(b, cl, 6)
        for f in FIELDS:
            np.testing.assert_array_equal(b.download(f), ref[f])
        b.close()


def test_bulk_copy_staging_batch(oracle_mod):
    from lydion_b200.m1 import batch_for_clouds, cloud_params
    clouds = W.batch_clouds(n_clouds=5, n_nu=32, sides=(9, 12, 17, 24), seed=9, x_max=100.0,
                            tau0_range=(1e4, 1e7), T_range=(3e2, 1e4))
    clouds[1].bc_z_top = W.BC_REFLECT
    clouds[2].bc_r_right = W.BC_REFLECT
    out = []
    for staging in (STAGING_LANES, STAGING_TMA):
        b = batch_for_clouds(clouds)
        b.set_tuning(8, 0, 0, 0, staging)
        assert b.tuning()[4] == staging
        h = b.batch_steps(8, cloud_params(clouds))
        out.append((h, [b.download_cloud(q, "J") for q in range(len(clouds))]))
        b.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    for x, y in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(x, y)


def test_bulk_copy_staging_headline_cloud(oracle_mod):
    """The 256 x 256 x 64 cloud: 20 fused steps with each staging, bit for bit."""
    cl = W.config_c2()
    _, a, b = _pair(oracle_mod, cl, seed=None)
    a.set_tuning(20, 0, 0, 3, STAGING_LANES)
    b.set_tuning(20, 0, 0, 3, STAGING_TMA)
    np.testing.assert_array_equal(_steps(a, cl, 20), _steps(b, cl, 20))
    for f in FIELDS:
        np.testing.assert_array_equal(a.download(f), b.download(f))
    a.close()
    b.close()


def test_unknown_staging_is_rejected(oracle_mod):
    from lydion_b200._lib import LYD_ERR_ARG, LydionError
    _, ctx = matched_pair(oracle_mod, CLOUDS["glf_outflow"]())
    with pytest.raises(LydionError) as e:
        ctx.set_tuning(16, 0, 0, 0, 7)
    assert e.value.code == LYD_ERR_ARG
    ctx.close()
