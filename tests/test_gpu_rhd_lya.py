"""The RHD-side Lyman-alpha block on the device (lyd_rhd_lya_prepare, lyd_rhd_lya_absorb)
against the oracle's restatement of PrepareLyaSubCycling! and the Lyman-alpha part of
AbsorptionStep (src/PhotoChemistryAndCooling/PhotoThermoChemistry.jl:2087-2155, 1580-1680), on
a seeded cloud with random gas and dust states, per-cell sub-steps that make some cells reject,
and two committed sub-steps in a row."""
import numpy as np
import pytest

from helpers import random_state
from lydion_b200 import workloads as W
from lydion_b200._lib import PREC_FP32, PREC_FP64, PREC_MIXED

pytestmark = pytest.mark.gpu

KAPPA_ABS, KAPPA_F, RHO_IGNORE = W.DUST_KAPPA_ABS, W.DUST_KAPPA_F, W.DUST_RHO_IGNORE
C_TILDE = 3e8


def matched(precision, seed, oracle_hvoigt=False):
    from oracle import oracle as O
    from lydion_b200.m1 import context_for_cloud
    cl = W.small_cloud(nr=10, nz=9, n_nu=24)
    sp, rho_d = W.rhd_gas_state(cl, seed)
    st = O.OracleState(cl)
    ctx = context_for_cloud(cl, precision=precision)
    acF, dF = O.rhd_lya_prepare(st, sp, rho_d, KAPPA_ABS, KAPPA_F, RHO_IGNORE, z=0.5)
    ctx.rhd_lya_prepare(sp["T"], sp["nHI"], sp["nH2"], sp["nHII"], sp["nHeI"], sp["ne"], sp["nOHx"], sp["nCHx"],
                        rho_d, KAPPA_ABS, KAPPA_F, RHO_IGNORE, z=0.5)
    if oracle_hvoigt:
        # the same H_voigt on both sides (the device's Voigt tables agree with the oracle's to
        # ~1e-11 on narrow bins, checked in test_prepare_matches_oracle), phi_nu over all bins
        ctx.upload("Hvoigt", st.Hvoigt)
        ctx.update_phi_nu(0, cl.n_nu - 1)
    J, Hr, HZ = random_state(cl, seed + 1, amp=1e-14)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
        getattr(st, name)[...] = a
        getattr(st, name + "_old")[...] = a
        ctx.upload(name, a)
        ctx.upload(name + "_old", a)
    # e_Lya of the previous accepted sub-step: the current 4 pi / c int J, perturbed
    e0 = 4 * np.pi / 2.99792458e10 * np.einsum("jik,k->ji", J, cl.freq.dnu)
    e0 = e0 * np.random.default_rng(seed + 2).uniform(0.5, 1.5, size=e0.shape)
    ctx.upload("e_Lya", e0)
    return cl, st, ctx, acF, dF, e0.copy()


def rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_prepare_matches_oracle(precision):
    cl, st, ctx, acF, dF, _ = matched(precision, 11)
    for name, ref in (("alpha", st.alpha), ("alpha_c", st.alpha_c), ("pd", st.pd), ("js", st.js), ("T", st.T),
                      ("alpha_cF", acF)):
        got = ctx.download(name)
        assert rel(got, ref) <= 1e-12, (name, rel(got, ref))
    # the Voigt look-up tables: the tolerance of the other H_voigt parity tests
    assert rel(ctx.download("Hvoigt"), st.Hvoigt) <= 1e-9
    # some dust was ignored and some cells carry a destruction probability and both emissivities
    assert np.any(dF[0] == 0.0) and np.any(st.pd > 0.0) and np.all(st.js > 0.0)
    ctx.close()


@pytest.mark.parametrize("precision,tol", [(PREC_FP64, 1e-12), (PREC_MIXED, 1e-12), (PREC_FP32, 2e-6)])
def test_absorb_two_committed_substeps(precision, tol):
    from oracle import oracle as O
    cl, st, ctx, acF, dF, e_or = matched(precision, 23, oracle_hvoigt=True)
    rng = np.random.default_rng(5)
    for call in range(2):
        # sub-steps spanning 1e-3 .. 1e3 absorption times: long ones reject
        dt_lya = 1.0 / (C_TILDE * (st.alpha_c + st.pd * st.alpha))
        dt = dt_lya * 10.0 ** rng.uniform(-3.0, 3.0, size=dt_lya.shape)
        ref = O.rhd_lya_absorb(st, acF, dF, dt, C_TILDE, e_or, commit=True)
        got = ctx.rhd_lya_absorb(dt, C_TILDE, commit=True)
        assert ref["reject"].any() and not ref["reject"].all(), call
        np.testing.assert_array_equal(got["reject"], ref["reject"])
        for k in ("e_new", "dt_lya"):
            assert rel(got[k], ref[k]) <= tol, (call, k, rel(got[k], ref[k]))
        # de is a relative change of e_Lya, resolved to the rounding of J and e (FP32 storage:
        # ~1e-7 of J)
        np.testing.assert_allclose(got["de"], ref["de"], rtol=tol, atol=1e-5 if precision == PREC_FP32 else 1e-12)
        scale = np.abs(ref["split"]).max()
        for k in ("dru_r", "dru_Z"):
            np.testing.assert_allclose(got[k], ref[k], rtol=tol, atol=tol * np.abs(ref[k]).max())
        np.testing.assert_allclose(got["split"], ref["split"], rtol=tol, atol=tol * scale)
        # the split adds up to the total
        np.testing.assert_allclose(got["split"][0::2].sum(0), got["dru_r"], rtol=1e-9, atol=1e-12 * scale)
        for name in ("J", "H_r", "H_Z", "J_old", "H_r_old", "H_Z_old"):
            a, b = ctx.download(name), getattr(st, name)
            np.testing.assert_allclose(a, b, rtol=tol, atol=tol * np.abs(b).max(), err_msg=f"{call} {name}")
        np.testing.assert_allclose(ctx.download("e_Lya"), e_or, rtol=tol, atol=0.0)
    ctx.close()


def test_absorb_needs_prepare():
    from lydion_b200._lib import LydionError
    from lydion_b200.m1 import context_for_cloud
    cl = W.small_cloud(nr=10, nz=9, n_nu=24)
    ctx = context_for_cloud(cl)
    with pytest.raises(LydionError):
        ctx.rhd_lya_absorb(np.full((cl.nz, cl.nr), 1e3), C_TILDE)
    ctx.close()


# (previous c~, c~_min): the cell maximum (~5.3e8 cm/s here) unclamped, capped at 4x the previous
# value, floored at 0.75x, and raised to c~_min
@pytest.mark.parametrize("ct_old,ct_min", [(3e8, 1e7), (1e7, 1e7), (3e9, 1e7), (1e9, 1e9)])
def test_find_rsl_matches_oracle(ct_old, ct_min):
    """FindRSL_LyaRT on the device against the oracle, on the seeded gas state with random flows
    and pressures, through each of its clamps."""
    from oracle import oracle as O
    cl, st, ctx, acF, dF, _ = matched(PREC_FP64, 31)
    rng = np.random.default_rng(9)
    shape = (cl.nz, cl.nr)
    sp, rho_d = W.rhd_gas_state(cl, 31)
    from lydion_b200 import constants as K
    nH = sp["nHI"] + sp["nHII"]
    hydro = {"u_r": 1e6 * rng.normal(size=shape), "u_Z": 1e6 * rng.normal(size=shape),
             "rho": nH * K.mH / K.X_H, "gamma_ad": np.full(shape, 5.0 / 3.0), "T": sp["T"],
             "xHII": sp["nHII"] / nH, "xH2": 0.5 * sp["nH2"] / nH}
    hydro["P"] = 2.0 * nH * K.kB * sp["T"] * rng.uniform(0.5, 2.0, size=shape)
    ref = O.find_rsl_lya(cl.geom, hydro, rho_d, st.pd, KAPPA_ABS, 4.0, K.X_H / K.mH, ct_old, ct_min)
    got = ctx.find_rsl_lya(ct_old, ct_min, hydro["u_r"], hydro["u_Z"], hydro["P"], hydro["rho"], hydro["gamma_ad"],
                           hydro["T"], hydro["xHII"], hydro["xH2"], rho_d, KAPPA_ABS)
    assert abs(got - ref) <= 1e-13 * ref, (got, ref)
    ctx.close()
