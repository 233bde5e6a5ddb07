"""Host-side pieces of the adjoint workflow (no GPU): the 64-point spectrum resampling, the
turbulent-cloud generator and the chain rules from the library's gradients to n_H, T, dust
and a per-cell velocity scale."""
import numpy as np

from lydion_b200 import adjoint as A
from lydion_b200 import constants as K
from lydion_b200 import workloads as W


def test_resampling_is_linear_interpolation():
    cl = W.small_cloud(nr=6, nz=5, n_nu=16)
    M, xs = A.spectrum_resampling(cl.freq, 64)
    xb = A.x_of_bins(cl.freq)
    s = np.sin(0.01 * xb) + 2.0
    np.testing.assert_allclose(M @ s, np.interp(xs, xb, s), rtol=1e-13)
    np.testing.assert_allclose(M.sum(1), 1.0, rtol=1e-14)


def test_gaussian_random_field_statistics():
    g = W.gaussian_random_field(128, 128, seed=3)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.0) < 1e-12
    # the spectrum falls as k^-11/3: a radially averaged power-law fit
    P = np.abs(np.fft.rfft2(g)) ** 2
    kz = np.fft.fftfreq(128)[:, None]
    kr = np.fft.rfftfreq(128)[None, :]
    k = np.hypot(kz, kr)
    m = (k > 0.02) & (k < 0.3)
    slope = np.polyfit(np.log(k[m]), np.log(P[m]), 1)[0]
    assert abs(slope - (-11.0 / 3.0)) < 0.3


def test_turbulent_cloud_fields():
    c = W.turbulent_cloud(nr=32, nz=32, n_nu=16, seed=11)
    inside = c.alpha > 0
    sigma0 = K.compute_sigma0(1e4)
    np.testing.assert_allclose(c.alpha[inside], c.n_H[inside] * sigma0, rtol=1e-14)
    np.testing.assert_allclose(c.alpha_c[inside], c.kappa_d * 0.01 * c.n_H[inside] * K.mH, rtol=1e-14)
    # kappa_d gives dust optical depth 1 across R_cl at the mean density
    assert abs(c.kappa_d * 0.01 * 100.0 * K.mH * K.pc - 1.0) < 1e-12


def test_chain_rules_match_their_definitions():
    c = W.turbulent_cloud(nr=12, nz=10, n_nu=16, seed=2)
    rng = np.random.default_rng(0)
    g = {k: rng.standard_normal((c.nz, c.nr)) for k in ("grad_alpha", "grad_alpha_c", "grad_T")}
    for f in A.VEL_FIELDS:
        g["grad_" + f] = rng.standard_normal((c.nz, c.nr))
    g["grad_u_r_star"] = rng.standard_normal((c.nz, c.nr + 1))
    g["grad_u_Z_star"] = rng.standard_normal((c.nz + 1, c.nr))
    out = A.physical_gradients(c, g)
    j, i = 4, 3
    # directional check: O linear in the inputs with the given gradients
    def O(cl):
        s = np.sum(g["grad_alpha"] * cl.alpha) + np.sum(g["grad_alpha_c"] * cl.alpha_c) + np.sum(g["grad_T"] * cl.T)
        for f in A.VEL_FIELDS:
            s += np.sum(g["grad_" + f] * getattr(cl, f))
        return s + np.sum(g["grad_u_r_star"] * cl.u_r_star) + np.sum(g["grad_u_Z_star"] * cl.u_Z_star)

    h = 1e-6
    def with_nH(s):
        cl = W.turbulent_cloud(nr=12, nz=10, n_nu=16, seed=2)
        n = cl.n_H[j, i] * (1 + s)
        cl.alpha[j, i] = n * K.compute_sigma0(cl.T[j, i])
        cl.alpha_c[j, i] = cl.kappa_d * 0.01 * n * K.mH
        return np.sum(g["grad_alpha"] * cl.alpha) + np.sum(g["grad_alpha_c"] * cl.alpha_c)
    d = (with_nH(h) - with_nH(-h)) / (2 * h * c.n_H[j, i])
    assert abs(d - out["grad_n_H"][j, i]) <= 1e-6 * abs(d)
    def with_v(s):
        cl = W.turbulent_cloud(nr=12, nz=10, n_nu=16, seed=2)
        A.scale_cell_velocity(cl, j, i, s)
        return O(cl) - np.sum(g["grad_T"] * cl.T)
    d = (with_v(h) - with_v(-h)) / (2 * h)
    assert abs(d - A.velocity_scale_gradient(c, g)[j, i]) <= 1e-6 * abs(d)
