"""Gradients of the static-cloud diagnostics through the adjoint of the step (lyd_adjoint_run).

The library returns the gradient of

    objective = w_MF * M_F(last step) + sum_k w_k * S_k(final J)

with respect to the step's own inputs: the line-centre opacity alpha, the continuum opacity
alpha_c, the temperature T (through the Doppler width and recoil of the frequency factors and,
when H_voigt was computed on the device, through H_voigt), the seven velocity inputs and the
initial state. This module adds what depends on how a user parametrises a cloud:

* the 64-point emergent spectrum: the 48-bin edge-ring spectrum linearly interpolated onto
  64 evenly spaced points in x = (nu - nu_0) / Doppler width; its vector-Jacobian product is
  the transpose of that interpolation applied to the 64 weights;
* n_H, T and dust: alpha = x_HI n_H sigma0(T) and alpha_c = kappa_d * 0.01 n_H m_H give
  dO/dn_H = sigma0 dO/dalpha + kappa_d 0.01 m_H dO/dalpha_c, dO/dT adds
  n_H dsigma0/dT dO/dalpha (sigma0 ~ T^-1/2), and dO/dkappa_d(cell) = 0.01 n_H m_H dO/dalpha_c;
* velocity: the gradient with respect to a per-cell scale of the cell's velocity (the cell's
  five velocity-gradient inputs and, shared half-and-half with the neighbour, its four face
  velocities u*).
"""
import numpy as np

from . import constants as K


def x_of_bins(freq, T_ref=1e4):
    """Bin-centre x = (nu_C - nu_0) / Doppler width at T_ref."""
    return (np.asarray(freq.nuC) - K.nu_lya) / K.compute_dnuD(T_ref)


def spectrum_resampling(freq, n_points=64, T_ref=1e4):
    """The (n_points, n_nu) matrix of linear interpolation from the bin-centre spectrum onto
    n_points evenly spaced x over the bin-centre range, and those x."""
    xb = x_of_bins(freq, T_ref)
    xs = np.linspace(xb[0], xb[-1], n_points)
    M = np.zeros((n_points, xb.size))
    for p, x in enumerate(xs):
        k = int(np.clip(np.searchsorted(xb, x) - 1, 0, xb.size - 2))
        t = (x - xb[k]) / (xb[k + 1] - xb[k])
        M[p, k] = 1.0 - t
        M[p, k + 1] = t
    return M, xs


def physical_gradients(cloud, g, x_HI=1.0, dust_to_gas=0.01):
    """dO/dn_H, dO/dT (total), dO/dkappa_d per cell from the library's gradients, for a cloud
    built with alpha = x_HI n_H sigma0(T) and alpha_c = kappa_d dust_to_gas n_H m_H."""
    T = cloud.T
    sigma0 = K.sigma0_prefact / (K.b_prefact * np.sqrt(T))      # compute_sigma0, per cell
    nH = cloud.n_H if cloud.n_H is not None else cloud.alpha / (x_HI * sigma0)
    inside = cloud.alpha > 0.0
    gnH = np.where(inside, x_HI * sigma0 * g["grad_alpha"] + cloud.kappa_d * dust_to_gas * K.mH * g["grad_alpha_c"], 0.0)
    gT = g["grad_T"] + np.where(inside, x_HI * nH * (-0.5 * sigma0 / T) * g["grad_alpha"], 0.0)
    gk = np.where(inside, dust_to_gas * nH * K.mH * g["grad_alpha_c"], 0.0)
    return {"grad_n_H": gnH, "grad_T_total": gT, "grad_kappa_d": gk}


VEL_FIELDS = ("dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ", "ur_over_r")


def velocity_scale_gradient(cloud, g):
    """dO/ds per cell for u -> (1 + s) u on the cell's velocity-gradient inputs and, with
    weight 1/2, on its four face velocities."""
    out = np.zeros((cloud.nz, cloud.nr))
    for f in VEL_FIELDS:
        out += g["grad_" + f] * getattr(cloud, f)
    ur = g["grad_u_r_star"] * cloud.u_r_star          # [j, f]
    uz = g["grad_u_Z_star"] * cloud.u_Z_star          # [f, i]
    out += 0.5 * (ur[:, :-1] + ur[:, 1:])
    out += 0.5 * (uz[:-1, :] + uz[1:, :])
    return out


def scale_cell_velocity(cloud, j, i, s):
    """Apply the per-cell velocity scale of velocity_scale_gradient to cloud (in place)."""
    for f in VEL_FIELDS:
        getattr(cloud, f)[j, i] *= 1.0 + s
    cloud.u_r_star[j, i] *= 1.0 + 0.5 * s
    cloud.u_r_star[j, i + 1] *= 1.0 + 0.5 * s
    cloud.u_Z_star[j, i] *= 1.0 + 0.5 * s
    cloud.u_Z_star[j + 1, i] *= 1.0 + 0.5 * s


def objective_weights(freq, w_MF=1.0, w64=None, T_ref=1e4):
    """(w_MF, per-bin weights) for an objective on M_F and the 64-point spectrum."""
    if w64 is None:
        return w_MF, None
    M, _ = spectrum_resampling(freq, len(w64), T_ref)
    return w_MF, M.T @ np.asarray(w64, dtype=np.float64)
