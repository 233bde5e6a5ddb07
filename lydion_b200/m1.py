"""Device-resident Lyman-alpha state: a thin object wrapper over one lyd_ctx.

Arrays cross the boundary in the reference's memory order (Julia column-major [k, i, j] ==
numpy C-order [j, i, k]); per-cell arrays are numpy [j, i]."""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import BC_OUTFLOW, BC_REFLECT, F, PREC_FP64, PREC_MIXED, check, lib


def _dp(a):
    return a.ctypes.data_as(_lib.P)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class M1Context:
    """One Lyman-alpha state on one GPU (see include/lydion_m1.h)."""

    def __init__(self, n_nu, n_r, n_z, kcore_min, kcore_max, alpha_floor, recoil=True, flux_method=0,
                 precision=PREC_FP64, keep_freq_factors=False, j_scale=0.0, device=0):
        self.n_nu, self.n_r, self.n_z = int(n_nu), int(n_r), int(n_z)
        self.precision = precision
        dims = _lib.Dims(self.n_nu, self.n_r, self.n_z, 0)
        cfg = _lib.Config(int(flux_method), int(bool(recoil)), int(precision), int(kcore_min), int(kcore_max),
                          int(bool(keep_freq_factors)), float(alpha_floor), float(j_scale), int(device))
        h = C.c_void_p()
        check(lib().lyd_create(C.byref(h), C.byref(dims), C.byref(cfg)))
        self._h = h
        self._keep = []

    # -- lifetime --------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().lyd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def _ck(self, rc):
        check(rc, self._h)

    # -- set-up ----------------------------------------------------------------------------
    def set_geometry(self, g):
        keep = [_c64(a) for a in (g.r, g.Z, g.rCoM, g.ZCoM, g.dV, g.inv_dV, g.A_r, g.A_Z, g.inv_r_cell,
                                  g.dr_L, g.dr_R, g.inv_dr_i_im1, g.inv_dr_ip1_i, g.inv_dr_ip2_ip1,
                                  g.dZ_L, g.dZ_R, g.inv_dZ_j_jm1, g.inv_dZ_jp1_j, g.inv_dZ_jp2_jp1)]
        p = [_dp(a) for a in keep]
        s = _lib.Geometry(*p[:14], (C.c_double * 10)(*g.dr_b), *p[14:], (C.c_double * 10)(*g.dZ_b))
        self._ck(lib().lyd_set_geometry(self._h, C.byref(s)))

    def set_freq_grid(self, fq):
        keep = [_c64(a) for a in (fq.nu, fq.nuC, fq.dnu, fq.inv_dnu, fq.inv_nuC)]
        s = _lib.FreqGrid(*[_dp(a) for a in keep])
        self._ck(lib().lyd_set_freq_grid(self._h, C.byref(s)))

    def upload(self, name, arr):
        a = _c64(arr)
        self._ck(lib().lyd_upload(self._h, F[name], _dp(a), a.size))

    def download(self, name, shape=None):
        if shape is None:
            if F[name] < 16:
                shape = (self.n_z, self.n_r, self.n_nu)
            elif name == "u_r_star":
                shape = (self.n_z, self.n_r + 1)
            elif name == "u_Z_star":
                shape = (self.n_z + 1, self.n_r)
            else:
                shape = (self.n_z, self.n_r)
        out = np.empty(shape, dtype=np.float64)
        self._ck(lib().lyd_download(self._h, F[name], _dp(out), out.size))
        return out

    def synchronize(self):
        self._ck(lib().lyd_synchronize(self._h))

    def stream(self):
        s = C.c_void_p()
        self._ck(lib().lyd_get_stream(self._h, C.byref(s)))
        return s.value

    # -- the step --------------------------------------------------------------------------
    def find_active_bins(self):
        a, b = C.c_int32(), C.c_int32()
        self._ck(lib().lyd_find_active_bins(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def advect(self, ctdt, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT, bc_z_top=BC_OUTFLOW, bc_r_left=BC_REFLECT):
        self._ck(lib().lyd_advect(self._h, float(ctdt), bc_r_left, bc_r_right, bc_z_bot, bc_z_top))

    def emission_absorption(self, c_tilde, dt):
        self._ck(lib().lyd_emission_absorption(self._h, float(c_tilde), float(dt)))

    def frequency_update(self, ctdt, update_freq_factors=True):
        self._ck(lib().lyd_frequency_update(self._h, float(ctdt), int(bool(update_freq_factors))))

    def update_J_and_H(self, dt, c_tilde, update_freq_factors=True, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                       bc_z_top=BC_OUTFLOW, bc_r_left=BC_REFLECT):
        self._ck(lib().lyd_update_J_and_H(self._h, float(dt), float(c_tilde), int(bool(update_freq_factors)),
                                          bc_r_left, bc_r_right, bc_z_bot, bc_z_top))

    def force_multiplier(self, dt, z_center, bc_z_bot=BC_REFLECT):
        out = np.zeros(4)
        self._ck(lib().lyd_force_multiplier(self._h, float(dt), float(z_center), bc_z_bot, _dp(out)))
        return out

    def f_esc(self, L_allspace, bc_z_bot=BC_REFLECT):
        f = C.c_double()
        self._ck(lib().lyd_f_esc(self._h, float(L_allspace), bc_z_bot, C.byref(f)))
        return f.value

    def reset_dru(self):
        self._ck(lib().lyd_reset_dru(self._h))

    def static_steps(self, n_steps, c_tilde, dt, z_center, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                     bc_z_top=BC_OUTFLOW, history=True):
        p = _lib.StepParams(float(c_tilde), float(dt), float(z_center), bc_r_right, bc_z_bot, bc_z_top, int(n_steps))
        if history:
            hist = (_lib.Diag * max(1, n_steps))()
            self._ck(lib().lyd_static_steps(self._h, C.byref(p), hist))
            return np.array([[d.M_F, d.M_F_radial_net, d.M_F_radial_out, d.L_tot, d.f_esc, d.kmin, d.kmax]
                             for d in hist[:n_steps]])
        self._ck(lib().lyd_static_steps(self._h, C.byref(p), None))
        return None

    def set_timing(self, on):
        self._ck(lib().lyd_set_timing(self._h, int(bool(on))))

    def timing(self):
        ms = np.zeros(3)
        self._ck(lib().lyd_get_timing(self._h, _dp(ms)))
        return ms

    # -- set-up helpers --------------------------------------------------------------------
    def update_hvoigt(self):
        self._ck(lib().lyd_update_hvoigt(self._h))

    def update_phi_nu(self, kmin, kmax):
        self._ck(lib().lyd_update_phi_nu(self._h, int(kmin), int(kmax)))

    def pd_lya(self, nHII, ne, nHI, nHeI, nH2, T, z=0.0):
        arrs = [_c64(np.ravel(a)) for a in (nHII, ne, nHI, nHeI, nH2, T)]
        out = np.empty(arrs[0].size)
        self._ck(lib().lyd_pd_lya(self._h, out.size, *[_dp(a) for a in arrs], float(z), _dp(out)))
        return out.reshape(np.shape(nHII))

    def cfl_dt(self, c_tilde, u_r, u_Z, cfl):
        a, b = _c64(u_r), _c64(u_Z)
        out = C.c_double()
        self._ck(lib().lyd_cfl_dt(self._h, float(c_tilde), _dp(a), _dp(b), float(cfl), C.byref(out)))
        return out.value

    def edge_spectra(self):
        n = lib().lyd_edge_count(self.n_r, self.n_z)
        raw = np.empty((n, self.n_nu)); norm = np.empty_like(raw)
        ri = (C.c_int32 * n)(); zi = (C.c_int32 * n)()
        self._ck(lib().lyd_edge_spectra(self._h, _dp(raw), _dp(norm), ri, zi))
        return raw, norm, np.array(ri[:]), np.array(zi[:])


def voigt_tables(n=200001, xmax=1000.0):
    """The device's Voigt look-up tables (host computation, no GPU needed): shape (5, n)."""
    out = np.empty((5, n))
    check(lib().lyd_voigt_tables(_dp(out), int(n), float(xmax)))
    return out


def context_for_cloud(cloud, precision=PREC_FP64, device=0, keep_freq_factors=False, j_scale=0.0,
                      hvoigt=None, phi_nu=None, alpha_F=None):
    """Create a context and upload every input of a workloads.StaticCloud.

    H_voigt is computed on the device (lyd_update_hvoigt) unless an array is given;
    phi_nu is derived on the device over the core bins (lyd_update_phi_nu) unless given;
    alpha_F is alpha*H_voigt (+ alpha_cF) unless given."""
    fq = cloud.freq
    ctx = M1Context(cloud.n_nu, cloud.nr, cloud.nz, fq.kcore_min, fq.kcore_max, cloud.alpha_floor,
                    recoil=cloud.recoil, flux_method=cloud.flux_method, precision=precision,
                    keep_freq_factors=keep_freq_factors, j_scale=j_scale, device=device)
    ctx.set_geometry(cloud.geom)
    ctx.set_freq_grid(fq)
    for name in ("alpha", "alpha_c", "pd", "js", "T", "dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ", "ur_over_r",
                 "u_r_star", "u_Z_star"):
        ctx.upload(name, getattr(cloud, name))
    if np.any(cloud.alpha_cF):
        ctx.upload("alpha_cF", cloud.alpha_cF)
    if hvoigt is None:
        ctx.update_hvoigt()
    else:
        ctx.upload("Hvoigt", hvoigt)
    if phi_nu is None:
        ctx.update_phi_nu(fq.kcore_min, fq.kcore_max)
    else:
        ctx.upload("phi_nu", phi_nu)
    if alpha_F is not None:
        ctx.upload("alpha_F", alpha_F)
    return ctx
