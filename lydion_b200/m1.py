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
                 precision=PREC_FP64, keep_freq_factors=False, j_scale=0.0, device=0, cartesian=False,
                 bc_r_left=BC_REFLECT):
        self.n_nu, self.n_r, self.n_z = int(n_nu), int(n_r), int(n_z)
        self.precision = precision
        dims = _lib.Dims(self.n_nu, self.n_r, self.n_z, 0)
        cfg = _lib.Config(int(flux_method), int(bool(recoil)), int(precision), int(kcore_min), int(kcore_max),
                          int(bool(keep_freq_factors)), float(alpha_floor), float(j_scale), int(device),
                          _lib.GEOM_CARTESIAN if cartesian else _lib.GEOM_CYLINDRICAL, int(bc_r_left))
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

    def download(self, name, shape=None, out=None):
        """Copy a field to the host. `out`, when given, is a C-contiguous float64 array of the
        field's size that receives the data in place (page-locked memory makes the copy a
        direct DMA); otherwise a new array is returned."""
        if out is not None:
            if out.dtype != np.float64 or not out.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous float64 array")
            self._ck(lib().lyd_download(self._h, F[name], _dp(out), out.size))
            return out
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

    def advect_jh(self, ctdt, kmin, kmax, update_jold, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                  bc_z_top=BC_OUTFLOW, bc_r_left=BC_REFLECT):
        """AdvectJandH! over bins kmin..kmax (0-based) with the J_old rule of update_jold."""
        self._ck(lib().lyd_advect_jh(self._h, float(ctdt), int(kmin), int(kmax), int(bool(update_jold)), bc_r_left,
                                     bc_r_right, bc_z_bot, bc_z_top))

    def emission_absorption(self, c_tilde, dt):
        self._ck(lib().lyd_emission_absorption(self._h, float(c_tilde), float(dt)))

    def frequency_update(self, ctdt, update_freq_factors=True):
        self._ck(lib().lyd_frequency_update(self._h, float(ctdt), int(bool(update_freq_factors))))

    def update_J_and_H(self, dt, c_tilde, update_freq_factors=True, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                       bc_z_top=BC_OUTFLOW, bc_r_left=BC_REFLECT):
        self._ck(lib().lyd_update_J_and_H(self._h, float(dt), float(c_tilde), int(bool(update_freq_factors)),
                                          bc_r_left, bc_r_right, bc_z_bot, bc_z_top))

    def force_multiplier(self, dt, z_center, bc_z_bot=BC_REFLECT, f_grav=None):
        """{M_F, net, out, L_tot}; with f_grav = (f_grav_r, f_grav_Z) the gravity method's
        {M_F, M_F_antigravity, net, out, L_tot}."""
        if f_grav is None:
            out = np.zeros(4)
            self._ck(lib().lyd_force_multiplier(self._h, float(dt), float(z_center), bc_z_bot, _dp(out)))
            return out
        gr, gz = _c64(f_grav[0]), _c64(f_grav[1])
        out = np.zeros(5)
        self._ck(lib().lyd_force_multiplier_gravity(self._h, float(dt), _dp(gr), _dp(gz), float(z_center), bc_z_bot,
                                                    _dp(out)))
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

    def static_step_host(self, J, H_r, H_Z, c_tilde, dt, z_center, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                         bc_z_top=BC_OUTFLOW, out=None, chunks=8):
        """One static-driver iteration on host state (lyd_static_step_host): J, H_r, H_Z (float64,
        C-contiguous, the lyd_upload layout) go up, the new state comes back into `out`
        (three arrays; may be the inputs themselves; new arrays when None), pipelined over
        `chunks` row chunks. Returns (J, H_r, H_Z, record) with the step's diagnostics record
        (M_F, M_F_radial_net, M_F_radial_out, L_tot, f_esc, kmin, kmax)."""
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in (J, H_r, H_Z)]
        outs = list(out) if out is not None else [np.empty_like(a) for a in ins]
        for a, b in zip(ins, outs):
            if b.dtype != np.float64 or not b.flags.c_contiguous or b.size != a.size:
                raise ValueError("outputs must be C-contiguous float64 arrays of the inputs' size")
        p = _lib.StepParams(float(c_tilde), float(dt), float(z_center), bc_r_right, bc_z_bot, bc_z_top, 1)
        d = _lib.Diag()
        self._ck(lib().lyd_static_step_host(self._h, C.byref(p), _dp(ins[0]), _dp(ins[1]), _dp(ins[2]),
                                             _dp(outs[0]), _dp(outs[1]), _dp(outs[2]), int(chunks), C.byref(d)))
        rec = np.array([d.M_F, d.M_F_radial_net, d.M_F_radial_out, d.L_tot, d.f_esc, d.kmin, d.kmax])
        return outs[0], outs[1], outs[2], rec

    def set_timing(self, on):
        self._ck(lib().lyd_set_timing(self._h, int(bool(on))))

    def timing(self):
        ms = np.zeros(3)
        self._ck(lib().lyd_get_timing(self._h, _dp(ms)))
        return ms

    def set_tuning(self, rows_per_tile=16, cells_per_block=0, solver=_lib.SOLVER_PCR, adv_ctas_per_sm=0,
                   adv_staging=_lib.STAGING_AUTO):
        t = _lib.Tuning(int(rows_per_tile), int(cells_per_block), int(solver), int(adv_ctas_per_sm), int(adv_staging))
        self._ck(lib().lyd_set_tuning(self._h, C.byref(t)))

    def tuning(self):
        """(rows_per_tile, cells_per_block, solver, adv_ctas_per_sm, adv_staging); cells_per_block
        < 0 when chosen automatically; adv_staging is the staging the advection uses
        (STAGING_LANES or STAGING_TMA)."""
        t = _lib.Tuning()
        self._ck(lib().lyd_get_tuning(self._h, C.byref(t)))
        return t.rows_per_tile, t.cells_per_block, t.solver, t.adv_ctas_per_sm, t.adv_staging

    # -- adjoint ---------------------------------------------------------------------------
    def adjoint(self, n_steps, c_tilde, dt, z_center, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                bc_z_top=BC_OUTFLOW, w_MF=1.0, w_spec=None, checkpoint_every=0, want=None, snapshots=0):
        """Gradients of  w_MF * M_F(last step) + sum_k w_spec[k] * S_k(final J)  over n_steps
        static-driver steps from the current state (lyd_adjoint_run); the context ends in
        the final state. checkpoint_every: 1 keeps every step, K > 1 a checkpoint every K steps,
        0 every step when it fits (else K = 100), < 0 the binomial schedule with `snapshots`
        snapshots (0: the fewest with at most two advances of any step). Returns a dict: objective, M_F, spectrum and the gradients
        grad_alpha, grad_alpha_c, grad_T, grad_Hv, grad_u_r_star, grad_u_Z_star,
        grad_dur_dr, grad_dur_dZ, grad_duZ_dr, grad_duZ_dZ, grad_ur_over_r, grad_J0,
        grad_H_r0, grad_H_Z0 (numpy arrays in the reference's memory order)."""
        nr, nz, nnu = self.n_r, self.n_z, self.n_nu
        p = _lib.StepParams(float(c_tilde), float(dt), float(z_center), bc_r_right, bc_z_bot, bc_z_top, int(n_steps))
        ws = None if w_spec is None else _c64(w_spec)
        cfg = _lib.AdjointCfg(p, int(checkpoint_every), int(snapshots), float(w_MF), _dp(ws) if ws is not None else None)
        shapes = {"objective": (1,), "M_F": (1,), "spectrum": (nnu,), "grad_alpha": (nz, nr),
                  "grad_alpha_c": (nz, nr), "grad_T": (nz, nr), "grad_Hv": (nz, nr, nnu),
                  "grad_u_r_star": (nz, nr + 1), "grad_u_Z_star": (nz + 1, nr),
                  "grad_J0": (nz, nr, nnu), "grad_H_r0": (nz, nr, nnu), "grad_H_Z0": (nz, nr, nnu)}
        du = ("grad_dur_dr", "grad_dur_dZ", "grad_duZ_dr", "grad_duZ_dZ", "grad_ur_over_r")
        res = {k: np.zeros(v) for k, v in shapes.items() if want is None or k in want or k in ("objective", "M_F", "spectrum")}
        for k in du:
            if want is None or k in want:
                res[k] = np.zeros((nz, nr))
        o = _lib.AdjointOut()
        for name in shapes:
            if name in res:
                setattr(o, name, _dp(res[name]))
        for q, k in enumerate(du):
            if k in res:
                o.grad_du[q] = _dp(res[k])
        self._ck(lib().lyd_adjoint_run(self._h, C.byref(cfg), C.byref(o)))
        res["objective"] = float(res["objective"][0])
        res["M_F"] = float(res["M_F"][0])
        return res

    def adjoint_timing(self):
        """ms of the last timed adjoint: forward sweep, recomputation (with the advection's
        tapes), 0 (reserved), frequency-step adjoint, advection adjoint."""
        ms = np.zeros(5)
        self._ck(lib().lyd_get_adjoint_timing(self._h, _dp(ms)))
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

    # -- Z-slab domain decomposition (see lydion_b200/domain.py) ---------------------------
    def dd_set_halo(self, h_bot, h_top):
        self._ck(lib().lyd_dd_set_halo(self._h, int(h_bot), int(h_top)))

    def dd_columns(self):
        return int(lib().lyd_dd_columns(self._h))

    def dd_find_active_partials(self, colsum):
        self._ck(lib().lyd_dd_find_active_partials(self._h, C.c_void_p(colsum.data_ptr())))

    def dd_step_partials(self, colsum, c_tilde, dt, z_center, bc_r_right=BC_OUTFLOW, bc_z_bot=BC_REFLECT,
                         bc_z_top=BC_OUTFLOW):
        p = _lib.StepParams(float(c_tilde), float(dt), float(z_center), bc_r_right, bc_z_bot, bc_z_top, 1)
        self._ck(lib().lyd_dd_step_partials(self._h, C.byref(p), C.c_void_p(colsum.data_ptr())))

    def dd_finish(self, colsum, step=True):
        """The next window (and the step's record) from the all-reduced column sums: returns
        [M_F, radial net, radial out, L, f_esc, kmin, kmax]."""
        d = _lib.Diag()
        self._ck(lib().lyd_dd_finish(self._h, C.c_void_p(colsum.data_ptr()), int(bool(step)), C.byref(d)))
        return [d.M_F, d.M_F_radial_net, d.M_F_radial_out, d.L_tot, d.f_esc, d.kmin, d.kmax]

    def dd_halo(self, side, pack, buf):
        self._ck(lib().lyd_dd_halo(self._h, int(side), int(bool(pack)), C.c_void_p(buf.data_ptr())))

    # -- RHD-side Lyman-alpha block --------------------------------------------------------
    def rhd_lya_prepare(self, T, nHI, nH2, nHII, nHeI, ne, nOHx, nCHx, rho_d, kappa_abs, kappa_F, rho_ignore,
                        z=0.0, ots=True, destruction=True):
        """PrepareLyaSubCycling! for every cell (lyd_rhd_lya_prepare): per-cell arrays of shape
        (n_z, n_r); rho_d (3, n_z, n_r) holds the silicate, carbonaceous and PAH dust densities."""
        arrs = [_c64(np.ravel(a)) for a in (T, nHI, nH2, nHII, nHeI, ne, nOHx, nCHx)]
        rho = _c64(np.reshape(rho_d, (3, -1)))
        if any(a.size != self.n_r * self.n_z for a in arrs) or rho.shape[1] != self.n_r * self.n_z:
            raise ValueError("per-cell arrays must have n_r * n_z entries")
        d = _lib.DustLya((C.c_double * 3)(*kappa_abs), (C.c_double * 3)(*kappa_F), float(rho_ignore))
        self._ck(lib().lyd_rhd_lya_prepare(self._h, *[_dp(a) for a in arrs], _dp(rho), C.byref(d), float(z),
                                           int(bool(ots)), int(bool(destruction))))

    def rhd_lya_absorb(self, dt, c_tilde, commit=False, results=True):
        """The Lyman-alpha block of AbsorptionStep for every cell over its own sub-step dt
        (lyd_rhd_lya_absorb). Returns the per-cell results as (n_z, n_r) arrays (split: 8 of them),
        or None without `results` (nothing is copied back)."""
        shape = (self.n_z, self.n_r)
        dts = _c64(np.broadcast_to(np.asarray(dt, dtype=np.float64), shape))
        if not results:
            self._ck(lib().lyd_rhd_lya_absorb(self._h, _dp(dts), float(c_tilde), int(bool(commit)), None))
            return None
        n = self.n_r * self.n_z
        rej = np.zeros(n, dtype=np.int32)
        res = {k: np.empty(n) for k in ("de", "e_new", "dru_r", "dru_Z", "dt_lya")}
        split = np.empty(8 * n)
        out = _lib.RhdLyaOut(rej.ctypes.data_as(C.POINTER(C.c_int32)), _dp(res["de"]), _dp(res["e_new"]),
                             _dp(res["dru_r"]), _dp(res["dru_Z"]), _dp(split), _dp(res["dt_lya"]))
        self._ck(lib().lyd_rhd_lya_absorb(self._h, _dp(dts), float(c_tilde), int(bool(commit)), C.byref(out)))
        r = {k: v.reshape(shape) for k, v in res.items()}
        r["reject"] = rej.reshape(shape).astype(bool)
        r["split"] = split.reshape((8,) + shape)
        return r

    def find_rsl_lya(self, c_tilde_old, c_tilde_min, u_r, u_Z, P, rho, gamma_ad, T, xHII, xH2, rho_d, kappa_abs,
                     eps_rsl=4.0, X_over_mH=None):
        """FindRSL_LyaRT (lyd_find_rsl_lya): the reduced speed of light the Lya transport needs."""
        from . import constants as K
        if X_over_mH is None:
            X_over_mH = K.X_H / K.mH
        arrs = [_c64(np.ravel(a)) for a in (u_r, u_Z, P, rho, gamma_ad, T, xHII, xH2)]
        rho = _c64(np.reshape(rho_d, (3, -1)))
        d = _lib.DustLya((C.c_double * 3)(*kappa_abs), (C.c_double * 3)(0.0, 0.0, 0.0), 0.0)
        out = C.c_double()
        self._ck(lib().lyd_find_rsl_lya(self._h, float(c_tilde_old), float(c_tilde_min), *[_dp(a) for a in arrs],
                                        _dp(rho), C.byref(d), float(eps_rsl), float(X_over_mH), C.byref(out)))
        return out.value

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


class M1Batch(M1Context):
    """Many independent clouds of uneven (n_r, n_z) on one GPU, sharing a frequency grid and a
    configuration (lyd_batch_create). Every step kernel covers all clouds in one launch."""

    def __init__(self, sizes, n_nu, kcore_min, kcore_max, alpha_floor, recoil=True, flux_method=0,
                 precision=PREC_FP64, keep_freq_factors=False, j_scale=0.0, device=0):
        self.sizes = [(int(a), int(b)) for a, b in sizes]
        self.n_clouds = len(self.sizes)
        self.n_nu = int(n_nu)
        self.n_r = self.n_z = None
        self.precision = precision
        nr = (C.c_int32 * self.n_clouds)(*[a for a, _ in self.sizes])
        nz = (C.c_int32 * self.n_clouds)(*[b for _, b in self.sizes])
        cfg = _lib.Config(int(flux_method), int(bool(recoil)), int(precision), int(kcore_min), int(kcore_max),
                          int(bool(keep_freq_factors)), float(alpha_floor), float(j_scale), int(device))
        h = C.c_void_p()
        check(lib().lyd_batch_create(C.byref(h), self.n_clouds, nr, nz, self.n_nu, C.byref(cfg)))
        self._h = h
        self._keep = []

    @property
    def cell_bins(self):
        n = C.c_int64()
        self._ck(lib().lyd_batch_info(self._h, None, C.byref(n)))
        return int(n.value)

    def set_geometry(self, g, cloud=0):
        keep = [_c64(a) for a in (g.r, g.Z, g.rCoM, g.ZCoM, g.dV, g.inv_dV, g.A_r, g.A_Z, g.inv_r_cell,
                                  g.dr_L, g.dr_R, g.inv_dr_i_im1, g.inv_dr_ip1_i, g.inv_dr_ip2_ip1,
                                  g.dZ_L, g.dZ_R, g.inv_dZ_j_jm1, g.inv_dZ_jp1_j, g.inv_dZ_jp2_jp1)]
        p = [_dp(a) for a in keep]
        s = _lib.Geometry(*p[:14], (C.c_double * 10)(*g.dr_b), *p[14:], (C.c_double * 10)(*g.dZ_b))
        self._ck(lib().lyd_set_geometry_cloud(self._h, int(cloud), C.byref(s)))

    def upload_cloud(self, cloud, name, arr):
        a = _c64(arr)
        self._ck(lib().lyd_upload_cloud(self._h, int(cloud), F[name], _dp(a), a.size))

    def download_cloud(self, cloud, name):
        nr, nz = self.sizes[cloud]
        if F[name] < 16:
            shape = (nz, nr, self.n_nu)
        elif name == "u_r_star":
            shape = (nz, nr + 1)
        elif name == "u_Z_star":
            shape = (nz + 1, nr)
        else:
            shape = (nz, nr)
        out = np.empty(shape, dtype=np.float64)
        self._ck(lib().lyd_download_cloud(self._h, int(cloud), F[name], _dp(out), out.size))
        return out

    def download(self, name, shape=None):
        raise TypeError("a batch downloads per cloud: use download_cloud(cloud, name)")

    def find_active_bins(self):
        a = (C.c_int32 * self.n_clouds)()
        b = (C.c_int32 * self.n_clouds)()
        self._ck(lib().lyd_find_active_bins(self._h, a, b))
        return np.array(a[:]), np.array(b[:])

    def batch_steps(self, n_steps, params, history=True, persistent=False, barrier_polls=1 << 24):
        """params: one (c_tilde, dt, z_center, bc_r_right, bc_z_bot, bc_z_top) per cloud.
        Returns the (n_steps, n_clouds, 7) records when history is set. `persistent` runs each
        step as one cooperative launch whose grid barriers give up after `barrier_polls` polls
        (lyd_batch_steps_persistent)."""
        arr = (_lib.CloudParams * self.n_clouds)()
        for q, (ct, dt, zc, br, bb, bt) in enumerate(params):
            arr[q] = _lib.CloudParams(float(ct), float(dt), float(zc), int(br), int(bb), int(bt), 0)
        if persistent:
            call = lambda h: lib().lyd_batch_steps_persistent(self._h, arr, int(n_steps), int(barrier_polls), h)
        else:
            call = lambda h: lib().lyd_batch_steps(self._h, arr, int(n_steps), h)
        if history:
            hist = (_lib.Diag * max(1, n_steps * self.n_clouds))()
            self._ck(call(hist))
            out = np.array([[d.M_F, d.M_F_radial_net, d.M_F_radial_out, d.L_tot, d.f_esc, d.kmin, d.kmax]
                            for d in hist[:n_steps * self.n_clouds]])
            return out.reshape(n_steps, self.n_clouds, 7)
        self._ck(call(None))
        return None

    def persistent_graph(self):
        """1 when the persistent step replays from a CUDA graph, -1 when it is launched directly
        (capture refused by the runtime), 0 before its first run."""
        g = C.c_int32(0)
        self._ck(lib().lyd_persistent_info(self._h, C.byref(g)))
        return g.value

    def edge_spectra(self, cloud=0):
        nr, nz = self.sizes[cloud]
        n = lib().lyd_edge_count(nr, nz)
        raw = np.empty((n, self.n_nu)); norm = np.empty_like(raw)
        ri = (C.c_int32 * n)(); zi = (C.c_int32 * n)()
        self._ck(lib().lyd_edge_spectra_cloud(self._h, int(cloud), _dp(raw), _dp(norm), ri, zi))
        return raw, norm, np.array(ri[:]), np.array(zi[:])


def pinned_zeros(shape):
    """A float64 array of zeros in page-locked host memory (lyd_host_alloc): its copies to and
    from a context run at the link's rate (about 55 GB/s each way on a B200 box, against
    ~10 GB/s through pageable memory) and overlap the step in static_step_host. The memory is
    released with the last array that views it."""
    import weakref
    n = int(np.prod(shape))
    p = C.c_void_p()
    check(lib().lyd_host_alloc(max(1, n) * 8, C.byref(p)))
    buf = (C.c_double * max(1, n)).from_address(p.value)
    weakref.finalize(buf, lib().lyd_host_free, p)
    a = np.frombuffer(buf, dtype=np.float64, count=n).reshape(shape)
    a[...] = 0.0
    return a


def batch_for_clouds(clouds, precision=PREC_FP64, device=0, keep_freq_factors=False, j_scale=0.0):
    """Create a batch context holding every workloads.StaticCloud of `clouds` (one shared
    frequency grid, configuration taken from the first cloud) and upload their inputs; H_voigt
    and phi_nu are computed on the device."""
    c0 = clouds[0]
    fq = c0.freq
    b = M1Batch([(c.nr, c.nz) for c in clouds], c0.n_nu, fq.kcore_min, fq.kcore_max, c0.alpha_floor,
                recoil=c0.recoil, flux_method=c0.flux_method, precision=precision,
                keep_freq_factors=keep_freq_factors, j_scale=j_scale, device=device)
    b.set_freq_grid(fq)
    for q, c in enumerate(clouds):
        if c.freq is not fq and not np.array_equal(c.freq.nu, fq.nu):
            raise ValueError("the clouds of a batch share one frequency grid")
        b.set_geometry(c.geom, q)
        for name in ("alpha", "alpha_c", "pd", "js", "T", "dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ", "ur_over_r",
                     "u_r_star", "u_Z_star", "alpha_cF"):
            b.upload_cloud(q, name, getattr(c, name))
    b.update_hvoigt()
    b.update_phi_nu(fq.kcore_min, fq.kcore_max)
    return b


def cloud_params(clouds):
    return [(c.c_tilde, c.dt, c.z_center, c.bc_r_right, c.bc_z_bot, c.bc_z_top) for c in clouds]


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
    cart = bool(getattr(cloud.geom, "cartesian", False))
    ctx = M1Context(cloud.n_nu, cloud.nr, cloud.nz, fq.kcore_min, fq.kcore_max, cloud.alpha_floor,
                    recoil=cloud.recoil, flux_method=cloud.flux_method, precision=precision,
                    keep_freq_factors=keep_freq_factors, j_scale=j_scale, device=device, cartesian=cart,
                    bc_r_left=getattr(cloud, "bc_r_left", BC_REFLECT))
    ctx.set_geometry(cloud.geom)
    ctx.set_freq_grid(fq)
    for name in ("alpha", "alpha_c", "pd", "js", "T", "dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ", "ur_over_r",
                 "u_r_star", "u_Z_star"):
        if cart and name == "ur_over_r":
            continue            # no u_r / r term on a Cartesian grid
        ctx.upload(name, getattr(cloud, name))
    if getattr(cloud, "species", None):
        # destruction probability from the cell's species densities, on the device (pd_Lya)
        sp = cloud.species
        cloud.pd = ctx.pd_lya(sp["nHII"], sp["ne"], sp["nHI"], sp["nHeI"], sp["nH2"], cloud.T)
        ctx.upload("pd", cloud.pd)
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
