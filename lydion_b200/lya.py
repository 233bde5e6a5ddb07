"""Drop-in replacements of the reference's Lyman-alpha step functions, with the Julia call
signatures (snake_case names; arrays in the reference's memory order, i.e. numpy [j, i, k]
for a Julia A[k, i, j]). Each call uploads its host arrays to a cached device context, runs
the CUDA kernels through the C ABI and writes the results back into the caller's arrays in
place, as the Julia functions mutate theirs.

    advect_lya!                      -> advect_lya                        (src/UpdateLyaJandH.jl:107)
    AdvectJandH!                     -> advect_J_and_H                    (src/AdvectJandH.jl:2227)
    LyαEmissionAbsorptionUpdate!     -> lya_emission_absorption_update     (src/ConstantsAndFunctions.jl:483)
    FrequencyUpdateJLyα_AllCells!    -> frequency_update_J_lya_all_cells   (src/UpdateLyaJandH.jl:231)
    UpdateLyαJandH!                  -> update_lya_J_and_H                 (src/UpdateLyaJandH.jl:409)
    Update_f_Lyα_MF_L_Lyα!           -> update_f_lya_MF_L_lya              (src/ConstantsAndFunctions.jl:588)
      (gravity method)               -> update_f_lya_MF_L_lya_gravity      (src/ConstantsAndFunctions.jl:691)
    Compute_f_esc_Lyα_Cylindrical    -> compute_f_esc_lya_cylindrical      (src/ConstantsAndFunctions.jl:969)
    FindActiveBins                   -> find_active_bins                   (src/UpdateLyaJandH.jl:47)
    pd_Lyα                           -> pd_lya                             (src/LymanAlphaDestruction.jl:43)
    GetRHDCFLTimeStep                -> get_rhd_cfl_time_step              (src/AdvectJandH.jl:29)

A caller that advances many steps should keep the state on the device instead
(m1.M1Context / lyd_static_steps); these functions pay a host<->device copy of every array
they touch on every call, exactly like a stateless drop-in.
"""
from dataclasses import dataclass, field

import numpy as np

from . import constants as K
from ._lib import BC_OUTFLOW, BC_REFLECT, FLUX_GLF, FLUX_HLL
from .m1 import M1Context

_SYM = {"Reflect": BC_REFLECT, "Outflow": BC_OUTFLOW, ":Reflect": BC_REFLECT, ":Outflow": BC_OUTFLOW}


def _bc(v):
    if isinstance(v, str):
        return _SYM[v]
    return int(v)


@dataclass
class LyaArrays:
    """The fields of LyaArrays{FluxMethod} (src/Structs.jl:23-124) the step touches."""
    c_tilde: float
    J: np.ndarray
    J_old: np.ndarray
    H_r: np.ndarray
    H_Z: np.ndarray
    H_r_old: np.ndarray
    H_Z_old: np.ndarray
    alpha: np.ndarray
    alpha_F: np.ndarray
    alpha_c: np.ndarray
    pd: np.ndarray
    js: np.ndarray
    Hvoigt: np.ndarray
    phi_nu: np.ndarray
    nu: np.ndarray
    nuC: np.ndarray
    dnu: np.ndarray
    inv_dnu: np.ndarray
    inv_nuC: np.ndarray
    kcore_min: int                  # 0-based
    kcore_max: int
    recoil: bool
    alpha_floor: float
    dru_r: np.ndarray
    dru_Z: np.ndarray
    f_r: np.ndarray
    f_Z: np.ndarray
    flux_method: int = FLUX_GLF
    M_F: float = 0.0
    M_F_radial_net: float = 0.0
    M_F_radial_out: float = 0.0
    L_lya: float = 0.0
    f_esc_lya: float = 0.0

    @property
    def N_nu(self):
        return self.nuC.size


def generate_lya_arrays_from_saved(c_tilde, freq, geom, T, Hvoigt, phi_nu, recoil=True, hll=False):
    """GenerateLyaArrays_FromSaved (src/SetupLymanAlphaArrays.jl:244-393) for a frequency grid
    `freq` (grid.FreqGrid), geometry `geom` and temperature T [j, i]; H_voigt and phi_nu are
    supplied (the reference computes them with Update_Hvoigt!/Update_phi_nu!; on the device
    use M1Context.update_hvoigt)."""
    nz, nr = T.shape
    n = freq.n_nu
    z3 = lambda: np.zeros((nz, nr, n))
    z2 = lambda: np.zeros((nz, nr))
    from .grid import alpha_floor
    return LyaArrays(c_tilde=c_tilde, J=z3(), J_old=z3(), H_r=z3(), H_Z=z3(), H_r_old=z3(), H_Z_old=z3(),
                     alpha=z2(), alpha_F=z3(), alpha_c=z2(), pd=z2(), js=z2(), Hvoigt=np.array(Hvoigt, dtype=float),
                     phi_nu=np.array(phi_nu, dtype=float), nu=freq.nu, nuC=freq.nuC, dnu=freq.dnu,
                     inv_dnu=freq.inv_dnu, inv_nuC=freq.inv_nuC, kcore_min=freq.kcore_min,
                     kcore_max=freq.kcore_max, recoil=recoil, alpha_floor=alpha_floor(geom),
                     dru_r=z2(), dru_Z=z2(), f_r=z2(), f_Z=z2(), flux_method=FLUX_HLL if hll else FLUX_GLF)


class _Cache:
    """One device context per (grid shape, flux method, recoil, core range, geometry)."""

    def __init__(self):
        self.key = None
        self.ctx = None

    def get(self, lya, geom):
        nz, nr, n = lya.J.shape
        key = (n, nr, nz, lya.flux_method, bool(lya.recoil), lya.kcore_min, lya.kcore_max, lya.alpha_floor,
               id(geom))
        if key != self.key:
            if self.ctx is not None:
                self.ctx.close()
            self.ctx = M1Context(n, nr, nz, lya.kcore_min, lya.kcore_max, lya.alpha_floor, recoil=lya.recoil,
                                 flux_method=lya.flux_method)
            self.ctx.set_geometry(geom)
            from .grid import FreqGrid
            self.ctx.set_freq_grid(FreqGrid(lya.nu, lya.nuC, lya.dnu, lya.inv_dnu, lya.inv_nuC, lya.kcore_min,
                                            lya.kcore_max))
            self.key = key
        return self.ctx


_cache = _Cache()


def _push_state(ctx, lya):
    for name in ("J", "J_old", "H_r", "H_Z", "H_r_old", "H_Z_old"):
        ctx.upload(name, getattr(lya, name))


def _pull_state(ctx, lya):
    for name in ("J", "J_old", "H_r", "H_Z", "H_r_old", "H_Z_old"):
        getattr(lya, name)[...] = ctx.download(name)


def _push_velocity(ctx, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r):
    for name, a in (("u_r_star", u_r_star), ("u_Z_star", u_Z_star), ("dur_dr", dur_dr), ("dur_dZ", dur_dZ),
                    ("duZ_dr", duZ_dr), ("duZ_dZ", duZ_dZ), ("ur_over_r", ur_over_r)):
        if a is not None:
            ctx.upload(name, a)


def find_active_bins(lya, geom):
    """FindActiveBins (src/UpdateLyaJandH.jl:47-97) -> (kmin, kmax), 0-based."""
    ctx = _cache.get(lya, geom)
    ctx.upload("J", lya.J)
    return ctx.find_active_bins()


def advect_lya(ctdt, lya, geom, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r,
               BC_r_left="Reflect", BC_r_right="Outflow", BC_Z_bot="Reflect", BC_Z_top="Outflow"):
    """AdvectLya! (src/UpdateLyaJandH.jl:107-171); mutates lya.J, J_old, H_r, H_Z, H_*_old."""
    ctx = _cache.get(lya, geom)
    _push_state(ctx, lya)
    ctx.upload("Hvoigt", lya.Hvoigt)
    ctx.upload("alpha_F", lya.alpha_F)
    _push_velocity(ctx, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    ctx.advect(ctdt, _bc(BC_r_right), _bc(BC_Z_bot), _bc(BC_Z_top), bc_r_left=_bc(BC_r_left))
    _pull_state(ctx, lya)


class _BandCache:
    """One device context per (bands, grid shape, flux method, geometry) for AdvectJandH!."""

    def __init__(self):
        self.key = None
        self.ctx = None

    def get(self, n, nr, nz, flux, geom):
        key = (n, nr, nz, flux, id(geom))
        if key != self.key:
            if self.ctx is not None:
                self.ctx.close()
            from .grid import FreqGrid, alpha_floor
            self.ctx = M1Context(n, nr, nz, 0, 0, alpha_floor(geom), recoil=False, flux_method=flux)
            self.ctx.set_geometry(geom)
            # the bands' frequencies are not read by the advection; any increasing grid will do
            nu = np.arange(n + 1, dtype=np.float64) + 1.0
            nuC = 0.5 * (nu[1:] + nu[:-1])
            dnu = np.diff(nu)
            self.ctx.set_freq_grid(FreqGrid(nu, nuC, dnu, 1.0 / dnu, 1.0 / nuC, 0, 0))
            self.key = key
        return self.ctx


_band_cache = _BandCache()


def advect_J_and_H(ctdt, alpha_F, J, J_old, H_r, H_Z, geom, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ,
                   ur_over_r, UpdateJold=True, BC_r_left="Reflect", BC_r_right="Outflow", BC_Z_bot="Reflect",
                   BC_Z_top="Outflow", kmin=0, kmax=None, FluxSolver="HLL"):
    """AdvectJandH! (src/AdvectJandH.jl:2227-2464) for any set of bands: advects bins
    kmin..kmax (0-based, default all) of J, H_r, H_Z with the flux opacities alpha_F; J_old
    becomes J when UpdateJold, and is left alone otherwise (the stellar/IR call of
    PhotoThermoChemistry.jl:3854-3868 passes UpdateJold = false). Mutates J, H_r, H_Z (and
    J_old)."""
    nz, nr, n = J.shape
    flux = FLUX_HLL if str(FluxSolver).strip(":").upper() == "HLL" else FLUX_GLF
    ctx = _band_cache.get(n, nr, nz, flux, geom)
    for name, a in (("J", J), ("H_r", H_r), ("H_Z", H_Z), ("J_old", J_old), ("alpha_F", alpha_F)):
        ctx.upload(name, a)
    _push_velocity(ctx, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    kmax = n - 1 if kmax is None else kmax
    ctx.advect_jh(ctdt, kmin, kmax, UpdateJold, _bc(BC_r_right), _bc(BC_Z_bot), _bc(BC_Z_top),
                  bc_r_left=_bc(BC_r_left))
    for name, a in (("J", J), ("H_r", H_r), ("H_Z", H_Z), ("J_old", J_old)):
        a[...] = ctx.download(name)


def lya_emission_absorption_update(J, J_old, H_r, H_Z, H_r_old, H_Z_old, js, phi_nu, Hvoigt, alpha, alpha_c,
                                   alpha_F, pd, dru_r, dru_Z, dnu, c_tilde, dt, *, lya, geom):
    """LyaEmissionAbsorptionUpdate! (src/ConstantsAndFunctions.jl:483-573). The Julia function
    takes the arrays one by one; the device context needs the grid, so `lya` and `geom` name
    the state the arrays belong to. Mutates J, J_old, H_r, H_Z, H_*_old, dru_r, dru_Z."""
    ctx = _cache.get(lya, geom)
    for name, a in (("J", J), ("J_old", J_old), ("H_r", H_r), ("H_Z", H_Z), ("H_r_old", H_r_old),
                    ("H_Z_old", H_Z_old), ("js", js), ("phi_nu", phi_nu), ("Hvoigt", Hvoigt), ("alpha", alpha),
                    ("alpha_c", alpha_c), ("alpha_F", alpha_F), ("pd", pd), ("dru_r", dru_r), ("dru_Z", dru_Z)):
        ctx.upload(name, a)
    ctx.emission_absorption(c_tilde, dt)
    for name, a in (("J", J), ("J_old", J_old), ("H_r", H_r), ("H_Z", H_Z), ("H_r_old", H_r_old),
                    ("H_Z_old", H_Z_old), ("dru_r", dru_r), ("dru_Z", dru_Z)):
        a[...] = ctx.download(name)


def frequency_update_J_lya_all_cells(ctdt, lya, T, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r,
                                     update_freq_factors=True, *, geom):
    """FrequencyUpdateJLya_AllCells! (src/UpdateLyaJandH.jl:231-391); mutates lya's J/H arrays."""
    ctx = _cache.get(lya, geom)
    _push_state(ctx, lya)
    for name, a in (("Hvoigt", lya.Hvoigt), ("alpha", lya.alpha), ("T", T)):
        ctx.upload(name, a)
    _push_velocity(ctx, None, None, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    ctx.frequency_update(ctdt, update_freq_factors)
    _pull_state(ctx, lya)


def update_lya_J_and_H(dt, c_tilde, lya, geom, T, update_freq_factors, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr,
                       duZ_dZ, ur_over_r, BC_r_left="Reflect", BC_r_right="Outflow", BC_Z_bot="Reflect",
                       BC_Z_top="Outflow"):
    """UpdateLyaJandH! (src/UpdateLyaJandH.jl:409-486): advection then frequency update."""
    ctx = _cache.get(lya, geom)
    _push_state(ctx, lya)
    for name, a in (("Hvoigt", lya.Hvoigt), ("alpha_F", lya.alpha_F), ("alpha", lya.alpha), ("T", T)):
        ctx.upload(name, a)
    _push_velocity(ctx, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    ctx.update_J_and_H(dt, c_tilde, update_freq_factors, _bc(BC_r_right), _bc(BC_Z_bot), _bc(BC_Z_top),
                       bc_r_left=_bc(BC_r_left))
    _pull_state(ctx, lya)


def update_f_lya_MF_L_lya(f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM, dt, z_center, BC_Z_bot="Reflect", *, lya,
                          geom):
    """Update_f_Lya_MF_L_Lya! (src/ConstantsAndFunctions.jl:588-674) ->
    (M_F, M_F_radial_net, M_F_radial_out, L_tot); fills f_r, f_Z."""
    ctx = _cache.get(lya, geom)
    for name, a in (("dru_r", dru_r), ("dru_Z", dru_Z), ("js", js)):
        ctx.upload(name, a)
    out = ctx.force_multiplier(dt, z_center, _bc(BC_Z_bot))
    f_r[...] = ctx.download("f_r")
    f_Z[...] = ctx.download("f_Z")
    return tuple(float(v) for v in out)


def update_f_lya_MF_L_lya_gravity(f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM, dt, f_grav_r, f_grav_Z, z_center,
                                  BC_Z_bot="Reflect", *, lya, geom):
    """The gravity method of Update_f_Lya_MF_L_Lya! (src/ConstantsAndFunctions.jl:691-804) ->
    (M_F, M_F_antigravity, M_F_radial_net, M_F_radial_out, L_tot); fills f_r, f_Z."""
    ctx = _cache.get(lya, geom)
    for name, a in (("dru_r", dru_r), ("dru_Z", dru_Z), ("js", js)):
        ctx.upload(name, a)
    out = ctx.force_multiplier(dt, z_center, _bc(BC_Z_bot), f_grav=(f_grav_r, f_grav_Z))
    f_r[...] = ctx.download("f_r")
    f_Z[...] = ctx.download("f_Z")
    return tuple(float(v) for v in out)


def compute_f_esc_lya_cylindrical(H_r, H_Z, A_r, A_Z, dnu, L_allspace, BC_Z_bot="Reflect", *, lya, geom):
    """Compute_f_esc_Lya_Cylindrical (src/ConstantsAndFunctions.jl:969-993)."""
    ctx = _cache.get(lya, geom)
    ctx.upload("H_r", H_r)
    ctx.upload("H_Z", H_Z)
    return ctx.f_esc(L_allspace, _bc(BC_Z_bot))


def pd_lya(nHII, ne, nHI, nHeI, nH2, T, z=0.0, *, lya, geom):
    """pd_Lya (src/LymanAlphaDestruction.jl:43-97), element-wise on the device."""
    return _cache.get(lya, geom).pd_lya(nHII, ne, nHI, nHeI, nH2, T, z)


def get_rhd_cfl_time_step(geom, c_tilde, u_r, u_Z, CFL, *, lya):
    """GetRHDCFLTimeStep (src/AdvectJandH.jl:29-68)."""
    return _cache.get(lya, geom).cfl_dt(c_tilde, u_r, u_Z, CFL)
