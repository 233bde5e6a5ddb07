"""Drop-in replacements of the reference's Lyman-alpha step functions with the Julia call
signatures: the same positional arguments in the same order, with the same defaults (snake_case
names; arrays in the reference's memory order, i.e. numpy [j, i, k] for a Julia A[k, i, j]).

    AdvectLyα!                       -> advect_lya                        (src/UpdateLyaJandH.jl:107)
    AdvectJandH!                     -> advect_J_and_H                    (src/AdvectJandH.jl:2227)
    LyαEmissionAbsorptionUpdate!     -> lya_emission_absorption_update     (src/ConstantsAndFunctions.jl:483)
    FrequencyUpdateJLyα_AllCells!    -> frequency_update_J_lya_all_cells   (src/UpdateLyaJandH.jl:231)
    UpdateLyαJandH!                  -> update_lya_J_and_H                 (src/UpdateLyaJandH.jl:409)
    Update_f_Lyα_MF_L_Lyα!           -> update_f_lya_MF_L_lya              (src/ConstantsAndFunctions.jl:588)
      (gravity method)               -> update_f_lya_MF_L_lya_gravity      (src/ConstantsAndFunctions.jl:691)
    Compute_f_esc_Lyα_Cylindrical    -> compute_f_esc_lya_cylindrical      (src/ConstantsAndFunctions.jl:969)
    Reset_Δρu!                       -> reset_dru                          (src/ConstantsAndFunctions.jl:809)
    FindActiveBins                   -> find_active_bins                   (src/UpdateLyaJandH.jl:47)
    pd_Lyα                           -> pd_lya                             (src/LymanAlphaDestruction.jl:43)
    GetRHDCFLTimeStep                -> get_rhd_cfl_time_step              (src/AdvectJandH.jl:29)

Device twins. Every LyaArrays gets one device context, its twin, holding the state and the
inputs on the GPU: generate_lya_arrays_from_saved makes it, or the first call that passes the
LyaArrays with its geometry. The functions the reference hands arrays only
(LyαEmissionAbsorptionUpdate!, Update_f_Lyα_MF_L_Lyα!, Compute_f_esc_Lyα_Cylindrical,
Reset_Δρu!) find the twin by the identity of the arrays they are given: the arrays of a
LyaArrays are registered with its twin (the Julia binding does the same with an IdDict, so the
reference's call sites stay as they are). Geometry arrays they are given (ΔV, rCoM, ZCoM, A_r,
A_Z) must be the twin's geometry, or hold its values.

Transfers.
  * Inputs the step only reads (H_voigt, phi_nu, alpha_F, alpha, alpha_c, p_d, js, T and the
    seven velocity fields) go to the device the first time an array object is passed for a
    field, and again only when another object is passed or after mark_dirty(array) -- a caller
    that changes such an array in place calls mark_dirty on it.
  * The state (J, J_old, H_r, H_Z, H_r_old, H_Z_old, dru_r, dru_Z, f_r, f_Z), in the default copy
    mode, goes up before every call that reads it and comes back into the caller's arrays after
    every call that writes it: the host arrays are always current, as with the reference's
    in-place mutation. After set_resident(lya) it stays on the device instead: sync_to_host(lya)
    brings it back, and mark_dirty(lya.J, ...) sends host edits before the next call.
"""
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import BC_OUTFLOW, BC_REFLECT, FLUX_GLF, FLUX_HLL
from .m1 import M1Context

_SYM = {"Reflect": BC_REFLECT, "Outflow": BC_OUTFLOW, ":Reflect": BC_REFLECT, ":Outflow": BC_OUTFLOW}


def _bc(v):
    if isinstance(v, str):
        return _SYM[v]
    return int(v)


@dataclass(eq=False)
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


STATE = ("J", "J_old", "H_r", "H_Z", "H_r_old", "H_Z_old")
_CELL_STATE = ("dru_r", "dru_Z", "f_r", "f_Z")
_LYA_INPUTS = ("alpha", "alpha_F", "alpha_c", "pd", "js", "Hvoigt", "phi_nu")


class _Twin:
    """The device side of one LyaArrays: a context, which array object each input field was
    last uploaded from, the fields to send again, and the bytes moved each way."""

    def __init__(self, lya, geom):
        from .grid import FreqGrid
        nz, nr, n = lya.J.shape
        self.lya, self.geom = lya, geom
        self.ctx = M1Context(n, nr, nz, lya.kcore_min, lya.kcore_max, lya.alpha_floor, recoil=lya.recoil,
                             flux_method=lya.flux_method, cartesian=bool(getattr(geom, "cartesian", False)))
        self.ctx.set_geometry(geom)
        self.ctx.set_freq_grid(FreqGrid(lya.nu, lya.nuC, lya.dnu, lya.inv_dnu, lya.inv_nuC, lya.kcore_min,
                                        lya.kcore_max))
        self.seen = {}           # input field -> the array object last uploaded for it
        self.dirty = set()       # fields to upload before their next use
        self.resident = False
        self.h2d = 0             # bytes uploaded / downloaded by the drop-in calls
        self.d2h = 0

    # inputs: once per array object, or when marked dirty
    def put_input(self, name, arr):
        if arr is None:
            return
        if self.seen.get(name) is arr and name not in self.dirty:
            return
        self.ctx.upload(name, arr)
        self.seen[name] = arr
        self.dirty.discard(name)
        self.h2d += np.asarray(arr).nbytes

    # state: every call in copy mode; in resident mode only what the host changed
    def put_state(self, pairs):
        for name, arr in pairs:
            if self.resident and name not in self.dirty:
                continue
            self.ctx.upload(name, arr)
            self.dirty.discard(name)
            self.h2d += arr.nbytes

    def get_state(self, pairs):
        if self.resident:
            return
        for name, arr in pairs:
            _download_into(self.ctx, name, arr)
            self.d2h += arr.nbytes

    def state_pairs(self, names):
        return [(n, getattr(self.lya, n)) for n in names]


def _download_into(ctx, name, arr):
    """Download a field into the caller's array in place (a temporary when the array is not a
    C-contiguous float64 array)."""
    if arr.dtype == np.float64 and arr.flags.c_contiguous:
        ctx.download(name, out=arr)
    else:
        arr[...] = ctx.download(name, shape=arr.shape)


_twins = {}      # id(LyaArrays) -> _Twin
_owners = {}     # id(array) -> (_Twin, field name, the array)


def _register(tw):
    for name in STATE + _CELL_STATE + _LYA_INPUTS:
        a = getattr(tw.lya, name)
        _owners[id(a)] = (tw, name, a)


def twin_of(lya, geom=None):
    """The device twin of `lya`, made (with `geom`) on first use."""
    tw = _twins.get(id(lya))
    if tw is not None and tw.lya is lya:
        if geom is not None and geom is not tw.geom:
            tw.ctx.set_geometry(geom)
            tw.geom = geom
            _register(tw)
        return tw
    if geom is None:
        raise ValueError("this LyaArrays has no device twin yet: make it with generate_lya_arrays_from_saved "
                         "or pass it with its geometry to advect_lya / update_lya_J_and_H first")
    tw = _Twin(lya, geom)
    _twins[id(lya)] = tw
    _register(tw)
    return tw


def _owner(arr, what):
    got = _owners.get(id(arr))
    if got is None or got[2] is not arr:
        raise ValueError(f"{what} is not an array of a LyaArrays with a device twin; "
                         "make the LyaArrays with generate_lya_arrays_from_saved")
    return got[0]


def _same_geometry(tw, name, arr):
    """An array the reference passes explicitly must be the twin's own geometry array (or
    hold the same values)."""
    mine = getattr(tw.geom, name)
    if arr is not mine and not np.array_equal(np.asarray(arr), mine):
        raise ValueError(f"{name} differs from the geometry of this LyaArrays' device twin")


def release(lya):
    """Drop the device twin of `lya` and its registrations."""
    tw = _twins.pop(id(lya), None)
    if tw is None:
        return
    for k in [k for k, v in _owners.items() if v[0] is tw]:
        del _owners[k]
    tw.ctx.close()


def set_resident(lya, on=True):
    """Keep the state of `lya` on the device between calls (True) or copy it every call (False,
    the default). Switching off brings the state back first."""
    tw = twin_of(lya)
    if tw.resident and not on:
        sync_to_host(lya)
    if on and not tw.resident:
        # the host arrays are the state to start from
        for name, arr in tw.state_pairs(STATE + _CELL_STATE):
            tw.ctx.upload(name, arr)
            tw.dirty.discard(name)
            tw.h2d += arr.nbytes
    tw.resident = bool(on)


def sync_to_host(lya):
    """Bring the device state of `lya` into its host arrays (resident mode)."""
    tw = twin_of(lya)
    for name, arr in tw.state_pairs(STATE + _CELL_STATE):
        _download_into(tw.ctx, name, arr)
        tw.d2h += arr.nbytes


def mark_dirty(*arrays):
    """Host edits of these arrays (state or inputs of a LyaArrays with a twin) go to the device
    before the next call that uses them."""
    for a in arrays:
        tw, name, _ = _owners.get(id(a), (None, None, None))
        if tw is None:
            raise ValueError("mark_dirty: not an array of a LyaArrays with a device twin")
        tw.dirty.add(name)


def transfer_bytes(lya):
    """(bytes uploaded, bytes downloaded) by the drop-in calls on `lya` so far."""
    tw = twin_of(lya)
    return tw.h2d, tw.d2h


def generate_lya_arrays_from_saved(c_tilde, freq, geom, T, Hvoigt, phi_nu, recoil=True, hll=False):
    """GenerateLyaArrays_FromSaved (src/SetupLymanAlphaArrays.jl:244-393) for a frequency grid
    `freq` (grid.FreqGrid), geometry `geom` and temperature T [j, i]; H_voigt and phi_nu are
    supplied (the reference computes them with Update_Hvoigt!/Update_phi_nu!). Makes the
    arrays' device twin. The cell-bin arrays are page-locked (m1.pinned_zeros), so the copies
    of the copy mode run at the link's rate."""
    from .m1 import pinned_zeros
    nz, nr = T.shape
    n = freq.n_nu
    z3 = lambda: pinned_zeros((nz, nr, n))

    def pinned_copy(a):
        out = pinned_zeros((nz, nr, n))
        out[...] = a
        return out
    z2 = lambda: np.zeros((nz, nr))
    from .grid import alpha_floor
    lya = LyaArrays(c_tilde=c_tilde, J=z3(), J_old=z3(), H_r=z3(), H_Z=z3(), H_r_old=z3(), H_Z_old=z3(),
                    alpha=z2(), alpha_F=z3(), alpha_c=z2(), pd=z2(), js=z2(), Hvoigt=pinned_copy(Hvoigt),
                    phi_nu=pinned_copy(phi_nu), nu=freq.nu, nuC=freq.nuC, dnu=freq.dnu,
                    inv_dnu=freq.inv_dnu, inv_nuC=freq.inv_nuC, kcore_min=freq.kcore_min,
                    kcore_max=freq.kcore_max, recoil=recoil, alpha_floor=alpha_floor(geom),
                    dru_r=z2(), dru_Z=z2(), f_r=z2(), f_Z=z2(), flux_method=FLUX_HLL if hll else FLUX_GLF)
    twin_of(lya, geom)
    return lya


def _put_velocity(tw, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r):
    for name, a in (("u_r_star", u_r_star), ("u_Z_star", u_Z_star), ("dur_dr", dur_dr), ("dur_dZ", dur_dZ),
                    ("duZ_dr", duZ_dr), ("duZ_dZ", duZ_dZ), ("ur_over_r", ur_over_r)):
        if a is not None and not (name == "ur_over_r" and getattr(tw.geom, "cartesian", False)):
            tw.put_input(name, a)


def _copy_old(lya):
    """The reference's phases end with J_old = J and H_old = H."""
    if lya.J_old is not lya.J:
        lya.J_old[...] = lya.J
        lya.H_r_old[...] = lya.H_r
        lya.H_Z_old[...] = lya.H_Z


def find_active_bins(lya, dV):
    """FindActiveBins (src/UpdateLyaJandH.jl:47-97) -> (kmin, kmax), 0-based."""
    tw = twin_of(lya)
    _same_geometry(tw, "dV", dV)
    tw.put_state(tw.state_pairs(("J",)))
    return tw.ctx.find_active_bins()


def advect_lya(ctdt, lya, geom, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r,
               BC_r_left="Reflect", BC_r_right="Outflow", BC_Z_bot="Reflect", BC_Z_top="Outflow"):
    """AdvectLya! (src/UpdateLyaJandH.jl:107-171); mutates lya.J, J_old, H_r, H_Z, H_*_old."""
    tw = twin_of(lya, geom)
    tw.put_state(tw.state_pairs(("J", "H_r", "H_Z")))
    tw.put_input("Hvoigt", lya.Hvoigt)
    tw.put_input("alpha_F", lya.alpha_F)
    _put_velocity(tw, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    tw.ctx.advect(ctdt, _bc(BC_r_right), _bc(BC_Z_bot), _bc(BC_Z_top), bc_r_left=_bc(BC_r_left))
    tw.get_state(tw.state_pairs(("J", "H_r", "H_Z")))
    if not tw.resident:
        _copy_old(lya)


def lya_emission_absorption_update(J, J_old, H_r, H_Z, H_r_old, H_Z_old, js, phi_nu, Hvoigt, alpha, alpha_c,
                                   alpha_F, pd, dru_r, dru_Z, dnu, c_tilde, dt):
    """LyaEmissionAbsorptionUpdate! (src/ConstantsAndFunctions.jl:483-573). Mutates J, J_old,
    H_r, H_Z, H_*_old, dru_r, dru_Z; the twin is the one J belongs to."""
    tw = _owner(J, "J")
    lya = tw.lya
    for name, a in (("J_old", J_old), ("H_r", H_r), ("H_Z", H_Z), ("H_r_old", H_r_old), ("H_Z_old", H_Z_old),
                    ("dru_r", dru_r), ("dru_Z", dru_Z)):
        if a is not getattr(lya, name):
            raise ValueError(f"{name} is not the {name} array of the LyaArrays J belongs to")
    if dnu is not lya.dnu and not np.array_equal(dnu, lya.dnu):
        raise ValueError("dnu differs from the frequency grid of this LyaArrays' device twin")
    tw.put_state(tw.state_pairs(STATE + ("dru_r", "dru_Z")))
    for name, a in (("js", js), ("phi_nu", phi_nu), ("Hvoigt", Hvoigt), ("alpha", alpha), ("alpha_c", alpha_c),
                    ("alpha_F", alpha_F), ("pd", pd)):
        tw.put_input(name, a)
    tw.ctx.emission_absorption(c_tilde, dt)
    tw.get_state(tw.state_pairs(("J", "H_r", "H_Z", "dru_r", "dru_Z")))
    if not tw.resident:
        _copy_old(lya)


def frequency_update_J_lya_all_cells(ctdt, lya, T, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r,
                                     update_freq_factors=True):
    """FrequencyUpdateJLya_AllCells! (src/UpdateLyaJandH.jl:231-391); mutates lya's J/H arrays."""
    tw = twin_of(lya)
    tw.put_state(tw.state_pairs(STATE))
    tw.put_input("Hvoigt", lya.Hvoigt)
    tw.put_input("alpha", lya.alpha)
    tw.put_input("T", T)
    _put_velocity(tw, None, None, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    tw.ctx.frequency_update(ctdt, update_freq_factors)
    tw.get_state(tw.state_pairs(("J", "H_r", "H_Z")))
    if not tw.resident:
        _copy_old(lya)


def update_lya_J_and_H(dt, c_tilde, lya, geom, T, update_freq_factors, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr,
                       duZ_dZ, ur_over_r, BC_r_left="Reflect", BC_r_right="Outflow", BC_Z_bot="Reflect",
                       BC_Z_top="Outflow"):
    """UpdateLyaJandH! (src/UpdateLyaJandH.jl:409-486): advection then frequency update."""
    tw = twin_of(lya, geom)
    tw.put_state(tw.state_pairs(("J", "H_r", "H_Z")))
    for name in ("Hvoigt", "alpha_F", "alpha"):
        tw.put_input(name, getattr(lya, name))
    tw.put_input("T", T)
    _put_velocity(tw, u_r_star, u_Z_star, dur_dr, dur_dZ, duZ_dr, duZ_dZ, ur_over_r)
    tw.ctx.update_J_and_H(dt, c_tilde, update_freq_factors, _bc(BC_r_right), _bc(BC_Z_bot), _bc(BC_Z_top),
                          bc_r_left=_bc(BC_r_left))
    tw.get_state(tw.state_pairs(("J", "H_r", "H_Z")))
    if not tw.resident:
        _copy_old(lya)


def _force_inputs(tw, f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM):
    lya = tw.lya
    for name, a in (("f_r", f_r), ("f_Z", f_Z), ("dru_Z", dru_Z)):
        if a is not getattr(lya, name):
            raise ValueError(f"{name} is not the {name} array of the LyaArrays dru_r belongs to")
    for name, a in (("dV", dV), ("rCoM", rCoM), ("ZCoM", ZCoM)):
        _same_geometry(tw, name, a)
    tw.put_state(tw.state_pairs(("dru_r", "dru_Z")))
    tw.put_input("js", js)


def update_f_lya_MF_L_lya(f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM, dt, z_center, BC_Z_bot="Reflect"):
    """Update_f_Lya_MF_L_Lya! (src/ConstantsAndFunctions.jl:588-674) ->
    (M_F, M_F_radial_net, M_F_radial_out, L_tot); fills f_r, f_Z."""
    tw = _owner(dru_r, "dru_r")
    _force_inputs(tw, f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM)
    out = tw.ctx.force_multiplier(dt, z_center, _bc(BC_Z_bot))
    tw.get_state(tw.state_pairs(("f_r", "f_Z")))
    return tuple(float(v) for v in out)


def update_f_lya_MF_L_lya_gravity(f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM, dt, f_grav_r, f_grav_Z, z_center,
                                  BC_Z_bot="Reflect"):
    """The gravity method of Update_f_Lya_MF_L_Lya! (src/ConstantsAndFunctions.jl:691-804) ->
    (M_F, M_F_antigravity, M_F_radial_net, M_F_radial_out, L_tot); fills f_r, f_Z."""
    tw = _owner(dru_r, "dru_r")
    _force_inputs(tw, f_r, f_Z, dru_r, dru_Z, js, dV, rCoM, ZCoM)
    out = tw.ctx.force_multiplier(dt, z_center, _bc(BC_Z_bot), f_grav=(f_grav_r, f_grav_Z))
    tw.get_state(tw.state_pairs(("f_r", "f_Z")))
    return tuple(float(v) for v in out)


def compute_f_esc_lya_cylindrical(H_r, H_Z, A_r, A_Z, dnu, L_allspace, BC_Z_bot="Reflect"):
    """Compute_f_esc_Lya_Cylindrical (src/ConstantsAndFunctions.jl:969-993)."""
    tw = _owner(H_r, "H_r")
    if H_Z is not tw.lya.H_Z:
        raise ValueError("H_Z is not the H_Z array of the LyaArrays H_r belongs to")
    for name, a in (("A_r", A_r), ("A_Z", A_Z)):
        _same_geometry(tw, name, a)
    if dnu is not tw.lya.dnu and not np.array_equal(dnu, tw.lya.dnu):
        raise ValueError("dnu differs from the frequency grid of this LyaArrays' device twin")
    tw.put_state(tw.state_pairs(("H_r", "H_Z")))
    return tw.ctx.f_esc(L_allspace, _bc(BC_Z_bot))


def reset_dru(dru_r, dru_Z):
    """Reset_Dru! (src/ConstantsAndFunctions.jl:809-816): zeroes both arrays, on the device and
    in the caller's arrays."""
    tw = _owner(dru_r, "dru_r")
    if dru_Z is not tw.lya.dru_Z:
        raise ValueError("dru_Z is not the dru_Z array of the LyaArrays dru_r belongs to")
    tw.ctx.reset_dru()
    if not tw.resident:
        dru_r[...] = 0.0
        dru_Z[...] = 0.0
    tw.dirty.discard("dru_r")
    tw.dirty.discard("dru_Z")


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
            self.geom = geom
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
    for name, a in (("u_r_star", u_r_star), ("u_Z_star", u_Z_star), ("dur_dr", dur_dr), ("dur_dZ", dur_dZ),
                    ("duZ_dr", duZ_dr), ("duZ_dZ", duZ_dZ), ("ur_over_r", ur_over_r)):
        if a is not None:
            ctx.upload(name, a)
    kmax = n - 1 if kmax is None else kmax
    ctx.advect_jh(ctdt, kmin, kmax, UpdateJold, _bc(BC_r_right), _bc(BC_Z_bot), _bc(BC_Z_top),
                  bc_r_left=_bc(BC_r_left))
    for name, a in (("J", J), ("H_r", H_r), ("H_Z", H_Z), ("J_old", J_old)):
        _download_into(ctx, name, a)


# ---- per-cell functions with no LyaArrays argument ----------------------------------------------
class _UtilityContexts:
    """Small contexts for the functions whose reference signature carries no LyaArrays:
    pd_Lya (any context serves: it is element-wise) and GetRHDCFLTimeStep (a context with
    the geometry of the interface coordinates it is given)."""

    def __init__(self):
        self.pd_ctx = None
        self.cfl = {}

    def for_pd(self):
        if self.pd_ctx is None:
            from .grid import uniform_cylindrical_geometry
            g = uniform_cylindrical_geometry(1.0, 1.0, 3, 3)
            self.pd_ctx = M1Context(4, 3, 3, 1, 2, 0.0, recoil=False)
            self.pd_ctx.set_geometry(g)
        return self.pd_ctx

    def for_cfl(self, r, Z):
        key = (np.asarray(r, dtype=np.float64).tobytes(), np.asarray(Z, dtype=np.float64).tobytes())
        ctx = self.cfl.get(key)
        if ctx is None:
            from .grid import cylindrical_geometry
            g = cylindrical_geometry(r, Z)
            ctx = M1Context(4, g.r.size - 1, g.Z.size - 1, 1, 2, 0.0, recoil=False)
            ctx.set_geometry(g)
            if len(self.cfl) > 8:
                for c in self.cfl.values():
                    c.close()
                self.cfl.clear()
            self.cfl[key] = ctx
        return ctx


_util = _UtilityContexts()


def pd_lya(nHII, ne, nHI, nHeI, nH2, T, z=0.0):
    """pd_Lya (src/LymanAlphaDestruction.jl:43-97) on the device, for scalars (returns a float,
    as the reference does) or element-wise for arrays of one shape."""
    out = _util.for_pd().pd_lya(*[np.asarray(a, dtype=np.float64) for a in (nHII, ne, nHI, nHeI, nH2, T)], z)
    return float(out) if np.ndim(out) == 0 else out


def get_rhd_cfl_time_step(r, Z, c_tilde, u_r, u_Z, CFL):
    """GetRHDCFLTimeStep (src/AdvectJandH.jl:29-68): the CFL step of a cylindrical grid with
    interface coordinates r (N_r + 1) and Z (N_Z + 1) and cell velocities u_r, u_Z [j, i]."""
    return _util.for_cfl(r, Z).cfl_dt(c_tilde, u_r, u_Z, CFL)


__all__ = ["LyaArrays", "generate_lya_arrays_from_saved", "advect_lya", "advect_J_and_H",
           "lya_emission_absorption_update", "frequency_update_J_lya_all_cells", "update_lya_J_and_H",
           "update_f_lya_MF_L_lya", "update_f_lya_MF_L_lya_gravity", "compute_f_esc_lya_cylindrical", "reset_dru",
           "find_active_bins", "pd_lya", "get_rhd_cfl_time_step", "set_resident", "sync_to_host", "mark_dirty",
           "transfer_bytes", "release", "twin_of", "_lib"]
