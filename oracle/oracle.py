"""ctypes front end of the CPU FP64 oracle (oracle/lydion_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, by __graft_entry__.smoke() as the checker, and by
bench.py's CPU-baseline leg. The product library never imports this module.

Parity status: the step is "parity unpinned" (the Julia reference cannot run in this
environment and no J/H golden vectors exist); the LAPACK dgtsv and the erf/Dawson Voigt
tables are pinned against scipy fixtures under tests/golden/.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liblydion_oracle.so")
_lib = None

P = C.POINTER(C.c_double)


def build():
    """Compile the oracle with its Makefile (gcc, OpenMP, no fast-math)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


class Geom(C.Structure):
    _fields_ = [("nr", C.c_int), ("nz", C.c_int), ("r", P), ("Z", P), ("rCoM", P), ("ZCoM", P),
                ("dV", P), ("inv_dV", P), ("A_r", P), ("A_Z", P), ("inv_r_cell", P),
                ("dr_L", P), ("dr_R", P), ("inv_dr_i_im1", P), ("inv_dr_ip1_i", P), ("inv_dr_ip2_ip1", P),
                ("dr_b", C.c_double * 10),
                ("dZ_L", P), ("dZ_R", P), ("inv_dZ_j_jm1", P), ("inv_dZ_jp1_j", P), ("inv_dZ_jp2_jp1", P),
                ("dZ_b", C.c_double * 10), ("bc_r_left", C.c_int)]


class Lya(C.Structure):
    _fields_ = [("nnu", C.c_int), ("nr", C.c_int), ("nz", C.c_int),
                ("J", P), ("J_old", P), ("H_r", P), ("H_Z", P), ("H_r_old", P), ("H_Z_old", P),
                ("alpha_F", P), ("Hvoigt", P), ("phi_nu", P),
                ("alpha", P), ("alpha_c", P), ("pd", P), ("js", P), ("T", P),
                ("dru_r", P), ("dru_Z", P), ("f_r", P), ("f_Z", P),
                ("nu", P), ("nuC", P), ("dnu", P), ("inv_dnu", P), ("inv_nuC", P),
                ("kcore_min", C.c_int), ("kcore_max", C.c_int), ("recoil", C.c_int), ("flux_method", C.c_int),
                ("alpha_floor", C.c_double),
                ("F_r", P), ("F_Z", P), ("F_r_Hr", P), ("F_Z_Hr", P), ("F_r_HZ", P), ("F_Z_HZ", P),
                ("K_iph", P), ("K_imh", P), ("Fkp", P), ("Fk", P), ("Fkm", P)]


class Vel(C.Structure):
    _fields_ = [("u_r_star", P), ("u_Z_star", P), ("dur_dr", P), ("dur_dZ", P), ("duZ_dr", P),
                ("duZ_dZ", P), ("ur_over_r", P)]


class VoigtLUT(C.Structure):
    _fields_ = [("xmax", C.c_double), ("xmin", C.c_double), ("inv_dx", C.c_double), ("nx", C.c_int),
                ("erf_y", P), ("dawson_y", P), ("gauss_y", P), ("xgauss_y", P), ("omx2gauss_y", P)]


def _declare(L):
    I, D = C.c_int, C.c_double
    sig = {
        "orc_minmod": (D, [D, D]), "orc_chi_L84": (D, [D]),
        "orc_D_edd": (None, [D, D, D, P]), "orc_D_edd_from_f_n": (None, [D, D, D, P]),
        "orc_hll_eigenvalues": (None, [D, D, P]),
        "orc_dgtsv": (I, [I, P, P, P, P]),
        "orc_pd_lya": (D, [D] * 7),
        "orc_compute_b": (D, [D]), "orc_compute_dnuD": (D, [D]), "orc_compute_a": (D, [D]),
        "orc_compute_sigma0": (D, [D]),
        "orc_voigt_H": (D, [C.c_void_p, D, D]), "orc_voigt_intH": (D, [C.c_void_p, D, D]),
        "orc_voigt_tophat": (D, [C.c_void_p, D, D, D, D]),
        "orc_update_hvoigt": (None, [C.c_void_p, C.c_void_p]),
        "orc_update_phi_nu": (None, [C.c_void_p, I, I]),
        "orc_find_active_bins": (None, [C.c_void_p, C.c_void_p, C.POINTER(I), C.POINTER(I)]),
        "orc_advect_jh": (None, [C.c_void_p, C.c_void_p, C.c_void_p, D, I, I, I, I, I, I]),
        "orc_advect_lya": (None, [C.c_void_p, C.c_void_p, C.c_void_p, D, I, I, I, C.POINTER(I), C.POINTER(I)]),
        "orc_emission_absorption": (None, [C.c_void_p, D, D]),
        "orc_update_freq_factors": (None, [C.c_void_p, C.c_void_p]),
        "orc_frequency_update_all_cells": (I, [C.c_void_p, C.c_void_p, D, I, C.POINTER(C.c_long)]),
        "orc_update_f_mf": (None, [C.c_void_p, C.c_void_p, D, D, I, P]),
        "orc_update_f_mf_gravity": (None, [C.c_void_p, C.c_void_p, D, P, P, D, I, P]),
        "orc_f_esc_lya": (D, [C.c_void_p, C.c_void_p, D, I]),
        "orc_reset_dru": (None, [C.c_void_p]),
        "orc_cfl_dt": (D, [C.c_void_p, D, P, P, D]),
        "orc_edge_count": (I, [I, I]),
        "orc_edge_spectra": (None, [C.c_void_p, P, P, C.POINTER(I), C.POINTER(I)]),
        "orc_static_step": (None, [C.c_void_p, C.c_void_p, C.c_void_p, D, D, D, I, I, I, P]),
        "orc_static_run": (None, [C.c_void_p, C.c_void_p, C.c_void_p, D, D, D, I, I, I, I, P]),
        "orc_num_threads": (I, []), "orc_set_num_threads": (None, [I]),
        "orc_prob_lya_sh95": (D, [D, D, I]), "orc_krec_hii": (D, [D, I]),
        "orc_js_rec_lya": (D, [D, D, D, I]), "orc_js_coll_lya": (D, [D, D, D]),
        "orc_rhd_lya_prepare_cell": (None, [P, C.c_void_p, D, I, I, P]),
        "orc_rhd_lya_absorb_cell": (I, [I, P, P, P, P, P, P, P, P, P, P, D, D, D, D, P]),
        "orc_find_rsl_lya": (D, [I, I] + [P] * 13 + [D, D, D, D]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(P)


_DUAL_PATH = os.path.join(_HERE, "build", "liblydion_oracle_dual.so")
_dual = None


def dual_lib():
    """The oracle compiled with dual numbers (lydion_oracle_dual.cpp): forward-mode derivatives."""
    global _dual
    if _dual is None:
        if not os.path.exists(_DUAL_PATH):
            build()
        _dual = C.CDLL(_DUAL_PATH)
        _dual.orcd_objective_tangent.restype = C.c_int
        _dual.orcd_objective_tangent.argtypes = [C.c_void_p] * 4 + [C.c_double] * 3 + [C.c_int] * 4 + \
            [C.c_double] + [P] * 7 + [P]
    return _dual


def objective_tangent(st, n_steps, w_MF=1.0, w_spec=None, seeds=None):
    """Forward-mode derivative of the static-driver objective w_MF * M_F(last step) +
    sum_k w_spec[k] S_k(final J) over n_steps from the initial state held by the OracleState
    `st` (its J, H_r, H_Z; H_voigt, phi_nu and alpha_F recomputed from T inside), along the
    direction `seeds`: a dict with any of alpha, alpha_c, T (numpy [j, i]), u_r_star, u_Z_star
    and J0. Returns (objective, directional derivative, M_F, its directional derivative)."""
    seeds = seeds or {}
    c = st.cloud
    keep = []

    def q(name):
        a = seeds.get(name)
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _p(a)

    ws = None if w_spec is None else np.ascontiguousarray(w_spec, dtype=np.float64)
    lut = st.lut or OracleLUT()
    out = np.zeros(4)
    dual_lib().orcd_objective_tangent(C.byref(st.s), C.byref(st.g), C.byref(st.v), lut.ref, c.c_tilde, c.dt,
                                      c.z_center, c.bc_r_right, c.bc_z_bot, c.bc_z_top, int(n_steps), float(w_MF),
                                      None if ws is None else _p(ws), q("alpha"), q("alpha_c"), q("T"),
                                      q("u_r_star"), q("u_Z_star"), q("J0"), _p(out))
    return tuple(float(x) for x in out)


# ---- Voigt look-up tables (src/FastInterpolations.jl:175-197) ----------------------------
XMAX_VOIGT = 1000.0
NX_VOIGT = 200001
_voigt_cache = {}


def voigt_tables(xmax=XMAX_VOIGT, nx=NX_VOIGT):
    """The five tables of CreateVoigtLUTs, tabulated with scipy's erf and Dawson integral
    (the stand-ins for SpecialFunctions.jl's erf/dawson)."""
    key = (xmax, nx)
    if key not in _voigt_cache:
        from scipy.special import erf, dawsn
        xmin = -xmax
        dx = (xmax - xmin) / (nx - 1)
        x = xmin + np.arange(nx, dtype=np.float64) * dx
        g = np.exp(-x * x)
        _voigt_cache[key] = dict(xmax=xmax, xmin=xmin, inv_dx=1.0 / dx, nx=nx,
                                 erf=np.ascontiguousarray(erf(x)), dawson=np.ascontiguousarray(dawsn(x)),
                                 gauss=g, xgauss=x * np.exp(-x * x), omx2gauss=(1.0 - 2.0 * (x * x)) * np.exp(-x * x))
    return _voigt_cache[key]


class OracleLUT:
    def __init__(self, xmax=XMAX_VOIGT, nx=NX_VOIGT):
        t = voigt_tables(xmax, nx)
        self._t = t
        self.s = VoigtLUT(t["xmax"], t["xmin"], t["inv_dx"], t["nx"], _p(t["erf"]), _p(t["dawson"]),
                          _p(t["gauss"]), _p(t["xgauss"]), _p(t["omx2gauss"]))

    @property
    def ref(self):
        return C.byref(self.s)


def geom_struct(geom, bc_r_left=0):
    keep = []

    def q(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _p(a)

    g = Geom(geom.nr, geom.nz, q(geom.r), q(geom.Z), q(geom.rCoM), q(geom.ZCoM), q(geom.dV), q(geom.inv_dV),
             q(geom.A_r), q(geom.A_Z), q(geom.inv_r_cell), q(geom.dr_L), q(geom.dr_R), q(geom.inv_dr_i_im1),
             q(geom.inv_dr_ip1_i), q(geom.inv_dr_ip2_ip1), (C.c_double * 10)(*geom.dr_b),
             q(geom.dZ_L), q(geom.dZ_R), q(geom.inv_dZ_j_jm1), q(geom.inv_dZ_jp1_j), q(geom.inv_dZ_jp2_jp1),
             (C.c_double * 10)(*geom.dZ_b), int(bc_r_left))
    return g, keep


class OracleState:
    """A LyaArrays restatement whose arrays are numpy buffers shared with the oracle.

    Arrays follow the reference's memory order: 3-D fields are numpy [j, i, k]."""

    FIELDS3 = ("J", "J_old", "H_r", "H_Z", "H_r_old", "H_Z_old", "alpha_F", "Hvoigt", "phi_nu",
               "Fkp", "Fk", "Fkm", "K_iph", "K_imh")

    def __init__(self, cloud, lut=None):
        lib()
        self.cloud = cloud
        nnu, nr, nz = cloud.n_nu, cloud.nr, cloud.nz
        z3 = lambda: np.zeros((nz, nr, nnu))
        for f in self.FIELDS3:
            setattr(self, f, z3())
        self.F_r = np.zeros((nz, nr + 1, nnu)); self.F_r_Hr = np.zeros_like(self.F_r); self.F_r_HZ = np.zeros_like(self.F_r)
        self.F_Z = np.zeros((nz + 1, nr, nnu)); self.F_Z_Hr = np.zeros_like(self.F_Z); self.F_Z_HZ = np.zeros_like(self.F_Z)
        self.alpha = np.ascontiguousarray(cloud.alpha, dtype=np.float64)
        self.alpha_c = np.ascontiguousarray(cloud.alpha_c, dtype=np.float64)
        self.pd = np.ascontiguousarray(cloud.pd, dtype=np.float64)
        self.js = np.ascontiguousarray(cloud.js, dtype=np.float64)
        self.T = np.ascontiguousarray(cloud.T, dtype=np.float64)
        self.dru_r = np.zeros((nz, nr)); self.dru_Z = np.zeros((nz, nr))
        self.f_r = np.zeros((nz, nr)); self.f_Z = np.zeros((nz, nr))
        fq = cloud.freq
        self._fq = [np.ascontiguousarray(a) for a in (fq.nu, fq.nuC, fq.dnu, fq.inv_dnu, fq.inv_nuC)]
        self.s = Lya(nnu, nr, nz, _p(self.J), _p(self.J_old), _p(self.H_r), _p(self.H_Z), _p(self.H_r_old),
                     _p(self.H_Z_old), _p(self.alpha_F), _p(self.Hvoigt), _p(self.phi_nu), _p(self.alpha),
                     _p(self.alpha_c), _p(self.pd), _p(self.js), _p(self.T), _p(self.dru_r), _p(self.dru_Z),
                     _p(self.f_r), _p(self.f_Z), *[_p(a) for a in self._fq], fq.kcore_min, fq.kcore_max,
                     int(cloud.recoil), int(cloud.flux_method), float(cloud.alpha_floor),
                     _p(self.F_r), _p(self.F_Z), _p(self.F_r_Hr), _p(self.F_Z_Hr), _p(self.F_r_HZ), _p(self.F_Z_HZ),
                     _p(self.K_iph), _p(self.K_imh), _p(self.Fkp), _p(self.Fk), _p(self.Fkm))
        self.g, self._gkeep = geom_struct(cloud.geom, getattr(cloud, "bc_r_left", 0))
        self._vel = [np.ascontiguousarray(a, dtype=np.float64) for a in
                     (cloud.u_r_star, cloud.u_Z_star, cloud.dur_dr, cloud.dur_dZ, cloud.duZ_dr, cloud.duZ_dZ,
                      cloud.ur_over_r)]
        self.v = Vel(*[_p(a) for a in self._vel])
        self.lut = lut

    # setup: src/FreqFactors.jl:24-51 and src/StaticCloudTest.jl:283-285
    def setup_profiles(self, lut=None):
        lut = lut or self.lut or OracleLUT()
        self.lut = lut
        lib().orc_update_hvoigt(lut.ref, C.byref(self.s))
        fq = self.cloud.freq
        lib().orc_update_phi_nu(C.byref(self.s), fq.kcore_min, fq.kcore_max)
        if np.any(self.cloud.alpha_cF):
            # RHD form, PhotoThermoChemistry.jl:2151
            self.alpha_F[...] = self.alpha[:, :, None] * self.Hvoigt + self.cloud.alpha_cF[:, :, None]
        else:
            # static-cloud form, src/StaticCloudTest.jl:283-285
            self.alpha_F[...] = self.alpha[:, :, None] * self.Hvoigt
        # UpdateFreqFactors! once at set-up, as the static driver does (src/StaticCloudTest.jl:309)
        lib().orc_update_freq_factors(C.byref(self.s), C.byref(self.v))

    def ref(self):
        return C.byref(self.s), C.byref(self.g), C.byref(self.v)

    def find_active_bins(self):
        a, b = C.c_int(), C.c_int()
        lib().orc_find_active_bins(C.byref(self.s), C.byref(self.g), C.byref(a), C.byref(b))
        return a.value, b.value

    def advect(self, ctdt):
        c = self.cloud
        a, b = C.c_int(), C.c_int()
        lib().orc_advect_lya(C.byref(self.s), C.byref(self.g), C.byref(self.v), ctdt, c.bc_r_right, c.bc_z_bot,
                             c.bc_z_top, C.byref(a), C.byref(b))
        return a.value, b.value

    def advect_jh(self, ctdt, kmin, kmax, update_jold):
        c = self.cloud
        lib().orc_advect_jh(C.byref(self.s), C.byref(self.g), C.byref(self.v), ctdt, int(update_jold), c.bc_r_right,
                            c.bc_z_bot, c.bc_z_top, int(kmin), int(kmax))

    def emission_absorption(self, c_tilde, dt):
        lib().orc_emission_absorption(C.byref(self.s), c_tilde, dt)

    def frequency_update(self, ctdt, update_ff=True):
        npiv = C.c_long(0)
        nfail = lib().orc_frequency_update_all_cells(C.byref(self.s), C.byref(self.v), ctdt, int(update_ff),
                                                     C.byref(npiv))
        return nfail, npiv.value

    def force_multiplier(self, dt):
        out = np.zeros(4)
        lib().orc_update_f_mf(C.byref(self.s), C.byref(self.g), dt, self.cloud.z_center, self.cloud.bc_z_bot, _p(out))
        return out

    def force_multiplier_gravity(self, dt, f_grav_r, f_grav_Z):
        out = np.zeros(5)
        gr = np.ascontiguousarray(f_grav_r, dtype=np.float64)
        gz = np.ascontiguousarray(f_grav_Z, dtype=np.float64)
        lib().orc_update_f_mf_gravity(C.byref(self.s), C.byref(self.g), dt, _p(gr), _p(gz), self.cloud.z_center,
                                      self.cloud.bc_z_bot, _p(out))
        return out

    def f_esc(self, L_all):
        return lib().orc_f_esc_lya(C.byref(self.s), C.byref(self.g), L_all, self.cloud.bc_z_bot)

    def step(self):
        c = self.cloud
        d = np.zeros(7)
        lib().orc_static_step(C.byref(self.s), C.byref(self.g), C.byref(self.v), c.c_tilde, c.dt, c.z_center,
                              c.bc_r_right, c.bc_z_bot, c.bc_z_top, _p(d))
        return d

    def run(self, n_steps):
        c = self.cloud
        d = np.zeros((n_steps, 7))
        lib().orc_static_run(C.byref(self.s), C.byref(self.g), C.byref(self.v), c.c_tilde, c.dt, c.z_center,
                             c.bc_r_right, c.bc_z_bot, c.bc_z_top, n_steps, _p(d))
        return d

    def edge_spectra(self):
        n = lib().orc_edge_count(self.cloud.nr, self.cloud.nz)
        raw = np.zeros((n, self.cloud.n_nu)); norm = np.zeros_like(raw)
        ri = (C.c_int * n)(); zi = (C.c_int * n)()
        lib().orc_edge_spectra(C.byref(self.s), _p(raw), _p(norm), ri, zi)
        return raw, norm, np.array(ri[:]), np.array(zi[:])


def dgtsv(dl, d, du, b):
    dl, d, du, b = (np.array(a, dtype=np.float64) for a in (dl, d, du, b))
    info = lib().orc_dgtsv(d.size, _p(dl), _p(d), _p(du), _p(b))
    return b, info


def scalar(name, *args):
    return getattr(lib(), name)(*args)


def vec_fn(name, *args, n=3):
    out = np.zeros(n)
    getattr(lib(), name)(*args, _p(out))
    return out


# ---- RHD-side Lyman-alpha block (oracle/lydion_oracle_rhd.c) -------------------------------
class DustLya(C.Structure):
    _fields_ = [("kappa_abs", C.c_double * 3), ("kappa_F", C.c_double * 3), ("rho_ignore", C.c_double)]


def rhd_lya_prepare(state, sp, rho_d, kappa_abs, kappa_F, rho_ignore, z=0.0, ots=True, destruction=True):
    """PrepareLyaSubCycling! on an OracleState: sp holds the per-cell arrays T, nHI, nH2, nHII,
    nHeI, ne, nOHx, nCHx ((n_z, n_r) each); rho_d is (3, n_z, n_r). Sets T, alpha, alpha_c, pd,
    js, H_voigt and phi_nu (all bins) on the state; returns alpha_cF and the dust flux opacities
    (3, n_z, n_r)."""
    d = DustLya((C.c_double * 3)(*kappa_abs), (C.c_double * 3)(*kappa_F), float(rho_ignore))
    nz, nr = state.T.shape
    acF = np.zeros((nz, nr))
    dF = np.zeros((3, nz, nr))
    out = np.zeros(8)
    names = ("T", "nHI", "nH2", "nHII", "nHeI", "ne", "nOHx", "nCHx")
    for j in range(nz):
        for i in range(nr):
            v = np.array([float(sp[n][j, i]) for n in names] + [float(rho_d[q][j, i]) for q in range(3)])
            lib().orc_rhd_lya_prepare_cell(_p(v), C.byref(d), float(z), int(bool(ots)), int(bool(destruction)),
                                           _p(out))
            state.T[j, i] = v[0]
            state.alpha[j, i], state.alpha_c[j, i], acF[j, i] = out[0], out[1], out[2]
            state.pd[j, i], state.js[j, i] = out[3], out[4]
            dF[:, j, i] = out[5:8]
    lut = state.lut or OracleLUT()
    state.lut = lut
    lib().orc_update_hvoigt(lut.ref, C.byref(state.s))
    lib().orc_update_phi_nu(C.byref(state.s), 0, state.cloud.n_nu - 1)
    return acF, dF


def rhd_lya_absorb(state, acF, dF, dt, c_tilde, e_lya, jeps=1e-60, commit=False):
    """The Lyman-alpha block of AbsorptionStep for every cell of an OracleState from its J_old /
    H_old over the per-cell sub-step dt; writes J, H (and, with commit, the accepted cells' old
    state and e_lya, or restores the rejected ones). Returns a dict of per-cell results."""
    nz, nr = state.T.shape
    nnu = state.cloud.n_nu
    dnu = np.ascontiguousarray(state.cloud.freq.dnu, dtype=np.float64)
    res = {k: np.zeros((nz, nr)) for k in ("de", "e_new", "dru_r", "dru_Z", "dt_lya")}
    res["split"] = np.zeros((8, nz, nr))
    res["reject"] = np.zeros((nz, nr), dtype=bool)
    out = np.zeros(13)
    cell = np.zeros(8)
    dt = np.broadcast_to(np.asarray(dt, dtype=np.float64), (nz, nr))
    for j in range(nz):
        for i in range(nr):
            cell[:] = [state.alpha[j, i], state.alpha_c[j, i], acF[j, i], state.pd[j, i], state.js[j, i],
                       dF[0, j, i], dF[1, j, i], dF[2, j, i]]
            row = lambda a: np.ascontiguousarray(a[j, i])
            Hv, phi = row(state.Hvoigt), row(state.phi_nu)
            Jo, Hro, HZo = row(state.J_old), row(state.H_r_old), row(state.H_Z_old)
            J, Hr, HZ = np.zeros(nnu), np.zeros(nnu), np.zeros(nnu)
            rej = lib().orc_rhd_lya_absorb_cell(nnu, _p(dnu), _p(Hv), _p(phi), _p(Jo), _p(Hro), _p(HZo), _p(J),
                                                _p(Hr), _p(HZ), _p(cell), float(dt[j, i]), float(c_tilde),
                                                float(e_lya[j, i]), float(jeps), _p(out))
            state.J[j, i], state.H_r[j, i], state.H_Z[j, i] = J, Hr, HZ
            res["reject"][j, i] = bool(rej)
            res["e_new"][j, i], res["de"][j, i], res["dru_r"][j, i], res["dru_Z"][j, i] = out[0], out[1], out[2], out[3]
            res["split"][:, j, i] = out[4:12]
            res["dt_lya"][j, i] = out[12]
            if commit:
                if rej:
                    state.J[j, i], state.H_r[j, i], state.H_Z[j, i] = Jo, Hro, HZo
                else:
                    state.J_old[j, i], state.H_r_old[j, i], state.H_Z_old[j, i] = J, Hr, HZ
                    e_lya[j, i] = out[0]
    return res


def find_rsl_lya(geom, hydro, rho_d, pd, kappa_abs, eps_rsl, X_over_mH, ct_old, ct_min):
    """FindRSL_LyaRT on one cloud: hydro holds u_r, u_Z, P, rho, gamma_ad, T, xHII, xH2 ((n_z, n_r) each)."""
    a = [np.ascontiguousarray(hydro[k], dtype=np.float64) for k in
         ("u_r", "u_Z", "P", "rho", "gamma_ad", "T", "xHII", "xH2")]
    rd = np.ascontiguousarray(rho_d, dtype=np.float64)
    pdc = np.ascontiguousarray(pd, dtype=np.float64)
    ka = np.ascontiguousarray(kappa_abs, dtype=np.float64)
    r = np.ascontiguousarray(geom.r, dtype=np.float64)
    Z = np.ascontiguousarray(geom.Z, dtype=np.float64)
    return lib().orc_find_rsl_lya(geom.nr, geom.nz, _p(r), _p(Z), *[_p(x) for x in a], _p(rd), _p(pdc), _p(ka),
                                  float(eps_rsl), float(X_over_mH), float(ct_old), float(ct_min))
