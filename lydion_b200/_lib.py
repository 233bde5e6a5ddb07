"""ctypes binding of liblydion_m1.so (the C ABI declared in include/lydion_m1.h).

There is no fallback: if the CUDA library is missing this module raises, and every step
call goes through the CUDA kernels."""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "liblydion_m1.so")

LYD_OK = 0
LYD_ERR_ARG, LYD_ERR_CUDA, LYD_ERR_NONFINITE, LYD_ERR_SOLVE, LYD_ERR_STATE, LYD_ERR_NOMEM = -1, -2, -3, -4, -5, -6
LYD_ERR_TIMEOUT = -7
BC_REFLECT, BC_OUTFLOW = 0, 1
FLUX_GLF, FLUX_HLL = 0, 1
GEOM_CYLINDRICAL, GEOM_CARTESIAN = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2

F = dict(J=0, J_old=1, H_r=2, H_Z=3, H_r_old=4, H_Z_old=5, Hvoigt=6, phi_nu=7, alpha_F=8,
         alpha=16, alpha_c=17, alpha_cF=18, pd=19, js=20, T=21, dur_dr=22, dur_dZ=23, duZ_dr=24, duZ_dZ=25,
         ur_over_r=26, dru_r=27, dru_Z=28, f_r=29, f_Z=30, e_Lya=31, u_r_star=40, u_Z_star=41)

P = C.POINTER(C.c_double)


class LydionError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lydion_m1 error {code}: {msg}")
        self.code = code


class Dims(C.Structure):
    _fields_ = [("n_nu", C.c_int32), ("n_r", C.c_int32), ("n_z", C.c_int32), ("reserved", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("flux_method", C.c_int32), ("recoil", C.c_int32), ("precision", C.c_int32),
                ("kcore_min", C.c_int32), ("kcore_max", C.c_int32), ("keep_freq_factors", C.c_int32),
                ("alpha_floor", C.c_double), ("j_scale", C.c_double), ("device", C.c_int32),
                ("geometry", C.c_int32), ("bc_r_left", C.c_int32), ("reserved", C.c_int32 * 5)]


class Geometry(C.Structure):
    _fields_ = [("r", P), ("Z", P), ("rCoM", P), ("ZCoM", P), ("dV", P), ("inv_dV", P), ("A_r", P), ("A_Z", P),
                ("inv_r_cell", P), ("dr_L", P), ("dr_R", P), ("inv_dr_i_im1", P), ("inv_dr_ip1_i", P),
                ("inv_dr_ip2_ip1", P), ("dr_bnd", C.c_double * 10), ("dZ_L", P), ("dZ_R", P),
                ("inv_dZ_j_jm1", P), ("inv_dZ_jp1_j", P), ("inv_dZ_jp2_jp1", P), ("dZ_bnd", C.c_double * 10)]


class FreqGrid(C.Structure):
    _fields_ = [("nu", P), ("nuC", P), ("dnu", P), ("inv_dnu", P), ("inv_nuC", P)]


class StepParams(C.Structure):
    _fields_ = [("c_tilde", C.c_double), ("dt", C.c_double), ("z_center", C.c_double), ("bc_r_right", C.c_int32),
                ("bc_z_bot", C.c_int32), ("bc_z_top", C.c_int32), ("n_steps", C.c_int32)]


class Diag(C.Structure):
    _fields_ = [("M_F", C.c_double), ("M_F_radial_net", C.c_double), ("M_F_radial_out", C.c_double),
                ("L_tot", C.c_double), ("f_esc", C.c_double), ("kmin", C.c_int32), ("kmax", C.c_int32)]


class CloudParams(C.Structure):
    _fields_ = [("c_tilde", C.c_double), ("dt", C.c_double), ("z_center", C.c_double), ("bc_r_right", C.c_int32),
                ("bc_z_bot", C.c_int32), ("bc_z_top", C.c_int32), ("reserved", C.c_int32)]


class Tuning(C.Structure):
    _fields_ = [("rows_per_tile", C.c_int32), ("cells_per_block", C.c_int32), ("solver", C.c_int32),
                ("adv_ctas_per_sm", C.c_int32), ("adv_staging", C.c_int32)]


STAGING_AUTO, STAGING_LANES, STAGING_TMA = 0, 1, 2


SOLVER_PCR, SOLVER_THOMAS = 0, 1


class AdjointCfg(C.Structure):
    _fields_ = [("step", StepParams), ("checkpoint_every", C.c_int32), ("snapshots", C.c_int32), ("w_MF", C.c_double),
                ("w_spec", P)]


class DustLya(C.Structure):
    _fields_ = [("kappa_abs", C.c_double * 3), ("kappa_F", C.c_double * 3), ("rho_ignore", C.c_double)]


class RhdLyaOut(C.Structure):
    _fields_ = [("reject", C.POINTER(C.c_int32)), ("de", P), ("e_new", P), ("dru_r", P), ("dru_Z", P),
                ("split", P), ("dt_lya", P)]


class AdjointOut(C.Structure):
    _fields_ = [("objective", P), ("M_F", P), ("spectrum", P), ("grad_alpha", P), ("grad_alpha_c", P), ("grad_T", P),
                ("grad_Hv", P), ("grad_u_r_star", P), ("grad_u_Z_star", P), ("grad_du", P * 5), ("grad_J0", P),
                ("grad_H_r0", P), ("grad_H_Z0", P)]

# name -> (restype, argtypes); this list is the ABI surface checked by the CPU tests
I32, D, SZ, VP = C.c_int32, C.c_double, C.c_size_t, C.c_void_p
SIGNATURES = {
    "lyd_create": (C.c_int, [C.POINTER(VP), C.POINTER(Dims), C.POINTER(Config)]),
    "lyd_destroy": (C.c_int, [VP]),
    "lyd_last_error": (C.c_char_p, [VP]),
    "lyd_abi_version": (C.c_int, []),
    "lyd_math_check": (C.c_int, [I32, P, P, SZ]),
    "lyd_host_alloc": (C.c_int, [SZ, C.POINTER(VP)]),
    "lyd_host_free": (C.c_int, [VP]),
    "lyd_set_geometry": (C.c_int, [VP, C.POINTER(Geometry)]),
    "lyd_set_freq_grid": (C.c_int, [VP, C.POINTER(FreqGrid)]),
    "lyd_upload": (C.c_int, [VP, I32, P, SZ]),
    "lyd_download": (C.c_int, [VP, I32, P, SZ]),
    "lyd_synchronize": (C.c_int, [VP]),
    "lyd_get_stream": (C.c_int, [VP, C.POINTER(VP)]),
    "lyd_find_active_bins": (C.c_int, [VP, C.POINTER(I32), C.POINTER(I32)]),
    "lyd_advect": (C.c_int, [VP, D, I32, I32, I32, I32]),
    "lyd_advect_jh": (C.c_int, [VP, D, I32, I32, I32, I32, I32, I32, I32]),
    "lyd_emission_absorption": (C.c_int, [VP, D, D]),
    "lyd_frequency_update": (C.c_int, [VP, D, I32]),
    "lyd_update_J_and_H": (C.c_int, [VP, D, D, I32, I32, I32, I32, I32]),
    "lyd_force_multiplier": (C.c_int, [VP, D, D, I32, P]),
    "lyd_force_multiplier_gravity": (C.c_int, [VP, D, P, P, D, I32, P]),
    "lyd_f_esc": (C.c_int, [VP, D, I32, P]),
    "lyd_reset_dru": (C.c_int, [VP]),
    "lyd_static_steps": (C.c_int, [VP, C.POINTER(StepParams), C.POINTER(Diag)]),
    "lyd_set_timing": (C.c_int, [VP, I32]),
    "lyd_get_timing": (C.c_int, [VP, P]),
    "lyd_batch_create": (C.c_int, [C.POINTER(VP), I32, C.POINTER(I32), C.POINTER(I32), I32, C.POINTER(Config)]),
    "lyd_batch_info": (C.c_int, [VP, C.POINTER(I32), C.POINTER(C.c_int64)]),
    "lyd_set_geometry_cloud": (C.c_int, [VP, I32, C.POINTER(Geometry)]),
    "lyd_upload_cloud": (C.c_int, [VP, I32, I32, P, SZ]),
    "lyd_download_cloud": (C.c_int, [VP, I32, I32, P, SZ]),
    "lyd_edge_spectra_cloud": (C.c_int, [VP, I32, P, P, C.POINTER(I32), C.POINTER(I32)]),
    "lyd_batch_steps": (C.c_int, [VP, C.POINTER(CloudParams), I32, C.POINTER(Diag)]),
    "lyd_batch_steps_persistent": (C.c_int, [VP, C.POINTER(CloudParams), I32, C.c_int64, C.POINTER(Diag)]),
    "lyd_static_step_host": (C.c_int, [VP, C.POINTER(StepParams), P, P, P, P, P, P, I32, C.POINTER(Diag)]),
    "lyd_persistent_info": (C.c_int, [VP, C.POINTER(I32)]),
    "lyd_set_tuning": (C.c_int, [VP, C.POINTER(Tuning)]),
    "lyd_get_tuning": (C.c_int, [VP, C.POINTER(Tuning)]),
    "lyd_adjoint_run": (C.c_int, [VP, C.POINTER(AdjointCfg), C.POINTER(AdjointOut)]),
    "lyd_get_adjoint_timing": (C.c_int, [VP, P]),
    "lyd_update_hvoigt": (C.c_int, [VP]),
    "lyd_update_phi_nu": (C.c_int, [VP, I32, I32]),
    "lyd_pd_lya": (C.c_int, [VP, SZ, P, P, P, P, P, P, D, P]),
    "lyd_rhd_lya_prepare": (C.c_int, [VP, P, P, P, P, P, P, P, P, P, C.POINTER(DustLya), D, I32, I32]),
    "lyd_rhd_lya_absorb": (C.c_int, [VP, P, D, I32, C.POINTER(RhdLyaOut)]),
    "lyd_find_rsl_lya": (C.c_int, [VP, D, D, P, P, P, P, P, P, P, P, P, C.POINTER(DustLya), D, D, P]),
    "lyd_dd_set_halo": (C.c_int, [VP, I32, I32]),
    "lyd_dd_columns": (C.c_int, [VP]),
    "lyd_dd_find_active_partials": (C.c_int, [VP, VP]),
    "lyd_dd_step_partials": (C.c_int, [VP, C.POINTER(StepParams), VP]),
    "lyd_dd_finish": (C.c_int, [VP, VP, I32, C.POINTER(Diag)]),
    "lyd_dd_halo": (C.c_int, [VP, I32, I32, VP]),
    "lyd_cfl_dt": (C.c_int, [VP, D, P, P, D, P]),
    "lyd_edge_count": (C.c_int, [I32, I32]),
    "lyd_edge_spectra": (C.c_int, [VP, P, P, C.POINTER(I32), C.POINTER(I32)]),
    "lyd_voigt_tables": (C.c_int, [P, I32, D]),
    "lyd_find_active_bins_noalloc": (C.c_int, [VP, VP, VP, I32, I32, I32, I32, I32, VP, C.POINTER(I32),
                                               C.POINTER(I32)]),
}

_lib = None


def lib():
    """Load liblydion_m1.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lydion_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc, ctx=None):
    if rc != LYD_OK:
        msg = lib().lyd_last_error(ctx).decode() if ctx else ""
        raise LydionError(rc, msg)
