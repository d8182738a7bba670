"""ctypes declarations of libbamrex_cuda.so (include/bamrex_cuda.h).

The shared library is the product: there is no Python or CPU fallback.  If
it is missing or fails to load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbamrex_cuda.so")

MAX_NCOMP = 8

# status codes
OK, ERR_ARG, ERR_OOM, ERR_NAN, ERR_TIMEOUT, ERR_CUDA, ERR_UNSUPPORTED, ERR_NOT_CONVERGED = range(8)
# NumericalMethods::Method (Source/NumericalMethods.H:10-19)
MUSCL_HANCOCK, HLLC, IMEX, RCM, SLIC, FORCE, LAX_FRIEDRICHS = range(7)
METHODS = {"muscl_hancock": MUSCL_HANCOCK, "hllc": HLLC, "imex": IMEX, "rcm": RCM, "slic": SLIC,
           "force": FORCE, "lax_friedrichs": LAX_FRIEDRICHS}
# Limiter (Source/Fluxes/Limiters.H:13)
MINBEE, VAN_LEER, VAN_ALBADA, SUPERBEE = range(4)
LIMITERS = {"minbee": MINBEE, "van_leer": VAN_LEER, "van_albada": VAN_ALBADA, "superbee": SUPERBEE}
# boundary kinds
BC_TRANSMISSIVE, BC_PERIODIC, BC_REFLECTIVE = range(3)
BCS = {"transmissive": BC_TRANSMISSIVE, "periodic": BC_PERIODIC, "reflective": BC_REFLECTIVE}
# level state precision
FP64, FP32_STORAGE = 0, 1
# rigid bodies: shapes (Source/Geometry), combinations, RigidBodyBCType
# (Source/BoundaryConditions/BCTypes.H:50-57), GFMFlag bits (Source/GFM/GFMFlag.H)
SDF_PLANE, SDF_SPHERE, SDF_CYLINDER = range(3)
SDF_UNION, SDF_INTERSECTION = range(2)
RB_REFLECTIVE, RB_NO_SLIP, RB_FOEXTRAP = range(3)
RB_BCS = {"reflective": RB_REFLECTIVE, "no_slip": RB_NO_SLIP, "foextrap": RB_FOEXTRAP}
GFM_GHOST, GFM_INTERFACE, GFM_FILL = 1, 2, 4


class BamrexError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("bamrex status %d: %s" % (status, message))
        self.status = status


class Box(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3)]

    @classmethod
    def make(cls, lo, hi):
        b = cls()
        for d in range(3):
            b.lo[d] = int(lo[d]) if d < len(lo) else 0
            b.hi[d] = int(hi[d]) if d < len(hi) else 0
        return b


class Array4(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_void_p),
        ("jstride", ctypes.c_longlong),
        ("kstride", ctypes.c_longlong),
        ("nstride", ctypes.c_longlong),
        ("begin", ctypes.c_int * 3),
        ("end", ctypes.c_int * 3),
        ("ncomp", ctypes.c_int),
    ]


class CParm(ctypes.Structure):
    _fields_ = [
        ("adiabatic", ctypes.c_double),
        ("eos_mu", ctypes.c_double),
        ("Pr", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("eta_prime", ctypes.c_double),
        ("T_prime", ctypes.c_double),
        ("S_eta", ctypes.c_double),
        ("epsilon", ctypes.c_double),
        ("Re", ctypes.c_double),
        ("R_spec", ctypes.c_double),
        ("cv", ctypes.c_double),
        ("cp", ctypes.c_double),
        ("adia", ctypes.c_double * 9),
        ("Reinv", ctypes.c_double),
        ("limiter", ctypes.c_int),
        ("limiter_indices", ctypes.c_uint * MAX_NCOMP),
        ("limit_on_primv", ctypes.c_ubyte * MAX_NCOMP),
        ("need_primitive_for_limiting", ctypes.c_ubyte),
    ]


class Region(ctypes.Structure):
    _fields_ = [("box", ctypes.c_int), ("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3), ("offset", ctypes.c_longlong)]


class LevelDesc(ctypes.Structure):
    _fields_ = [
        ("spacedim", ctypes.c_int),
        ("domain", Box),
        ("prob_lo", ctypes.c_double * 3),
        ("prob_hi", ctypes.c_double * 3),
        ("bc_lo", ctypes.c_int * 3),
        ("bc_hi", ctypes.c_int * 3),
        ("boxes", ctypes.POINTER(Box)),
        ("nboxes", ctypes.c_int),
        ("ngrow", ctypes.c_int),
        ("method", ctypes.c_int),
        ("cfl", ctypes.c_double),
        ("parm", CParm),
        ("x_segment", ctypes.c_int),
        ("s_segment", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("x_mode", ctypes.c_int),
        ("staging", ctypes.c_int),
        ("staging_dir", ctypes.c_int * 3),
    ]


# x-sweep kernels (BAMREX_XSWEEP_*)
XSWEEP_AUTO, XSWEEP_ROWS, XSWEEP_MARCH = 0, 1, 2
# sweep input staging (BAMREX_STAGING_*)
STAGING_AUTO, STAGING_REGISTERS, STAGING_TMA, STAGING_WAVE = 0, 1, 2, 3

MAX_LEVELS = 8
# linear-operator boundary types (amrex::LinOpBCType subset)
LINOP_PERIODIC, LINOP_NEUMANN, LINOP_DIRICHLET = range(3)
# preconditioners of the flexible solve
PRECOND_NETWORK, PRECOND_NETWORK_VCYCLE, PRECOND_VCYCLE, PRECOND_VCYCLE_NETWORK = range(4)


class HelmholtzDesc(ctypes.Structure):
    _fields_ = [
        ("spacedim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("prob_lo", ctypes.c_double * 3),
        ("prob_hi", ctypes.c_double * 3),
        ("bc_lo", ctypes.c_int * 3),
        ("bc_hi", ctypes.c_int * 3),
        ("max_levels", ctypes.c_int),
        ("nu1", ctypes.c_int),
        ("nu2", ctypes.c_int),
        ("bottom_sweeps", ctypes.c_int),
    ]


# IMEX settings (BAMREX_IMEX_*) and fields of the last step
IMEX_RUSANOV, IMEX_MUSCL_RUSANOV = 0, 1
ENTH_REUSE_PRESSURE, ENTH_CONSERVATIVE, ENTH_CONSERVATIVE_EX = 0, 1, 2
KE_CONSERVATIVE, KE_EX, KE_SPLIT = 0, 1, 2
SP111, SSP222, SASSP322, SASSP332, SSP433 = range(5)
(FIELD_UEX, FIELD_ENTHALPY, FIELD_KE, FIELD_RHS, FIELD_PRESSURE, FIELD_FLUX_X, FIELD_FLUX_Y,
 FIELD_FLUX_Z) = range(8)


class ImexDesc(ctypes.Structure):
    _fields_ = [
        ("spacedim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("prob_lo", ctypes.c_double * 3),
        ("prob_hi", ctypes.c_double * 3),
        ("bc_lo", ctypes.c_int * 3),
        ("bc_hi", ctypes.c_int * 3),
        ("parm", CParm),
        ("advection_flux", ctypes.c_int),
        ("enthalpy_method", ctypes.c_int),
        ("ke_method", ctypes.c_int),
        ("cfl", ctypes.c_double),
        ("tol_rel", ctypes.c_double),
        ("tol_abs", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("tableau", ctypes.c_int),
    ]


class Sdf(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("center", ctypes.c_double * 3),
        ("axis", ctypes.c_double * 3),
        ("radius", ctypes.c_double),
        ("fluid_inside", ctypes.c_int),
    ]


class BodyDesc(ctypes.Structure):
    _fields_ = [
        ("nshapes", ctypes.c_int),
        ("combine", ctypes.c_int),
        ("shapes", Sdf * 2),
        ("rb_bc", ctypes.c_int),
        ("stencil", ctypes.c_int),
        ("fill_diagonals", ctypes.c_int),
    ]


class AmrDesc(ctypes.Structure):
    _fields_ = [
        ("base", LevelDesc),
        ("max_level", ctypes.c_int),
        ("ref_ratio", ctypes.c_int),
        ("blocking_factor", ctypes.c_int),
        ("max_grid_size", ctypes.c_int),
        ("n_error_buf", ctypes.c_int),
        ("n_proper", ctypes.c_int),
        ("grid_eff", ctypes.c_double),
        ("regrid_int", ctypes.c_int),
        ("do_reflux", ctypes.c_int),
        ("phigrad_var", ctypes.c_int),
        ("phigrad_var_is_primv", ctypes.c_int),
        ("phigrad", ctypes.c_double * MAX_LEVELS),
        ("max_phigrad_lev", ctypes.c_int),
        ("phierr_var", ctypes.c_int),
        ("phierr_var_is_primv", ctypes.c_int),
        ("phierr", ctypes.c_double * MAX_LEVELS),
        ("max_phierr_lev", ctypes.c_int),
        ("max_int_lev", ctypes.c_int),
        ("lstol", ctypes.c_double * MAX_LEVELS),
        ("max_box_lev", ctypes.c_int),
        ("box_lo", ctypes.c_double * 3),
        ("box_hi", ctypes.c_double * 3),
    ]


class TagDesc(ctypes.Structure):
    _fields_ = [
        ("do_err", ctypes.c_int), ("err_var", ctypes.c_int), ("err_var_is_primv", ctypes.c_int),
        ("phierr", ctypes.c_double),
        ("do_grad", ctypes.c_int), ("grad_var", ctypes.c_int), ("grad_var_is_primv", ctypes.c_int),
        ("phigrad", ctypes.c_double),
        ("do_box", ctypes.c_int), ("box_lo", ctypes.c_double * 3), ("box_hi", ctypes.c_double * 3),
        ("do_interface", ctypes.c_int), ("lstol", ctypes.c_double),
    ]


class AmrStepping(ctypes.Structure):
    _fields_ = [
        ("coarse_steps", ctypes.c_int),
        ("have_dt", ctypes.c_int),
        ("nlevels", ctypes.c_int),
        ("dt_level", ctypes.c_double * MAX_LEVELS),
    ]


# Every symbol include/bamrex_cuda.h declares, with (restype, argtypes).
_vp, _i, _d, _ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
_dp = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "bamrex_abi_version": (_i, []),
    "bamrex_release_memory": (_i, []),
    "bamrex_last_error": (ctypes.c_char_p, []),
    "bamrex_status_string": (ctypes.c_char_p, [_i]),
    "bamrex_profile_enable": (_i, [_i]),
    "bamrex_profile_reset": (_i, []),
    "bamrex_profile_report": (_i, [ctypes.c_char_p, _i, ctypes.POINTER(ctypes.c_int)]),
    "bamrex_parm_set_defaults": (_i, [ctypes.POINTER(CParm), _i]),
    "bamrex_parm_init": (_i, [ctypes.POINTER(CParm)]),
    "bamrex_compute_flux": (_i, [_i, _i, _i, _d, ctypes.POINTER(Box), Array4, Array4, _dp, _d,
                                 ctypes.POINTER(CParm), _vp]),
    "bamrex_compute_flux_LR": (_i, [_i, _i, _i, _d, ctypes.POINTER(Box), Array4, Array4, Array4, _dp, _d,
                                    ctypes.POINTER(CParm), _vp]),
    "bamrex_sweep_update": (_i, [_i, _i, ctypes.POINTER(Box), Array4, Array4, Array4, _dp, _d, _vp]),
    "bamrex_conservative_update": (_i, [_i, ctypes.POINTER(Box), Array4, Array4, ctypes.POINTER(Array4), _d,
                                        _dp, _vp]),
    "bamrex_sweep_box": (_i, [_i, _i, _i, ctypes.POINTER(Box), Array4, Array4, Array4, _dp, _d,
                              ctypes.POINTER(CParm), _vp]),
    "bamrex_level_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(LevelDesc), _vp]),
    "bamrex_level_destroy": (_i, [_vp]),
    "bamrex_level_last_error": (ctypes.c_char_p, [_vp]),
    "bamrex_level_num_cells": (_ll, [_vp]),
    "bamrex_level_stream": (_vp, [_vp]),
    "bamrex_level_x_mode": (_i, [_vp]),
    "bamrex_level_staging": (_i, [_vp, _i]),
    "bamrex_level_fab": (_i, [_vp, _i, ctypes.POINTER(Array4)]),
    "bamrex_level_copy_in": (_i, [_vp, _vp]),
    "bamrex_level_copy_out": (_i, [_vp, _vp]),
    "bamrex_level_sync": (_i, [_vp]),
    "bamrex_level_conserved_sums": (_i, [_vp, _dp]),
    "bamrex_level_fill_boundary": (_i, [_vp]),
    "bamrex_level_advance": (_i, [_vp, _d, _d, _i, _i, _dp]),
    "bamrex_level_est_time_step": (_i, [_vp, _dp]),
    "bamrex_level_run": (_i, [_vp, _i, _d, _i, _dp, ctypes.POINTER(_i)]),
    "bamrex_level_run_async": (_i, [_vp, _i, _d, _i, _d]),
    "bamrex_level_run_wait": (_i, [_vp, _dp, ctypes.POINTER(_i)]),
    "bamrex_level_set_timing": (_i, [_vp, _i]),
    "bamrex_level_counters": (_i, [_vp, ctypes.POINTER(_ll), _dp, ctypes.POINTER(_ll)]),
    "bamrex_level_reset_counters": (_i, [_vp]),
    "bamrex_level_sweep_times": (_i, [_vp, _dp, ctypes.POINTER(_ll)]),
    "bamrex_conserved_sums_noalloc": (_i, [_i, ctypes.POINTER(Box), ctypes.POINTER(Array4), _i, _dp, _dp, _vp]),
    "bamrex_level_set_halo": (_i, [_vp, _i, ctypes.POINTER(Region), _i, ctypes.POINTER(Region), _i]),
    "bamrex_level_halo_pack": (_i, [_vp, _i, _vp]),
    "bamrex_level_halo_unpack": (_i, [_vp, _i, _vp]),
    "bamrex_level_fill_dir": (_i, [_vp, _i]),
    "bamrex_level_sweep_dir": (_i, [_vp, _i, _d, _i]),
    "bamrex_level_wave_speed": (_i, [_vp, _dp]),
    "bamrex_level_dist_begin": (_i, [_vp, _d, _d]),
    "bamrex_level_wave_speed_async": (_i, [_vp, _vp]),
    "bamrex_level_dist_dt": (_i, [_vp, _vp, _i]),
    "bamrex_level_fill_dir_device": (_i, [_vp, _i]),
    "bamrex_level_sweep_dir_device": (_i, [_vp, _i, _i]),
    "bamrex_level_set_sweep_split": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_int), _i]),
    "bamrex_level_sweep_dir_device_part": (_i, [_vp, _i, _i, _i]),
    "bamrex_level_dist_end": (_i, [_vp, _dp, _dp, ctypes.POINTER(ctypes.c_int)]),
    "bamrex_level_step_host": (_i, [_vp, _vp, _vp, _d, _i, _dp]),
    "bamrex_level_run_host": (_i, [_vp, _vp, _i, _d, _i, _dp, _dp]),
    "bamrex_level_host_slabs": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_int)]),
    "bamrex_level_set_body": (_i, [_vp, ctypes.POINTER(BodyDesc)]),
    "bamrex_level_fill_body_ghosts": (_i, [_vp]),
    "bamrex_level_body_field": (_i, [_vp, _i, _dp]),
    "bamrex_level_body_counts": (_i, [_vp, ctypes.POINTER(_ll), ctypes.POINTER(_ll)]),
    "bamrex_level_tag": (_i, [_vp, _i, _i, _d, _i, _i, _i, _d, ctypes.c_char_p]),
    "bamrex_level_tag_ex": (_i, [_vp, _vp, ctypes.c_char_p]),
    "bamrex_coupling_create": (_i, [ctypes.POINTER(_vp), _vp, _vp, _i]),
    "bamrex_coupling_destroy": (_i, [_vp]),
    "bamrex_coupling_save_coarse_old": (_i, [_vp, _d, _d]),
    "bamrex_coupling_fill_patch": (_i, [_vp, _d]),
    "bamrex_coupling_fill_coarse_patch": (_i, [_vp]),
    "bamrex_coupling_reflux": (_i, [_vp]),
    "bamrex_coupling_avg_down": (_i, [_vp]),
    "bamrex_coupling_covered_sums": (_i, [_vp, _dp]),
    "bamrex_coupling_register": (_i, [_vp, _i, _dp, ctypes.POINTER(_i)]),
    "bamrex_cluster_tags": (_i, [_i, ctypes.POINTER(Box), ctypes.POINTER(_i), ctypes.POINTER(Box), _i, ctypes.c_char_p,
                                 _i, _i, _i, _i, _i, _d, ctypes.POINTER(Box), _i, ctypes.POINTER(_i)]),
    "bamrex_amr_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(AmrDesc), _vp]),
    "bamrex_amr_destroy": (_i, [_vp]),
    "bamrex_amr_last_error": (ctypes.c_char_p, [_vp]),
    "bamrex_amr_finest_level": (_i, [_vp]),
    "bamrex_amr_level": (_vp, [_vp, _i]),
    "bamrex_amr_boxes": (_i, [_vp, _i, ctypes.POINTER(Box), _i, ctypes.POINTER(_i)]),
    "bamrex_amr_set_level_boxes": (_i, [_vp, _i, ctypes.POINTER(Box), _i]),
    "bamrex_amr_regrid": (_i, [_vp, _i, _d]),
    "bamrex_amr_avg_down_all": (_i, [_vp]),
    "bamrex_amr_coarse_step": (_i, [_vp, _d, _dp, _dp]),
    "bamrex_amr_set_regrid_int": (_i, [_vp, _i]),
    "bamrex_amr_set_graph": (_i, [_vp, _i]),
    "bamrex_amr_graph_stats": (_i, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong),
                                    ctypes.POINTER(ctypes.c_longlong)]),
    "bamrex_amr_set_body": (_i, [_vp, ctypes.POINTER(BodyDesc)]),
    "bamrex_amr_get_stepping": (_i, [_vp, ctypes.POINTER(AmrStepping)]),
    "bamrex_amr_set_stepping": (_i, [_vp, ctypes.POINTER(AmrStepping)]),
    "bamrex_amr_dt_level": (_i, [_vp, _dp]),
    "bamrex_amr_conserved_sums": (_i, [_vp, _dp]),
    "bamrex_helmholtz_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(HelmholtzDesc), _vp]),
    "bamrex_helmholtz_destroy": (_i, [_vp]),
    "bamrex_helmholtz_last_error": (ctypes.c_char_p, [_vp]),
    "bamrex_helmholtz_num_levels": (_i, [_vp]),
    "bamrex_helmholtz_set_scalars": (_i, [_vp, _d, _d, _d]),
    "bamrex_helmholtz_set_acoeffs": (_i, [_vp, _vp, _d]),
    "bamrex_helmholtz_set_bcoeffs": (_i, [_vp, _vp, _vp, _vp]),
    "bamrex_helmholtz_set_bcoeffs_from_cell": (_i, [_vp, _vp]),
    "bamrex_helmholtz_set_ccoeffs": (_i, [_vp, _vp]),
    "bamrex_helmholtz_apply": (_i, [_vp, _vp, _vp]),
    "bamrex_helmholtz_smooth": (_i, [_vp, _vp, _vp, _i]),
    "bamrex_helmholtz_vcycle": (_i, [_vp, _vp, _vp]),
    "bamrex_helmholtz_solve": (_i, [_vp, _vp, _vp, _d, _d, _i, _i, ctypes.POINTER(_i), _dp]),
    "bamrex_helmholtz_launches": (_ll, [_vp]),
    "bamrex_precnet_create": (_i, [ctypes.POINTER(_vp), _i, _i, _i, ctypes.c_ulonglong, _vp]),
    "bamrex_precnet_destroy": (_i, [_vp]),
    "bamrex_precnet_last_error": (ctypes.c_char_p, [_vp]),
    "bamrex_precnet_num_params": (_i, [_vp]),
    "bamrex_precnet_resize": (_i, [_vp, _i, _i, _i]),
    "bamrex_precnet_get_weights": (_i, [_vp, _vp]),
    "bamrex_precnet_set_weights": (_i, [_vp, _vp]),
    "bamrex_precnet_forward": (_i, [_vp, _vp, _vp]),
    "bamrex_precnet_backward": (_i, [_vp, _vp, _vp]),
    "bamrex_precnet_train_step": (_i, [_vp, _vp, _vp, ctypes.c_float, _dp]),
    "bamrex_precnet_set_tensor_cores": (_i, [_vp, _i]),
    "bamrex_helmholtz_solve_learned": (_i, [_vp, _vp, _i, _vp, _vp, _d, _d, _i, _i, ctypes.POINTER(_i),
                                            ctypes.POINTER(_i), _dp, ctypes.POINTER(_i)]),
    "bamrex_imex_create": (_i, [ctypes.POINTER(_vp), ctypes.POINTER(ImexDesc), _vp]),
    "bamrex_imex_destroy": (_i, [_vp]),
    "bamrex_imex_last_error": (ctypes.c_char_p, [_vp]),
    "bamrex_imex_set_state": (_i, [_vp, _vp, _vp]),
    "bamrex_imex_get_state": (_i, [_vp, _vp, _vp]),
    "bamrex_imex_est_time_step": (_i, [_vp, _dp]),
    "bamrex_imex_step": (_i, [_vp, _d, ctypes.POINTER(_i), _dp]),
    "bamrex_imex_set_precnet": (_i, [_vp, _vp, _i]),
    "bamrex_imex_operator": (_vp, [_vp]),
    "bamrex_imex_field": (_i, [_vp, _i, _vp, ctypes.POINTER(_ll)]),
    "bamrex_imex_launches": (_ll, [_vp]),
}

_LIB = None


def lib() -> ctypes.CDLL:
    """Load libbamrex_cuda.so (raises if it is absent: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libbamrex_cuda.so is not built (%s); run `python -m bamrex_b200.build`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def profile_enable(on=True) -> bool:
    """Turn the library's host-side region timers on or off; returns the
    previous setting."""
    return bool(lib().bamrex_profile_enable(1 if on else 0))


def profile_reset() -> None:
    lib().bamrex_profile_reset()


def profile_report() -> list:
    """The region timers as [(name, calls, total_s, avg_ms, max_ms)], largest
    total first."""
    need = ctypes.c_int(0)
    lib().bamrex_profile_report(None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(max(1, need.value))
    lib().bamrex_profile_report(buf, len(buf), ctypes.byref(need))
    rows = []
    for line in buf.value.decode().splitlines()[1:]:
        name, calls, total, avg, mx = line.rsplit(" ", 4)
        rows.append((name, int(calls), float(total), float(avg), float(mx)))
    return rows


def check(rc: int, level_handle=None, amr_handle=None) -> None:
    if rc == OK:
        return
    L = lib()
    msg = L.bamrex_last_error().decode()
    if level_handle is not None:
        lm = L.bamrex_level_last_error(level_handle)
        if lm:
            msg = lm.decode() or msg
    if amr_handle is not None:
        am = L.bamrex_amr_last_error(amr_handle)
        if am:
            msg = am.decode() or msg
    raise BamrexError(rc, msg or L.bamrex_status_string(rc).decode())
