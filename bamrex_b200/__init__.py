"""bamrex_b200: the explicit finite-volume path of BAMReX on B200 (sm_100a).

MUSCL-Hancock reconstruction with half-step evolution, HLLC / SLIC / FORCE /
Lax-Friedrichs interface fluxes, the split conservative update, ghost fill
and the CFL reduction, in hand-written CUDA kernels behind the C ABI of
``libbamrex_cuda.so`` (include/bamrex_cuda.h).  This package holds the build
recipe (``bamrex_b200.build``), the ctypes binding (``_abi``), the Python
mirror of the reference's level surface (``level``) and seeded problem
generators (``problems``).
"""
from . import problems
from ._abi import (XSWEEP_AUTO, XSWEEP_MARCH, XSWEEP_ROWS, STAGING_AUTO, STAGING_REGISTERS, STAGING_TMA, STAGING_WAVE, BC_PERIODIC, BC_REFLECTIVE, BC_TRANSMISSIVE, FORCE, FP32_STORAGE, FP64, HLLC, LAX_FRIEDRICHS,
                   LIMITERS, METHODS, MINBEE, MUSCL_HANCOCK, SLIC, SUPERBEE, VAN_ALBADA, VAN_LEER, BamrexError, lib,
                   SDF_PLANE, SDF_SPHERE, SDF_CYLINDER, SDF_UNION, SDF_INTERSECTION, RB_REFLECTIVE, RB_NO_SLIP,
                   RB_FOEXTRAP, RB_BCS, GFM_GHOST, GFM_INTERFACE, GFM_FILL, profile_enable, profile_report,
                   profile_reset)
from .level import (Level, Packing, Parm, compute_flux, compute_flux_LR, conservative_update, decompose,
                    sweep_box, sweep_update)

__all__ = [
    "Level", "Packing", "Parm", "compute_flux", "compute_flux_LR", "conservative_update", "decompose", "sweep_box",
    "sweep_update", "problems", "lib", "BamrexError", "XSWEEP_AUTO", "XSWEEP_ROWS", "XSWEEP_MARCH", "STAGING_AUTO", "STAGING_REGISTERS", "STAGING_TMA", "STAGING_WAVE", "MUSCL_HANCOCK", "HLLC", "SLIC", "FORCE", "LAX_FRIEDRICHS",
    "METHODS", "LIMITERS", "MINBEE", "VAN_LEER", "VAN_ALBADA", "SUPERBEE", "BC_TRANSMISSIVE", "BC_PERIODIC",
    "BC_REFLECTIVE", "SDF_PLANE", "SDF_SPHERE", "SDF_CYLINDER", "SDF_UNION", "SDF_INTERSECTION", "RB_REFLECTIVE",
    "RB_NO_SLIP", "RB_FOEXTRAP", "RB_BCS", "GFM_GHOST", "GFM_INTERFACE", "GFM_FILL", "profile_enable",
    "profile_report", "profile_reset",
]
