"""Python mirror of the first-order IMEX step over the C ABI.

``Imex`` is one box covering the domain, stepped by advance_imex_rk with the
SP111 tableau and the linearised pressure equation
(Source/IMEX/IMEX_RK.cpp:23-86, Source/IMEX/IMEX_O1.cpp:19-176); the
settings mirror IMEXSettings (Source/IMEX/IMEXSettings.H).  All work runs in
libbamrex_cuda.so (imex.cu); the pressure equation is solved by the
library's Helmholtz operator, optionally with the learned preconditioner.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import (ENTH_REUSE_PRESSURE, IMEX_RUSANOV, KE_EX, BamrexError, ImexDesc, check, lib)
from .level import Parm


class Imex:
    def __init__(self, spacedim, n, prob_lo, prob_hi, parm: Parm, bc_lo=None, bc_hi=None,
                 advection_flux=IMEX_RUSANOV, enthalpy_method=ENTH_REUSE_PRESSURE, ke_method=KE_EX, cfl=0.5,
                 tol_rel=0.0, tol_abs=0.0, max_iter=0, tableau=0, stream=None):
        self.D = spacedim
        self.NC = spacedim + 2
        self.n = tuple(n) + (1,) * (3 - len(n))
        d = ImexDesc()
        d.spacedim = spacedim
        for q in range(3):
            d.n[q] = self.n[q]
            d.prob_lo[q] = float(prob_lo[q]) if q < len(prob_lo) else 0.0
            d.prob_hi[q] = float(prob_hi[q]) if q < len(prob_hi) else 1.0
            d.bc_lo[q] = int(bc_lo[q]) if bc_lo is not None and q < len(bc_lo) else 0
            d.bc_hi[q] = int(bc_hi[q]) if bc_hi is not None and q < len(bc_hi) else 0
        d.parm = parm.to_c()
        d.advection_flux, d.enthalpy_method, d.ke_method = advection_flux, enthalpy_method, ke_method
        d.cfl, d.tol_rel, d.tol_abs, d.max_iter, d.tableau = cfl, tol_rel, tol_abs, max_iter, tableau
        self.dx = [(d.prob_hi[q] - d.prob_lo[q]) / self.n[q] for q in range(spacedim)]
        self._h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        check(lib().bamrex_imex_create(ctypes.byref(self._h), ctypes.byref(d), st))
        self.shape = (self.n[2], self.n[1], self.n[0])

    def close(self):
        if self._h:
            lib().bamrex_imex_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != 0:
            m = lib().bamrex_imex_last_error(self._h)
            raise BamrexError(rc, (m or b"").decode() or lib().bamrex_last_error().decode())

    def set_state(self, U, p=None):
        """U: (D+2, nz, ny, nx) conserved state; p: (nz, ny, nx) pressure or
        None (from the state)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.NC,) + self.shape
        pp = None
        if p is not None:
            p = np.ascontiguousarray(p, dtype=np.float64)
            assert p.shape == self.shape
            pp = ctypes.c_void_p(p.ctypes.data)
        self._ck(lib().bamrex_imex_set_state(self._h, ctypes.c_void_p(U.ctypes.data), pp))

    def get_state(self):
        U = np.empty((self.NC,) + self.shape)
        p = np.empty(self.shape)
        self._ck(lib().bamrex_imex_get_state(self._h, ctypes.c_void_p(U.ctypes.data), ctypes.c_void_p(p.ctypes.data)))
        return U, p

    def est_time_step(self) -> float:
        dt = ctypes.c_double()
        self._ck(lib().bamrex_imex_est_time_step(self._h, ctypes.byref(dt)))
        return dt.value

    def step(self, dt):
        """One IMEX step; returns (pressure-solve iterations, relative residual)."""
        it = ctypes.c_int()
        rr = ctypes.c_double()
        self._ck(lib().bamrex_imex_step(self._h, dt, ctypes.byref(it), ctypes.byref(rr)))
        return it.value, rr.value

    def set_precnet(self, net, mode=_abi.PRECOND_NETWORK_VCYCLE):
        self._ck(lib().bamrex_imex_set_precnet(self._h, net._h if net is not None else None, mode))

    def field(self, which):
        """An intermediate field of the last step as an array (see
        BAMREX_IMEX_FIELD_* for the grids)."""
        cnt = ctypes.c_longlong()
        self._ck(lib().bamrex_imex_field(self._h, which, None, ctypes.byref(cnt)))
        out = np.empty(cnt.value)
        self._ck(lib().bamrex_imex_field(self._h, which, ctypes.c_void_p(out.ctypes.data), ctypes.byref(cnt)))
        D, (nz, ny, nx) = self.D, self.shape
        g = lambda m, d: m + (2 if d < D else 0)
        if which in (_abi.FIELD_UEX, _abi.FIELD_ENTHALPY):
            shp = (g(nz, 2), g(ny, 1), g(nx, 0))
            return out.reshape(((self.NC,) if which == _abi.FIELD_UEX else ()) + shp)
        if which in (_abi.FIELD_KE, _abi.FIELD_RHS, _abi.FIELD_PRESSURE):
            return out.reshape(self.shape)
        d = which - _abi.FIELD_FLUX_X
        shp = [nz, ny, nx]
        shp[2 - d] += 1
        return out.reshape((self.NC,) + tuple(shp))

    @property
    def launches(self):
        return lib().bamrex_imex_launches(self._h)
