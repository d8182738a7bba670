"""Python mirror of the pressure Helmholtz operator (MLABecLaplacianGrad,
Source/LinearSolver/MLALaplacianGrad.H) and its solve (setup_pressure_op /
solve_pressure, Source/IMEX/IMEX_O1.cpp:570-640) over the C ABI.

Vectors are numpy float64 arrays of shape (nz, ny, nx) (nz = 1 in 2D), or
CUDA tensors of the same shape; face coefficients have one more entry along
their direction.  All work runs in libbamrex_cuda.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._abi import HelmholtzDesc, LINOP_PERIODIC, check, lib


def _ptr(a):
    """(pointer, keep-alive) of a numpy array or a CUDA tensor."""
    if a is None:
        return None, None
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous()
        return ctypes.c_void_p(a.data_ptr()), a
    arr = np.ascontiguousarray(a, dtype=np.float64)
    return ctypes.c_void_p(arr.ctypes.data), arr


class Helmholtz:
    """y = A a x - B div(b grad x) + C c . grad x on one box covering the
    domain, with a multigrid hierarchy for smoothing and solves."""

    def __init__(self, spacedim, n, prob_lo=None, prob_hi=None, bc_lo=None, bc_hi=None, max_levels=0, nu1=2,
                 nu2=2, bottom_sweeps=16, stream=None):
        self.D = spacedim
        self.n = tuple(int(x) for x in n) + (1,) * (3 - len(n))
        d = HelmholtzDesc()
        d.spacedim = spacedim
        for q in range(3):
            d.n[q] = self.n[q]
            d.prob_lo[q] = float(prob_lo[q]) if prob_lo is not None and q < len(prob_lo) else 0.0
            d.prob_hi[q] = float(prob_hi[q]) if prob_hi is not None and q < len(prob_hi) else 1.0
            d.bc_lo[q] = int(bc_lo[q]) if bc_lo is not None and q < len(bc_lo) else LINOP_PERIODIC
            d.bc_hi[q] = int(bc_hi[q]) if bc_hi is not None and q < len(bc_hi) else LINOP_PERIODIC
        d.max_levels, d.nu1, d.nu2, d.bottom_sweeps = max_levels, nu1, nu2, bottom_sweeps
        self._h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        check(lib().bamrex_helmholtz_create(ctypes.byref(self._h), ctypes.byref(d), st))
        self.shape = (self.n[2], self.n[1], self.n[0])

    def close(self):
        if self._h:
            lib().bamrex_helmholtz_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != 0:
            msg = lib().bamrex_helmholtz_last_error(self._h)
            from ._abi import BamrexError
            raise BamrexError(rc, (msg or b"").decode() or lib().bamrex_last_error().decode())

    @property
    def num_levels(self):
        return lib().bamrex_helmholtz_num_levels(self._h)

    def face_shape(self, d):
        s = list(self.shape)
        s[2 - d] += 1
        return tuple(s)

    # MLABecLaplacianGrad set-up
    def setScalars(self, a, b, c=0.0):
        self._ck(lib().bamrex_helmholtz_set_scalars(self._h, a, b, c))

    def setACoeffs(self, alpha):
        if np.isscalar(alpha):
            self._ck(lib().bamrex_helmholtz_set_acoeffs(self._h, None, float(alpha)))
        else:
            p, keep = _ptr(alpha)
            self._ck(lib().bamrex_helmholtz_set_acoeffs(self._h, p, 0.0))

    def setBCoeffs(self, faces):
        ps = [_ptr(f) for f in faces] + [(None, None)] * (3 - len(faces))
        self._ck(lib().bamrex_helmholtz_set_bcoeffs(self._h, ps[0][0], ps[1][0], ps[2][0]))

    def setBCoeffsFromCell(self, beta_cc):
        p, keep = _ptr(beta_cc)
        self._ck(lib().bamrex_helmholtz_set_bcoeffs_from_cell(self._h, p))

    def setCCoeffs(self, c):
        p, keep = _ptr(c)
        self._ck(lib().bamrex_helmholtz_set_ccoeffs(self._h, p))

    # operations
    def apply(self, x):
        xp, kx = _ptr(x)
        y = np.empty(self.shape)
        self._ck(lib().bamrex_helmholtz_apply(self._h, xp, ctypes.c_void_p(y.ctypes.data)))
        return y

    def smooth(self, phi, rhs, redblack):
        out = np.array(phi, dtype=np.float64, copy=True)
        rp, kr = _ptr(rhs)
        self._ck(lib().bamrex_helmholtz_smooth(self._h, ctypes.c_void_p(out.ctypes.data), rp, redblack))
        return out

    def vcycle(self, r):
        rp, kr = _ptr(r)
        z = np.empty(self.shape)
        self._ck(lib().bamrex_helmholtz_vcycle(self._h, ctypes.c_void_p(z.ctypes.data), rp))
        return z

    def solve(self, rhs, x0=None, tol_rel=1e-12, tol_abs=0.0, max_iter=1000, use_graph=True):
        """BiCGStab + V-cycle; returns (x, iterations, relative residual)."""
        x = np.zeros(self.shape) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        rp, kr = _ptr(rhs)
        it = ctypes.c_int()
        rr = ctypes.c_double()
        self._ck(lib().bamrex_helmholtz_solve(self._h, ctypes.c_void_p(x.ctypes.data), rp, tol_rel, tol_abs, max_iter,
                                              1 if use_graph else 0, ctypes.byref(it), ctypes.byref(rr)))
        return x, it.value, rr.value

    def solve_device(self, x, rhs, tol_rel=1e-12, tol_abs=0.0, max_iter=1000, use_graph=True):
        """The same on CUDA tensors (x updated in place)."""
        it = ctypes.c_int()
        rr = ctypes.c_double()
        self._ck(lib().bamrex_helmholtz_solve(self._h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(rhs.data_ptr()),
                                              tol_rel, tol_abs, max_iter, 1 if use_graph else 0, ctypes.byref(it),
                                              ctypes.byref(rr)))
        return it.value, rr.value

    def launches(self):
        return lib().bamrex_helmholtz_launches(self._h)


def _main(argv=None):
    """python -m bamrex_b200.helmholtz [--n N] [--solves K]: the low-Mach
    pressure solve (lognormal density, beta = 1/rho) on the device, timed."""
    import argparse
    import time

    import torch

    from . import problems
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--tol", type=float, default=1e-8)
    a = ap.parse_args(argv)
    p = problems.low_mach_pressure_problem(n=a.n)
    h = Helmholtz(2, (a.n, a.n))
    h.setScalars(1.0, p["B"], 0.0)
    h.setACoeffs(p["a"])
    h.setBCoeffsFromCell(p["beta_cc"])
    rhs = torch.from_numpy(p["rhs"].copy()).cuda()
    x = torch.zeros_like(rhs)
    for k in range(a.solves):
        x.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, rr = h.solve_device(x, rhs, tol_rel=a.tol)
        torch.cuda.synchronize()
        print("solve %d: %d iterations, relative residual %.2e, %.2f ms" % (k, it, rr, 1e3 * (time.perf_counter() - t0)))
    h.close()


if __name__ == "__main__":
    _main()
