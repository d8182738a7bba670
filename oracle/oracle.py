"""TEST INFRASTRUCTURE ONLY -- ctypes front end of the CPU oracle.

The oracle (bamrex_oracle.c) is a plain-C restatement of BAMReX's explicit
finite-volume path.  It is the parity checker for the CUDA kernels and the
timed CPU baseline; it is never part of the product path.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.

Layout conventions follow amrex::Array4 (Source/Fluxes/Fluxes.H call surface):
a box's fab covers the valid box grown by ``ngrow`` in every active
direction, components slowest, i fastest.  Global ("domain") arrays used by
the tests are numpy arrays of shape (NC, nz, ny, nx) indexed from the domain
lower corner.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# NumericalMethods::Method (Source/NumericalMethods.H:10-19)
MUSCL_HANCOCK, HLLC, IMEX, RCM, SLIC, FORCE, LAX_FRIEDRICHS = range(7)
# Limiter enum order (Source/Fluxes/Limiters.H:13)
MINBEE, VAN_LEER, VAN_ALBADA, SUPERBEE = range(4)
LIMITERS = {"minbee": MINBEE, "van_leer": VAN_LEER, "van_albada": VAN_ALBADA, "superbee": SUPERBEE}
# boundary kinds
TRANSMISSIVE, PERIODIC, REFLECTIVE = range(3)
MAX_NCOMP = 8


class _OParm(ctypes.Structure):
    _fields_ = [
        ("adiabatic", ctypes.c_double),
        ("epsilon", ctypes.c_double),
        ("limiter", ctypes.c_int),
        ("limiter_indices", ctypes.c_uint * MAX_NCOMP),
        ("limit_on_primv", ctypes.c_ubyte * MAX_NCOMP),
        ("need_primitive_for_limiting", ctypes.c_ubyte),
    ]


class _OA4(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.POINTER(ctypes.c_double)),
        ("jstride", ctypes.c_longlong),
        ("kstride", ctypes.c_longlong),
        ("nstride", ctypes.c_longlong),
        ("begin", ctypes.c_int * 3),
        ("end", ctypes.c_int * 3),
        ("ncomp", ctypes.c_int),
    ]


class _OLevel(ctypes.Structure):
    _fields_ = [
        ("D", ctypes.c_int),
        ("nboxes", ctypes.c_int),
        ("ngrow", ctypes.c_int),
        ("dom_lo", ctypes.c_int * 3),
        ("dom_hi", ctypes.c_int * 3),
        ("bc_lo", ctypes.c_int * 3),
        ("bc_hi", ctypes.c_int * 3),
        ("dx", ctypes.c_double * 3),
        ("boxes", ctypes.POINTER(ctypes.c_int)),
        ("offsets", ctypes.POINTER(ctypes.c_longlong)),
        ("strides", ctypes.POINTER(ctypes.c_longlong)),
    ]


_LIBS: dict[bool, ctypes.CDLL] = {}
# The timing build (fast=True): the committed x86-64-v3 library, or one
# compiled for this host's CPU by use_native_build().
_FAST = {"path": os.path.join(_HERE, "liboracle_fast.so"), "march": "x86-64-v3"}


def use_native_build() -> str:
    """Compile the timing build with -march=native (the reference's own flag,
    CMakeLists.txt:8) for the CPU this process runs on, into a temporary
    directory, and use it for every later fast=True call.  Returns the -march
    value in use ("native", or "x86-64-v3" when the compile fails or the
    timing library is already loaded)."""
    import tempfile
    if True in _LIBS:
        return _FAST["march"]
    d = tempfile.mkdtemp(prefix="bamrex_oracle_native_")
    out = os.path.join(d, "liboracle_native.so")
    r = subprocess.run(["gcc", "-O3", "-funroll-loops", "-march=native", "-fPIC", "-shared", "-fopenmp", "-o", out,
                        os.path.join(_HERE, "bamrex_oracle.c")], capture_output=True)
    if r.returncode == 0 and os.path.exists(out):
        _FAST.update(path=out, march="native")
    return _FAST["march"]


def host_cpu() -> dict:
    """Model name and the widest x86 vector extension of this host's CPU."""
    model, flags = "unknown", set()
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    isa = "avx512" if "avx512f" in flags else ("avx2" if "avx2" in flags else "sse")
    return {"model": model, "isa": isa}


def build(force: bool = False) -> None:
    """Compile the oracle libraries in place (make)."""
    targets = [os.path.join(_HERE, n) for n in ("liboracle.so", "liboracle_fast.so")]
    src = os.path.join(_HERE, "bamrex_oracle.c")
    if force or any(not os.path.exists(t) or os.path.getmtime(t) < os.path.getmtime(src) for t in targets):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib(fast: bool = False) -> ctypes.CDLL:
    if fast in _LIBS:
        return _LIBS[fast]
    build()
    L = ctypes.CDLL(_FAST["path"] if fast else os.path.join(_HERE, "liboracle.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    L.oracle_consv_from_primv.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, dp]
    L.oracle_primv_from_consv.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, dp]
    L.oracle_euler_flux.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, dp]
    L.oracle_wave_speed_toro.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, dp]
    L.oracle_hllc_face.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double, dp]
    L.oracle_slope_limit.argtypes = [ctypes.c_int, ctypes.c_double]
    L.oracle_slope_limit.restype = ctypes.c_double
    L.oracle_minmod.argtypes = [ctypes.c_double, ctypes.c_double]
    L.oracle_minmod.restype = ctypes.c_double
    L.oracle_compute_flux.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, _OA4, _OA4, dp,
                                      ctypes.c_double, ctypes.POINTER(_OParm)]
    L.oracle_compute_flux.restype = ctypes.c_int
    L.oracle_compute_flux_LR.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip, _OA4, _OA4, _OA4,
                                         dp, ctypes.c_double, ctypes.POINTER(_OParm)]
    L.oracle_compute_flux_LR.restype = ctypes.c_int
    L.oracle_sweep_update.argtypes = [ctypes.c_int, ctypes.c_int, ip, ip, _OA4, _OA4, _OA4, dp, ctypes.c_double]
    L.oracle_conservative_update.argtypes = [ctypes.c_int, ip, ip, _OA4, _OA4, ctypes.POINTER(_OA4),
                                             ctypes.c_double, dp]
    L.oracle_fill_boundary.argtypes = [ctypes.POINTER(_OLevel), dp]
    L.oracle_fill_boundary.restype = ctypes.c_int
    L.oracle_max_wave_speed.argtypes = [ctypes.POINTER(_OLevel), dp, ctypes.c_double, ctypes.c_double]
    L.oracle_max_wave_speed.restype = ctypes.c_double
    L.oracle_est_time_step.argtypes = [ctypes.POINTER(_OLevel), dp, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double]
    L.oracle_est_time_step.restype = ctypes.c_double
    ppd = ctypes.POINTER(dp)
    ppll = ctypes.POINTER(ctypes.POINTER(ctypes.c_longlong))
    L.oracle_advance_explicit.argtypes = [ctypes.POINTER(_OLevel), dp, dp, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.POINTER(_OParm), ppd, ppll, ppll, ctypes.c_int]
    L.oracle_advance_explicit.restype = ctypes.c_int
    L.oracle_sweep_dir.argtypes = [ctypes.POINTER(_OLevel), dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(_OParm)]
    L.oracle_sweep_dir.restype = ctypes.c_int
    L.oracle_num_threads.restype = ctypes.c_int
    _LIBS[fast] = L
    return L


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iv(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


@dataclass
class Parm:
    """The explicit-path fields of the reference Parm (Source/System/Parm.H:14-61)
    with FluidSystem::set_parm_defaults (Source/System/FluidSystem.cpp:52-71)."""
    D: int
    adiabatic: float = 1.4
    epsilon: float = 1.0
    limiter: int = VAN_LEER
    limiter_indices: list = field(default=None)
    limit_on_primv: list = field(default=None)

    def __post_init__(self):
        if self.limiter_indices is None:
            self.limiter_indices = [1 + self.D] * MAX_NCOMP  # UInd::E
        if self.limit_on_primv is None:
            self.limit_on_primv = [False] * MAX_NCOMP

    def to_c(self) -> _OParm:
        p = _OParm()
        p.adiabatic = self.adiabatic
        p.epsilon = self.epsilon
        p.limiter = self.limiter
        for n in range(MAX_NCOMP):
            p.limiter_indices[n] = int(self.limiter_indices[n])
            p.limit_on_primv[n] = 1 if self.limit_on_primv[n] else 0
        p.need_primitive_for_limiting = 1 if any(self.limit_on_primv[: self.D + 2]) else 0
        return p


def array4(a: np.ndarray, begin) -> _OA4:
    """View a C-contiguous (ncomp, nz, ny, nx) float64 array as an Array4 whose
    first cell is ``begin``."""
    assert a.ndim == 4
    v = _OA4()
    v.p = _dp(a)
    nc, nz, ny, nx = a.shape
    v.jstride, v.kstride, v.nstride = nx, nx * ny, nx * ny * nz
    for d in range(3):
        v.begin[d] = int(begin[d])
    v.end[0], v.end[1], v.end[2] = begin[0] + nx, begin[1] + ny, begin[2] + nz
    v.ncomp = nc
    return v


# ---------------------------------------------------------------- pointwise
def consv_from_primv(D, q, adia, eps):
    q = np.ascontiguousarray(q, dtype=np.float64)
    u = np.zeros(D + 2)
    lib().oracle_consv_from_primv(D, _dp(q), adia, eps, _dp(u))
    return u


def primv_from_consv(D, u, adia, eps):
    u = np.ascontiguousarray(u, dtype=np.float64)
    q = np.zeros(D + 2)
    lib().oracle_primv_from_consv(D, _dp(u), adia, eps, _dp(q))
    return q


def euler_flux(D, dir, u, adia, eps):
    u = np.ascontiguousarray(u, dtype=np.float64)
    f = np.zeros(D + 2)
    lib().oracle_euler_flux(D, dir, _dp(u), adia, eps, _dp(f))
    return f


def wave_speed_toro(D, dir, uL, uR, adia, eps):
    uL = np.ascontiguousarray(uL, dtype=np.float64)
    uR = np.ascontiguousarray(uR, dtype=np.float64)
    out = np.zeros(3)
    lib().oracle_wave_speed_toro(D, dir, _dp(uL), _dp(uR), adia, adia, eps, _dp(out))
    return out  # S_L, S_R, S_*


def hllc_face(D, dir, uL, uR, adia, eps):
    uL = np.ascontiguousarray(uL, dtype=np.float64)
    uR = np.ascontiguousarray(uR, dtype=np.float64)
    f = np.zeros(D + 2)
    lib().oracle_hllc_face(D, dir, _dp(uL), _dp(uR), adia, eps, _dp(f))
    return f


def slope_limit(limiter, r):
    return lib().oracle_slope_limit(limiter, float(r))


def minmod(a, b):
    return lib().oracle_minmod(float(a), float(b))


# ---------------------------------------------------------------- box level
def compute_flux(D, method, dir, lo, hi, consv, consv_begin, dx, dt, parm: Parm):
    """Fluxes.H-style per-box flux.  ``consv`` is (NC, nz, ny, nx) starting at
    ``consv_begin``; returns the flux array on surroundingNodes(box, dir) and
    its begin corner."""
    NC = D + 2
    fhi = list(hi)
    fhi[dir] += 1
    shape = (NC, fhi[2] - lo[2] + 1, fhi[1] - lo[1] + 1, fhi[0] - lo[0] + 1)
    flux = np.full(shape, np.nan)
    cp = parm.to_c()
    rc = lib().oracle_compute_flux(D, method, dir, _iv(lo), _iv(hi), array4(flux, lo), array4(consv, consv_begin),
                                   _dp(np.asarray(dx, dtype=np.float64)), dt, ctypes.byref(cp))
    if rc != 0:
        raise ValueError("unsupported method")
    return flux


def compute_flux_LR(D, kind, dir, lo, hi, cL, cR, begin, dx, dt, parm: Parm):
    NC = D + 2
    fhi = list(hi)
    fhi[dir] += 1
    shape = (NC, fhi[2] - lo[2] + 1, fhi[1] - lo[1] + 1, fhi[0] - lo[0] + 1)
    flux = np.full(shape, np.nan)
    cp = parm.to_c()
    rc = lib().oracle_compute_flux_LR(D, kind, dir, _iv(lo), _iv(hi), array4(flux, lo), array4(cL, begin),
                                      array4(cR, begin), _dp(np.asarray(dx, dtype=np.float64)), dt,
                                      ctypes.byref(cp))
    if rc != 0:
        raise ValueError("unsupported kind")
    return flux


# ---------------------------------------------------------------- level
def decompose(D, dom_lo, dom_hi, max_grid_size):
    """Chop the domain into boxes of at most ``max_grid_size`` cells per side
    (list of (lo, hi) triples)."""
    ranges = []
    for d in range(3):
        if d >= D:
            ranges.append([(0, 0)])
            continue
        r = []
        s = dom_lo[d]
        while s <= dom_hi[d]:
            e = min(s + max_grid_size - 1, dom_hi[d])
            r.append((s, e))
            s = e + 1
        ranges.append(r)
    boxes = []
    for (zl, zh) in ranges[2]:
        for (yl, yh) in ranges[1]:
            for (xl, xh) in ranges[0]:
                boxes.append(((xl, yl, zl), (xh, yh, zh)))
    return boxes


class LevelLayout:
    """All fabs of one level in one flat float64 buffer."""

    def __init__(self, D, dom_lo, dom_hi, boxes, ngrow, dx, bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)):
        self.D, self.NC, self.ngrow = D, D + 2, ngrow
        self.dom_lo = tuple(int(x) for x in dom_lo)
        self.dom_hi = tuple(int(x) for x in dom_hi)
        self.boxes = [(tuple(int(x) for x in lo), tuple(int(x) for x in hi)) for lo, hi in boxes]
        self.dx = tuple(float(x) for x in dx) + (1.0,) * (3 - len(dx))
        self.bc_lo, self.bc_hi = tuple(bc_lo), tuple(bc_hi)
        offs, strides, begins, shapes = [], [], [], []
        off = 0
        for lo, hi in self.boxes:
            g = [ngrow if d < D else 0 for d in range(3)]
            b = [lo[d] - g[d] for d in range(3)]
            n = [hi[d] - lo[d] + 1 + 2 * g[d] for d in range(3)]
            offs.append(off)
            strides += [n[0], n[0] * n[1], n[0] * n[1] * n[2]]
            begins.append(b)
            shapes.append((self.NC, n[2], n[1], n[0]))
            off += self.NC * n[0] * n[1] * n[2]
        self.size = off
        self.offsets = np.array(offs, dtype=np.int64)
        self.strides = np.array(strides, dtype=np.int64)
        self.begins, self.shapes = begins, shapes
        self._boxes_c = np.array([list(lo) + list(hi) for lo, hi in self.boxes], dtype=np.int32).ravel()
        L = _OLevel()
        L.D, L.nboxes, L.ngrow = D, len(self.boxes), ngrow
        for d in range(3):
            L.dom_lo[d], L.dom_hi[d] = self.dom_lo[d], self.dom_hi[d]
            L.bc_lo[d], L.bc_hi[d] = int(self.bc_lo[d]), int(self.bc_hi[d])
            L.dx[d] = self.dx[d]
        L.boxes = self._boxes_c.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        L.offsets = self.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
        L.strides = self.strides.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
        self._c = L

    def alloc(self) -> np.ndarray:
        return np.full(self.size, np.nan)

    def fab(self, buf, b) -> np.ndarray:
        nc, nz, ny, nx = self.shapes[b]
        o = int(self.offsets[b])
        return buf[o:o + nc * nz * ny * nx].reshape(self.shapes[b])

    def domain_shape(self):
        n = [self.dom_hi[d] - self.dom_lo[d] + 1 for d in range(3)]
        return (self.NC, n[2], n[1], n[0])

    def scatter(self, buf, glob):
        """Copy a global (NC, nz, ny, nx) array into the valid cells of every fab."""
        for b, (lo, hi) in enumerate(self.boxes):
            f = self.fab(buf, b)
            bg = self.begins[b]
            f[:, lo[2] - bg[2]:hi[2] - bg[2] + 1, lo[1] - bg[1]:hi[1] - bg[1] + 1, lo[0] - bg[0]:hi[0] - bg[0] + 1] = \
                glob[:, lo[2] - self.dom_lo[2]:hi[2] - self.dom_lo[2] + 1,
                     lo[1] - self.dom_lo[1]:hi[1] - self.dom_lo[1] + 1,
                     lo[0] - self.dom_lo[0]:hi[0] - self.dom_lo[0] + 1]

    def gather(self, buf) -> np.ndarray:
        glob = np.full(self.domain_shape(), np.nan)
        for b, (lo, hi) in enumerate(self.boxes):
            f = self.fab(buf, b)
            bg = self.begins[b]
            glob[:, lo[2] - self.dom_lo[2]:hi[2] - self.dom_lo[2] + 1,
                 lo[1] - self.dom_lo[1]:hi[1] - self.dom_lo[1] + 1,
                 lo[0] - self.dom_lo[0]:hi[0] - self.dom_lo[0] + 1] = \
                f[:, lo[2] - bg[2]:hi[2] - bg[2] + 1, lo[1] - bg[1]:hi[1] - bg[1] + 1, lo[0] - bg[0]:hi[0] - bg[0] + 1]
        return glob

    # -- oracle calls
    def fill_boundary(self, buf, fast=False) -> int:
        return lib(fast).oracle_fill_boundary(ctypes.byref(self._c), _dp(buf))

    def max_wave_speed(self, buf, adia, eps, fast=False) -> float:
        return lib(fast).oracle_max_wave_speed(ctypes.byref(self._c), _dp(buf), adia, eps)

    def est_time_step(self, buf, adia, eps, cfl, fast=False) -> float:
        return lib(fast).oracle_est_time_step(ctypes.byref(self._c), _dp(buf), adia, eps, cfl)

    def advance_explicit(self, S1, S2, time, dt, method, parm: Parm, nthreads=0, fast=False):
        """One split step (advance_explicit).  S1 must be ghost-filled; S2 is
        scratch.  The result is left in S1."""
        cp = parm.to_c()
        rc = lib(fast).oracle_advance_explicit(ctypes.byref(self._c), _dp(S1), _dp(S2), time, dt, method,
                                               ctypes.byref(cp), None, None, None, nthreads)
        if rc != 0:
            raise ValueError("oracle advance failed")

    def sweep_dir(self, Sin, Sout, d, dt, method, parm: Parm, fast=False):
        """One sweep in direction d: Sout's valid cells from ghost-filled Sin."""
        cp = parm.to_c()
        if lib(fast).oracle_sweep_dir(ctypes.byref(self._c), _dp(Sin), _dp(Sout), d, dt, method, ctypes.byref(cp)) != 0:
            raise ValueError("oracle sweep failed")

    def advance_explicit_fluxes(self, S1, S2, time, dt, method, parm: Parm, nthreads=0, fast=False):
        """advance_explicit that also returns the fluxes of every sweep:
        out[d][b] is a (NC, nz, ny, nx) array on surroundingNodes(box b, d)
        (the reference's fluxes[d] MultiFab, unscaled)."""
        cp = parm.to_c()
        bufs, offs, strs, shapes = [], [], [], []
        for d in range(3):
            if d >= self.D:
                bufs.append(np.zeros(1))
                offs.append(np.zeros(max(1, len(self.boxes)), dtype=np.int64))
                strs.append(np.zeros(3 * max(1, len(self.boxes)), dtype=np.int64))
                shapes.append([])
                continue
            o, st, sh, acc = [], [], [], 0
            for lo, hi in self.boxes:
                n = [hi[q] - lo[q] + 1 + (1 if q == d else 0) for q in range(3)]
                o.append(acc)
                st += [n[0], n[0] * n[1], n[0] * n[1] * n[2]]
                sh.append((self.NC, n[2], n[1], n[0]))
                acc += self.NC * n[0] * n[1] * n[2]
            bufs.append(np.full(acc, np.nan))
            offs.append(np.array(o, dtype=np.int64))
            strs.append(np.array(st, dtype=np.int64))
            shapes.append(sh)
        dp = ctypes.POINTER(ctypes.c_double)
        llp = ctypes.POINTER(ctypes.c_longlong)
        fo = (dp * 3)(*[_dp(b) for b in bufs])
        oo = (llp * 3)(*[o.ctypes.data_as(llp) for o in offs])
        so = (llp * 3)(*[s.ctypes.data_as(llp) for s in strs])
        rc = lib(fast).oracle_advance_explicit(ctypes.byref(self._c), _dp(S1), _dp(S2), time, dt, method,
                                               ctypes.byref(cp), fo, oo, so, nthreads)
        if rc != 0:
            raise ValueError("oracle advance failed")
        out = []
        for d in range(self.D):
            per = []
            for b, sh in enumerate(shapes[d]):
                o = int(offs[d][b])
                per.append(bufs[d][o:o + int(np.prod(sh))].reshape(sh))
            out.append(per)
        return out


def num_threads(fast=False) -> int:
    return lib(fast).oracle_num_threads()


def run_level(layout: LevelLayout, glob0, parm: Parm, method, cfl, nsteps=None, stop_time=None,
              fixed_dt=None, nthreads=0, fast=False):
    """Driver restating Amr::coarseTimeStep for one level: initial dt from
    estTimeStep (computeInitialDt, Source/AmrLevelAdv.cpp:487-532), then per
    step FillPatch + advance_explicit + computeNewDt (:537-619) with the
    stop-time clamp.  Returns (final global state, time, list of dts)."""
    S1, S2 = layout.alloc(), layout.alloc()
    layout.scatter(S1, glob0)
    layout.fill_boundary(S1, fast)
    time = 0.0

    def new_dt(buf, t):
        if fixed_dt is not None:
            return fixed_dt
        dt0 = layout.est_time_step(buf, parm.adiabatic, parm.epsilon, cfl, fast)
        if stop_time is not None and stop_time >= 0.0:
            eps = 0.001 * dt0
            if t + dt0 > stop_time - eps:
                dt0 = stop_time - t
        return dt0

    dt = new_dt(S1, time)
    dts = []
    step = 0
    while True:
        if nsteps is not None and step >= nsteps:
            break
        if stop_time is not None and time >= stop_time:
            break
        S2[:] = S1
        layout.advance_explicit(S1, S2, time, dt, method, parm, nthreads, fast)
        layout.fill_boundary(S1, fast)
        time += dt
        dts.append(dt)
        step += 1
        dt = new_dt(S1, time)
    return layout.gather(S1), time, dts
