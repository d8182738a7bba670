"""Python mirror of the reference's level-advance surface over the C ABI.

``Level`` follows AmrLevelAdv for the explicit methods
(Source/AmrLevelAdv.H:110-120, Source/AmrLevelAdv_advance.cpp:21-439,
Source/AmrLevelAdv.cpp:395-619): ``advance(time, dt, iteration, ncycle)``,
``estTimeStep()``, and ``run()`` for the coarse-step loop with the device
computing each new dt.  The per-box functions mirror Source/Fluxes/Fluxes.H.
All device work happens in libbamrex_cuda.so; this module only builds
arguments, so a missing library raises instead of falling back.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import Array4, Box, CParm, LevelDesc, check, lib


@dataclass
class Parm:
    """The Parm fields read by the explicit path (Source/System/Parm.H:14-61);
    unset fields take FluidSystem::set_parm_defaults."""
    spacedim: int
    adiabatic: float = 1.4
    epsilon: float = 1.0
    limiter: int = _abi.VAN_LEER
    limiter_indices: list = field(default=None)
    limit_on_primv: list = field(default=None)

    def to_c(self) -> CParm:
        p = CParm()
        check(lib().bamrex_parm_set_defaults(ctypes.byref(p), self.spacedim))
        p.adiabatic = self.adiabatic
        p.epsilon = self.epsilon
        p.limiter = int(self.limiter)
        if self.limiter_indices is not None:
            for n, v in enumerate(self.limiter_indices):
                p.limiter_indices[n] = int(v)
        if self.limit_on_primv is not None:
            for n, v in enumerate(self.limit_on_primv):
                p.limit_on_primv[n] = 1 if v else 0
        check(lib().bamrex_parm_init(ctypes.byref(p)))
        return p


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(getattr(stream, "cuda_stream"))


def array4_of(t, begin) -> Array4:
    """Array4 view of a contiguous (ncomp, nz, ny, nx) float64 device tensor
    whose first element is the cell ``begin``."""
    assert t.dim() == 4 and t.is_contiguous(), "expected a contiguous (ncomp, nz, ny, nx) tensor"
    nc, nz, ny, nx = t.shape
    a = Array4()
    a.p = t.data_ptr()
    a.jstride, a.kstride, a.nstride = nx, nx * ny, nx * ny * nz
    for d in range(3):
        a.begin[d] = int(begin[d])
    a.end[0], a.end[1], a.end[2] = int(begin[0]) + nx, int(begin[1]) + ny, int(begin[2]) + nz
    a.ncomp = nc
    return a


def _dx3(dx):
    v = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    for d, x in enumerate(dx):
        v[d] = float(x)
    return v


# ----------------------------------------------------------- per-box calls
def compute_flux(method, dir, spacedim, bx, flux, flux_begin, consv, consv_begin, dx, dt, parm: Parm,
                 stream=None, time=0.0):
    """compute_{MUSCL_hancock,HLLC,SLIC,force,LF}_flux on one box
    (Source/Fluxes/Fluxes.H); ``flux``/``consv`` are device tensors."""
    b = Box.make(*bx)
    cp = parm.to_c()
    check(lib().bamrex_compute_flux(method, dir, spacedim, time, ctypes.byref(b), array4_of(flux, flux_begin),
                                    array4_of(consv, consv_begin), _dx3(dx), dt, ctypes.byref(cp),
                                    _stream_ptr(stream)))


def compute_flux_LR(kind, dir, spacedim, bx, flux, flux_begin, cL, cR, c_begin, dx, dt, parm: Parm, stream=None,
                    time=0.0):
    b = Box.make(*bx)
    cp = parm.to_c()
    check(lib().bamrex_compute_flux_LR(kind, dir, spacedim, time, ctypes.byref(b), array4_of(flux, flux_begin),
                                       array4_of(cL, c_begin), array4_of(cR, c_begin), _dx3(dx), dt,
                                       ctypes.byref(cp), _stream_ptr(stream)))


def sweep_box(method, dir, spacedim, bx, Uout, out_begin, Uin, in_begin, dx, dt, parm: Parm, flux=None,
              flux_begin=None, stream=None):
    b = Box.make(*bx)
    cp = parm.to_c()
    fa = array4_of(flux, flux_begin) if flux is not None else Array4()
    check(lib().bamrex_sweep_box(method, dir, spacedim, ctypes.byref(b), array4_of(Uout, out_begin),
                                 array4_of(Uin, in_begin), fa, _dx3(dx), dt, ctypes.byref(cp), _stream_ptr(stream)))


def sweep_update(dir, spacedim, bx, Uout, out_begin, Uin, in_begin, flux, flux_begin, dx, dt, stream=None):
    b = Box.make(*bx)
    check(lib().bamrex_sweep_update(dir, spacedim, ctypes.byref(b), array4_of(Uout, out_begin),
                                    array4_of(Uin, in_begin), array4_of(flux, flux_begin), _dx3(dx), dt,
                                    _stream_ptr(stream)))


def conservative_update(spacedim, bx, out, out_begin, inp, in_begin, fluxes, flux_begins, dt, idx, stream=None):
    b = Box.make(*bx)
    arr = (Array4 * 3)()
    for d in range(spacedim):
        arr[d] = array4_of(fluxes[d], flux_begins[d])
    check(lib().bamrex_conservative_update(spacedim, ctypes.byref(b), array4_of(out, out_begin),
                                           array4_of(inp, in_begin), arr, dt, _dx3(idx), _stream_ptr(stream)))


# ----------------------------------------------------------- packing
def decompose(spacedim, dom_lo, dom_hi, max_grid_size):
    """Chop the domain into boxes of at most max_grid_size cells per side."""
    ranges = []
    for d in range(3):
        if d >= spacedim:
            ranges.append([(0, 0)])
            continue
        r, s = [], dom_lo[d]
        while s <= dom_hi[d]:
            e = min(s + max_grid_size - 1, dom_hi[d])
            r.append((s, e))
            s = e + 1
        ranges.append(r)
    return [((xl, yl, zl), (xh, yh, zh)) for (zl, zh) in ranges[2] for (yl, yh) in ranges[1]
            for (xl, xh) in ranges[0]]


class Packing:
    """Map between a global (NC, nz, ny, nx) array and the packed box-major
    layout of bamrex_level_copy_in/out."""

    def __init__(self, spacedim, dom_lo, boxes):
        self.NC = spacedim + 2
        self.dom_lo = tuple(dom_lo) + (0,) * (3 - len(dom_lo))
        self.boxes = boxes
        self.offsets = []
        off = 0
        for lo, hi in boxes:
            n = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1)
            self.offsets.append(off)
            off += n * self.NC
        self.size = off

    def _slices(self, lo, hi):
        L = self.dom_lo
        return (slice(None), slice(lo[2] - L[2], hi[2] - L[2] + 1), slice(lo[1] - L[1], hi[1] - L[1] + 1),
                slice(lo[0] - L[0], hi[0] - L[0] + 1))

    def pack(self, glob, out=None):
        out = np.empty(self.size) if out is None else out
        if len(self.boxes) == 1:
            out[:] = glob.reshape(-1) if glob.flags["C_CONTIGUOUS"] else np.ascontiguousarray(glob).reshape(-1)
            return out
        for (lo, hi), o in zip(self.boxes, self.offsets):
            blk = glob[self._slices(lo, hi)]
            out[o:o + blk.size] = blk.reshape(-1)
        return out

    def unpack(self, packed, glob=None):
        shape0 = None
        if glob is None:
            his = np.max(np.array([hi for _, hi in self.boxes]), axis=0)
            n = [his[d] - self.dom_lo[d] + 1 for d in range(3)]
            shape0 = (self.NC, n[2], n[1], n[0])
            glob = np.empty(shape0)
        for (lo, hi), o in zip(self.boxes, self.offsets):
            sl = self._slices(lo, hi)
            shp = (self.NC, hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1)
            glob[sl] = packed[o:o + int(np.prod(shp))].reshape(shp)
        return glob


# ----------------------------------------------------------- level
def body_desc(shapes, combine=_abi.SDF_UNION, rb_bc=_abi.RB_REFLECTIVE, stencil=2, fill_diagonals=False):
    """bamrex_body_desc of one or two shape dicts (kind, center, axis,
    radius, fluid_inside)."""
    if isinstance(shapes, dict):
        shapes = [shapes]
    d = _abi.BodyDesc()
    d.nshapes = len(shapes)
    d.combine = int(combine)
    for n, sh in enumerate(shapes):
        f = d.shapes[n]
        f.kind = int(sh["kind"])
        for q in range(3):
            c = sh.get("center", (0.0, 0.0, 0.0))
            a = sh.get("axis", (0.0, 0.0, 1.0))
            f.center[q] = float(c[q]) if q < len(c) else 0.0
            f.axis[q] = float(a[q]) if q < len(a) else 0.0
        f.radius = float(sh.get("radius", 0.0))
        f.fluid_inside = 1 if sh.get("fluid_inside", False) else 0
    d.rb_bc = int(rb_bc)
    d.stencil = int(stencil)
    d.fill_diagonals = 1 if fill_diagonals else 0
    return d


class Level:
    """One AMR level on the device (all boxes in one box table)."""

    def __init__(self, spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm: Parm, method=_abi.MUSCL_HANCOCK,
                 cfl=0.9, ngrow=2, bc_lo=None, bc_hi=None, stream=None, x_segment=0, s_segment=0,
                 precision=_abi.FP64, x_mode=_abi.XSWEEP_AUTO, staging=_abi.STAGING_AUTO, staging_dir=(0, 0, 0)):
        self.D, self.NC = spacedim, spacedim + 2
        self.boxes = [(tuple(lo) + (0,) * (3 - len(lo)), tuple(hi) + (0,) * (3 - len(hi))) for lo, hi in boxes]
        self.dom_lo = tuple(dom_lo) + (0,) * (3 - len(dom_lo))
        self.dom_hi = tuple(dom_hi) + (0,) * (3 - len(dom_hi))
        self.parm, self.method, self.cfl = parm, method, cfl
        d = LevelDesc()
        d.spacedim = spacedim
        d.domain = Box.make(self.dom_lo, self.dom_hi)
        for q in range(3):
            d.prob_lo[q] = float(prob_lo[q]) if q < len(prob_lo) else 0.0
            d.prob_hi[q] = float(prob_hi[q]) if q < len(prob_hi) else 1.0
            d.bc_lo[q] = int(bc_lo[q]) if bc_lo is not None and q < len(bc_lo) else 0
            d.bc_hi[q] = int(bc_hi[q]) if bc_hi is not None and q < len(bc_hi) else 0
        self._boxes_c = (Box * len(self.boxes))(*[Box.make(lo, hi) for lo, hi in self.boxes])
        d.boxes = self._boxes_c
        d.nboxes = len(self.boxes)
        d.ngrow = ngrow
        d.method = method
        d.cfl = cfl
        d.parm = parm.to_c()
        d.x_segment = x_segment
        d.s_segment = s_segment
        d.precision = precision
        d.x_mode = x_mode
        d.staging = staging
        for i in range(3):
            d.staging_dir[i] = int(staging_dir[i])
        self.precision = precision
        self._h = ctypes.c_void_p()
        check(lib().bamrex_level_create(ctypes.byref(self._h), ctypes.byref(d), _stream_ptr(stream)))
        self.packing = Packing(spacedim, self.dom_lo, self.boxes)
        self.ncells = lib().bamrex_level_num_cells(self._h)
        self.dx = [(float(prob_hi[q]) - float(prob_lo[q])) / (self.dom_hi[q] - self.dom_lo[q] + 1)
                   for q in range(spacedim)]
        self._owned = True

    @classmethod
    def wrap(cls, handle, spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, method, cfl, precision):
        """A non-owning view of a level created elsewhere (an AMR hierarchy)."""
        self = cls.__new__(cls)
        self.D, self.NC = spacedim, spacedim + 2
        self.boxes = [(tuple(lo) + (0,) * (3 - len(lo)), tuple(hi) + (0,) * (3 - len(hi))) for lo, hi in boxes]
        self.dom_lo = tuple(dom_lo) + (0,) * (3 - len(dom_lo))
        self.dom_hi = tuple(dom_hi) + (0,) * (3 - len(dom_hi))
        self.parm, self.method, self.cfl, self.precision = parm, method, cfl, precision
        self._h = ctypes.c_void_p(handle)
        self.packing = Packing(spacedim, self.dom_lo, self.boxes)
        self.ncells = lib().bamrex_level_num_cells(self._h)
        self.dx = [(float(prob_hi[q]) - float(prob_lo[q])) / (self.dom_hi[q] - self.dom_lo[q] + 1)
                   for q in range(spacedim)]
        self._owned = False
        return self

    # lifetime
    def close(self):
        if self._h and getattr(self, "_owned", True):
            lib().bamrex_level_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        check(rc, self._h)

    # data movement
    def copy_in_ptr(self, ptr: int):
        self._ck(lib().bamrex_level_copy_in(self._h, ctypes.c_void_p(ptr)))

    def copy_out_ptr(self, ptr: int):
        self._ck(lib().bamrex_level_copy_out(self._h, ctypes.c_void_p(ptr)))

    def set_state(self, glob: np.ndarray):
        """Upload a global (NC, nz, ny, nx) float64 array (synchronous)."""
        packed = np.ascontiguousarray(self.packing.pack(glob))
        self.copy_in_ptr(packed.ctypes.data)
        self.sync()

    def get_state(self) -> np.ndarray:
        packed = np.empty(self.packing.size)
        self.copy_out_ptr(packed.ctypes.data)
        self.sync()
        return self.packing.unpack(packed)

    def step_host_ptr(self, in_ptr: int, out_ptr: int, dt: float, nslabs: int = 0) -> float:
        """One step of a host-resident packed state (bamrex_level_step_host):
        uploads, sweeps and downloads overlap in slabs.  Returns the CFL time
        step estimate of the result."""
        nxt = ctypes.c_double()
        self._ck(lib().bamrex_level_step_host(self._h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), float(dt),
                                              int(nslabs), ctypes.byref(nxt)))
        return nxt.value

    def run_host_ptr(self, ptr: int, nsteps: int, dt0: float, time: float = 0.0, nslabs: int = 0):
        """nsteps host round-trip steps of the packed state at ptr, in place
        (bamrex_level_run_host).  Returns (time, next dt)."""
        t, nxt = ctypes.c_double(time), ctypes.c_double()
        self._ck(lib().bamrex_level_run_host(self._h, ctypes.c_void_p(ptr), int(nsteps), float(dt0), int(nslabs),
                                             ctypes.byref(t), ctypes.byref(nxt)))
        return t.value, nxt.value

    def host_slabs(self, nslabs: int = 0) -> int:
        """Slabs the host steps stream this level in for nslabs (0: not
        streamed; bamrex_level_host_slabs)."""
        n = ctypes.c_int()
        self._ck(lib().bamrex_level_host_slabs(self._h, int(nslabs), ctypes.byref(n)))
        return n.value

    def sync(self):
        self._ck(lib().bamrex_level_sync(self._h))

    @property
    def x_mode(self) -> int:
        """The x-sweep kernel in use: XSWEEP_ROWS or XSWEEP_MARCH."""
        return lib().bamrex_level_x_mode(self._h)

    def staging(self, d) -> int:
        """The kernel of the sweep of direction d: STAGING_REGISTERS,
        STAGING_TMA or STAGING_WAVE."""
        return lib().bamrex_level_staging(self._h, int(d))

    def stream_handle(self) -> int:
        """The cudaStream_t the level works on (as an integer)."""
        return lib().bamrex_level_stream(self._h) or 0

    def fab(self, b) -> Array4:
        a = Array4()
        self._ck(lib().bamrex_level_fab(self._h, b, ctypes.byref(a)))
        return a

    # the reference's level surface
    def fill_boundary(self):
        self._ck(lib().bamrex_level_fill_boundary(self._h))

    def tag(self, grad_var=0, grad_threshold=0.0, grad_var_is_primv=False, err_var=None, phierr=0.0,
            err_var_is_primv=False) -> np.ndarray:
        """errorEst tags (1 = refine) of the valid cells in packed order."""
        buf = ctypes.create_string_buffer(int(self.ncells))
        self._ck(lib().bamrex_level_tag(self._h, int(grad_var), 1 if grad_var_is_primv else 0, float(grad_threshold),
                                        0 if err_var is None else 1, int(err_var or 0), 1 if err_var_is_primv else 0,
                                        float(phierr), buf))
        return np.frombuffer(buf.raw, dtype=np.uint8).copy()

    def tag_ex(self, grad_var=0, grad_threshold=0.0, grad_var_is_primv=False, err_var=None, phierr=0.0,
               err_var_is_primv=False, box=None, lstol=None) -> np.ndarray:
        """Every errorEst criterion (bamrex_level_tag_ex): as tag, plus
        box=(lo, hi) in physical coordinates (box_error) and, on a level with
        a rigid body, lstol (interface_error; None: off); ghost_error clears
        solid cells away from the interface whenever the level has a body."""
        t = _abi.TagDesc()
        t.do_err, t.err_var = (0, 0) if err_var is None else (1, int(err_var))
        t.err_var_is_primv, t.phierr = 1 if err_var_is_primv else 0, float(phierr)
        t.do_grad, t.grad_var = (1 if grad_threshold > 0 else 0), int(grad_var)
        t.grad_var_is_primv, t.phigrad = 1 if grad_var_is_primv else 0, float(grad_threshold)
        if box is not None:
            t.do_box = 1
            for q in range(3):
                t.box_lo[q] = float(box[0][q]) if q < len(box[0]) else 0.0
                t.box_hi[q] = float(box[1][q]) if q < len(box[1]) else 0.0
        if lstol is not None:
            t.do_interface, t.lstol = 1, float(lstol)
        buf = ctypes.create_string_buffer(int(self.ncells))
        self._ck(lib().bamrex_level_tag_ex(self._h, ctypes.byref(t), buf))
        return np.frombuffer(buf.raw, dtype=np.uint8).copy()

    # rigid body by the ghost-fluid method
    def set_body(self, shapes, combine=_abi.SDF_UNION, rb_bc=_abi.RB_REFLECTIVE, stencil=2, fill_diagonals=False):
        """A static rigid body (bamrex_level_set_body).  shapes: one or two
        dicts with kind (SDF_PLANE / SDF_SPHERE / SDF_CYLINDER), center, axis
        (plane normal out of the body / cylinder axis), radius, fluid_inside;
        None removes the body."""
        if shapes is None:
            self._ck(lib().bamrex_level_set_body(self._h, None))
            return
        d = body_desc(shapes, combine, rb_bc, stencil, fill_diagonals)
        self._ck(lib().bamrex_level_set_body(self._h, ctypes.byref(d)))

    def fill_body_ghosts(self):
        """The rigid-body ghost fill on the current state (FillRBGhostCells)."""
        self._ck(lib().bamrex_level_fill_body_ghosts(self._h))

    def body_field(self, which) -> np.ndarray:
        """Level set (0), normal component d (1 + d) or GFM flags (-1) of the
        valid cells as a global (nz, ny, nx) array."""
        out = np.empty(int(self.ncells))
        self._ck(lib().bamrex_level_body_field(self._h, int(which), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        his = np.max(np.array([hi for _, hi in self.boxes]), axis=0)
        n = [his[d] - self.dom_lo[d] + 1 for d in range(3)]
        glob = np.full((n[2], n[1], n[0]), np.nan)
        o = 0
        L = self.dom_lo
        for lo, hi in self.boxes:
            shp = (hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1)
            m = shp[0] * shp[1] * shp[2]
            glob[lo[2] - L[2]:hi[2] - L[2] + 1, lo[1] - L[1]:hi[1] - L[1] + 1, lo[0] - L[0]:hi[0] - L[0] + 1] = \
                out[o:o + m].reshape(shp)
            o += m
        return glob

    def body_counts(self):
        """(interface ghost cells, body cells swept by the extrapolation)."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        self._ck(lib().bamrex_level_body_counts(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def conserved_sums(self):
        """sum(U) * cell volume per component (FP64, fixed order)."""
        out = (ctypes.c_double * self.NC)()
        self._ck(lib().bamrex_level_conserved_sums(self._h, out))
        return np.array(list(out))

    def advance(self, time, dt, iteration=1, ncycle=1) -> float:
        out = ctypes.c_double()
        self._ck(lib().bamrex_level_advance(self._h, time, dt, iteration, ncycle, ctypes.byref(out)))
        return out.value

    def estTimeStep(self) -> float:
        out = ctypes.c_double()
        self._ck(lib().bamrex_level_est_time_step(self._h, ctypes.byref(out)))
        return out.value

    def run(self, nsteps, stop_time=-1.0, use_graph=True, time=0.0):
        t = ctypes.c_double(time)
        n = ctypes.c_int(0)
        self._ck(lib().bamrex_level_run(self._h, nsteps, stop_time, 1 if use_graph else 0, ctypes.byref(t),
                                        ctypes.byref(n)))
        return t.value, n.value

    def run_async(self, nsteps, stop_time=-1.0, use_graph=True, time=0.0):
        self._ck(lib().bamrex_level_run_async(self._h, nsteps, stop_time, 1 if use_graph else 0, time))

    def run_wait(self):
        t = ctypes.c_double()
        n = ctypes.c_int(0)
        self._ck(lib().bamrex_level_run_wait(self._h, ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    # measurement
    def set_timing(self, on=True):
        self._ck(lib().bamrex_level_set_timing(self._h, 1 if on else 0))

    def counters(self):
        a, b, c = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_longlong()
        self._ck(lib().bamrex_level_counters(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def reset_counters(self):
        self._ck(lib().bamrex_level_reset_counters(self._h))

    def sweep_times(self):
        """Per-direction (ms, launches) of the timed sweep kernels."""
        ms = (ctypes.c_double * 3)()
        n = (ctypes.c_longlong * 3)()
        self._ck(lib().bamrex_level_sweep_times(self._h, ms, n))
        return [(ms[d], n[d]) for d in range(self.D)]


def main(argv=None):
    """Step a synthetic level on cuda:0 (for timing and profiling runs):

        python -m bamrex_b200.level [--dim 2] [--n 4096] [--max-grid-size 0]
            [--staging 0] [--x-mode 0] [--steps 4] [--fp32]

    2D: the four-quadrant Riemann problem (minbee); 3D: seeded random cells
    (minbee); MUSCL-Hancock + HLLC, CFL 0.8, transmissive.  Prints the
    kernel of each direction's sweep, the sweep times per direction and the
    whole step (graph-replayed steps, host clock around synchronised runs)."""
    import argparse
    import json
    import time

    from . import problems
    ap = argparse.ArgumentParser(prog="python -m bamrex_b200.level")
    ap.add_argument("--dim", type=int, default=2, choices=(2, 3))
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--max-grid-size", type=int, default=0)
    ap.add_argument("--staging", type=int, default=_abi.STAGING_AUTO)
    ap.add_argument("--x-mode", type=int, default=_abi.XSWEEP_AUTO)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--fp32", action="store_true")
    a = ap.parse_args(argv)
    D, n = a.dim, a.n
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    u0 = problems.quadrant_2d(n) if D == 2 else problems.random_states(3, (n, n, n), seed=5)
    lev = Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, decompose(D, (0, 0, 0), hi, a.max_grid_size or n),
                Parm(D, limiter=_abi.MINBEE), method=_abi.MUSCL_HANCOCK, cfl=0.8, staging=a.staging, x_mode=a.x_mode,
                precision=_abi.FP32_STORAGE if a.fp32 else _abi.FP64)
    try:
        lev.set_state(u0)
        lev.set_timing(True)
        lev.run(a.steps, use_graph=False)
        out = {"kernels": [lev.staging(d) for d in range(D)],
               "ms_per_sweep": [ms / max(1, k) for ms, k in lev.sweep_times()]}
        lev.set_timing(False)
        lev.set_state(u0)
        lev.run(2)
        lev.sync()
        t0 = time.perf_counter()
        lev.run(a.steps)
        lev.sync()
        ms = (time.perf_counter() - t0) * 1e3 / max(1, a.steps)
        out["ms_per_step"] = ms
        out["cell_updates_per_s"] = float(n) ** D / (ms * 1e-3)
    finally:
        lev.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
