"""Python mirror of the AMR layer around AmrLevelAdv over the C ABI.

``Coupling`` is the pair of AMReX objects the reference uses between two
levels (FluxRegister, FillPatch / FillCoarsePatch with cell_cons_interp,
average_down; Source/AmrLevelAdv_advance.cpp:108, 192-254,
Source/AmrLevelAdv.cpp:371, 918-987).  ``Amr`` is the subcycled hierarchy
(Amr::coarseTimeStep with AmrLevelAdv::computeInitialDt / computeNewDt /
post_timestep / errorEst, Source/AmrLevelAdv.cpp:487-832).  Every level is a
device ``Level``; all work runs in libbamrex_cuda.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import AmrDesc, Box, LevelDesc, check, lib
from .level import Level, Parm


def _boxes3(boxes):
    return [(tuple(lo) + (0,) * (3 - len(lo)), tuple(hi) + (0,) * (3 - len(hi))) for lo, hi in boxes]


class Coupling:
    """Coarse/fine coupling of two device levels (refinement ratio 2 or 4)."""

    def __init__(self, crse: Level, fine: Level, ref_ratio=2):
        self.crse, self.fine, self.ratio = crse, fine, ref_ratio
        self._h = ctypes.c_void_p()
        check(lib().bamrex_coupling_create(ctypes.byref(self._h), crse._h, fine._h, ref_ratio))

    def close(self):
        if self._h:
            lib().bamrex_coupling_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def save_coarse_old(self, t_old, t_new):
        check(lib().bamrex_coupling_save_coarse_old(self._h, t_old, t_new))

    def fill_patch(self, time):
        check(lib().bamrex_coupling_fill_patch(self._h, time))

    def fill_coarse_patch(self):
        check(lib().bamrex_coupling_fill_coarse_patch(self._h))

    def reflux(self):
        check(lib().bamrex_coupling_reflux(self._h))

    def avg_down(self):
        check(lib().bamrex_coupling_avg_down(self._h))

    def covered_sums(self):
        out = (ctypes.c_double * self.crse.NC)()
        check(lib().bamrex_coupling_covered_sums(self._h, out))
        return np.array(list(out))

    def register(self, d):
        n = ctypes.c_int()
        check(lib().bamrex_coupling_register(self._h, d, None, ctypes.byref(n)))
        buf = np.zeros(self.crse.NC * n.value)
        if n.value:
            check(lib().bamrex_coupling_register(self._h, d, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                 ctypes.byref(n)))
        return buf.reshape(self.crse.NC, n.value)


def cluster_tags(spacedim, dom_lo, dom_hi, boxes, tags, ref_ratio=2, blocking_factor=8, max_grid_size=32,
                 n_error_buf=2, n_proper=1, grid_eff=0.7, periodic=(0, 0, 0)):
    """Level l+1 boxes from level-l tags (host-side grid generation)."""
    boxes = _boxes3(boxes)
    dom = Box.make(dom_lo, dom_hi)
    cb = (Box * len(boxes))(*[Box.make(lo, hi) for lo, hi in boxes])
    per = (ctypes.c_int * 3)(*[int(p) for p in periodic])
    n_blk = 1  # at most one new box per blocked cell
    for d in range(spacedim):
        n_blk *= (dom_hi[d] - dom_lo[d] + 1) // max(1, blocking_factor // ref_ratio)
    out = (Box * max(1, n_blk))()
    nout = ctypes.c_int()
    t = np.ascontiguousarray(tags, dtype=np.uint8).tobytes()
    check(lib().bamrex_cluster_tags(spacedim, ctypes.byref(dom), per, cb, len(boxes), t, ref_ratio, blocking_factor,
                                    max_grid_size, n_error_buf, n_proper, grid_eff, out, len(out), ctypes.byref(nout)))
    return [(tuple(out[i].lo), tuple(out[i].hi)) for i in range(nout.value)]


class Amr:
    """A subcycled AMR hierarchy of device levels."""

    def __init__(self, spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm: Parm, method=_abi.MUSCL_HANCOCK,
                 cfl=0.9, ngrow=2, bc_lo=None, bc_hi=None, precision=_abi.FP64, max_level=1, ref_ratio=2,
                 blocking_factor=8, max_grid_size=32, n_error_buf=2, n_proper=1, grid_eff=0.7, regrid_int=0,
                 do_reflux=True, phigrad=None, phigrad_var=0, phigrad_var_is_primv=False, phierr=None, phierr_var=0,
                 phierr_var_is_primv=False, max_int_lev=-1, lstol=None, max_box_lev=-1, refine_box=None,
                 staging=_abi.STAGING_AUTO, stream=None):
        self.D = spacedim
        self.parm, self.method, self.cfl, self.precision = parm, method, cfl, precision
        self.ratio = ref_ratio
        self.dom_lo = tuple(dom_lo) + (0,) * (3 - len(dom_lo))
        self.dom_hi = tuple(dom_hi) + (0,) * (3 - len(dom_hi))
        self.prob_lo = [float(x) for x in prob_lo]
        self.prob_hi = [float(x) for x in prob_hi]
        self.bc_lo = tuple(bc_lo) if bc_lo is not None else (0, 0, 0)
        self.bc_hi = tuple(bc_hi) if bc_hi is not None else (0, 0, 0)
        d = AmrDesc()
        b = d.base
        b.spacedim = spacedim
        b.domain = Box.make(self.dom_lo, self.dom_hi)
        for q in range(3):
            b.prob_lo[q] = self.prob_lo[q] if q < len(self.prob_lo) else 0.0
            b.prob_hi[q] = self.prob_hi[q] if q < len(self.prob_hi) else 1.0
            b.bc_lo[q] = int(self.bc_lo[q]) if q < len(self.bc_lo) else 0
            b.bc_hi[q] = int(self.bc_hi[q]) if q < len(self.bc_hi) else 0
        bx = _boxes3(boxes)
        self._boxes0 = (Box * len(bx))(*[Box.make(lo, hi) for lo, hi in bx])
        b.boxes = self._boxes0
        b.nboxes = len(bx)
        b.ngrow = ngrow
        b.method = method
        b.cfl = cfl
        b.parm = parm.to_c()
        b.precision = precision
        b.staging = staging  # sweep kernels of every level (bamrex_level_desc.staging)
        d.max_level = max_level
        d.ref_ratio = ref_ratio
        d.blocking_factor = blocking_factor
        d.max_grid_size = max_grid_size
        d.n_error_buf = n_error_buf
        d.n_proper = n_proper
        d.grid_eff = grid_eff
        d.regrid_int = regrid_int
        d.do_reflux = 1 if do_reflux else 0
        d.phigrad_var = phigrad_var
        d.phigrad_var_is_primv = 1 if phigrad_var_is_primv else 0
        phigrad = list(phigrad or [])
        for i, v in enumerate(phigrad[:_abi.MAX_LEVELS]):
            d.phigrad[i] = v
        d.max_phigrad_lev = len(phigrad)
        d.phierr_var = phierr_var
        d.phierr_var_is_primv = 1 if phierr_var_is_primv else 0
        phierr = list(phierr or [])
        for i, v in enumerate(phierr[:_abi.MAX_LEVELS]):
            d.phierr[i] = v
        d.max_phierr_lev = len(phierr)
        # interface tagging (tagging.max_int_lev / lstol) and box tagging
        # (tagging.max_box_lev / box_x, box_y, box_z as refine_box = (lo, hi))
        d.max_int_lev = int(max_int_lev)
        for i, v in enumerate(list(lstol or [])[:_abi.MAX_LEVELS]):
            d.lstol[i] = v
        d.max_box_lev = int(max_box_lev)
        if refine_box is not None:
            for q in range(3):
                d.box_lo[q] = float(refine_box[0][q]) if q < len(refine_box[0]) else 0.0
                d.box_hi[q] = float(refine_box[1][q]) if q < len(refine_box[1]) else 0.0
        self._desc = d
        self._h = ctypes.c_void_p()
        st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        check(lib().bamrex_amr_create(ctypes.byref(self._h), ctypes.byref(d), st))
        self.time = 0.0

    def close(self):
        if self._h:
            lib().bamrex_amr_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        check(rc, amr_handle=self._h)

    # structure
    @property
    def finest_level(self) -> int:
        return lib().bamrex_amr_finest_level(self._h)

    def domain(self, lev):
        f = self.ratio ** lev
        lo = tuple(self.dom_lo[d] * f if d < self.D else 0 for d in range(3))
        hi = tuple((self.dom_hi[d] + 1) * f - 1 if d < self.D else 0 for d in range(3))
        return lo, hi

    def boxes(self, lev):
        n = ctypes.c_int()
        self._ck(lib().bamrex_amr_boxes(self._h, lev, None, 0, ctypes.byref(n)))
        out = (Box * max(1, n.value))()
        self._ck(lib().bamrex_amr_boxes(self._h, lev, out, n.value, ctypes.byref(n)))
        return [(tuple(out[i].lo), tuple(out[i].hi)) for i in range(n.value)]

    def level(self, lev) -> Level:
        h = lib().bamrex_amr_level(self._h, lev)
        if not h:
            raise IndexError("no level %d" % lev)
        lo, hi = self.domain(lev)
        return Level.wrap(h, self.D, lo, hi, self.prob_lo, self.prob_hi, self.boxes(lev), self.parm, self.method,
                          self.cfl, self.precision)

    def set_level_boxes(self, lev, boxes):
        bx = _boxes3(boxes)
        arr = (Box * len(bx))(*[Box.make(lo, hi) for lo, hi in bx])
        self._ck(lib().bamrex_amr_set_level_boxes(self._h, lev, arr, len(bx)))

    def regrid(self, lbase=0, time=None):
        self._ck(lib().bamrex_amr_regrid(self._h, lbase, self.time if time is None else time))

    def avg_down_all(self):
        self._ck(lib().bamrex_amr_avg_down_all(self._h))

    # data
    def cell_centres(self, lev):
        """Cell-centre coordinates (x, y, z) arrays of level lev's domain."""
        lo, hi = self.domain(lev)
        out = []
        for d in range(3):
            n = hi[d] - lo[d] + 1
            if d < self.D:
                dx = (self.prob_hi[d] - self.prob_lo[d]) / n
                out.append(self.prob_lo[d] + (np.arange(n) + 0.5) * dx)
            else:
                out.append(np.zeros(1))
        return out

    def set_state(self, lev, glob):
        self.level(lev).set_state(glob)

    def get_state(self, lev) -> np.ndarray:
        """Level lev on its whole domain (NaN outside its boxes)."""
        L = self.level(lev)
        lo, hi = self.domain(lev)
        n = [hi[d] - lo[d] + 1 for d in range(3)]
        glob = np.full((self.D + 2, n[2], n[1], n[0]), np.nan)
        packed = np.empty(L.packing.size)
        L.copy_out_ptr(packed.ctypes.data)
        L.sync()
        return L.packing.unpack(packed, glob)

    def init(self, fn, time=0.0):
        """Initial hierarchy (Amr::initialInit): level 0 from fn(amr, 0),
        then repeatedly tag the finest level, build the next one and fill
        it from fn(amr, lev) (initData); finally average down (post_init)."""
        self.set_state(0, fn(self, 0))
        lev = 0
        while lev < self._desc.max_level:
            self.regrid(lev, time)
            if self.finest_level <= lev:
                break
            lev += 1
            self.set_state(lev, fn(self, lev))
        self.avg_down_all()
        self.time = time

    # time stepping
    def coarse_step(self, stop_time=-1.0) -> float:
        t = ctypes.c_double(self.time)
        dt = ctypes.c_double()
        self._ck(lib().bamrex_amr_coarse_step(self._h, stop_time, ctypes.byref(t), ctypes.byref(dt)))
        self.time = t.value
        return dt.value

    def run(self, nsteps, stop_time=-1.0):
        dts = []
        for _ in range(nsteps):
            if stop_time >= 0 and self.time >= stop_time:
                break
            dts.append(self.coarse_step(stop_time))
        return dts

    @property
    def coarse_steps(self) -> int:
        """Coarse steps taken (Amr::levelSteps(0)); a restart keeps counting."""
        st = _abi.AmrStepping()
        self._ck(lib().bamrex_amr_get_stepping(self._h, ctypes.byref(st)))
        return st.coarse_steps

    def set_regrid_int(self, n):
        self._ck(lib().bamrex_amr_set_regrid_int(self._h, n))

    def set_graph(self, on: bool):
        """Coarse steps replayed as CUDA graphs with the time steps on the
        device (bamrex_amr_set_graph; on by default)."""
        self._ck(lib().bamrex_amr_set_graph(self._h, 1 if on else 0))

    def graph_stats(self):
        """(graphs captured, coarse steps replayed, kernel nodes of the
        current levels' graph) (bamrex_amr_graph_stats)."""
        c, r, k = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
        self._ck(lib().bamrex_amr_graph_stats(self._h, ctypes.byref(c), ctypes.byref(r), ctypes.byref(k)))
        return c.value, r.value, k.value

    def set_body(self, shapes, combine=_abi.SDF_UNION, rb_bc=_abi.RB_REFLECTIVE, stencil=2, fill_diagonals=False):
        """A static rigid body on every level, present and future
        (bamrex_amr_set_body); None removes it."""
        from .level import body_desc
        if shapes is None:
            self._ck(lib().bamrex_amr_set_body(self._h, None))
            return
        d = body_desc(shapes, combine, rb_bc, stencil, fill_diagonals)
        self._ck(lib().bamrex_amr_set_body(self._h, ctypes.byref(d)))

    def dt_level(self):
        out = (ctypes.c_double * _abi.MAX_LEVELS)()
        self._ck(lib().bamrex_amr_dt_level(self._h, out))
        return [out[i] for i in range(self.finest_level + 1)]

    def conserved_sums(self):
        out = (ctypes.c_double * (self.D + 2))()
        self._ck(lib().bamrex_amr_conserved_sums(self._h, out))
        return np.array(list(out))


def chop_drawn(boxes, choices, rng, D=3):
    """Boxes cut so each piece's sides are at most a max_grid_size drawn per
    box from `choices` (all multiples of the blocking factor)."""
    out = []
    for lo, hi in boxes:
        m = int(rng.choice(choices))
        pieces = [(list(lo), list(hi))]
        for d in range(D):
            nxt = []
            for plo, phi in pieces:
                a = plo[d]
                while a <= phi[d]:
                    b = min(phi[d], a + m - 1)
                    qlo, qhi = list(plo), list(phi)
                    qlo[d], qhi[d] = a, b
                    nxt.append((qlo, qhi))
                    a = b + 1
            pieces = nxt
        out += [(tuple(a), tuple(b)) for a, b in pieces]
    return out


BLAST_BOX_SIZES = (16, 32, 48, 64)


def blast_hierarchy(n0, precision=_abi.FP64, seed=20261203, stream=None, staging=_abi.STAGING_AUTO):
    """The 3D spherical blast (p 10 inside r < 0.2, 0.1 outside, rho 1) on a
    3-level hierarchy: base n0^3 on [0,1]^3, ratio 2, blocking factor 8,
    grad_error on rho >= 0.1, MUSCL-Hancock/minbee, CFL 0.8, boxes cut to a
    max_grid_size drawn per box from {16, 32, 48, 64}.  The levels form
    during four coarse steps with a regrid every 2 (the density is uniform
    at t = 0), then their boxes are redrawn; returns the hierarchy with
    regridding switched off and the random generator."""
    from . import problems
    hi = (n0 - 1,) * 3
    rng = np.random.default_rng(seed)
    base = chop_drawn([((0, 0, 0), hi)], BLAST_BOX_SIZES, rng)
    A = Amr(3, (0, 0, 0), hi, [0.0] * 3, [1.0] * 3, base, Parm(3, limiter=_abi.MINBEE), cfl=0.8, max_level=2,
            ref_ratio=2, blocking_factor=8, max_grid_size=64, n_error_buf=2, grid_eff=0.7, regrid_int=2,
            phigrad=[0.1, 0.1], phigrad_var=0, precision=precision, staging=staging, stream=stream)
    A.set_state(0, problems.blast_3d(n0, radius=0.2))
    for _ in range(4):
        A.coarse_step()
    old = [A.boxes(lev) for lev in range(A.finest_level + 1)]
    for lev in range(1, len(old)):
        A.set_level_boxes(lev, chop_drawn(old[lev], BLAST_BOX_SIZES, rng))
    A.set_regrid_int(0)
    return A, rng


def main(argv=None):
    """Coarse steps of the 3D blast hierarchy on cuda:0 (for timing and
    profiling runs):

        python -m bamrex_b200.amr [--n 256] [--steps 4] [--fp32] [--regrid-int K] [--profile]

    Prints the levels' cells, boxes and sweep kernels and the time per
    coarse step (host clock around synchronised steps); --regrid-int K
    regrids every K coarse steps during the timed steps, --profile adds the
    library's region timers (bamrex_profile_report) over those steps."""
    import argparse
    import json
    import time

    import torch
    ap = argparse.ArgumentParser(prog="python -m bamrex_b200.amr")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--regrid-int", type=int, default=0)
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--staging", type=int, default=_abi.STAGING_AUTO, help="sweep kernels of every level")
    ap.add_argument("--warm-steps", type=int, default=0, help="untimed coarse steps on fixed grids first")
    a = ap.parse_args(argv)
    A, _ = blast_hierarchy(a.n, _abi.FP32_STORAGE if a.fp32 else _abi.FP64, staging=a.staging)
    try:
        for _ in range(a.warm_steps):
            A.coarse_step()
        A.set_regrid_int(a.regrid_int)
        if a.profile:
            _abi.profile_enable(True)
            _abi.profile_reset()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("amr_coarse_steps")
        t0 = time.perf_counter()
        for _ in range(a.steps):
            A.coarse_step()
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        torch.cuda.nvtx.range_pop()
        out = {"cells": [sum(int(np.prod([h[d] - l[d] + 1 for d in range(3)])) for l, h in A.boxes(lev))
                         for lev in range(A.finest_level + 1)],
               "boxes": [len(A.boxes(lev)) for lev in range(A.finest_level + 1)],
               "kernels": [[A.level(lev).staging(d) for d in range(3)] for lev in range(A.finest_level + 1)],
               "ms_per_coarse_step": el / max(1, a.steps) * 1e3}
        if a.profile:
            out["regions"] = [{"name": n, "calls": c, "total_s": round(t, 6), "max_ms": round(m, 3)}
                              for n, c, t, _, m in _abi.profile_report()]
    finally:
        A.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
