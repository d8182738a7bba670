"""Checkpoints of a device hierarchy, and restart from them: the
reference's amr.checkPoint() (Source/main.cpp:96-99, every amr.check_int
coarse steps and at the end) with AmrLevelAdv::checkPoint / restart
(Source/AmrLevelAdv.cpp:95-113), which hand the levels' state to AMReX.

A checkpoint keeps what the next coarse step reads: every level's boxes and
the conserved state of its valid cells, the time, the coarse steps taken
(they time the regrids) and each level's time step (a step right after a
regrid takes the smaller of the new estimate and the old step).  Ghost
cells, the coarse level's old time level, flux registers and the rigid
body's fields are rebuilt by the next step, so a restarted run continues the
original bit for bit.

Layout (a directory, AMReX-like):

    <dir>/Header             "bamrex-b200-checkpoint 1", dimension, time,
                             finest level, refinement ratio, coarse steps,
                             whether a time step is set, the time step of
                             every level, then per level its domain and
                             boxes (one per line, cell indices)
    <dir>/Level_<l>/Cell_H   the level's MultiFab on disk, written by the
    <dir>/Level_<l>/Cell_D_00000
                             plotfile writer (AMReX's VisMF layout; exact
                             IEEE doubles in the host's byte order)
"""
from __future__ import annotations

import os

import numpy as np

from ._abi import AmrStepping, lib
from .plotfile import _read_level, _write_level

MAGIC = "bamrex-b200-checkpoint 1"


def _fmt(x) -> str:
    return repr(float(x))


def write_checkpoint(path, amr) -> None:
    """Write the checkpoint of a device hierarchy (amr: bamrex_b200.amr.Amr)
    into the directory `path`."""
    st = AmrStepping()
    amr._ck(lib().bamrex_amr_get_stepping(amr._h, st))
    D, finest = amr.D, amr.finest_level
    os.makedirs(path, exist_ok=True)
    hdr = [MAGIC, str(D), _fmt(amr.time), str(finest), str(amr.ratio), str(st.coarse_steps), str(st.have_dt),
           " ".join(_fmt(st.dt_level[l]) for l in range(st.nlevels))]
    for lev in range(finest + 1):
        dlo, dhi = amr.domain(lev)
        boxes = amr.boxes(lev)
        glob = amr.get_state(lev)
        fabs = []
        for lo, hi in boxes:
            sl = tuple(slice(lo[d] - dlo[d], hi[d] - dlo[d] + 1) if d < D else slice(0, 1) for d in (2, 1, 0))
            fabs.append(np.ascontiguousarray(glob[(slice(None),) + sl]))
        _write_level(os.path.join(path, "Level_%d" % lev), D, boxes, fabs, D + 2)
        hdr.append("%d %d" % (lev, len(boxes)))
        hdr.append(" ".join(str(v) for v in tuple(dlo) + tuple(dhi)))
        hdr += [" ".join(str(v) for v in tuple(lo) + tuple(hi)) for lo, hi in boxes]
    with open(os.path.join(path, "Header"), "w") as f:
        f.write("\n".join(hdr) + "\n")


def read_checkpoint(path) -> dict:
    """The contents of a checkpoint directory: dimension, time, ratio,
    coarse steps, have_dt, dt per level, and per level (domain, boxes,
    fabs) with fabs the (NC, nz, ny, nx) arrays of the boxes' valid cells."""
    with open(os.path.join(path, "Header")) as f:
        lines = f.read().split("\n")
    if lines[0].strip() != MAGIC:
        raise ValueError("%s is not a bamrex-b200 checkpoint" % path)
    D, time, finest, ratio = int(lines[1]), float(lines[2]), int(lines[3]), int(lines[4])
    steps, have_dt = int(lines[5]), int(lines[6])
    dts = [float(x) for x in lines[7].split()]
    pos = 8
    levels = []
    for lev in range(finest + 1):
        l_, nb = (int(x) for x in lines[pos].split())
        if l_ != lev:
            raise ValueError("%s: level %d out of order" % (path, l_))
        v = [int(x) for x in lines[pos + 1].split()]
        dom = (tuple(v[:3]), tuple(v[3:]))
        boxes = []
        for b in range(nb):
            w = [int(x) for x in lines[pos + 2 + b].split()]
            boxes.append((tuple(w[:3]), tuple(w[3:])))
        pos += 2 + nb
        fboxes, fabs = _read_level(os.path.join(path, "Level_%d" % lev), D, D + 2)
        if [tuple(map(tuple, fb)) for fb in fboxes] != [tuple(map(tuple, b)) for b in boxes]:
            raise ValueError("%s: level %d boxes disagree with its MultiFab" % (path, lev))
        levels.append((dom, boxes, fabs))
    return {"D": D, "time": time, "ratio": ratio, "coarse_steps": steps, "have_dt": have_dt, "dt_level": dts,
            "levels": levels}


def restore(amr, ck) -> None:
    """Put a checkpoint (read_checkpoint) into a hierarchy whose base level
    already has the checkpoint's boxes: the finer levels' boxes, every
    level's state, the time and the stepping state."""
    D = amr.D
    if ck["D"] != D or ck["ratio"] != amr.ratio:
        raise ValueError("checkpoint of a %dD hierarchy with ratio %d" % (ck["D"], ck["ratio"]))
    base = [tuple(map(tuple, b)) for b in ck["levels"][0][1]]
    if [tuple(map(tuple, b)) for b in amr.boxes(0)] != base:
        raise ValueError("the hierarchy's base level must have the checkpoint's boxes (make it with restart_amr)")
    for lev in range(1, len(ck["levels"])):
        amr.set_level_boxes(lev, ck["levels"][lev][1])
    for lev, (dom, boxes, fabs) in enumerate(ck["levels"]):
        dlo, dhi = amr.domain(lev)
        n = [dhi[d] - dlo[d] + 1 for d in range(3)]
        glob = np.zeros((D + 2, n[2], n[1], n[0]))
        for (lo, hi), fab in zip(boxes, fabs):
            sl = tuple(slice(lo[d] - dlo[d], hi[d] - dlo[d] + 1) if d < D else slice(0, 1) for d in (2, 1, 0))
            glob[(slice(None),) + sl] = fab
        amr.set_state(lev, glob)
    st = AmrStepping()
    st.coarse_steps = ck["coarse_steps"]
    st.have_dt = ck["have_dt"]
    st.nlevels = len(ck["dt_level"])
    for lev, v in enumerate(ck["dt_level"]):
        st.dt_level[lev] = v
    amr._ck(lib().bamrex_amr_set_stepping(amr._h, st))
    amr.time = ck["time"]


def restart_amr(path, make):
    """A hierarchy continuing the checkpoint at `path`: make(base_boxes)
    builds the device hierarchy (the run's settings, the checkpoint's base
    level boxes), then restore() fills it."""
    ck = read_checkpoint(path)
    amr = make(ck["levels"][0][1])
    try:
        restore(amr, ck)
    except Exception:
        amr.close()
        raise
    return amr


__all__ = ["write_checkpoint", "read_checkpoint", "restore", "restart_amr", "MAGIC"]
