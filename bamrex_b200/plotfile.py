"""AMReX plotfiles of a hierarchy (the reference's writePlotFile,
Source/AmrLevelAdv.cpp:117-135, hands its state to AMReX's
AmrLevel::writePlotFile). With a rigid body the reference first refills
the cells inside the body by first-order extrapolation for nicer pictures;
write_amr_plotfile writes them as the last step's rigid-body fill left
them. The fluid cells are the same either way.

Layout (AMReX's native plotfile format, "HyperCLaw-V1.1", restated from
its published description):

    <dir>/Header             variable names, dimension, time, finest
                             level, problem box, ratios, level domains,
                             level steps, cell sizes, then per level its
                             boxes in physical coordinates and the path
                             of its MultiFab
    <dir>/Level_<l>/Cell_H   VisMF header: version, layout, components,
                             ghost width, the box array, the file and
                             byte offset of every box, per-box minima
                             and maxima of every component
    <dir>/Level_<l>/Cell_D_00000
                             per box: a FAB header line naming the real
                             format (IEEE double, byte order) and the
                             box, then every component's values with
                             i fastest

The state is written in the host's byte order, which the FAB header
records. read_plotfile reads such a directory back.
"""
from __future__ import annotations

import os
import sys

import numpy as np

_FORMAT = "(64 11 52 0 1 12 0 1023)"
_ORDER = {"little": "(8, (8 7 6 5 4 3 2 1))", "big": "(8, (1 2 3 4 5 6 7 8))"}


def _box_str(D, lo, hi):
    f = lambda v: "(" + ",".join(str(int(x)) for x in v[:D]) + ")"
    return "(%s %s %s)" % (f(lo), f(hi), f((0,) * D))


def _real(x) -> str:
    return repr(float(x))


def write_plotfile(path, spacedim, time, prob_lo, prob_hi, levels, varnames, ref_ratio=2, level_steps=None):
    """Write a plotfile directory.

    levels: one entry per level, (domain_lo, domain_hi, boxes, fabs) where
    boxes are (lo, hi) cell index triples and fabs the matching
    (ncomp, nz, ny, nx) float64 arrays of each box's valid cells."""
    D = spacedim
    ncomp = len(varnames)
    nlev = len(levels)
    level_steps = list(level_steps) if level_steps is not None else [0] * nlev
    os.makedirs(path, exist_ok=True)
    dx = []
    for lev, (dlo, dhi, _, _) in enumerate(levels):
        dx.append([(prob_hi[d] - prob_lo[d]) / (dhi[d] - dlo[d] + 1) for d in range(D)])
    hdr = ["HyperCLaw-V1.1", str(ncomp)] + list(varnames) + [str(D), _real(time), str(nlev - 1)]
    hdr.append(" ".join(_real(x) for x in prob_lo[:D]) + " ")
    hdr.append(" ".join(_real(x) for x in prob_hi[:D]) + " ")
    hdr.append(" ".join(str(ref_ratio) for _ in range(nlev - 1)) + (" " if nlev > 1 else ""))
    hdr.append(" ".join(_box_str(D, dlo, dhi) for dlo, dhi, _, _ in levels) + " ")
    hdr.append(" ".join(str(s) for s in level_steps) + " ")
    for lev in range(nlev):
        hdr.append(" ".join(_real(x) for x in dx[lev]) + " ")
    hdr += ["0", "0"]  # Cartesian coordinates; no boundary cells written
    for lev, (dlo, dhi, boxes, fabs) in enumerate(levels):
        if len(boxes) != len(fabs):
            raise ValueError("level %d: %d boxes but %d fabs" % (lev, len(boxes), len(fabs)))
        hdr.append("%d %d %s" % (lev, len(boxes), _real(time)))
        hdr.append(str(level_steps[lev]))
        for lo, hi in boxes:
            for d in range(D):
                x0 = prob_lo[d] + lo[d] * dx[lev][d]
                x1 = prob_lo[d] + (hi[d] + 1) * dx[lev][d]
                hdr.append("%s %s" % (_real(x0), _real(x1)))
        hdr.append("Level_%d/Cell" % lev)
        _write_level(os.path.join(path, "Level_%d" % lev), D, boxes, fabs, ncomp)
    with open(os.path.join(path, "Header"), "w") as f:
        f.write("\n".join(hdr) + "\n")


def _write_level(ldir, D, boxes, fabs, ncomp):
    os.makedirs(ldir, exist_ok=True)
    order = _ORDER[sys.byteorder]
    offsets, mins, maxs = [], [], []
    with open(os.path.join(ldir, "Cell_D_00000"), "wb") as f:
        for (lo, hi), fab in zip(boxes, fabs):
            a = np.ascontiguousarray(fab, dtype=np.float64)
            shape = tuple(hi[d] - lo[d] + 1 if d < D else 1 for d in (2, 1, 0))
            if a.shape != (ncomp,) + shape:
                raise ValueError("fab of box %s..%s has shape %s, expected %s" % (lo, hi, a.shape, (ncomp,) + shape))
            offsets.append(f.tell())
            f.write(("FAB (%s,%s)%s %d\n" % ("(8, " + _FORMAT + ")", order, _box_str(D, lo, hi), ncomp)).encode())
            f.write(a.tobytes())
            flat = a.reshape(ncomp, -1)
            mins.append(flat.min(axis=1))
            maxs.append(flat.max(axis=1))
    n = len(boxes)
    lines = ["1", "0", str(ncomp), "0", "(%d 0" % n]
    lines += [_box_str(D, lo, hi) for lo, hi in boxes]
    lines += [")", str(n)]
    lines += ["FabOnDisk: Cell_D_00000 %d" % o for o in offsets]
    lines += ["", "%d,%d" % (n, ncomp)]
    lines += ["".join(_real(v) + "," for v in m) for m in mins]
    lines += ["", "%d,%d" % (n, ncomp)]
    lines += ["".join(_real(v) + "," for v in m) for m in maxs]
    with open(os.path.join(ldir, "Cell_H"), "w") as f:
        f.write("\n".join(lines) + "\n")


def _parse_box(s):
    parts = s.replace("(", " ").replace(")", " ").split()
    vals = [[int(x) for x in p.split(",")] for p in parts]
    pad = (0,) * (3 - len(vals[0]))
    return tuple(vals[0]) + pad, tuple(vals[1]) + pad


def read_plotfile(path):
    """{'varnames', 'spacedim', 'time', 'prob_lo', 'prob_hi', 'ref_ratio',
    'level_steps', 'levels': [(domain_lo, domain_hi, boxes, fabs)]} of a
    plotfile directory written by write_plotfile."""
    with open(os.path.join(path, "Header")) as f:
        lines = f.read().split("\n")
    it = iter(lines)
    if next(it) != "HyperCLaw-V1.1":
        raise ValueError("not a HyperCLaw-V1.1 plotfile")
    ncomp = int(next(it))
    varnames = [next(it) for _ in range(ncomp)]
    D = int(next(it))
    time = float(next(it))
    nlev = int(next(it)) + 1
    prob_lo = [float(x) for x in next(it).split()]
    prob_hi = [float(x) for x in next(it).split()]
    ratios = [int(x) for x in next(it).split()]
    dom_line = next(it)
    doms = [_parse_box(s) for s in _split_boxes(dom_line)]
    steps = [int(x) for x in next(it).split()]
    for _ in range(nlev):
        next(it)
    next(it), next(it)
    levels = []
    for lev in range(nlev):
        _, nb, _ = next(it).split()
        next(it)
        for _ in range(int(nb) * D):
            next(it)
        rel = next(it)
        boxes, fabs = _read_level(os.path.join(path, os.path.dirname(rel)), D, ncomp)
        levels.append((doms[lev][0], doms[lev][1], boxes, fabs))
    return dict(varnames=varnames, spacedim=D, time=time, prob_lo=prob_lo, prob_hi=prob_hi,
                ref_ratio=ratios[0] if ratios else None, level_steps=steps, levels=levels)


def _split_boxes(line):
    out, depth, cur = [], 0, ""
    for ch in line:
        if ch == "(":
            depth += 1
        if depth > 0:
            cur += ch
        if ch == ")":
            depth -= 1
            if depth == 0:
                out.append(cur)
                cur = ""
    return out


def _read_level(ldir, D, ncomp):
    with open(os.path.join(ldir, "Cell_H")) as f:
        lines = f.read().split("\n")
    n = int(lines[4].split()[0].lstrip("("))
    boxes = [_parse_box(lines[5 + b]) for b in range(n)]
    fod = [l.split() for l in lines[7 + n:7 + 2 * n]]
    fabs = []
    for (lo, hi), (_, fname, off) in zip(boxes, fod):
        with open(os.path.join(ldir, fname), "rb") as f:
            f.seek(int(off))
            head = f.readline().decode()
            if _FORMAT not in head:
                raise ValueError("unsupported FAB real format: %s" % head.strip())
            little = _ORDER["little"] in head
            shape = tuple(hi[d] - lo[d] + 1 if d < D else 1 for d in (2, 1, 0))
            cnt = ncomp * int(np.prod(shape))
            a = np.frombuffer(f.read(8 * cnt), dtype="<f8" if little else ">f8")
        fabs.append(a.astype(np.float64).reshape((ncomp,) + shape))
    return boxes, fabs


def amr_plot_levels(amr):
    """(levels, varnames, level ratio) of a device hierarchy for
    write_plotfile: every level's valid boxes with their conserved state."""
    D = amr.D
    names = ["density"] + ["mom_" + "xyz"[d] for d in range(D)] + ["energy"]
    levels = []
    for lev in range(amr.finest_level + 1):
        dlo, dhi = amr.domain(lev)
        glob = amr.get_state(lev)
        boxes = amr.boxes(lev)
        fabs = []
        for lo, hi in boxes:
            sl = tuple(slice(lo[d] - dlo[d], hi[d] - dlo[d] + 1) if d < D else slice(0, 1) for d in (2, 1, 0))
            fabs.append(np.ascontiguousarray(glob[(slice(None),) + sl]))
        levels.append((dlo, dhi, boxes, fabs))
    return levels, names


def write_amr_plotfile(path, amr, step=0):
    """The plotfile of a device hierarchy's current state (conserved
    variables density, mom_x.., energy on every level)."""
    levels, names = amr_plot_levels(amr)
    write_plotfile(path, amr.D, amr.time, amr.prob_lo, amr.prob_hi, levels, names, ref_ratio=amr.ratio,
                   level_steps=[step * amr.ratio ** l for l in range(len(levels))])
