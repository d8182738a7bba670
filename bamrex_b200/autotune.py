"""Autotuner for the sweep launches of a level: per direction the sweep
kernel (how it stages its input and shares the stencil: the L2-loading row
or marching kernels, the TMA-staged per-warp march, or the TMA-staged block
wavefront) and then the work-item shape (segment lengths along the sweep)
are chosen by timing the candidates on the device with the level's own
sweep timing events, and remembered per configuration (device, dimension,
precision, method, box shapes, library version) in a small JSON cache.

The library's own choice (a slot-step cost model for the kernel, segments
that keep every resident unit busy) is the starting point; the tuner keeps
it unless a candidate is measurably faster.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

from . import _abi

X_CANDIDATES = (32, 64, 128, 256, 512, 1024, 2048)
S_CANDIDATES = (16, 24, 32, 48, 64, 96, 128, 256)
# (staging, x_mode) of each kernel kind tried; x_mode only matters for the
# L2-loading x sweep
KINDS = {"rows": (_abi.STAGING_REGISTERS, _abi.XSWEEP_ROWS), "march": (_abi.STAGING_REGISTERS, _abi.XSWEEP_MARCH),
         "tma": (_abi.STAGING_TMA, _abi.XSWEEP_AUTO), "wave": (_abi.STAGING_WAVE, _abi.XSWEEP_AUTO)}
_CACHE_VERSION = 2


def _cache_path():
    base = os.environ.get("BAMREX_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "bamrex_b200")
    return os.path.join(base, "sweep_tuning.json")


def config_key(spacedim, boxes, precision, method, parm, device_name):
    shapes = sorted({tuple(hi[d] - lo[d] + 1 for d in range(3)) for lo, hi in boxes})
    raw = json.dumps([_CACHE_VERSION, _abi.lib().bamrex_abi_version(), device_name, spacedim, precision, method,
                      parm.limiter, parm.adiabatic, len(boxes), shapes])
    return hashlib.sha1(raw.encode()).hexdigest()


def _time_level(make_level, u0, steps, **kw):
    lev = make_level(**kw)
    try:
        kinds = [lev.staging(d) for d in range(lev.D)]
        lev.set_state(u0)
        lev.run(1, use_graph=False)
        lev.set_timing(True)
        lev.reset_counters()
        lev.run(steps, use_graph=False)
        times = [ms / max(1, n) for ms, n in lev.sweep_times()]
    finally:
        lev.close()
    return times, kinds


def tune_sweeps(spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, u0, method=0, precision=0, bc_lo=None,
                bc_hi=None, steps=3, use_cache=True, log=None):
    """Best sweep set-up for this level configuration: a dict with
    staging_dir (per direction), x_mode, x_segment, s_segment (0: the
    library's choice), and the measured table {candidate: [ms per sweep by
    direction]}."""
    import torch

    from .level import Level
    dev = torch.cuda.get_device_name()
    key = config_key(spacedim, boxes, precision, method, parm, dev)
    path = _cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return cache[key]

    def make(staging_dir=(0, 0, 0), x_mode=0, x_segment=0, s_segment=0):
        return Level(spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, method=method, cfl=0.8, bc_lo=bc_lo,
                     bc_hi=bc_hi, x_segment=x_segment, s_segment=s_segment, precision=precision,
                     staging_dir=staging_dir, x_mode=x_mode)

    D = spacedim
    base, base_kinds = _time_level(make, u0, steps)
    table = {"auto": base}
    # kernel per direction: every direction swept by one kind at a time
    best = {d: ("auto", base[d]) for d in range(D)}
    for name, (staging, xm) in KINDS.items():
        if name in ("rows", "march") and D == 1:
            continue
        try:
            t, _ = _time_level(make, u0, steps, staging_dir=(staging,) * 3, x_mode=xm)
        except _abi.BamrexError:
            continue  # the TMA kinds serve the fast path only
        table[name] = t
        for d in range(D):
            if name == "rows" and d > 0:
                continue  # the y / z sweeps of "rows" are the marching kernels of "march"
            if t[d] < 0.98 * best[d][1]:
                best[d] = (name, t[d])
    staging_dir = [0, 0, 0]
    x_mode = 0
    for d in range(D):
        name = best[d][0]
        if name == "auto":
            staging_dir[d] = base_kinds[d]
        else:
            staging_dir[d] = KINDS[name][0]
            if d == 0 and name in ("rows", "march"):
                x_mode = KINDS[name][1]
    cfg = {"staging_dir": staging_dir, "x_mode": x_mode}
    cur, _ = _time_level(make, u0, steps, **cfg)
    # segment lengths for the chosen kernels
    best_x, best_x_ms = 0, cur[0]
    max_len = max(hi[0] - lo[0] + 1 for lo, hi in boxes)
    for xs in X_CANDIDATES:
        if xs > max(32, max_len):
            continue
        t, _ = _time_level(make, u0, steps, x_segment=xs, **cfg)
        table["x%d" % xs] = t
        if t[0] < 0.98 * best_x_ms:
            best_x, best_x_ms = xs, t[0]
    best_s = 0
    if D > 1:
        best_s_ms = sum(cur[1:])
        for ss in S_CANDIDATES:
            t, _ = _time_level(make, u0, steps, x_segment=best_x, s_segment=ss, **cfg)
            table["s%d" % ss] = t
            if sum(t[1:]) < 0.98 * best_s_ms:
                best_s, best_s_ms = ss, sum(t[1:])
    res = {"staging_dir": staging_dir, "x_mode": x_mode, "x_segment": best_x, "s_segment": best_s,
           "auto_kinds": base_kinds, "table": table}
    if log:
        log("autotune %s: kernels %s, x_segment %s, s_segment %s" % (key[:8], staging_dir[:D], best_x or "auto",
                                                                     best_s or "auto"))
    if use_cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache[key] = res
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f)
        os.replace(tmp, path)
    return res


def tune_segments(spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, u0, method=0, precision=0, bc_lo=None,
                  bc_hi=None, steps=3, use_cache=True, log=None):
    """The segment lengths tune_sweeps picks (for the kernels it picks) and
    its measured table."""
    r = tune_sweeps(spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, u0, method, precision, bc_lo, bc_hi,
                    steps, use_cache, log)
    return r["x_segment"], r["s_segment"], r["table"]


KIND_NAMES = {_abi.STAGING_REGISTERS: "registers", _abi.STAGING_TMA: "tma", _abi.STAGING_WAVE: "wave"}


def segment_table_summary(table):
    """Compact {candidate: total sweep ms} for reports."""
    return {k: round(float(np.sum(v)), 4) for k, v in table.items()}
