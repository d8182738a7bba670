"""Autotuner for the sweep launches of a level: the work-item shape (the
x-segment length of the row-marching x sweep and the column-segment length
of the strided y/z sweeps) is chosen by timing the candidates on the device
with the level's own sweep timing events, and remembered per configuration
(device, dimension, precision, method, box shapes) in a small JSON cache.

The default choice inside the library (segments long enough to give every
resident warp about six items) is the starting point; the tuner keeps it
unless a candidate is measurably faster.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

X_CANDIDATES = (32, 64, 128, 256, 512, 1024, 2048)
S_CANDIDATES = (16, 24, 32, 48, 64, 96, 128, 256)


def _cache_path():
    base = os.environ.get("BAMREX_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "bamrex_b200")
    return os.path.join(base, "sweep_segments.json")


def config_key(spacedim, boxes, precision, method, parm, device_name):
    shapes = sorted({tuple(hi[d] - lo[d] + 1 for d in range(3)) for lo, hi in boxes})
    raw = json.dumps([device_name, spacedim, precision, method, parm.limiter, parm.adiabatic, len(boxes), shapes])
    return hashlib.sha1(raw.encode()).hexdigest()


def _time_level(make_level, u0, x_seg, s_seg, steps):
    lev = make_level(x_seg, s_seg)
    try:
        lev.set_state(u0)
        lev.run(1, use_graph=False)
        lev.set_timing(True)
        lev.reset_counters()
        lev.run(steps, use_graph=False)
        times = [ms / max(1, n) for ms, n in lev.sweep_times()]
    finally:
        lev.close()
    return times


def tune_segments(spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, u0, method=0, precision=0, bc_lo=None,
                  bc_hi=None, steps=3, use_cache=True, log=None):
    """Best (x_segment, s_segment) for this level configuration, and the
    measured table {candidate: [ms per sweep by direction]}."""
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
            c = cache[key]
            return c["x_segment"], c["s_segment"], c.get("table", {})

    def make(xs, ss):
        return Level(spacedim, dom_lo, dom_hi, prob_lo, prob_hi, boxes, parm, method=method, cfl=0.8, bc_lo=bc_lo,
                     bc_hi=bc_hi, x_segment=xs, s_segment=ss, precision=precision)

    base = _time_level(make, u0, 0, 0, steps)
    table = {"auto": base}
    best_x, best_x_ms = 0, base[0]
    best_s, best_s_ms = 0, (sum(base[1:]) if spacedim > 1 else 0.0)
    max_len = max(hi[0] - lo[0] + 1 for lo, hi in boxes)
    for xs in X_CANDIDATES:
        if xs > max(32, max_len):
            continue
        t = _time_level(make, u0, xs, best_s or 0, steps)
        table["x%d" % xs] = t
        if t[0] < 0.98 * best_x_ms:
            best_x, best_x_ms = xs, t[0]
    if spacedim > 1:
        for ss in S_CANDIDATES:
            t = _time_level(make, u0, best_x, ss, steps)
            table["s%d" % ss] = t
            if sum(t[1:]) < 0.98 * best_s_ms:
                best_s, best_s_ms = ss, sum(t[1:])
    if log:
        log("autotune %s: x_segment %s, s_segment %s" % (key[:8], best_x or "auto", best_s or "auto"))
    if use_cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache[key] = {"x_segment": best_x, "s_segment": best_s, "table": table}
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f)
        os.replace(tmp, path)
    return best_x, best_s, table


def segment_table_summary(table):
    """Compact {candidate: total sweep ms} for reports."""
    return {k: float(np.sum(v)) for k, v in table.items()}
