#!/usr/bin/env python
"""Throughput of the explicit finite-volume path on B200.

Workload (one "step" = one full split time step, x sweep then y sweep, of
the whole grid, with the device-side CFL reduction and dt update):
2D four-quadrant Riemann problem, 4096 x 4096 cells on [0,1]^2, gamma 1.4,
seeded quadrant states (rho ~ U[0.1,1.5], u,v ~ U[-1,1], p ~ U[0.03,1.5])
with a 1e-3 relative white-noise density perturbation, MUSCL-Hancock with
the minbee limiter + HLLC, CFL 0.8, transmissive boundaries, FP64.

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU
restatement of the reference path (oracle/, the reference itself cannot be
built without AMReX) on the host cores instead.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s"
NC2D = 4


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4096, help="cells per side")
    ap.add_argument("--max-grid-size", type=int, default=0, help="box size (0: one box per rank)")
    ap.add_argument("--graph", type=int, default=0, help="1: time the CUDA-graph replay instead")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--e2e-slabs", type=int, default=0, help="slabs of the streamed host steps (0: the library picks)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-storage variant")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-imex", action="store_true", help="skip the IMEX pressure-solve comparison")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default sweep segments")
    ap.add_argument("--x-mode", type=int, default=0, help="x-sweep kernel: 0 automatic, 1 warp per row, 2 thread per row")
    ap.add_argument("--no-amr", action="store_true", help="skip the 3D AMR blast sample")
    ap.add_argument("--amr-n", type=int, default=256, help="base cells per side of the AMR blast sample")
    ap.add_argument("--amr-steps", type=int, default=100, help="timed coarse steps of the AMR blast sample (fixed grids)")
    ap.add_argument("--amr-regrid-steps", type=int, default=10,
                    help="timed coarse steps of the AMR blast sample with a regrid every 2")
    ap.add_argument("--imex-n", type=int, default=2048, help="cells per side of the IMEX pressure problem")
    ap.add_argument("--no-body", action="store_true", help="skip the ghost-fluid rigid-body sample")
    ap.add_argument("--body-cases", default="2d,3d,3d_amr", help="rigid-body cases to run (2d, 3d, 3d_amr)")
    ap.add_argument("--body-amr-n", type=int, nargs=3, default=[512, 512, 128],
                    help="base cells of the two-level rigid-body sample")
    ap.add_argument("--body-amr-steps", type=int, default=50, help="timed coarse steps of the two-level rigid-body sample")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity checks against the oracle")
    ap.add_argument("--split", action="store_true",
                    help="run the multi-rank (split-level, NCCL) path also on one rank")
    ap.add_argument("--fp32-oracle-steps", type=int, default=10,
                    help="steps of the FP32-storage L1 comparison with the FP64 oracle (0: skip)")
    return ap.parse_args()


def workload_config(n, boxes, mgs, extra=None):
    cfg = {
        "workload": "2D four-quadrant Riemann problem %dx%d, MUSCL-Hancock/minbee + HLLC, CFL 0.8, transmissive, "
                    "FP64, 1 step = x sweep + y sweep + CFL/dt" % (n, n),
        "cells": n * n,
        "boxes": boxes,
        "max_grid_size": mgs,
        "l2": "inputs larger than L2: %.0f MB state per buffer > 126 MB" % (NC2D * 8 * n * n / 1e6),
        "seed": 20261203,
    }
    if extra:
        cfg.update(extra)
    return cfg


KIND_NAMES = {1: "registers", 2: "tma", 3: "wave"}


def sweep_kernel_name(D, d, kind, x_rows):
    if kind == 3:
        return "sweep_wave_kernel<%d,%d>" % (D, d)
    if kind == 2:
        return "sweep_tma_kernel<%d,%d>" % (D, d)
    return "sweep_x_kernel<%d>" % D if (d == 0 and x_rows) else "sweep_s_kernel<%d,%d>" % (D, d)


def parity_check(lev, u_start, n, steps_from):
    """One step of the bench's own level (its kernels and segments) against
    the oracle from the same input: relative L-infinity per component and
    relative conserved totals (the drop-in bar: 1e-12 and 1e-13)."""
    import numpy as np

    from oracle import oracle as o
    hi = (n - 1, n - 1, 0)
    lay = o.LevelLayout(2, (0, 0, 0), hi, o.decompose(2, (0, 0, 0), hi, 64), 2, [1.0 / n, 1.0 / n])
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u_start)
    lay.fill_boundary(S1)
    dt_ref = lay.est_time_step(S1, 1.4, 1.0, 0.8)
    S2[:] = S1
    lay.advance_explicit(S1, S2, 0.0, dt_ref, o.MUSCL_HANCOCK, o.Parm(2, limiter=o.MINBEE))
    ref = lay.gather(S1)
    lev.set_state(u_start)
    dt = lev.estTimeStep()
    lev.advance(0.0, dt_ref)
    got = lev.get_state()
    linf = [float(np.max(np.abs(got[c] - ref[c])) / np.max(np.abs(ref[c]))) for c in range(4)]
    tot = [float(abs(got[c].sum() - ref[c].sum()) / np.abs(ref[c]).sum()) for c in range(4)]
    return {"from": steps_from, "rel_linf": linf, "rel_totals": tot, "dt_rel": abs(dt - dt_ref) / dt_ref,
            "pass": max(linf) <= 1e-12 and max(tot) <= 1e-13 and abs(dt - dt_ref) <= 1e-14 * dt_ref}


def fp32_l1_vs_oracle(n, u0, steps, lev32):
    """FP32-storage state after `steps` steps of the oracle's dt sequence
    against the FP64 oracle: relative L1 of density and energy."""
    import numpy as np

    from oracle import oracle as o
    hi = (n - 1, n - 1, 0)
    lay = o.LevelLayout(2, (0, 0, 0), hi, o.decompose(2, (0, 0, 0), hi, 64), 2, [1.0 / n, 1.0 / n])
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u0)
    P = o.Parm(2, limiter=o.MINBEE)
    lev32.set_state(u0)
    t = 0.0
    for _ in range(steps):
        lay.fill_boundary(S1, fast=True)
        dt = lay.est_time_step(S1, 1.4, 1.0, 0.8, fast=True)
        S2[:] = S1
        lay.advance_explicit(S1, S2, t, dt, o.MUSCL_HANCOCK, P, fast=True)
        lev32.advance(t, dt)
        t += dt
    ref, got = lay.gather(S1), lev32.get_state()
    return {"steps": steps, "rel_l1_rho": float(np.abs(got[0] - ref[0]).sum() / np.abs(ref[0]).sum()),
            "rel_l1_E": float(np.abs(got[3] - ref[3]).sum() / np.abs(ref[3]).sum()),
            "reference": "FP64 oracle (optimised build), same dt sequence"}


def parity_scalars(parity):
    """The parity figures as flat config entries."""
    if not parity:
        return {}
    out = {}
    for k in ("fp64_step_from_initial", "fp64_step_from_timed_state"):
        if k in parity:
            out["parity_%s_rel_linf" % k[5:]] = max(parity[k]["rel_linf"])
            out["parity_%s_rel_totals" % k[5:]] = max(parity[k]["rel_totals"])
    if "fp32_storage" in parity:
        out["parity_fp32_l1_rho"] = parity["fp32_storage"]["rel_l1_rho"]
        out["parity_fp32_l1_E"] = parity["fp32_storage"]["rel_l1_E"]
    return out


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, interval_ms=50):
        self.index, self.interval_ms = index, interval_ms
        self.proc, self.lines, self.marks = None, [], []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", str(self.interval_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.time(), ln.strip()))

    def mark(self, name):
        self.marks.append((name, time.time()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        rows = []
        for ts, ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((ts, float(f[1]), float(f[2]), f))
            except ValueError:
                continue
        inside = [r for r in rows if t0 <= r[0] <= t1]
        window = "timed region"
        if not inside:
            inside = rows
            window = "whole run (no sample fell inside the timed region)"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, _, _, f in inside:
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[1] for r in inside), "sm_max_mhz": max(r[2] for r in inside),
                "reasons": sorted(reasons), "samples": len(inside), "window": window}


# ------------------------------------------------------------------ helpers
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kind):
    """DRAM bytes per cell per sweep launch from the committed ncu summary
    (profiles/sweep_*.md, line 'dram_bytes_per_cell_<kind>: X'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith(".md"):
            continue
        m = re.search(r"dram_bytes_per_cell_%s:\s*([0-9.]+)" % kind, open(os.path.join(pdir, fn)).read())
        if m:
            return float(m.group(1))
    return None


def cpu_baseline_run(n_full, seconds, warm_steps=0, fixed_steps=None):
    """Time the CPU restatement (oracle/, optimised build, all host threads)
    on the same workload with the reference's 64x64 boxes.  The sample is
    the full grid when one step fits the time budget, else a smaller square
    grid of the same problem.  Returns a dict (value in cell-updates/s)."""
    import numpy as np

    from bamrex_b200 import problems
    from oracle import oracle as o

    march = o.use_native_build()
    cpu = o.host_cpu()
    threads = o.num_threads(fast=True)

    def setup(n):
        hi = (n - 1, n - 1, 0)
        boxes = o.decompose(2, (0, 0, 0), hi, 64)
        lay = o.LevelLayout(2, (0, 0, 0), hi, boxes, 2, [1.0 / n, 1.0 / n])
        S1, S2 = lay.alloc(), lay.alloc()
        lay.scatter(S1, problems.quadrant_2d(n))
        lay.fill_boundary(S1, fast=True)
        return lay, S1, S2

    parm = o.Parm(2, limiter=o.MINBEE)

    def step(lay, S1, S2, t, dt):
        S2[:] = S1
        lay.advance_explicit(S1, S2, t, dt, o.MUSCL_HANCOCK, parm, fast=True)
        lay.fill_boundary(S1, fast=True)
        return lay.est_time_step(S1, 1.4, 1.0, 0.8, fast=True)

    # calibrate on 512^2
    lay, S1, S2 = setup(512)
    dt = lay.est_time_step(S1, 1.4, 1.0, 0.8, fast=True)
    t0 = time.perf_counter()
    dt = step(lay, S1, S2, 0.0, dt)
    rate = 512 * 512 / (time.perf_counter() - t0)
    steps_wanted = fixed_steps if fixed_steps is not None else None
    n = n_full
    total = steps_wanted + warm_steps if steps_wanted else 1
    while n > 512 and total * n * n / rate > seconds:
        n //= 2
    lay, S1, S2 = setup(n)
    dt = lay.est_time_step(S1, 1.4, 1.0, 0.8, fast=True)
    t = 0.0
    for _ in range(warm_steps):
        dt_new = step(lay, S1, S2, t, dt)
        t += dt
        dt = dt_new
    steps = 0
    t0 = time.perf_counter()
    while True:
        dt_new = step(lay, S1, S2, t, dt)
        t += dt
        dt = dt_new
        steps += 1
        el = time.perf_counter() - t0
        if fixed_steps is not None:
            if steps >= fixed_steps:
                break
        elif el >= seconds or steps >= 50:
            break
    el = time.perf_counter() - t0
    value = n * n * steps / el
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "elapsed_s": el, "steps": steps,
            "n": n, "cpu_model": cpu["model"], "isa": cpu["isa"], "march": march,
            "sample": "%d step(s) of the same 2D quadrant problem at %dx%d (64x64 boxes, the reference's "
                      "max_grid_size), CPU restatement of the reference path, -O3 -funroll-loops -march=%s "
                      "(host %s, %s), OpenMP over boxes, %d threads"
                      % (steps, n, n, march, cpu["model"], cpu["isa"], threads)}


# ------------------------------------------------------------------ arms
def imex_pressure_run(n):
    """The 2D IMEX pressure solve at n^2 (lognormal density, Mach 0.01):
    plain BiCGStab + multigrid V-cycle against FGMRES with the learned
    preconditioner, both to 1e-8 relative residual; the network is trained
    here on 2000 pairs from the plain solver (256^2 patches, what one V-cycle
    leaves of random right-hand sides)."""
    import numpy as np
    import torch

    from bamrex_b200 import problems
    from bamrex_b200._abi import PRECOND_NETWORK_VCYCLE, PRECOND_VCYCLE, PRECOND_VCYCLE_NETWORK
    from bamrex_b200.helmholtz import Helmholtz
    from bamrex_b200.learned import PrecNet, make_training_pairs, solve_learned_device, train

    p = problems.low_mach_pressure_problem(n=n)
    h = Helmholtz(2, (n, n))
    h.setScalars(1.0, p["B"], 0.0)
    h.setACoeffs(p["a"])
    h.setBCoeffsFromCell(p["beta_cc"])
    rhs = torch.from_numpy(p["rhs"].copy()).cuda()
    x = torch.zeros_like(rhs)

    def timed(fn, reps=3):
        best, out = None, None
        for _ in range(reps):
            x.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        return best * 1e3, out

    h.solve_device(x, rhs, tol_rel=1e-8)  # graph build
    plain_ms, (pit, prr) = timed(lambda: h.solve_device(x, rhs, tol_rel=1e-8))
    t0 = time.time()
    # pairs of what one V-cycle leaves (residual, error): the network of the
    # two combined modes corrects a V-cycle (raw (residual, error) pairs made
    # FGMRES take 21-29 iterations instead of 13-14 at 2048^2)
    X, Y = make_training_pairs(2000, n=256, seed=7, after_vcycle=True)
    t_pairs = time.time() - t0
    net = PrecNet(256, 256, batch=8, seed=1)
    t0 = time.time()
    losses = train(net, X, Y, epochs=6, batch=8, lr=2e-3)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    net.resize(n, n, 1)
    learned = {}
    for name, mode in (("network+vcycle", PRECOND_NETWORK_VCYCLE), ("vcycle+network", PRECOND_VCYCLE_NETWORK),
                       ("vcycle_only", PRECOND_VCYCLE)):
        ms, (it, fit, rr, fb) = timed(lambda: solve_learned_device(h, net if mode != PRECOND_VCYCLE else None, x, rhs,
                                                                   tol_rel=1e-8, max_iter=100, restart=30, mode=mode), 2)
        learned[name] = {"ms": ms, "fgmres_iterations": it, "fallback_iterations": fit, "rel_residual": rr,
                         "fell_back": fb}
    best = min(("network+vcycle", "vcycle+network"), key=lambda k: learned[k]["ms"])
    h.close()
    step = imex_step_run(n, net, {"network+vcycle": PRECOND_NETWORK_VCYCLE,
                                  "vcycle+network": PRECOND_VCYCLE_NETWORK}[best])
    net.close()
    return {
        "workload": "2D IMEX pressure solve %dx%d, lognormal density (log-sigma 1, correlation 32 cells), beta = 1/rho, "
                    "Mach 0.01, periodic, target relative residual 1e-8" % (n, n),
        "plain": {"solver": "BiCGStab + multigrid V-cycle (GSRB 2+2, CUDA graph per iteration)", "ms": plain_ms,
                  "iterations": pit, "rel_residual": prr},
        "learned": {"solver": "FGMRES(30) + network (4 levels, 16 channels, 3x3, BF16 weights, FP32 accumulation)",
                    "best_mode": best, "modes": learned, "train_pairs": 2000, "pairs": "after one V-cycle",
                    "pairs_seconds": t_pairs,
                    "train_seconds": t_train, "train_loss_first_last": [float(np.mean(losses[:10])),
                                                                        float(np.mean(losses[-10:]))]},
        "learned_over_plain_time": learned[best]["ms"] / plain_ms,
        "target_ratio": 0.5,
        "imex_step": step,
    }


def imex_step_run(n, net, mode, steps=5):
    """Full first-order IMEX steps (bamrex_imex: Rusanov advection, enthalpy
    from the previous pressure, explicit kinetic energy, pressure solve to
    1e-8, fluxes, update) on the 2D low-Mach state at n^2, periodic, CFL 0.8
    on the advective speed: ms per step with the plain and with the learned
    pressure solve."""
    import torch

    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.imex import Imex

    U, p = problems.low_mach_state(n)
    out = {"workload": "2D low-Mach IMEX step %dx%d: lognormal density (log-sigma 1, correlation 32 cells), "
                       "velocity the curl of a random stream function at peak 0.01, p = 1/gamma, epsilon 1, periodic, "
                       "Rusanov advection, enthalpy from the previous pressure, explicit kinetic energy, pressure solve "
                       "to 1e-8, advective CFL 0.8" % (n, n), "steps": steps}
    for name in ("plain", "learned"):
        im = Imex(2, (n, n), [0.0, 0.0], [1.0, 1.0], bx.Parm(2, adiabatic=1.4, epsilon=1.0), bc_lo=[1, 1],
                  bc_hi=[1, 1], cfl=0.8, tol_rel=1e-8)
        if name == "learned":
            im.set_precnet(net, mode)
        im.set_state(U, p)
        im.step(im.est_time_step())  # builds the solver's graphs
        im.set_state(U, p)
        its = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            it, rr = im.step(im.est_time_step())
            its.append(it)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / steps
        out[name] = {"ms_per_step": ms, "solve_iterations": its, "last_rel_residual": rr}
        im.close()
    out["learned_over_plain_step_time"] = out["learned"]["ms_per_step"] / out["plain"]["ms_per_step"]
    return out


def amr_blast_run(n0, coarse_steps, precision, regrid_steps=None):
    """The 3D spherical blast on a 3-level hierarchy (ratio 2, blocking
    factor 8, max_grid_size drawn per box from {16,32,48,64}, grad_error on
    rho >= 0.1, regrid every 2 coarse steps, subcycling): cell-updates/s
    over `coarse_steps` coarse steps after the levels have formed."""
    import torch

    import bamrex_b200 as bx
    from bamrex_b200.amr import blast_hierarchy

    A, _ = blast_hierarchy(n0, precision)
    cells = [sum(int(np.prod([h[d] - l[d] + 1 for d in range(3)])) for l, h in A.boxes(lev))
             for lev in range(A.finest_level + 1)]
    nboxes = [len(A.boxes(lev)) for lev in range(A.finest_level + 1)]
    updates_per_step = sum(c * 2 ** lev for lev, c in enumerate(cells))
    s0 = A.conserved_sums()
    # stepping alone (fixed grids), then with a regrid every 2 coarse steps
    A.set_regrid_int(0)
    # the host-driven coarse step (every launch from the host, dt read back
    # per level) for comparison, then the graph-replayed one (warmed up: the
    # first step after a change of the levels is host-driven, the next two
    # capture the graphs of the two buffer states of the 3D base level)
    n_host = min(20, coarse_steps)
    A.set_graph(False)
    A.coarse_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_host):
        A.coarse_step()
    torch.cuda.synchronize()
    dt_host = time.perf_counter() - t0
    A.set_graph(True)
    for _ in range(3):
        A.coarse_step()
    caps0, reps0, _ = A.graph_stats()
    torch.cuda.synchronize()
    # an NVTX range lets a profiler capture exactly these steps
    # (ncu --nvtx --nvtx-include "amr_fixed_steps_fp64/")
    torch.cuda.nvtx.range_push("amr_fixed_steps_" + ("fp64" if precision == bx.FP64 else "fp32"))
    t0 = time.perf_counter()
    for _ in range(coarse_steps):
        A.coarse_step()
    torch.cuda.synchronize()
    dt_fixed = time.perf_counter() - t0
    torch.cuda.nvtx.range_pop()
    caps1, reps1, kernels = A.graph_stats()
    s1 = A.conserved_sums()
    kinds = [[A.level(lev).staging(d) for d in range(3)] for lev in range(A.finest_level + 1)]
    A.set_regrid_int(2)
    nr = coarse_steps if regrid_steps is None else regrid_steps
    t0 = time.perf_counter()
    for _ in range(nr):
        A.coarse_step()
    torch.cuda.synchronize()
    dt_regrid = time.perf_counter() - t0
    A.close()
    return {"cells_per_level": cells, "boxes_per_level": nboxes, "coarse_steps": coarse_steps,
            "ms_per_coarse_step": dt_fixed / coarse_steps * 1e3,
            "cell_updates_per_s": updates_per_step * coarse_steps / dt_fixed,
            "coarse_step_graph": {
                "replayed_steps": reps1 - reps0, "captures_in_timed_steps": caps1 - caps0,
                "kernel_nodes_per_graph": kernels,
                "launches_per_coarse_step": (len(cells) - 1) + 2,
                "launches_note": "per coarse step: the max wave speed of each level but the finest (its own comes "
                                 "fused with its last sweep), the device dt kernel, one graph launch",
                "host_driven_ms_per_coarse_step": dt_host / n_host * 1e3,
                "host_driven_kernel_launches_per_coarse_step": kernels + (len(cells) - 1)},
            "sweep_kernels_per_level": [",".join(KIND_NAMES[k] for k in kk) for kk in kinds],
            "coarse_steps_with_regrid": nr,
            "ms_per_coarse_step_with_regrid_every_2": dt_regrid / nr * 1e3,
            "mass_drift_rel": float(abs(s1[0] - s0[0]) / abs(s0[0]))}


def rigid_body_run(D, n, mgs, precision, steps=10, vortex=False):
    """A static cylinder of radius 0.1 at the domain centre (axis z),
    ghost-fluid reflective wall, in a free stream (Mach 0.3), or with
    vortex=True the low-Mach configuration: an isentropic vortex (strength
    0.5, core 0.05, peak swirl Mach ~0.06) carried by a Mach 0.05 free
    stream from upstream of the cylinder.  Step time with and without the body and the rigid-body ghost
    fill alone (interface cells, D + 1 extrapolation rounds, boundary
    fills)."""
    import torch

    import bamrex_b200 as bx
    from bamrex_b200.level import decompose

    boxes = decompose(D, (0,) * D, tuple(x - 1 for x in n), mgs)
    # cubic cells: the domain is [0, 1] along x
    lev = bx.Level(D, (0,) * D, tuple(x - 1 for x in n), [0.0] * D, [n[d] / n[0] for d in range(D)], boxes, bx.Parm(D),
                   cfl=0.8, ngrow=4, precision=precision)
    shp = (n[2] if D > 2 else 1, n[1], n[0])
    gamma = 1.4
    hi_phys = [n[d] / n[0] for d in range(D)]
    if vortex:
        from bamrex_b200 import problems
        U = problems.isentropic_vortex(D, n, [0.0] * D, hi_phys, centre=(0.25, 0.5), strength=0.5, scale=0.05,
                                       vel_bg=(0.05 * np.sqrt(gamma), 0.0, 0.0), adiabatic=gamma)
    else:
        U = np.zeros((D + 2,) + shp)
        u0 = 0.3 * np.sqrt(gamma)
        U[0] = 1.0
        U[1] = u0
        U[D + 1] = 1.0 / (gamma - 1) + 0.5 * u0 * u0
    lev.set_state(U)
    dt = lev.estTimeStep()

    def ms_per_step(k, fn):
        lev.sync()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(k):
            fn()
        lev.sync()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) * 1e3 / k

    ms_per_step(2, lambda: lev.advance(0.0, dt))
    plain = ms_per_step(steps, lambda: lev.advance(0.0, dt))
    t0 = time.perf_counter()
    lev.set_body(dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.5), axis=(0, 0, 1), radius=0.1))
    setup = (time.perf_counter() - t0) * 1e3
    ms_per_step(2, lambda: lev.advance(0.0, dt))
    body = ms_per_step(steps, lambda: lev.advance(0.0, dt))
    fill = ms_per_step(steps, lev.fill_body_ghosts)
    iface, swept = lev.body_counts()
    lev.close()
    ncells = int(np.prod(n))
    flow = ("isentropic vortex (strength 0.5, core 0.05) in a Mach 0.05 free stream" if vortex
            else "free stream Mach 0.3")
    return {"workload": "%s %s, max_grid_size %d, %s, %s past a cylinder r 0.1 (reflective wall)" % (
                "x".join(str(x) for x in n), "3D" if D == 3 else "2D", mgs,
                "FP32 storage" if precision == bx.FP32_STORAGE else "FP64", flow),
            "boxes": len(boxes), "interface_cells": iface, "swept_cells": swept,
            "ms_per_step_plain": plain, "ms_per_step_with_body": body, "ms_rigid_body_fill": fill,
            "set_up_ms": setup, "cell_updates_per_s_with_body": ncells / (body * 1e-3)}


def rigid_body_amr_run(n=(512, 512, 128), mgs=32, steps=50, l1_steps=10):
    """The 3D low-Mach rigid-body configuration on two AMR levels: an
    isentropic vortex (strength 0.5, core 0.05) carried by a Mach 0.05 free
    stream towards a static cylinder (r 0.1, axis z, reflective ghost-fluid
    wall), base n cells (cubic cells, x on [0, 1]) in boxes of mgs, level 1
    where errorEst's interface_error tags (|level set| <= 3 coarse cells),
    ghost_error clearing the solid; FP32 storage, explicit
    MUSCL-Hancock/HLLC coarse steps with subcycling (replayed as graphs).
    Level 1 starts from the coarse interpolation of the base level.  The
    FP32-storage density / energy L1 is taken against the FP64 hierarchy of
    the same grids after l1_steps coarse steps to the same time."""
    import torch

    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.amr import Amr
    from bamrex_b200.level import decompose

    D = 3
    hi = tuple(x - 1 for x in n)
    phys = [n[d] / n[0] for d in range(D)]
    gamma = 1.4
    U0 = problems.isentropic_vortex(D, n, [0.0] * D, phys, centre=(0.25, 0.5), strength=0.5, scale=0.05,
                                    vel_bg=(0.05 * np.sqrt(gamma), 0.0, 0.0), adiabatic=gamma)

    def make(prec):
        A = Amr(D, (0, 0, 0), hi, [0.0] * D, phys, decompose(D, (0, 0, 0), hi, mgs), bx.Parm(D), cfl=0.8, ngrow=4,
                precision=prec, max_level=1, blocking_factor=8, max_grid_size=mgs, n_error_buf=2, grid_eff=0.7,
                max_int_lev=1, lstol=[3.0 / n[0]])
        A.set_body(dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.5 * phys[2]), axis=(0, 0, 1), radius=0.1))
        A.set_state(0, U0)
        t0 = time.perf_counter()
        A.regrid(0, 0.0)
        A.avg_down_all()
        torch.cuda.synchronize()
        return A, (time.perf_counter() - t0) * 1e3

    A, regrid_ms = make(bx.FP32_STORAGE)
    cells = [sum(int(np.prod([h[d] - l[d] + 1 for d in range(3)])) for l, h in A.boxes(lev))
             for lev in range(A.finest_level + 1)]
    nboxes = [len(A.boxes(lev)) for lev in range(A.finest_level + 1)]
    updates_per_step = sum(c * 2 ** lev for lev, c in enumerate(cells))
    s0 = A.conserved_sums()
    for _ in range(3):
        A.coarse_step()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        A.coarse_step()
    torch.cuda.synchronize()
    dt_run = time.perf_counter() - t0
    s1 = A.conserved_sums()
    caps, reps, kern = A.graph_stats()
    iface = [A.level(lev).body_counts()[0] for lev in range(A.finest_level + 1)]
    A.close()
    # FP32 storage against FP64 on the same grids, to the same time
    A64, _ = make(bx.FP64)
    for _ in range(l1_steps):
        A64.coarse_step()
    t_end = A64.time
    A32, _ = make(bx.FP32_STORAGE)
    for _ in range(l1_steps):
        if A32.time < t_end:
            A32.coarse_step(t_end)
    l1 = {}
    same_grids = [A32.boxes(lev) for lev in range(A32.finest_level + 1)] == \
        [A64.boxes(lev) for lev in range(A64.finest_level + 1)]
    for lev in range(A64.finest_level + 1):
        a, b = A32.get_state(lev), A64.get_state(lev)
        m = ~np.isnan(b[0])
        for name, c in (("rho", 0), ("E", D + 1)):
            l1["level%d_rel_l1_%s" % (lev, name)] = float(np.abs(a[c][m] - b[c][m]).sum() / np.abs(b[c][m]).sum())
    l1["time"] = t_end
    l1["fp32_time"] = A32.time
    l1["same_grids"] = same_grids
    l1["reference"] = ("FP64 hierarchy of the same grids on the device (its path matches the oracle to 1e-12 "
                       "per substep at the test sizes)")
    A32.close()
    A64.close()
    return {"workload": "3D %s base, max_grid_size %d, 2 levels (ratio 2, blocking factor 8) around a cylinder r 0.1 "
                        "by interface tagging (|level set| <= 3 coarse cells), FP32 storage, isentropic vortex "
                        "(strength 0.5, core 0.05) in a Mach 0.05 free stream, reflective ghost-fluid wall, explicit "
                        "MUSCL-Hancock/HLLC, CFL 0.8, subcycling" % ("x".join(str(x) for x in n), mgs),
            "cells_per_level": cells, "boxes_per_level": nboxes, "interface_cells_per_level": iface,
            "coarse_steps": steps, "ms_per_coarse_step": dt_run / steps * 1e3,
            "cell_updates_per_s": updates_per_step * steps / dt_run, "regrid_ms": regrid_ms,
            "graph": {"captures": caps, "replayed_steps": reps, "kernel_nodes_per_graph": kern},
            "mass_drift_rel": float(abs(s1[0] - s0[0]) / abs(s0[0])),
            "fp32_vs_fp64": l1,
            "not_built": "the IMEX pressure step of this configuration (IMEX runs on one box covering the domain)"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    r = cpu_baseline_run(args.n, seconds=120.0, warm_steps=args.warmup, fixed_steps=args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": args.gpus,
        "steps": r["steps"], "warmup": args.warmup, "ms_per_step": 1e3 * r["elapsed_s"] / r["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded four-quadrant initial state)",
        "config": workload_config(args.n, None, 64, {"sample_n": r["n"], "threads": r["cores"]}),
        "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"], "cpu_model": r["cpu_model"], "isa": r["isa"], "march": r["march"]},
        "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference needs the AMReX library (not available offline), so its CPU path runs as the "
                "line-by-line restatement in oracle/",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import bamrex_b200 as bx
    from bamrex_b200 import problems

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the timing build of the CPU baseline for this host's CPU, before
        # anything loads the oracle's default timing build
        from oracle import oracle as o
        o.use_native_build()

    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev_index = torch.cuda.current_device()
    n = args.n
    D = 2
    hi = (n - 1, n - 1, 0)
    mgs = args.max_grid_size if args.max_grid_size > 0 else n
    boxes = bx.decompose(D, (0, 0, 0), hi, mgs)
    u0 = problems.quadrant_2d(n)
    stream = torch.cuda.Stream()
    parm = bx.Parm(D, limiter=bx.MINBEE)
    setup = {"staging_dir": (0, 0, 0), "x_mode": args.x_mode, "x_segment": 0, "s_segment": 0}
    tuned = None
    if not args.no_autotune:
        from bamrex_b200.autotune import segment_table_summary, tune_sweeps
        r = tune_sweeps(D, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], boxes, parm, u0, steps=3)
        setup = {k: r[k] for k in setup}
        tuned = {"kernels": [KIND_NAMES[k] for k in r["staging_dir"][:D]], "x_segment": r["x_segment"] or "library",
                 "s_segment": r["s_segment"] or "library",
                 "library_choice": [KIND_NAMES[k] for k in r["auto_kinds"]],
                 "candidates_ms_per_step": segment_table_summary(r["table"])}
    lev = bx.Level(D, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], boxes, parm, method=bx.MUSCL_HANCOCK, cfl=0.8,
                   stream=stream, **setup)
    kinds = [lev.staging(d) for d in range(D)]
    x_rows = lev.x_mode == bx.XSWEEP_ROWS
    lev.set_state(u0)
    use_graph = bool(args.graph)

    # warm-up (also builds the CUDA graphs)
    lev.run(args.warmup, use_graph=use_graph)
    lev.run(1, use_graph=not use_graph)
    lev.set_state(u0)

    clocks = ClockSampler(dev_index)
    clocks.start()
    time.sleep(0.3)
    lev.set_timing(not use_graph)
    lev.reset_counters()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.time()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        lev.run_async(args.steps, use_graph=use_graph)
        ev1.record(stream)
    t_end, steps_done = lev.run_wait()
    torch.cuda.synchronize()
    t_wall1 = time.time()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    launches, sweep_ms, sweep_launches = lev.counters()
    lev.set_timing(False)
    u_fp64 = lev.get_state() if (rank == 0 and (not args.no_fp32 or not args.no_parity)) else None
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    assert steps_done == args.steps, (steps_done, args.steps)

    # e2e through the public API with host buffers: every step the state goes
    # host -> device, one step + its CFL estimate, device -> host
    # (bamrex_level_run_host: slabs streamed, the copies in both directions
    # overlap each other, the sweeps and the neighbouring steps' copies).
    pk = lev.packing
    host = torch.empty(pk.size, dtype=torch.float64, pin_memory=True)
    host.numpy()[:] = pk.pack(u0)
    hptr = host.data_ptr()
    dt = lev.estTimeStep()
    # one untimed step: the host step's streams, events and output staging
    # are created on first use
    lev.run_host_ptr(hptr, 1, dt, 0.0, args.e2e_slabs)
    e2e_slabs = lev.host_slabs(args.e2e_slabs)
    host.numpy()[:] = pk.pack(u0)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_e0 = time.time()
    with torch.cuda.stream(stream):
        e0.record(stream)
        tsim = 0.0
        tsim, dt = lev.run_host_ptr(hptr, args.e2e_steps, dt, 0.0, args.e2e_slabs)
        e1.record(stream)
    lev.sync()
    t_e1 = time.time()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    clocks.stop()
    # the copy roof of that path on this host: one state-sized pinned upload
    # and download at once (two streams), best of 3
    pcie = None
    if rank == 0:
        e2e_bytes = 8 * pk.size
        dev_buf = torch.empty(pk.size, dtype=torch.float64, device="cuda")
        host_dn = torch.empty(pk.size, dtype=torch.float64, pin_memory=True)
        s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()
        dev_src = torch.zeros(pk.size, dtype=torch.float64, device="cuda")
        best = 1e30
        for _ in range(3):
            torch.cuda.synchronize()
            c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c0.record()
            s_up.wait_stream(torch.cuda.current_stream())
            s_dn.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s_up):
                dev_buf.copy_(host, non_blocking=True)
            with torch.cuda.stream(s_dn):
                host_dn.copy_(dev_src, non_blocking=True)
            torch.cuda.current_stream().wait_stream(s_up)
            torch.cuda.current_stream().wait_stream(s_dn)
            c1.record()
            torch.cuda.synchronize()
            best = min(best, c0.elapsed_time(c1))
        roof_gbs = 2 * e2e_bytes / (best * 1e-3) / 1e9
        got_gbs = 2 * e2e_bytes * args.e2e_steps / (e2e_ms * 1e-3) / 1e9
        pcie = {"bidirectional_copy_GBps": roof_gbs, "achieved_GBps": got_gbs, "frac": got_gbs / roof_gbs,
                "how": "one %d-byte pinned host->device and device->host copy at once on two streams, best of 3; "
                       "achieved = (h2d + d2h bytes) x steps / e2e time" % e2e_bytes}
        del dev_buf, host_dn, dev_src
    # parity of the timed level itself (its kernels and segments) against
    # the oracle, one step from the initial state and one from the state the
    # timed steps reached
    parity = None
    if rank == 0 and world == 1 and not args.no_parity:
        parity = {"fp64_step_from_initial": parity_check(lev, u0, n, "initial state"),
                  "fp64_step_from_timed_state": parity_check(lev, u_fp64, n, "after the %d timed steps" % args.steps),
                  "bar": "rel L-inf <= 1e-12 per component, conserved totals <= 1e-13, dt <= 1e-14"}
    lev.close()

    # FP32-storage variant on the same workload: throughput, roofline, and
    # density / energy L1 error against the FP64 oracle (and the FP64 path)
    fp32 = None
    if u_fp64 is not None and not args.no_fp32:
        setup32 = {"x_mode": args.x_mode}
        if not args.no_autotune:
            from bamrex_b200.autotune import tune_sweeps
            r32 = tune_sweeps(D, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], boxes, parm, u0, precision=bx.FP32_STORAGE,
                              steps=3)
            setup32 = {k: r32[k] for k in ("staging_dir", "x_mode", "x_segment", "s_segment")}
        lev32 = bx.Level(D, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], boxes, bx.Parm(D, limiter=bx.MINBEE),
                         method=bx.MUSCL_HANCOCK, cfl=0.8, stream=stream, precision=bx.FP32_STORAGE, **setup32)
        kinds32 = [lev32.staging(d) for d in range(D)]
        lev32.set_state(u0)
        lev32.run(args.warmup, use_graph=use_graph)
        lev32.set_state(u0)
        lev32.set_timing(not use_graph)
        lev32.reset_counters()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            f0.record(stream)
            lev32.run_async(args.steps, use_graph=use_graph)
            f1.record(stream)
        lev32.run_wait()
        torch.cuda.synchronize()
        ms32 = f0.elapsed_time(f1)
        _, sweep_ms32, sweep_n32 = lev32.counters()
        u32 = lev32.get_state()
        lev32.set_timing(False)
        l1o = fp32_l1_vs_oracle(n, u0, args.fp32_oracle_steps, lev32) if args.fp32_oracle_steps > 0 else None
        lev32.close()
        if parity is not None and l1o is not None:
            parity["fp32_storage"] = l1o
        l1 = lambda a, b: float(np.abs(a - b).sum() / np.abs(b).sum())  # noqa: E731
        peak, _ = measured_peaks()
        ach32 = (2 * NC2D * 4 * n * n) / ((sweep_ms32 / sweep_n32) / 1e3) / 1e9 if sweep_n32 else None
        fp32 = {"value": n * n * args.steps / (ms32 / 1e3), "unit": METRIC, "ms_per_step": ms32 / args.steps,
                "roofline": {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s",
                             "frac": ach32 / peak if ach32 else None, "algorithmic_bytes_per_cell_sweep": 32},
                "kernels": ",".join(KIND_NAMES[k] for k in kinds32),
                "rel_l1_rho_vs_fp64_path": l1(u32[0], u_fp64[0]), "rel_l1_E_vs_fp64_path": l1(u32[3], u_fp64[3]),
                "l1_fp64_path": "the FP64 path after the same %d steps" % args.steps,
                "l1_vs_fp64_oracle": l1o}

    cells = n * n
    value = world * cells * args.steps / (ms / 1e3)
    e2e_value = world * cells * args.e2e_steps / (e2e_ms / 1e3)
    state_bytes = NC2D * 8 * cells

    roofline = None
    if sweep_launches:
        peak, peak_kind = measured_peaks()
        per_launch_s = (sweep_ms / sweep_launches) / 1e3
        alg_bytes = 2 * NC2D * 8 * cells  # read U once + write U once per sweep
        achieved = alg_bytes / per_launch_s / 1e9
        traffic = profiled_traffic("mhm2d")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": (traffic * cells) if traffic else None,
                    "kernel": " + ".join(sweep_kernel_name(2, d, kinds[d], x_rows) for d in range(D))
                    + " (both sweeps, averaged)",
                    "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": per_launch_s * 1e3,
                    "sweep_share_of_step": sweep_ms / ms if ms > 0 else None,
                    "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind if peak_kind == "measured"
                    else "fallback 6650 GB/s"}
        if fp32:
            roofline["fp32_storage_frac"] = fp32["roofline"]["frac"]
            roofline["fp32_storage_achieved"] = fp32["roofline"]["achieved"]
            roofline["fp32_storage_value"] = fp32["value"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_baseline_run(n, args.cpu_seconds)
        cpu = {k: r[k] for k in ("value", "unit", "cores", "kind", "sample", "cpu_model", "isa", "march")}

    imex = None
    if rank == 0 and world == 1 and not args.no_imex:
        imex = imex_pressure_run(args.imex_n)
    amr = None
    if rank == 0 and world == 1 and not args.no_amr:
        amr = {"workload": "3D spherical blast (p 10 inside r < 0.2, 0.1 outside, rho 1), base %d^3, 3 levels, "
                           "ratio 2, blocking factor 8, max_grid_size drawn per box from {16,32,48,64}, grad_error "
                           "on rho >= 0.1, MUSCL-Hancock/minbee, CFL 0.8, subcycling" % args.amr_n,
               "fp64": amr_blast_run(args.amr_n, args.amr_steps, bx.FP64, args.amr_regrid_steps),
               "fp32_storage": amr_blast_run(args.amr_n, args.amr_steps, bx.FP32_STORAGE, args.amr_regrid_steps)}

    body = None
    if rank == 0 and world == 1 and not args.no_body:
        cases = args.body_cases.split(",")
        body = {}
        if "2d" in cases:
            body["2d"] = rigid_body_run(2, (2048, 2048), 64, bx.FP64)
        if "3d" in cases:
            body["3d_fp32_storage"] = rigid_body_run(3, (512, 512, 128), 32, bx.FP32_STORAGE, steps=5, vortex=True)
        if "3d_amr" in cases:
            body["3d_amr"] = rigid_body_amr_run(tuple(args.body_amr_n), steps=args.body_amr_steps)

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded four-quadrant initial state, generated on the host)",
        "config": workload_config(n, len(boxes), mgs, {"graph_replay": use_graph, "parallelism": "single",
                                                        "kernels": ",".join(KIND_NAMES[k] for k in kinds),
                                                        "autotune": tuned,
                                                        **parity_scalars(parity)}),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes + 8,
                "path": "bamrex_level_run_host: every step the whole state host -> device and device -> host "
                        "(pinned), %d slabs streamed (uploads, sweeps, downloads overlapped within and across "
                        "steps; one strided copy per slab and direction), dt from the CFL estimate on the device"
                        % e2e_slabs,
                "steps": args.e2e_steps, "pcie_roof": pcie},
        "gpu_launches": launches,
        "clocks": clocks.summary(t_wall0, t_wall1),
        "fp32_storage": fp32,
        "imex_pressure_solve": imex,
        "amr_blast3d": amr,
        "rigid_body": body,
        "parity": parity,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_ours_dist(args, rank, world, local_rank):
    """N ranks, one GPU each: the domain is N blocks of n x n stacked in y
    (weak scaling), one block per rank; halos cross ranks over NCCL between
    sweeps and the max wave speed is all-reduced over the ranks in a device
    buffer every step, the next dt computed from it on the device, so the
    host enqueues the timed steps without waiting."""
    import torch
    import torch.distributed as dist

    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.distributed import DeviceEngine, DistLevel, partition

    torch.cuda.set_device(local_rank)
    dev_index = torch.cuda.current_device()
    n = args.n
    D = 2
    hi = (n - 1, n * world - 1, 0)
    boxes = bx.decompose(D, (0, 0, 0), hi, n)
    owners = partition(boxes, world)
    mine = [boxes[b] for b in range(len(boxes)) if owners[b] == rank]
    block = problems.quadrant_2d(n)
    glob = np.zeros((4, 1, n * world, n))
    for b, (lo, bhi) in enumerate(boxes):
        if owners[b] == rank:
            glob[:, :, lo[1]:bhi[1] + 1, :] = block
    lev = bx.Level(D, (0, 0, 0), hi, [0.0, 0.0], [1.0, float(world)], mine, bx.Parm(D, limiter=bx.MINBEE),
                   method=bx.MUSCL_HANCOCK, cfl=0.8)
    stream = torch.cuda.ExternalStream(lev.stream_handle())  # the level's own stream
    lev.set_state(glob)
    del glob
    dl = DistLevel(DeviceEngine(lev), D, (0, 0, 0), hi, boxes, owners, 2, (0, 0, 0), (0, 0, 0), lev.dx, 0.8, rank,
                   world, dist)
    dl.run_device(args.warmup)
    lev.set_timing(True)
    lev.reset_counters()
    clocks = ClockSampler(dev_index)
    clocks.start()
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.time()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    dl.run_device(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    t_wall1 = time.time()
    ms = ev0.elapsed_time(ev1)
    launches, sweep_ms, sweep_launches = lev.counters()
    t = torch.tensor([ms], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    cells = n * n * world
    value = cells * args.steps / (ms / 1e3)
    # end to end: each step copies this rank's state in from pinned host
    # memory, steps, and copies it back out
    nloc = lev.packing.size
    h_in = torch.empty(nloc, dtype=torch.float64, pin_memory=True)
    h_out = torch.empty(nloc, dtype=torch.float64, pin_memory=True)
    lev.copy_out_ptr(h_in.data_ptr())
    lev.sync()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        lev.copy_in_ptr(h_in.data_ptr())
        dl.run_device(1)
        lev.copy_out_ptr(h_out.data_ptr())
        lev.sync()
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = cells * args.e2e_steps / float(t.item())
    roofline = None
    if sweep_launches:
        peak, peak_kind = measured_peaks()
        per_launch_s = (sweep_ms / sweep_launches) / 1e3
        alg_bytes = 2 * NC2D * 8 * lev.ncells
        achieved = alg_bytes / per_launch_s / 1e9
        traffic = profiled_traffic("mhm2d")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": (traffic * lev.ncells) if traffic else None,
                    "kernel": "sweep kernels of rank 0 (both sweeps, averaged)",
                    "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": per_launch_s * 1e3,
                    "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind}
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded four-quadrant state per %dx%d block, generated on the host)" % (n, n),
        "config": {"workload": "2D four-quadrant Riemann problem, %d blocks of %dx%d stacked in y (one per GPU), "
                               "MUSCL-Hancock/minbee + HLLC, CFL 0.8, transmissive" % (world, n, n),
                   "cells": cells, "boxes": len(boxes), "l2": "inputs larger than L2", "seed": 20261203,
                   "parallelism": "domain decomposition: halo exchange over NCCL between sweeps, max wave speed "
                                  "all-reduced on the device, dt computed on the device"},
        "roofline": roofline,
        "cpu_baseline": None,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": nloc * 8 * world,
                "d2h_bytes_per_step": nloc * 8 * world + 48,
                "path": "per rank: bamrex_level_copy_in (pinned host) + split step with NCCL halos + "
                        "bamrex_level_copy_out", "steps": args.e2e_steps},
        "gpu_launches": launches,
        "clocks": clocks.summary(t_wall0, t_wall1),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1 or args.split:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29531")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        try:
            return run_ours_dist(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
