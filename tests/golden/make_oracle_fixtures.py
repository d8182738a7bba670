"""Generate the committed oracle fixtures tests/golden/oracle_fixtures.npz.

Each case is a seeded initial state advanced by the CPU oracle (the C
restatement in oracle/, parity build) through the reference's level step:
FillPatch, the split sweeps of advance_explicit, and estTimeStep / the
stop-time clamp.  The GPU tests compare the CUDA path against these arrays;
the CPU tests check that the oracle still reproduces them.

Usage: python tests/golden/make_oracle_fixtures.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bamrex_b200 import problems  # noqa: E402  (seeded generators, host only)
from oracle import oracle as o  # noqa: E402

# name: (D, n per dim, max_grid_size, method, limiter, bc, cfl, nsteps, generator)
CASES = {
    "sod400_1step": (1, 400, 100, o.MUSCL_HANCOCK, o.VAN_LEER, o.TRANSMISSIVE, 0.9, 1, "sod"),
    "sod400_20steps": (1, 400, 400, o.MUSCL_HANCOCK, o.VAN_LEER, o.TRANSMISSIVE, 0.9, 20, "sod"),
    "quadrant64_1step": (2, 64, 32, o.MUSCL_HANCOCK, o.MINBEE, o.TRANSMISSIVE, 0.8, 1, "quadrant"),
    "quadrant64_slic_1step": (2, 64, 64, o.SLIC, o.VAN_LEER, o.TRANSMISSIVE, 0.8, 1, "quadrant"),
    "random48_periodic_3steps": (2, 48, 16, o.MUSCL_HANCOCK, o.SUPERBEE, o.PERIODIC, 0.5, 3, "random2"),
    "blast16_1step": (3, 16, 8, o.MUSCL_HANCOCK, o.VAN_LEER, o.TRANSMISSIVE, 0.8, 1, "blast"),
}


def initial(gen, D, n):
    if gen == "sod":
        return problems.sod_1d(n)
    if gen == "quadrant":
        return problems.quadrant_2d(n, seed=problems.DEFAULT_SEED)
    if gen == "random2":
        return problems.random_states(2, (1, n, n), seed=7)
    if gen == "blast":
        return problems.blast_3d(n, radius=0.25)
    raise KeyError(gen)


def run_case(name):
    D, n, mgs, method, lim, bc, cfl, nsteps, gen = CASES[name]
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = o.decompose(D, (0, 0, 0), hi, mgs)
    lay = o.LevelLayout(D, (0, 0, 0), hi, boxes, 2, [1.0 / n] * D, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
    parm = o.Parm(D, adiabatic=1.4, limiter=lim)
    u0 = initial(gen, D, n)
    u1, t, dts = o.run_level(lay, u0, parm, method, cfl, nsteps=nsteps)
    return u0, u1, np.array(dts)


def main():
    out = {}
    for name in CASES:
        u0, u1, dts = run_case(name)
        out[name + "/u0"] = u0
        out[name + "/u1"] = u1
        out[name + "/dts"] = dts
        print(name, u1.shape, dts)
    np.savez_compressed(os.path.join(HERE, "oracle_fixtures.npz"), **out)


if __name__ == "__main__":
    main()
