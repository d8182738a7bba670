"""CPU checks of the oracle's level driver: it reproduces the committed
fixtures, conserves totals with periodic boundaries, is independent of the
box decomposition, and converges on the Sod problem."""
import os

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def fixtures():
    return np.load(os.path.join(ROOT, "tests", "golden", "oracle_fixtures.npz"))


def test_oracle_reproduces_fixtures(oracle, fixtures):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mk", os.path.join(ROOT, "tests", "golden", "make_oracle_fixtures.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    for name in mk.CASES:
        u0, u1, dts = mk.run_case(name)
        np.testing.assert_array_equal(u0, fixtures[name + "/u0"])
        np.testing.assert_array_equal(u1, fixtures[name + "/u1"])
        np.testing.assert_array_equal(dts, fixtures[name + "/dts"])


def _level(o, D, n, mgs, bc):
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = o.decompose(D, (0, 0, 0), hi, mgs)
    return o.LevelLayout(D, (0, 0, 0), hi, boxes, 2, [1.0 / n] * D, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)


@pytest.mark.parametrize("method", [0, 1, 4, 5, 6])
def test_periodic_conservation(oracle, method):
    from bamrex_b200 import problems
    o = oracle
    lay = _level(o, 2, 32, 16, o.PERIODIC)
    u0 = problems.random_states(2, (1, 32, 32), seed=11)
    u1, _, _ = o.run_level(lay, u0, o.Parm(2), method, 0.5, nsteps=3)
    t0, t1 = u0.sum(axis=(1, 2, 3)), u1.sum(axis=(1, 2, 3))
    assert np.all(np.abs(t1 - t0) <= 1e-13 * np.abs(t0).max())


def test_decomposition_invariance(oracle):
    from bamrex_b200 import problems
    o = oracle
    u0 = problems.quadrant_2d(40, seed=5)
    ref = None
    for mgs in (40, 16, 8):
        lay = _level(o, 2, 40, mgs, o.TRANSMISSIVE)
        u1, _, _ = o.run_level(lay, u0, o.Parm(2, limiter=o.MINBEE), o.MUSCL_HANCOCK, 0.8, nsteps=2)
        if ref is None:
            ref = u1
        np.testing.assert_array_equal(u1, ref)


def test_sod_shock_position(oracle):
    """Sod (C1) to t=0.2: the shock sits near x = 0.85 (exact 0.8504), the
    contact near 0.685 and the density plateau between matches the exact
    star-state density 0.2656 (rho*_R) to a few percent."""
    from bamrex_b200 import problems
    o = oracle
    lay = _level(o, 1, 400, 400, o.TRANSMISSIVE)
    u1, t, dts = o.run_level(lay, problems.sod_1d(400), o.Parm(1), o.MUSCL_HANCOCK, 0.9, stop_time=0.2)
    assert abs(t - 0.2) < 1e-12
    rho = u1[0, 0, 0]
    x = (np.arange(400) + 0.5) / 400
    shock = x[np.argmax(rho < 0.5 * (0.2656 + 0.125))]
    assert abs(shock - 0.8504) < 0.01
    plateau = rho[(x > 0.72) & (x < 0.82)]
    assert np.all(np.abs(plateau - 0.2656) < 0.01)
