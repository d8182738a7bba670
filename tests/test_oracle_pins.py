"""Pin the CPU oracle on the reference's own known-answer tests.

Every expected value and tolerance below comes from the BAMReX test sources
(extracted into tests/golden/reference_known_answers.json by
tests/golden/make_golden.py):
  Tests/HLLC01.cpp:8-66 + Tests/hllc_test.H   Toro (1994) wave-speed estimates
  Tests/Euler01.cpp:9-66 + Tests/BoxTest.H     prim<->cons, max wave speed
  Tests/Limiters01.cpp:5-16                    minmod
"""
import numpy as np
import pytest


def _state(D, primv3):
    """Embed a 1D (rho, u, p) fixture as a D-dimensional primitive state
    (the fixture's AMREX_D_DECL(u, 0, 0))."""
    rho, u, p = primv3
    return np.array([rho, u] + [0.0] * (D - 1) + [p])


@pytest.mark.parametrize("D", [1, 2, 3])
def test_toro_wave_speed_estimates(oracle, golden, D):
    for f in golden["toro_wave_speeds"]:
        g, eps = f["adiabatic"], f["epsilon"]
        uL = oracle.consv_from_primv(D, _state(D, f["primv_L"]), g, eps)
        uR = oracle.consv_from_primv(D, _state(D, f["primv_R"]), g, eps)
        sL, sR, ss = oracle.wave_speed_toro(D, 0, uL, uR, g, eps)
        k = f["speed_scale"]
        assert abs(sL - f["exp_To_S_L"] * k) <= f["tol"]["S_L"] * k, f["name"]
        assert abs(sR - f["exp_To_S_R"] * k) <= f["tol"]["S_R"] * k, f["name"]
        assert abs(ss - f["exp_To_S_interm"] * k) <= f["tol"]["S_interm"] * k, f["name"]


@pytest.mark.parametrize("D", [1, 2, 3])
def test_prim_cons_conversions(oracle, golden, D):
    bt = golden["box_test"]
    g, eps, tol = bt["adiabatic"], bt["epsilon"], bt["tol"]
    fx = bt["dims"][str(D)]
    for side in ("L", "R"):
        u = oracle.consv_from_primv(D, fx["primv_" + side], g, eps)
        np.testing.assert_allclose(u, fx["consv_" + side], rtol=0, atol=tol)
        q = oracle.primv_from_consv(D, fx["consv_" + side], g, eps)
        np.testing.assert_allclose(q, fx["primv_" + side], rtol=0, atol=tol)


@pytest.mark.parametrize("D", [2, 3])
def test_max_wave_speed_split_grid(oracle, golden, D):
    """Euler01.cpp MaxWaveSpeed: BoxTest::setup(true), a 4^D domain split into
    2^D-cell boxes, cells with all indices < 2 holding consv_L."""
    bt = golden["box_test"]
    g, eps = bt["adiabatic"], bt["epsilon"]
    fx = bt["dims"][str(D)]
    n = bt["layout"]["ncell"]
    lo, hi = (0, 0, 0), tuple((n - 1) if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, lo, hi, bt["layout"]["split"])
    lay = oracle.LevelLayout(D, lo, hi, boxes, 2, [1.0 / n] * D)
    glob = np.zeros(lay.domain_shape())
    for k in range(glob.shape[1]):
        for j in range(glob.shape[2]):
            for i in range(glob.shape[3]):
                inside = i < 2 and j < 2 and (k < 2 or D < 3)
                glob[:, k, j, i] = fx["consv_L"] if inside else fx["consv_R"]
    buf = lay.alloc()
    lay.scatter(buf, glob)
    assert lay.fill_boundary(buf) == 0
    got = lay.max_wave_speed(buf, g, eps)
    exp = golden["box_test"]["max_wave_speed"][str(D)]
    assert abs(got - exp) <= bt["max_wave_speed"]["rtol"] * exp


def test_minmod(oracle, golden):
    for a, b, c in golden["minmod"]:
        assert oracle.minmod(a, b) == c


def test_limiter_functions_properties(oracle):
    """Limiters.H:29-73: every limiter is 0 for r<=0, 1 at r=1, and bounded by 2."""
    for lim in range(4):
        assert oracle.slope_limit(lim, -1.0) == 0.0
        assert oracle.slope_limit(lim, 0.0) == 0.0
        assert abs(oracle.slope_limit(lim, 1.0) - 1.0) < 1e-15
        for r in np.linspace(0.01, 10, 50):
            assert 0.0 <= oracle.slope_limit(lim, r) <= 2.0
