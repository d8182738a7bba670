"""The IMEX step on the device (bamrex_imex, imex.cu) against
the CPU restatement (oracle/imex_oracle.py) and against the assertions of
the reference's own IMEX tests (Tests/IMEX_O1_01.cpp).

Around the pressure solve the device step reproduces the restatement to
1e-14 relative (the same operations in the same order); the pressure itself
is held to the solve tolerance through the restatement's operator."""
import numpy as np
import pytest

from conftest import ROOT  # noqa: F401

pytestmark = pytest.mark.gpu

ADIA, EPS = 1.6, 0.5


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def make(D, n, bc, method, enth, ke, gamma=ADIA, eps=EPS, **kw):
    import bamrex_b200 as bx
    from bamrex_b200.imex import Imex
    parm = bx.Parm(D, adiabatic=gamma, epsilon=eps)
    return Imex(D, [n] * D, [0.0] * D, [1.0] * D, parm, bc_lo=[bc] * 3, bc_hi=[bc] * 3, advection_flux=method,
                enthalpy_method=enth, ke_method=ke, **kw)


def box_test_state(D, n=4):
    from test_imex_cpu import box_test_state as bts
    return bts(D, n)


def smooth_state(D, n, seed):
    from test_imex_cpu import _smooth_state
    return _smooth_state(D, n, seed)


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("enth", [0, 1, 2])
def test_split_ke_energy_match(torch_cuda, D, enth):
    """SplitKEEnergyMatch (Tests/IMEX_O1_01.cpp:56-114) on the device:
    E_new = p/(gamma-1) + eps/(2 rho^n) m^n . m^new to 1e-12 relative."""
    U, p = box_test_state(D)
    im = make(D, 4, 0, 0, enth, 2)
    im.set_state(U, p)
    it, rr = im.step(0.01)
    assert rr <= 1e-12
    out, pn = im.get_state()
    dot = U[1] * out[1]
    for d in range(1, D):
        dot = dot + U[1 + d] * out[1 + d]
    expected = pn / (ADIA - 1) + 0.5 * EPS / U[0] * dot
    assert np.all(np.abs(out[1 + D] - expected) <= np.abs(expected) * 1e-12)
    im.close()


@pytest.mark.parametrize("D", [2, 3])
def test_explicit_ke_energy_match(torch_cuda, D):
    """ExplicitKEEnergyMatch (Tests/IMEX_O1_01.cpp:200-259) on the device."""
    import bamrex_b200._abi as A
    U, p = box_test_state(D)
    im = make(D, 4, 0, 0, 0, 1)
    im.set_state(U, p)
    im.step(0.01)
    out, pn = im.get_state()
    ex = im.field(A.FIELD_UEX)[(slice(None),) + tuple(slice(1, -1) if s > 1 else slice(None)
                                                       for s in im.field(A.FIELD_UEX).shape[1:])]
    m2 = ex[1] * ex[1]
    for d in range(1, D):
        m2 = m2 + ex[1 + d] * ex[1 + d]
    expected = pn / (ADIA - 1) + 0.5 * EPS / ex[0] * m2
    assert np.all(np.abs(out[1 + D] - expected) <= np.abs(expected) * 1e-12)
    im.close()


CASES = [
    # D, n, bc, method, enthalpy method, ke method
    (2, 32, 1, 0, 0, 1),
    (2, 32, 1, 1, 0, 2),
    (2, 24, 0, 1, 1, 0),
    (2, 20, 2, 0, 2, 2),
    (2, 16, 2, 1, 0, 1),
    (3, 12, 1, 1, 0, 2),
    (3, 10, 0, 0, 2, 1),
    (3, 8, 2, 1, 1, 2),
]


@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_step_matches_restatement(torch_cuda, case):
    """One step on a smooth state: with the device's pressure given, the
    restatement reproduces the explicit update, enthalpy, kinetic energy,
    pressure source, fluxes and new state to 1e-14; the device pressure
    solves the restatement's operator to the solve tolerance."""
    import bamrex_b200._abi as A
    from oracle import imex_oracle as IO
    D, n, bc, method, enth, ke = case
    U, p = smooth_state(D, n, 11)
    im = make(D, n, bc, method, enth, ke)
    im.set_state(U, p)
    dt = 0.5 * im.est_time_step()
    it, rr = im.step(dt)
    assert rr <= 1e-12
    out, pn = im.get_state()
    r = IO.imex_step(U, p, D, [1.0 / n] * D, dt, ADIA, EPS, [bc] * 3, [bc] * 3, method, enth, ke, p_new=pn)
    assert rel(im.field(A.FIELD_UEX), r["Uex"]) <= 1e-14
    assert rel(im.field(A.FIELD_ENTHALPY), r["enth"]) <= 1e-14
    assert rel(im.field(A.FIELD_KE), r["ke"]) <= 1e-14
    assert rel(im.field(A.FIELD_RHS), r["rhs"]) <= 1e-14
    for d in range(D):
        assert rel(im.field(A.FIELD_FLUX_X + d), r["fluxes"][d]) <= 1e-14, d
    for c in range(D + 2):
        assert rel(out[c], r["U"][c]) <= 1e-14, c
    res = r["rhs"] - r["op"].apply(pn)
    assert np.sqrt((res ** 2).sum()) <= 2e-12 * np.sqrt((r["rhs"] ** 2).sum())
    im.close()


def test_time_step_matches(torch_cuda):
    from oracle import imex_oracle as IO
    U, p = smooth_state(2, 32, 5)
    im = make(2, 32, 1, 0, 0, 1, cfl=0.7)
    im.set_state(U, p)
    assert abs(im.est_time_step() - IO.advective_time_step(U, 2, [1 / 32] * 2, 0.7)) <= 1e-15 * im.est_time_step()
    im.close()


@pytest.mark.parametrize("method,ke", [(0, 1), (1, 2)])
def test_periodic_run_conserves_and_tracks_restatement(torch_cuda, method, ke):
    """Ten steps on a periodic 48^2 domain: totals kept to round-off, and the
    state within 1e-9 of the restatement run with its own pressure solves
    (the two solvers agree to their tolerance, not bit for bit)."""
    from oracle import imex_oracle as IO
    D, n = 2, 48
    U, p = smooth_state(D, n, 2)
    im = make(D, n, 1, method, 0, ke)
    im.set_state(U, p)
    Ur, pr = U.copy(), p.copy()
    tot0 = U.sum(axis=(1, 2, 3))
    for _ in range(10):
        dt = im.est_time_step()
        assert abs(dt - IO.advective_time_step(Ur, D, [1 / n] * D, 0.5)) <= 1e-9 * dt
        im.step(dt)
        rr = IO.imex_step(Ur, pr, D, [1 / n] * D, dt, ADIA, EPS, [1] * 3, [1] * 3, method, 0, ke)
        Ur, pr = rr["U"], rr["p"]
    out, pn = im.get_state()
    scale = np.abs(U).sum(axis=(1, 2, 3))
    assert np.all(np.abs(out.sum(axis=(1, 2, 3)) - tot0) <= 1e-12 * scale)
    for c in range(D + 2):
        assert rel(out[c], Ur[c]) <= 1e-9
    assert rel(pn, pr) <= 1e-8
    im.close()


def test_learned_pressure_solve_in_the_step(torch_cuda):
    """The step with the learned preconditioner (an untrained network:
    FGMRES falls back to the plain solve when needed) reaches the same
    tolerance and the same state as the plain step."""
    from bamrex_b200.learned import PrecNet
    D, n = 2, 64
    U, p = smooth_state(D, n, 4)
    a = make(D, n, 1, 0, 0, 1)
    b = make(D, n, 1, 0, 0, 1)
    net = PrecNet(n, n, batch=1, seed=3)
    b.set_precnet(net)
    for im in (a, b):
        im.set_state(U, p)
    dt = a.est_time_step()
    _, ra = a.step(dt)
    _, rb = b.step(dt)
    assert ra <= 1e-12 and rb <= 1e-12
    ua, pa = a.get_state()
    ub, pb = b.get_state()
    assert rel(pb, pa) <= 1e-9
    for c in range(D + 2):
        assert rel(ub[c], ua[c]) <= 1e-10
    for x in (a, b, net):
        x.close()


def test_errors(torch_cuda):
    import bamrex_b200 as bx
    from bamrex_b200 import BamrexError
    with pytest.raises(BamrexError):
        make(2, 1, 0, 0, 0, 1)  # fewer cells than ghost layers
    with pytest.raises(BamrexError):
        make(2, 8, 0, 5, 0, 1)  # unknown advection flux
    im = make(2, 8, 1, 0, 0, 1, max_iter=1, tol_rel=1e-30)
    U, p = smooth_state(2, 8, 1)
    im.set_state(U, p)
    with pytest.raises(BamrexError) as e:
        im.step(0.01)
    assert e.value.status == bx._abi.ERR_NOT_CONVERGED
    out, _ = im.get_state()
    np.testing.assert_array_equal(out, U)  # the state is left unchanged
    im.close()


TABLEAUX = ["SP111", "SSP222", "SASSP322", "SASSP332", "SSP433"]
RK_CASES = [(tab, m, ke) for tab in TABLEAUX for (m, ke) in ((0, 1), (1, 2), (0, 0))]


@pytest.mark.parametrize("case", RK_CASES, ids=[str(c) for c in RK_CASES])
def test_rk_step_matches_restatement(torch_cuda, case):
    """One step of every tableau (stage states, stage pressures, stage
    fluxes, weighted flux sum, update) against the restatement with its own
    solves, both to 1e-13: the states agree to 1e-10, the periodic totals are
    kept to round-off."""
    from oracle import imex_oracle as IO
    tab, method, ke = case
    D, n = 2, 24
    U, p = smooth_state(D, n, 9)
    im = make(D, n, 1, method, 0, ke, tol_rel=1e-13, tableau=TABLEAUX.index(tab))
    im.set_state(U, p)
    dt = im.est_time_step()
    it, rr = im.step(dt)
    assert rr <= 1e-13
    out, pn = im.get_state()
    r = IO.imex_rk_step(U, p, D, [1 / n] * D, dt, ADIA, EPS, [1] * 3, [1] * 3, method, 0, ke, tab, tol_rel=1e-14)
    for c in range(D + 2):
        assert rel(out[c], r["U"][c]) <= 1e-10, c
    assert rel(pn, r["p"]) <= 1e-9
    scale = np.abs(U).sum(axis=(1, 2, 3))
    assert np.all(np.abs(out.sum(axis=(1, 2, 3)) - U.sum(axis=(1, 2, 3))) <= 1e-12 * scale)
    im.close()


@pytest.mark.parametrize("D", [2, 3])
def test_rk_3d_and_reflective(torch_cuda, D):
    """SSP433 with MUSCL-Rusanov and the explicit kinetic energy on a
    reflective (2D) or transmissive (3D) box tracks the restatement."""
    from oracle import imex_oracle as IO
    n = 16 if D == 2 else 8
    bc = 2 if D == 2 else 0
    U, p = smooth_state(D, n, 13)
    im = make(D, n, bc, 1, 2, 1, tol_rel=1e-13, tableau=4)
    im.set_state(U, p)
    dt = 0.5 * im.est_time_step()
    im.step(dt)
    out, pn = im.get_state()
    r = IO.imex_rk_step(U, p, D, [1 / n] * D, dt, ADIA, EPS, [bc] * 3, [bc] * 3, 1, 2, 1, "SSP433", tol_rel=1e-14)
    for c in range(D + 2):
        assert rel(out[c], r["U"][c]) <= 1e-10, c
    im.close()
