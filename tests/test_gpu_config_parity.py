"""Parity at the benchmark's own size: the 2D four-quadrant problem on
4096^2 cells (MUSCL-Hancock/minbee + HLLC, CFL 0.8, transmissive), as the
bench times it, against the CPU oracle.

Per step from identical inputs (AmrLevelAdv::advance_explicit,
Source/AmrLevelAdv_advance.cpp:261-360): relative L-infinity per component
<= 1e-12 and conserved totals <= 1e-13 relative; the time step of
estTimeStep (Source/AmrLevelAdv.cpp:395-477) within 1e-14.  The oracle runs
the reference's 64x64 boxes (results do not depend on the box layout); the
device runs one 4096^2 box with each x-sweep kernel, and 4096 boxes of
64^2.  The FP32-storage variant reports its density and energy L1 error
against the FP64 oracle after five steps of the oracle's dt sequence."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 4096
LINF = 1e-12
TOTALS = 1e-13


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def c2(oracle):
    """Initial state, the oracle's first step and its dt."""
    from bamrex_b200 import problems
    u0 = problems.quadrant_2d(N)
    lay = _layout(oracle)
    dt, u1 = _oracle_step(oracle, lay, u0)
    return {"u0": u0, "dt": dt, "u1": u1, "lay": lay}


def _layout(oracle):
    hi = (N - 1, N - 1, 0)
    return oracle.LevelLayout(2, (0, 0, 0), hi, oracle.decompose(2, (0, 0, 0), hi, 64), 2, [1.0 / N] * 2)


def _oracle_step(oracle, lay, u, dt=None):
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u)
    lay.fill_boundary(S1)
    if dt is None:
        dt = lay.est_time_step(S1, 1.4, 1.0, 0.8)
    S2[:] = S1
    lay.advance_explicit(S1, S2, 0.0, dt, oracle.MUSCL_HANCOCK, oracle.Parm(2, limiter=oracle.MINBEE))
    return dt, lay.gather(S1)


def _level(mgs, x_mode=0, precision=0, staging=0):
    import bamrex_b200 as bx
    hi = (N - 1, N - 1, 0)
    return bx.Level(2, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], bx.decompose(2, (0, 0, 0), hi, mgs),
                    bx.Parm(2, limiter=bx.MINBEE), method=bx.MUSCL_HANCOCK, cfl=0.8, x_mode=x_mode,
                    precision=precision, staging=staging)


def _check(got, ref, what):
    vol = 1.0 / N ** 2
    for c in range(4):
        e = float(np.max(np.abs(got[c] - ref[c])) / np.max(np.abs(ref[c])))
        assert e <= LINF, (what, "component", c, e)
        tg, tr = got[c].sum() * vol, ref[c].sum() * vol
        scale = np.abs(ref[c]).sum() * vol
        assert abs(tg - tr) <= TOTALS * scale, (what, "total", c, tg, tr)


@pytest.mark.parametrize("mgs,x_mode,staging", [(N, 1, 1), (N, 2, 1), (N, 0, 2), (N, 0, 3), (64, 0, 1), (64, 0, 2),
                                                 (64, 0, 3)],
                         ids=["one_box_xrows", "one_box_xmarch", "one_box_tma", "one_box_wave", "box64", "box64_tma",
                              "box64_wave"])
def test_c2_steps_match_oracle(torch_cuda, oracle, c2, mgs, x_mode, staging):
    """Two steps at 4096^2: the first from the initial state, the second from
    the device's own result (the oracle takes the same input); the sweeps
    load through L2 (either x kernel) or are staged by TMA."""
    lev = _level(mgs, x_mode, staging=staging)
    assert lev.staging(0) == staging and lev.staging(1) == staging
    lev.set_state(c2["u0"])
    dt = lev.estTimeStep()
    assert abs(dt - c2["dt"]) <= 1e-14 * c2["dt"], (dt, c2["dt"])
    lev.advance(0.0, dt)
    u1 = lev.get_state()
    _check(u1, c2["u1"], "step 1")
    dt2 = lev.estTimeStep()
    lev.advance(dt, dt2)
    u2 = lev.get_state()
    lev.close()
    _, ref2 = _oracle_step(oracle, c2["lay"], u1, dt2)
    _check(u2, ref2, "step 2")


def test_c2_fp32_storage_l1_vs_fp64_oracle(torch_cuda, oracle, c2):
    """FP32 storage on 4096^2 with the oracle's dt sequence: density and
    energy L1 error against the FP64 oracle after five steps."""
    import bamrex_b200 as bx
    lay = c2["lay"]
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, c2["u0"])
    P = oracle.Parm(2, limiter=oracle.MINBEE)
    lev = _level(N, 0, bx.FP32_STORAGE)
    lev.set_state(c2["u0"])
    t = 0.0
    for _ in range(5):
        lay.fill_boundary(S1)
        dt = lay.est_time_step(S1, 1.4, 1.0, 0.8)
        S2[:] = S1
        lay.advance_explicit(S1, S2, t, dt, oracle.MUSCL_HANCOCK, P)
        lev.advance(t, dt)
        t += dt
    ref = lay.gather(S1)
    got = lev.get_state()
    lev.close()
    l1 = [float(np.abs(got[c] - ref[c]).sum() / np.abs(ref[c]).sum()) for c in (0, 3)]
    print("FP32 storage 4096^2, 5 steps, L1 vs FP64 oracle: rho %.3e E %.3e" % tuple(l1))
    assert l1[0] < 1e-5 and l1[1] < 1e-5
