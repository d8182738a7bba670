"""The FP32-storage variant (state and fluxes in FP32; CFL/dt reduction and
conserved sums in FP64) against the FP64 oracle, and the conserved-sums
reduction of both precisions.

FP32 has no bit-level bar; what is checked and reported is the density and
energy L1 error relative to the FP64 oracle (sum |u32 - u64| / sum |u64|)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def _levels(oracle, D, n, mgs, bc, limiter, cfl, precision):
    import bamrex_b200 as bx
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
    lay = oracle.LevelLayout(D, (0, 0, 0), hi, boxes, 2, [1.0 / n] * D, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
    lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D, limiter=limiter), cfl=cfl,
                   bc_lo=(bc,) * 3, bc_hi=(bc,) * 3, precision=precision)
    return lay, lev


# Bounds on the relative L1 error after 10 steps.  In the 3D blast the
# difference to FP64 stays ~1e-8 for five steps, then grows to ~1e-4 in the
# shell around the initial discontinuity (0.2 < r < 0.4), with the IEEE
# float functions of the general kernels as well as with the fast ones, so
# its bound is wider.
@pytest.mark.parametrize("D,n,mgs,limiter,gen,bound", [(1, 400, 100, 1, "sod", 1e-5), (2, 128, 64, 0, "quadrant", 1e-5),
                                                       (3, 32, 16, 1, "blast", 2e-3)])
def test_fp32_storage_l1_vs_fp64_oracle(torch_cuda, oracle, D, n, mgs, limiter, gen, bound):
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    u0 = {"sod": lambda: problems.sod_1d(n), "quadrant": lambda: problems.quadrant_2d(n),
          "blast": lambda: problems.blast_3d(n, radius=0.25)}[gen]()
    nsteps = 10
    lay, lev = _levels(oracle, D, n, mgs, 0, limiter, 0.8, bx.FP32_STORAGE)
    ref, t_ref, dts = oracle.run_level(lay, u0, oracle.Parm(D, limiter=limiter), oracle.MUSCL_HANCOCK, 0.8,
                                       nsteps=nsteps)
    # (a) the oracle's dt sequence: the error of FP32 storage and arithmetic alone
    lev.set_state(u0)
    t = 0.0
    for dt in dts:
        lev.advance(t, dt)
        t += dt
    same_dt = lev.get_state()
    # (b) the FP32 level's own device dt (max wave speed of the FP32 state)
    lev.set_state(u0)
    t32, steps = lev.run(nsteps)
    own_dt = lev.get_state()
    lev.close()
    assert steps == nsteps
    assert abs(t32 - t_ref) <= 1e-3 * t_ref
    e = [_l1(same_dt[0], ref[0]), _l1(same_dt[D + 1], ref[D + 1]), _l1(own_dt[0], ref[0]),
         _l1(own_dt[D + 1], ref[D + 1])]
    print("FP32-storage L1 vs FP64 oracle (%dD, %d steps): same dt: rho %.3e E %.3e | own dt (time %+.1e): "
          "rho %.3e E %.3e" % (D, nsteps, e[0], e[1], t32 / t_ref - 1, e[2], e[3]))
    assert e[0] < bound and e[1] < bound
    assert e[2] < 1e-2 and e[3] < 1e-2


def test_conserved_sums_fp64_and_fp32(torch_cuda, oracle):
    """Totals sum(U) dV: FP64 level equals the oracle's totals, periodic runs
    conserve them (FP64 to 1e-13, FP32 storage to FP32 rounding), and the
    reduction is deterministic."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    D, n = 2, 96
    u0 = problems.random_states(2, (1, n, n), seed=3)
    vol = (1.0 / n) ** 2
    tot0 = u0.sum(axis=(1, 2, 3)) * vol
    scale = np.abs(u0).sum(axis=(1, 2, 3)) * vol
    for prec, tol in ((bx.FP64, 1e-13), (bx.FP32_STORAGE, 1e-6)):
        lay, lev = _levels(oracle, D, n, 32, oracle.PERIODIC, 1, 0.5, prec)
        lev.set_state(u0)
        s0 = lev.conserved_sums()
        if prec == bx.FP64:
            np.testing.assert_allclose(s0, tot0, rtol=0, atol=1e-14 * scale.max())
        lev.run(5)
        s1, s1b = lev.conserved_sums(), lev.conserved_sums()
        np.testing.assert_array_equal(s1, s1b)
        assert np.all(np.abs(s1 - s0) <= tol * scale), (prec, s1 - s0)
        lev.close()


def test_fp32_level_fab_is_refused(torch_cuda, oracle):
    """bamrex_array4 describes doubles only, so an FP32-storage level does not
    hand out its float fabs as one (a consumer would read past the buffer)."""
    import ctypes

    import bamrex_b200 as bx
    from bamrex_b200._abi import ERR_UNSUPPORTED, Array4, lib
    lay, lev = _levels(oracle, 2, 64, 32, 0, 1, 0.8, bx.FP32_STORAGE)
    a = Array4()
    assert lib().bamrex_level_fab(lev._h, 0, ctypes.byref(a)) == ERR_UNSUPPORTED
    assert b"FP32-storage" in lib().bamrex_last_error()
    assert not a.p
    lev.close()
    lay, lev = _levels(oracle, 2, 64, 32, 0, 1, 0.8, bx.FP64)
    assert lib().bamrex_level_fab(lev._h, 0, ctypes.byref(a)) == 0 and a.p
    lev.close()
