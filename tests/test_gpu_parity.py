"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Bar: FP64 results within 1e-12 relative L-infinity per
component per step, from identical inputs; conserved totals within 1e-13.
Relative L-infinity = max|gpu - ref| / max|ref| for each component.
"""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

RTOL_STEP = 1e-12     # per step, relative L-infinity per component
RTOL_TOTAL = 1e-13    # conserved totals


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def rel_linf(got, ref):
    got = np.asarray(got)
    ref = np.asarray(ref)
    errs = []
    for n in range(ref.shape[0]):
        scale = np.max(np.abs(ref[n]))
        scale = scale if scale > 0 else 1.0
        errs.append(np.max(np.abs(got[n] - ref[n])) / scale)
    return max(errs)


def _box_input(D, shape, ngrow, seed, jump=True):
    """Random physical conserved states on the valid box grown by ngrow in
    every active direction, with a density/pressure jump across the middle."""
    from bamrex_b200 import problems
    gshape = [shape[d] + 2 * ngrow if d < D else 1 for d in range(3)]
    u = problems.random_states(D, (gshape[2], gshape[1], gshape[0]), seed=seed)
    if jump:
        q = u.copy()
        half = gshape[0] // 2
        u[:, :, :, half:] *= 0.35
        u[D + 1, :, :, half:] = q[D + 1, :, :, half:] * 0.2
    return u


def _lim_cases():
    return [(0, 0), (0, 1), (0, 2), (0, 3), (4, 0), (4, 1), (1, 1), (5, 1), (6, 1)]


@pytest.mark.parametrize("gamma", [1.4, 1.6])
@pytest.mark.parametrize("D", [1, 2, 3])
@pytest.mark.parametrize("method,limiter", _lim_cases())
def test_compute_flux_per_box(torch_cuda, oracle, D, method, limiter, gamma):
    """compute_*_flux (Fluxes.H) on one box, every direction, vs the oracle.
    gamma 1.4 takes the fast MUSCL-Hancock kernels (1/z = 7), gamma 1.6 the
    general ones."""
    torch = torch_cuda
    import bamrex_b200 as bx
    shape = [37, 23, 11][:D] + [1] * (3 - D)
    ng = 2
    lo = (3, -2, 5)[:D] + (0,) * (3 - D)
    hi = tuple(lo[d] + shape[d] - 1 if d < D else 0 for d in range(3))
    begin = tuple(lo[d] - ng if d < D else 0 for d in range(3))
    u = _box_input(D, shape, ng, seed=100 + D * 10 + method + limiter)
    dx = [0.01, 0.02, 0.015][:D]
    dt = 0.3 * min(dx) / 4.0
    parm_o = oracle.Parm(D, adiabatic=gamma, limiter=limiter)
    parm_g = bx.Parm(D, adiabatic=gamma, limiter=limiter)
    ut = torch.tensor(u, device="cuda")
    for d in range(D):
        ref = oracle.compute_flux(D, method, d, lo, hi, u, begin, dx, dt, parm_o)
        ft = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
        bx.compute_flux(method, d, D, (lo, hi), ft, lo, ut, begin, dx, dt, parm_g)
        torch.cuda.synchronize()
        got = ft.cpu().numpy()
        assert np.isfinite(got).all()
        err = rel_linf(got, ref)
        assert err <= RTOL_STEP, (D, method, limiter, d, err)


@pytest.mark.parametrize("D", [2, 3])
def test_primitive_limiting(torch_cuda, oracle, D):
    """limit_on_primv / per-component limiting variables
    (CalcLimitingVal.H:9-22): density limited on p, momenta on velocities."""
    torch = torch_cuda
    import bamrex_b200 as bx
    shape = [19, 13, 7][:D] + [1] * (3 - D)
    lo = (0, 0, 0)
    hi = tuple(shape[d] - 1 if d < D else 0 for d in range(3))
    begin = tuple(-2 if d < D else 0 for d in range(3))
    u = _box_input(D, shape, 2, seed=77)
    idx = [1 + D] + [1 + d for d in range(D)] + [1 + D] + [0] * (8 - D - 2)
    prim = [True] + [True] * D + [False] + [False] * (8 - D - 2)
    dx = [0.01] * D
    dt = 0.001
    po = oracle.Parm(D, limiter=0, limiter_indices=idx, limit_on_primv=prim)
    pg = bx.Parm(D, limiter=0, limiter_indices=idx, limit_on_primv=prim)
    ut = torch.tensor(u, device="cuda")
    for d in range(D):
        ref = oracle.compute_flux(D, 0, d, lo, hi, u, begin, dx, dt, po)
        ft = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
        bx.compute_flux(0, d, D, (lo, hi), ft, lo, ut, begin, dx, dt, pg)
        torch.cuda.synchronize()
        assert rel_linf(ft.cpu().numpy(), ref) <= RTOL_STEP


@pytest.mark.parametrize("D", [1, 2, 3])
@pytest.mark.parametrize("kind", [1, 5])
def test_compute_flux_LR(torch_cuda, oracle, D, kind):
    torch = torch_cuda
    import bamrex_b200 as bx
    shape = [17, 9, 6][:D] + [1] * (3 - D)
    lo = (0, 0, 0)
    hi = tuple(shape[d] - 1 if d < D else 0 for d in range(3))
    begin = tuple(-1 if d < D else 0 for d in range(3))
    uL = _box_input(D, shape, 1, seed=5, jump=False)
    uR = _box_input(D, shape, 1, seed=6, jump=True)
    dx = [0.02] * D
    dt = 0.002
    for d in range(D):
        ref = oracle.compute_flux_LR(D, kind, d, lo, hi, uL, uR, begin, dx, dt, oracle.Parm(D))
        ft = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
        bx.compute_flux_LR(kind, d, D, (lo, hi), ft, lo, torch.tensor(uL, device="cuda"),
                           torch.tensor(uR, device="cuda"), begin, dx, dt, bx.Parm(D))
        torch.cuda.synchronize()
        assert rel_linf(ft.cpu().numpy(), ref) <= RTOL_STEP


@pytest.mark.parametrize("D", [1, 2, 3])
def test_sweep_box_fused_equals_flux_plus_update(torch_cuda, oracle, D):
    """bamrex_sweep_box (flux + update in one kernel, with flux output) vs the
    oracle's compute_MUSCL_hancock_flux followed by the sweep update
    (AmrLevelAdv_advance.cpp:330-341); and the stand-alone update kernels."""
    torch = torch_cuda
    import bamrex_b200 as bx
    from oracle.oracle import array4, lib as olib, _dp, _iv
    shape = [70, 21, 9][:D] + [1] * (3 - D)
    lo = (0, 0, 0)
    hi = tuple(shape[d] - 1 if d < D else 0 for d in range(3))
    begin = tuple(-2 if d < D else 0 for d in range(3))
    u = _box_input(D, shape, 2, seed=9)
    dx = [0.01, 0.02, 0.03][:D]
    dt = 0.0007
    ut = torch.tensor(u, device="cuda")
    for d in range(D):
        flux = oracle.compute_flux(D, 0, d, lo, hi, u, begin, dx, dt, oracle.Parm(D))
        out_ref = np.zeros((D + 2,) + tuple(shape[::-1]))
        olib().oracle_sweep_update(D, d, _iv(lo), _iv(hi), array4(out_ref, lo), array4(u, begin), array4(flux, lo),
                                   _dp(np.array(dx + [1.0] * (3 - D))), dt)
        out = torch.zeros(out_ref.shape, dtype=torch.float64, device="cuda")
        ft = torch.full(flux.shape, float("nan"), dtype=torch.float64, device="cuda")
        bx.sweep_box(0, d, D, (lo, hi), out, lo, ut, begin, dx, dt, bx.Parm(D), flux=ft, flux_begin=lo)
        torch.cuda.synchronize()
        assert rel_linf(ft.cpu().numpy(), flux) <= RTOL_STEP
        assert rel_linf(out.cpu().numpy(), out_ref) <= RTOL_STEP
        # the stand-alone sweep update kernel on the oracle's flux
        out2 = torch.zeros_like(out)
        bx.sweep_update(d, D, (lo, hi), out2, lo, ut, begin, torch.tensor(flux, device="cuda"), lo, dx, dt)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out2.cpu().numpy(), out_ref)


@pytest.mark.parametrize("D", [1, 2, 3])
def test_unsplit_conservative_update(torch_cuda, oracle, D):
    torch = torch_cuda
    import bamrex_b200 as bx
    from oracle.oracle import array4, lib as olib, _dp, _iv, _OA4
    rng = np.random.default_rng(3)
    shape = [9, 7, 5][:D] + [1] * (3 - D)
    lo = (1, 2, 3)[:D] + (0,) * (3 - D)
    hi = tuple(lo[d] + shape[d] - 1 if d < D else 0 for d in range(3))
    u = rng.standard_normal((D + 2,) + tuple(shape[::-1]))
    fl = []
    for d in range(D):
        s = list(shape)
        s[d] += 1
        fl.append(rng.standard_normal((D + 2,) + tuple(s[::-1])))
    dt, idx = 0.01, [3.0, 5.0, 7.0]
    ref = np.zeros_like(u)
    arr = (_OA4 * 3)(*[array4(fl[d], lo) for d in range(D)] + [_OA4()] * (3 - D))
    olib().oracle_conservative_update(D, _iv(lo), _iv(hi), array4(ref, lo), array4(u, lo), arr, dt, _dp(np.array(idx)))
    out = torch.zeros(u.shape, dtype=torch.float64, device="cuda")
    bx.conservative_update(D, (lo, hi), out, lo, torch.tensor(u, device="cuda"), lo,
                           [torch.tensor(f, device="cuda") for f in fl], [lo] * D, dt, idx)
    torch.cuda.synchronize()
    assert rel_linf(out.cpu().numpy(), ref) <= 1e-14


# ------------------------------------------------------------------ levels
def _make_levels(oracle, D, n, mgs, bc, method, limiter, cfl, x_mode=0, staging=0):
    import bamrex_b200 as bx
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
    lay = oracle.LevelLayout(D, (0, 0, 0), hi, boxes, 2, [1.0 / n] * D, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
    lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D, limiter=limiter), method=method,
                   cfl=cfl, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3, x_mode=x_mode, staging=staging)
    return lay, lev


LEVEL_CASES = [
    # D, n, max_grid_size, bc, method, limiter, cfl, initial
    (1, 400, 400, 0, 0, 1, 0.9, "sod"),
    (1, 400, 64, 0, 0, 1, 0.9, "sod"),
    (2, 96, 32, 0, 0, 0, 0.8, "quadrant"),
    (2, 96, 96, 0, 0, 0, 0.8, "quadrant"),
    (2, 64, 16, 1, 0, 3, 0.5, "random"),
    (2, 64, 32, 2, 0, 1, 0.5, "random"),
    (2, 64, 64, 0, 4, 1, 0.8, "quadrant"),
    (2, 64, 32, 0, 1, 1, 0.8, "quadrant"),
    (2, 64, 32, 1, 5, 1, 0.8, "random"),
    (2, 64, 32, 1, 6, 1, 0.8, "random"),
    (3, 24, 8, 0, 0, 1, 0.8, "blast"),
    (3, 24, 24, 2, 0, 2, 0.5, "random"),
]


def _initial(kind, D, n):
    from bamrex_b200 import problems
    if kind == "sod":
        return problems.sod_1d(n)
    if kind == "quadrant":
        return problems.quadrant_2d(n)
    if kind == "blast":
        return problems.blast_3d(n, radius=0.25)
    return problems.random_states(D, tuple(n if d < D else 1 for d in (2, 1, 0)), seed=21)


def _fast_path(D, method):
    # MUSCL-Hancock with the default energy limiting and gamma 1.4 in 2D/3D:
    # the configurations the TMA-staged sweeps serve
    return D >= 2 and method == 0


@pytest.mark.parametrize("x_mode,staging", [(1, 1), (2, 1), (0, 2), (0, 3)], ids=["xrows", "xmarch", "tma", "wave"])
@pytest.mark.parametrize("case", LEVEL_CASES, ids=[str(c) for c in LEVEL_CASES])
def test_level_step_parity(torch_cuda, oracle, case, x_mode, staging):
    """AmrLevelAdv::advance (one split step) on a whole level: same dt from
    estTimeStep, then the state after the step, vs the oracle; with either
    x-sweep kernel loading through L2 (warp per row segment, thread per row),
    and with every sweep staged by TMA where that path exists."""
    import bamrex_b200 as bx
    D, n, mgs, bc, method, lim, cfl, init = case
    tma = staging in (bx.STAGING_TMA, bx.STAGING_WAVE)
    if tma and not _fast_path(D, method):
        pytest.skip("no TMA-staged sweep for this configuration")
    lay, lev = _make_levels(oracle, D, n, mgs, bc, method, lim, cfl, x_mode, staging)
    if tma:
        assert all(lev.staging(d) == staging for d in range(D))
    else:
        assert lev.x_mode == (x_mode if D > 1 else 1)
        assert all(lev.staging(d) == bx.STAGING_REGISTERS for d in range(D))
    u0 = _initial(init, D, n)
    # oracle
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u0)
    lay.fill_boundary(S1)
    parm = oracle.Parm(D, limiter=lim)
    dt_ref = lay.est_time_step(S1, 1.4, 1.0, cfl)
    S2[:] = S1
    lay.advance_explicit(S1, S2, 0.0, dt_ref, method, parm)
    ref = lay.gather(S1)
    # gpu
    lev.set_state(u0)
    dt = lev.estTimeStep()
    assert abs(dt - dt_ref) <= 1e-14 * dt_ref
    lev.advance(0.0, dt_ref)
    got = lev.get_state()
    err = rel_linf(got, ref)
    assert err <= RTOL_STEP, err
    # conserved totals, relative to the component's magnitude sum (a total
    # that is zero by symmetry has no scale of its own)
    tg, tr = got.sum(axis=(1, 2, 3)), ref.sum(axis=(1, 2, 3))
    scale = np.abs(ref).sum(axis=(1, 2, 3))
    assert np.all(np.abs(tg - tr) <= RTOL_TOTAL * scale), (tg, tr)
    # the fused CFL reduction of the last sweep equals the oracle's estTimeStep
    dt2 = lev.estTimeStep()
    dt2_ref = lay.est_time_step(S1, 1.4, 1.0, cfl)
    assert abs(dt2 - dt2_ref) <= 1e-14 * dt2_ref
    lev.close()


@pytest.fixture(scope="module")
def fixtures():
    return np.load(os.path.join(ROOT, "tests", "golden", "oracle_fixtures.npz"))


def test_against_committed_fixtures(torch_cuda, oracle, fixtures):
    """The committed oracle fixtures (tests/golden/make_oracle_fixtures.py)
    reproduced by the device-dt run loop."""
    import importlib.util
    import bamrex_b200 as bx
    spec = importlib.util.spec_from_file_location("mk", os.path.join(ROOT, "tests", "golden", "make_oracle_fixtures.py"))
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    for name, (D, n, mgs, method, lim, bc, cfl, nsteps, gen) in mk.CASES.items():
        hi = tuple(n - 1 if d < D else 0 for d in range(3))
        boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
        lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D, limiter=lim), method=method, cfl=cfl,
                       bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
        lev.set_state(fixtures[name + "/u0"])
        t, steps = lev.run(nsteps)
        assert steps == nsteps
        dts = fixtures[name + "/dts"]
        assert abs(t - dts.sum()) <= 1e-13 * dts.sum(), name
        got = lev.get_state()
        # errors of one step compound over the run; the per-step bar applies
        # per step, the run is held to nsteps times it
        err = rel_linf(got, fixtures[name + "/u1"])
        assert err <= RTOL_STEP * max(1, nsteps), (name, err)
        lev.close()


def test_sod_run_to_stop_time(torch_cuda, oracle):
    """C1: 1D Sod to t = 0.2 with the stop-time clamp, device-computed dt."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    D, n = 1, 400
    lay, lev = _make_levels(oracle, D, n, 400, 0, 0, 1, 0.9)
    u0 = problems.sod_1d(n)
    ref, t_ref, dts = oracle.run_level(lay, u0, oracle.Parm(D), 0, 0.9, stop_time=0.2)
    lev.set_state(u0)
    t, steps = lev.run(10000, stop_time=0.2)
    assert steps == len(dts)
    assert abs(t - t_ref) <= 1e-14
    got = lev.get_state()
    assert rel_linf(got, ref) <= 1e-10
    lev.close()


def test_graph_replay_and_decomposition_are_exact(torch_cuda, oracle):
    """The CUDA-graph step replay equals direct launches bit for bit, and the
    result does not depend on the box decomposition."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    D, n = 2, 128
    u0 = problems.quadrant_2d(n)
    outs = []
    for mgs, graph in ((128, False), (128, True), (32, True), (48, False)):
        hi = (n - 1, n - 1, 0)
        boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
        lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D, limiter=0), cfl=0.8)
        lev.set_state(u0)
        lev.run(5, use_graph=graph)
        outs.append(lev.get_state())
        lev.close()
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("method,limiter", [(0, 0), (0, 2), (4, 1), (1, 1), (6, 1)])
def test_x_sweep_kernels_agree(torch_cuda, oracle, D, method, limiter):
    """The two x-sweep kernels evaluate the same scheme functions per cell;
    the compiler may contract multiply-adds differently in each, so a level
    run three steps with either agrees to the per-step bar times the steps
    (both are also held to the oracle by test_level_step_parity), on ragged
    boxes (widths and heights that are not multiples of 32); the automatic
    choice takes the thread-per-row kernel for narrow boxes."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    n = 100 if D == 2 else 36
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, 24 if D == 2 else 12)
    u0 = problems.random_states(D, tuple(n if d < D else 1 for d in (2, 1, 0)), seed=5)
    outs = []
    for mode in (bx.XSWEEP_ROWS, bx.XSWEEP_MARCH, bx.XSWEEP_AUTO):
        lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D, limiter=limiter), method=method,
                       cfl=0.6, bc_lo=(1,) * 3, bc_hi=(1,) * 3, x_mode=mode)
        if mode == bx.XSWEEP_AUTO:
            assert lev.x_mode == bx.XSWEEP_MARCH
        lev.set_state(u0)
        lev.run(3, use_graph=False)
        outs.append(lev.get_state())
        lev.close()
    for o in outs[1:]:
        assert rel_linf(o, outs[0]) <= 3 * RTOL_STEP
    # a single wide box keeps the row kernel
    lev = bx.Level(2, (0, 0, 0), (4095, 4095, 0), [0.0, 0.0], [1.0, 1.0], [((0, 0, 0), (4095, 4095, 0))],
                   bx.Parm(2), cfl=0.6)
    assert lev.x_mode == bx.XSWEEP_ROWS
    lev.close()


def _ragged_boxes_2d():
    """96^2 in boxes whose x neighbours sometimes hold a whole halo slab and
    sometimes split it between two boxes."""
    boxes = []
    for ylo, yhi in ((0, 31), (32, 63), (64, 95)):
        boxes.append(((0, ylo, 0), (47, yhi, 0)))
    for xlo, xhi in ((48, 71), (72, 95)):
        for ylo, yhi in ((0, 47), (48, 95)):
            boxes.append(((xlo, ylo, 0), (xhi, yhi, 0)))
    return boxes


@pytest.mark.parametrize("D,bc,precision", [(2, 0, 0), (2, 1, 0), (2, 2, 0), (2, 1, 1), (3, 0, 0), (3, 1, 1)],
                         ids=["2d-transmissive", "2d-periodic", "2d-reflective", "2d-periodic-fp32",
                              "3d-transmissive", "3d-periodic-fp32"])
def test_x_halos_read_from_neighbours_are_exact(torch_cuda, oracle, D, bc, precision):
    """The marching x sweep reads the x halo of a box from the same-level
    box that holds all of it, and the step's x ghost fill leaves those
    slabs out: a level in many boxes (ragged in 2D, where some halos are
    split between two boxes and keep the ghost copy; the domain sides keep
    their boundary fill) steps bit for bit like the same level in one box."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    n = 96 if D == 2 else 36
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = _ragged_boxes_2d() if D == 2 else oracle.decompose(D, (0, 0, 0), hi, 12)
    u0 = problems.random_states(D, tuple(n if d < D else 1 for d in (2, 1, 0)), seed=11)
    outs = []
    for bxs in ([((0, 0, 0), hi)], boxes):
        lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, bxs, bx.Parm(D, limiter=1), cfl=0.6,
                       bc_lo=(bc,) * 3, bc_hi=(bc,) * 3, x_mode=bx.XSWEEP_MARCH, staging=bx.STAGING_REGISTERS,
                       precision=precision)
        lev.set_state(u0)
        lev.run(3, use_graph=False)
        outs.append(lev.get_state())
        lev.close()
    np.testing.assert_array_equal(outs[1], outs[0])
