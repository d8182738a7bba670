"""GPU parity of the ghost-fluid rigid body (bamrex_level_set_body /
bamrex_level_fill_body_ghosts / advance with a body, through the C ABI)
against the CPU restatement oracle/gfm_oracle.py.

Bars: the level set, normals and flags are the same formulas in the same
operation order (no FMA contraction on either side): equal to the last bit.
The ghost fill and the step carry pow() of the exact Riemann solver and the
reference's long-double quotient of the extrapolation (a unit in the last
place each): 1e-12 relative L-infinity per component, the per-step bar of
the explicit path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def rel_linf(got, ref):
    errs = []
    for n in range(ref.shape[0]):
        scale = np.max(np.abs(ref[n]))
        errs.append(np.max(np.abs(got[n] - ref[n])) / (scale if scale > 0 else 1.0))
    return max(errs)


def _split(D, n, nb):
    """nb boxes along x (then y for nb == 4; 2 x 2 x 2 for nb == 8)."""
    if nb == 8 and D == 3:
        h = [x // 2 for x in n]
        return [(tuple(c[d] * h[d] for d in range(3)), tuple((c[d] + 1) * h[d] - 1 for d in range(3)))
                for c in [(i, j, k) for k in range(2) for j in range(2) for i in range(2)]]
    if nb == 4 and D >= 2:
        hx, hy = n[0] // 2, n[1] // 2
        out = []
        for j in range(2):
            for i in range(2):
                lo = [i * hx, j * hy] + [0] * (D - 2)
                hi = [(i + 1) * hx - 1, (j + 1) * hy - 1] + [n[d] - 1 for d in range(2, D)]
                out.append((tuple(lo), tuple(hi)))
        return out
    h = n[0] // nb
    return [(tuple([i * h] + [0] * (D - 1)),
             tuple([(i + 1) * h - 1 if i < nb - 1 else n[0] - 1] + [n[d] - 1 for d in range(1, D)])) for i in range(nb)]


def _pad(t):
    return tuple(t) + (0,) * (3 - len(t))


def _make(oracle, D, n, nb, ngrow=4, bc=0, method=0, cfl=0.8):
    import bamrex_b200 as bx
    boxes = _split(D, n, nb)
    dx = [1.0 / n[d] for d in range(D)]
    lay = oracle.LevelLayout(D, (0, 0, 0), _pad([x - 1 for x in n]), [(_pad(lo), _pad(hi)) for lo, hi in boxes], ngrow,
                             dx, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
    lev = bx.Level(D, (0,) * D, tuple(x - 1 for x in n), [0.0] * D, [1.0] * D, boxes, bx.Parm(D), method=method, cfl=cfl,
                   ngrow=ngrow, bc_lo=[bc] * D, bc_hi=[bc] * D)
    return lay, lev


def _flow(D, n, seed, gamma=1.4):
    """A free stream with smooth random perturbations (physical everywhere)."""
    rng = np.random.default_rng(seed)
    shape = (n[2] if D > 2 else 1, n[1] if D > 1 else 1, n[0])
    rho = 1.0 + 0.1 * rng.random(shape)
    vel = [0.3 + 0.05 * rng.standard_normal(shape)] + [0.05 * rng.standard_normal(shape) for _ in range(D - 1)]
    p = 1.0 + 0.1 * rng.random(shape)
    U = np.zeros((D + 2,) + shape)
    U[0] = rho
    ke = np.zeros(shape)
    for d in range(D):
        U[1 + d] = rho * vel[d]
        ke += vel[d] ** 2
    U[1 + D] = p / (gamma - 1) + 0.5 * rho * ke
    return U


def _shapes(case):
    """(gpu shape dicts, oracle shapes, combine)."""
    from oracle import gfm_oracle as G
    import bamrex_b200 as bx
    if case == "cylinder":
        s = [dict(kind=bx.SDF_CYLINDER, center=(0.52, 0.47, 0.0), axis=(0, 0, 1), radius=0.21)]
        comb = bx.SDF_UNION
    elif case == "sphere":
        s = [dict(kind=bx.SDF_SPHERE, center=(0.5, 0.45, 0.55), radius=0.27)]
        comb = bx.SDF_UNION
    elif case == "corner_sphere":
        s = [dict(kind=bx.SDF_SPHERE, center=(0.5, 0.5, 0.5), radius=0.17)]
        comb = bx.SDF_UNION
    elif case == "big_cylinder":
        s = [dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.0), axis=(0, 0, 1), radius=0.45)]
        comb = bx.SDF_UNION
    elif case == "big_sphere":
        s = [dict(kind=bx.SDF_SPHERE, center=(0.5, 0.5, 0.5), radius=0.47)]
        comb = bx.SDF_UNION
    elif case == "two_cylinders":
        s = [dict(kind=bx.SDF_CYLINDER, center=(0.3, 0.5, 0.0), axis=(0, 0, 1), radius=0.15),
             dict(kind=bx.SDF_CYLINDER, center=(0.62, 0.41, 0.0), axis=(0, 0, 1), radius=0.17)]
        comb = bx.SDF_UNION
    else:  # a half disc: the intersection of a cylinder and a plane
        s = [dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.0), axis=(0, 0, 1), radius=0.25),
             dict(kind=bx.SDF_PLANE, center=(0.45, 0.5, 0.0), axis=(-1.0, 0.3, 0.0))]
        comb = bx.SDF_INTERSECTION
    so = [G.make_shape(x["kind"], x.get("center", (0, 0, 0)), x.get("axis", (0, 0, 1)), x.get("radius", 0.0),
                       x.get("fluid_inside", False)) for x in s]
    return s, so, comb


LS_CASES = [(2, (40, 36), 3, "cylinder", 2, False), (2, (32, 32), 4, "two_cylinders", 3, True),
            (2, (36, 36), 2, "half_disc", 2, False), (3, (16, 14, 12), 2, "sphere", 2, False),
            (3, (12, 12, 12), 1, "cylinder", 3, True)]


@pytest.mark.parametrize("case", LS_CASES, ids=lambda c: "%dd-%s" % (c[0], c[3]))
def test_levelset_normals_flags(torch_cuda, oracle, case):
    """Level set, normals and GFM flags on every valid cell, bit for bit."""
    from oracle import gfm_oracle as G
    D, n, nb, shape, stencil, diag = case
    lay, lev = _make(oracle, D, n, nb)
    s, so, comb = _shapes(shape)
    lev.set_body(s, combine=comb, stencil=stencil, fill_diagonals=diag)
    body = G.Body(lay, so, comb, (0.0,) * D, stencil=stencil, fill_diagonals=diag)
    for which in range(D + 1):
        np.testing.assert_array_equal(lev.body_field(which), body.field(which))
    np.testing.assert_array_equal(lev.body_field(-1), body.field(-1))
    fl = body.field(-1).astype(int)
    ni, ns = lev.body_counts()
    assert ni == int(np.sum(((fl & G.GHOST) != 0) & ((fl & G.INTERFACE) != 0)))
    assert ns == int(np.sum(((fl & G.GHOST) != 0) & ((fl & G.INTERFACE) == 0)))
    assert ni > 0 and ns > 0
    lev.close()


FILL_CASES = [(2, (40, 36), 3, "cylinder", 0), (2, (40, 36), 3, "cylinder", 1), (2, (40, 36), 3, "cylinder", 2),
              (2, (32, 32), 4, "two_cylinders", 0), (2, (36, 36), 2, "half_disc", 0), (3, (16, 14, 12), 2, "sphere", 0),
              (3, (16, 14, 12), 2, "sphere", 2),
              # the body's centre on the corner of eight boxes
              (3, (16, 16, 16), 8, "corner_sphere", 0),
              (3, (32, 32, 32), 8, "corner_sphere", 0),
              # single boxes with large swept regions: a cp.async ring of four
              # records per thread (96^2, 20^3)
              (2, (96, 96), 1, "big_cylinder", 0),
              (3, (20, 20, 20), 1, "big_sphere", 0),
              # a 28^3 box: values fit, a ring of two records per thread
              # does not (the next record in registers instead)
              (3, (28, 28, 28), 1, "big_sphere", 0),
              # one 32^3 box whose swept region with its halo exceeds shared
              # memory in FP64: the global-memory sweep kernel
              (3, (32, 32, 32), 1, "big_sphere", 0)]


@pytest.mark.parametrize("case", FILL_CASES, ids=lambda c: "%dd-%s-rb%d" % (c[0], c[3], c[4]))
def test_body_ghost_fill(torch_cuda, oracle, case):
    """FillRBGhostCells (interface cells, inter-box fill, fast-sweeping
    extrapolation, boundary fill) vs the oracle."""
    from oracle import gfm_oracle as G
    D, n, nb, shape, rb = case
    lay, lev = _make(oracle, D, n, nb)
    s, so, comb = _shapes(shape)
    u0 = _flow(D, n, seed=7 + rb)
    lev.set_body(s, combine=comb, rb_bc=rb)
    lev.set_state(u0)
    lev.fill_body_ghosts()
    got = lev.get_state()
    body = G.Body(lay, so, comb, (0.0,) * D)
    buf = lay.alloc()
    lay.scatter(buf, u0)
    lay.fill_boundary(buf)
    assert G.fill_rb(lay, buf, body, rb, 1.4, 1.0) == 0
    ref = lay.gather(buf)
    assert not np.allclose(ref, u0)
    err = rel_linf(got, ref)
    assert err <= RTOL, err
    lev.close()


@pytest.mark.parametrize("case", [(2, (40, 36), 3, "cylinder", 0, 0), (2, (32, 32), 4, "two_cylinders", 2, 0),
                                  (2, (40, 36), 3, "cylinder", 1, 1), (3, (16, 14, 12), 2, "sphere", 0, 0)],
                         ids=lambda c: "%dd-%s-rb%d-m%d" % (c[0], c[3], c[4], c[5]))
def test_step_with_body(torch_cuda, oracle, case):
    """AmrLevelAdv::advance with a rigid body: FillPatch, FillRBGhostCells,
    fill_consv_boundary, then the split sweeps, vs the oracle."""
    from oracle import gfm_oracle as G
    D, n, nb, shape, rb, method = case
    lay, lev = _make(oracle, D, n, nb, method=method)
    s, so, comb = _shapes(shape)
    u0 = _flow(D, n, seed=31 + rb)
    lev.set_body(s, combine=comb, rb_bc=rb)
    lev.set_state(u0)
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u0)
    lay.fill_boundary(S1)
    dt = lay.est_time_step(S1, 1.4, 1.0, 0.8)
    body = G.Body(lay, so, comb, (0.0,) * D)
    G.fill_rb(lay, S1, body, rb, 1.4, 1.0)
    S2[:] = S1
    lay.advance_explicit(S1, S2, 0.0, dt, method, oracle.Parm(D))
    ref = lay.gather(S1)
    lev.advance(0.0, dt)
    got = lev.get_state()
    err = rel_linf(got, ref)
    assert err <= RTOL, err
    lev.close()


def test_run_with_body_graph(torch_cuda, oracle):
    """Three device-stepped steps (CUDA graph, device dt) with a body equal
    three oracle steps with estTimeStep between them."""
    from oracle import gfm_oracle as G
    D, n = 2, (40, 36)
    lay, lev = _make(oracle, D, n, 3)
    s, so, comb = _shapes("cylinder")
    u0 = _flow(D, n, seed=5)
    lev.set_body(s, combine=comb)
    lev.set_state(u0)
    t, steps = lev.run(3, use_graph=True)
    got = lev.get_state()
    body = G.Body(lay, so, comb, (0.0,) * D)
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u0)
    lay.fill_boundary(S1)
    time = 0.0
    for _ in range(3):
        dt = lay.est_time_step(S1, 1.4, 1.0, 0.8)
        G.fill_rb(lay, S1, body, G.REFLECTIVE, 1.4, 1.0)
        S2[:] = S1
        lay.advance_explicit(S1, S2, time, dt, 0, oracle.Parm(D))
        lay.fill_boundary(S1)
        time += dt
    assert steps == 3
    assert abs(t - time) <= 1e-13 * time
    err = rel_linf(got, lay.gather(S1))
    assert err <= 3 * RTOL, err
    lev.close()


def test_body_removed_restores_plain_step(torch_cuda, oracle):
    """set_body(None) leaves the plain explicit step."""
    D, n = 2, (32, 32)
    lay, lev = _make(oracle, D, n, 2)
    s, _, comb = _shapes("cylinder")
    u0 = _flow(D, n, seed=3)
    lev.set_body(s, combine=comb)
    lev.set_body(None)
    assert lev.body_counts() == (0, 0)
    lev.set_state(u0)
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u0)
    lay.fill_boundary(S1)
    dt = lay.est_time_step(S1, 1.4, 1.0, 0.8)
    S2[:] = S1
    lay.advance_explicit(S1, S2, 0.0, dt, 0, oracle.Parm(D))
    lev.advance(0.0, dt)
    assert rel_linf(lev.get_state(), lay.gather(S1)) <= RTOL
    lev.close()


def test_body_argument_errors(torch_cuda, oracle):
    import bamrex_b200 as bx
    s, _, comb = _shapes("cylinder")
    _, lev2 = _make(oracle, 2, (32, 32), 2, ngrow=3)
    with pytest.raises(bx.BamrexError) as e:
        lev2.set_body(s)
    assert e.value.status == bx._abi.ERR_ARG
    lev2.close()
    _, lev = _make(oracle, 2, (32, 32), 2, ngrow=4)
    with pytest.raises(bx.BamrexError):
        lev.set_body(s, stencil=5)
    with pytest.raises(bx.BamrexError):
        lev.set_body([dict(kind=bx.SDF_PLANE, center=(0.5, 0.5), axis=(0, 0, 0))])
    with pytest.raises(bx.BamrexError):
        lev.fill_body_ghosts()
    lev.close()


def _smooth_state(D, n, seed):
    from bamrex_b200 import problems
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    g = np.meshgrid(*([x] * D), indexing="ij")
    shp = (1,) * (3 - D) + (n,) * D
    ph = rng.uniform(0, 2 * np.pi, 3)
    q = np.zeros((D + 2,) + shp)
    q[0] = np.transpose(1 + 0.2 * np.sin(2 * np.pi * g[0] + ph[0]) * np.cos(2 * np.pi * g[-1] + ph[1])).reshape(shp)
    q[D + 1] = np.transpose(1 + 0.1 * np.cos(2 * np.pi * g[-1] + ph[2])).reshape(shp)
    q[1] = 0.3
    return problems.consv_from_primv(D, q, 1.4)


@pytest.mark.parametrize("D", [2, 3])
def test_hierarchy_with_body_matches_oracle(torch_cuda, oracle, D):
    """Subcycled coarse steps of a hierarchy with a rigid body on every level
    (coarse/fine ghost fill, then the rigid-body fill, then the sweeps, flux
    registers, reflux, average_down) against the restatement driven on the
    same grids: three levels and a cylinder in 2D, two levels and a sphere
    on the corner of eight boxes in 3D.

    The 3D case limits every component on its own ratio. With the default
    (every component limited on the energy's ratio) the limiter's 0/0 branch
    (a limiting variable flat to the last bit selects phi(1), one flat to
    rounding an arbitrary ratio) makes the step discontinuous in the last bit
    of the energy next to the body, and the device's fast sweeps round
    differently from the restatement (test_gfm_cpu.py,
    test_oracle_body_limiter_sensitivity: a 1e-15 change of the restatement's
    own input moves its result by 1e-8)."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import Amr
    from oracle import gfm_oracle as G
    from oracle.amr_oracle import OAmr
    n = 32 if D == 2 else 16
    hi0 = tuple(n - 1 if d < D else 0 for d in range(3))
    levels = [oracle.decompose(D, (0, 0, 0), hi0, n // 2)]
    lo1, hi1 = n // 2, n + n // 2 - 1
    levels.append(oracle.decompose(D, tuple(lo1 if d < D else 0 for d in range(3)),
                                   tuple(hi1 if d < D else 0 for d in range(3)), n // 2))
    if D == 2:
        lo2, hi2 = 2 * lo1 + n // 2, 2 * hi1 + 1 - n // 2
        levels.append(oracle.decompose(D, tuple(lo2 if d < D else 0 for d in range(3)),
                                       tuple(hi2 if d < D else 0 for d in range(3)), n // 2))
    if D == 2:
        shape = dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.0), axis=(0, 0, 1), radius=0.1)
    else:
        shape = dict(kind=bx.SDF_SPHERE, center=(0.5, 0.5, 0.5), radius=0.17)
    so = [G.make_shape(shape["kind"], shape["center"], shape.get("axis", (0, 0, 1)), shape["radius"])]
    own = list(range(D + 2)) + [1 + D] * (6 - D) if D == 3 else None
    A = Amr(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, levels[0], bx.Parm(D, limiter=1, limiter_indices=own),
            cfl=0.8, max_level=len(levels) - 1, blocking_factor=8, max_grid_size=64, ngrow=4)
    for l in range(1, len(levels)):
        A.set_level_boxes(l, levels[l])
    A.set_body(shape)
    OA = OAmr(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, levels, oracle.Parm(D, limiter=1, limiter_indices=own),
              oracle.MUSCL_HANCOCK, 0.8, ngrow=4)
    OA.set_bodies(so, 0, (0.0,) * D, G.REFLECTIVE, 1.4)
    for l in range(len(levels)):
        u = _smooth_state(D, n * 2 ** l, 11)
        A.set_state(l, u)
        OA.levels[l].set_dense(u)
    A.avg_down_all()
    OA.avg_down_all()
    for s in range(2):
        if s:
            for l in range(len(levels)):
                OA.levels[l].set_dense(A.get_state(l))
        dt = A.coarse_step()
        odt = OA.coarse_step()
        assert abs(dt - odt) <= 1e-12 * odt
        for l in range(len(levels)):
            got, ref = A.get_state(l), OA.levels[l].dense()
            m = ~np.isnan(ref)
            e = float(np.max(np.abs(got[m] - ref[m])) / np.max(np.abs(ref[m])))
            assert e <= 1e-12 * 2 ** l, (s, l, e)
    A.close()


@pytest.mark.parametrize("D", [2, 3])
def test_tagging_with_body_matches_oracle(torch_cuda, oracle, D):
    """errorEst on a level with a rigid body (bamrex_level_tag_ex): grad_error,
    box_error and interface_error, then ghost_error clearing the solid cells
    away from the interface, identical to the restatement
    (oracle.amr_oracle.tag_level + tag_level_extra on the restated level set
    and flags); bamrex_level_tag on the same level applies ghost_error."""
    from oracle import gfm_oracle as G
    from oracle.amr_oracle import OLevel, tag_level, tag_level_extra
    n = (48, 48) if D == 2 else (24, 24, 24)
    nb = 3 if D == 2 else 8
    lay, lev = _make(oracle, D, n, nb)
    s, so, comb = _shapes("cylinder" if D == 2 else "sphere")
    u0 = _flow(D, n, seed=9)
    lev.set_body(s, combine=comb)
    lev.set_state(u0)
    box = ((0.1, 0.6, 0.2), (0.35, 0.9, 0.7))
    t = lev.tag_ex(grad_var=0, grad_threshold=0.08, box=box, lstol=0.05)
    t_plain = lev.tag(grad_var=0, grad_threshold=0.08)
    t_box = lev.tag_ex(box=box)
    lev.close()
    boxes = [(_pad(lo), _pad(hi)) for lo, hi in _split(D, n, nb)]
    dx = [1.0 / n[d] for d in range(D)] + [1.0] * (3 - D)
    o = OLevel(D, (0, 0, 0), _pad([x - 1 for x in n]), boxes, 2, dx, (0, 0, 0), (0, 0, 0))
    o.set_dense(u0)
    o.lay.fill_boundary(o.S)
    body = G.Body(lay, so, comb, (0.0,) * D)
    ls, fl = body.field(0), body.field(-1).astype(np.int64)
    base = tag_level(o, grad_var=0, grad_threshold=0.08)
    want = tag_level_extra(base, boxes, (0, 0, 0), D, dx, (0.0, 0.0, 0.0), box=box, ls=ls, flags=fl, lstol=0.05)
    np.testing.assert_array_equal(t, want)
    np.testing.assert_array_equal(t_plain, tag_level_extra(base, boxes, (0, 0, 0), D, dx, (0.0, 0.0, 0.0), ls=ls,
                                                           flags=fl))
    np.testing.assert_array_equal(t_box, tag_level_extra(np.zeros_like(base), boxes, (0, 0, 0), D, dx,
                                                         (0.0, 0.0, 0.0), box=box, ls=ls, flags=fl))
    # every criterion decides some cells
    solid = ((fl & 1) != 0) & ((fl & 2) == 0)
    assert solid.sum() > 0 and 0 < t.sum() < t.size and t_box.sum() > 0
    assert t.sum() != t_plain.sum()


def test_hierarchy_regrid_around_body(torch_cuda):
    """Interface tagging drives the regrid of a hierarchy with a rigid body
    (tagging.max_int_lev / lstol): level 1 covers every level-0 cell at the
    interface or within lstol of it, and no coarse cell deep in the solid
    is tagged (ghost_error) - the fine boxes stay near the interface."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import Amr
    D, n = 2, 64
    hi = (n - 1, n - 1, 0)
    A = Amr(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, [((0, 0, 0), hi)], bx.Parm(D), cfl=0.8, ngrow=4, max_level=1,
            blocking_factor=8, max_grid_size=32, n_error_buf=1, max_int_lev=1, lstol=[0.03])
    A.set_body(dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.0), axis=(0, 0, 1), radius=0.25))
    A.set_state(0, _flow(D, (n, n), seed=4))
    A.regrid(0, 0.0)
    assert A.finest_level == 1
    ls = A.level(0).body_field(0)[0]
    fl = A.level(0).body_field(-1)[0].astype(np.int64)
    covered = np.zeros((n, n), dtype=bool)
    for lo, hi1 in A.boxes(1):
        covered[lo[1] // 2:hi1[1] // 2 + 1, lo[0] // 2:hi1[0] // 2 + 1] = True
    want = ((fl & 2) != 0) | (np.abs(ls) <= 0.03)
    assert want.sum() > 0 and covered[want].all()
    # deep in the solid (a disc of radius 0.1 about the centre) nothing is refined
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    deep = (X - 0.5) ** 2 + (Y - 0.5) ** 2 < 0.1 ** 2
    assert not covered[deep].any()
    A.close()


def test_extrapolation_limit_shared_by_levels(torch_cuda, oracle):
    """Two levels whose rigid-body sweeps need different amounts of shared
    memory (both above the default 48 KB): setting up the smaller one after
    the larger must not break the larger one's fill (the limit belongs to
    the kernel, not to a level); its step equals the step of the same level
    made alone."""
    def run(extra):
        _, a = _make(oracle, 3, (24, 24, 24), 1)
        s, _, comb = _shapes("big_sphere")
        a.set_body(s, combine=comb)
        b = None
        if extra:
            _, b = _make(oracle, 3, (20, 20, 20), 1)
            b.set_body(s, combine=comb)
        a.set_state(_flow(3, (24, 24, 24), seed=2))
        a.advance(0.0, 1e-3)
        got = a.get_state()
        a.close()
        if b is not None:
            b.close()
        return got
    np.testing.assert_array_equal(run(True), run(False))
