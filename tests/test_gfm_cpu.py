"""The ghost-fluid rigid-body restatement (oracle/gfm_oracle.py) pinned to
the reference's own tests: GFM flags (Tests/GFMFlag01.cpp, GFMFlag02.cpp),
bilinear interpolation (Tests/Interp01.cpp) and the exact Riemann solver on
Toro's five problems (Tests/ExactRiemann01.cpp, Tests/UnitDomainTest.H);
then properties of the rigid-body fill that need no GPU."""
import math

import numpy as np
import pytest

from oracle import gfm_oracle as G


def _layout(D, n, boxes=None, ngrow=3, bc=0, L=1.0):
    from oracle import oracle as O
    pad = (0,) * (3 - D)
    dom_hi = tuple(x - 1 for x in n) + pad
    boxes = [(tuple(lo) + pad, tuple(hi) + pad) for lo, hi in (boxes or [((0,) * D, dom_hi[:D])])]
    dx = [L / n[d] for d in range(D)]
    return O.LevelLayout(D, (0, 0, 0), dom_hi, boxes, ngrow, dx, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)


# ---- flags ----------------------------------------------------------------

def _flags(lay, body):
    return body.field(-1)[0].astype(int)


def test_flags_diagonal_interface():
    """GFMFlag01: body below the diagonal y <= x of a 5x5 unit grid."""
    lay = _layout(2, (5, 5), ngrow=2)
    dx = 0.2

    def ls(i, j, k):
        x = (i + 0.5) * dx
        y = (j + 0.5) * dx - 1e-10
        return (x - y) / math.sqrt(2)

    body = G.Body(lay, None, 0, (0, 0), stencil=2, ls_fn=ls)
    F = _flags(lay, body)
    for j in range(5):
        for i in range(5):
            f = F[j, i]
            assert bool(f & G.GHOST) == (i >= j)
            assert bool(f & G.INTERFACE) == (i == j or j == i + 1)
            assert bool(f & G.FILL) == (i >= j and i <= j + 1)


def _staircase(i, j, k):
    # body where j < ((i + 1) / 2) * 2 with C integer division
    return 1.0 if j < int((i + 1) / 2) * 2 else -1.0


def test_flags_staircase_stencil3():
    """GFMFlag02 staircase with fill_info.stencil = 3."""
    lay = _layout(2, (5, 5), ngrow=3)
    body = G.Body(lay, None, 0, (0, 0), stencil=3, ls_fn=_staircase)
    F = _flags(lay, body)
    for j in range(5):
        for i in range(5):
            f = F[j, i]
            ghost = j < int((i + 1) / 2) * 2
            assert bool(f & G.GHOST) == ghost
            assert bool(f & G.INTERFACE) == (i == j or j == i + 1 or j == i - 1)
            assert bool(f & G.FILL) == (not ((i == 4 and j == 0) or not ghost))


def test_flags_staircase_diagonals():
    """GFMFlag02 staircase with stencil 2 and fill_diagonals."""
    lay = _layout(2, (5, 5), ngrow=3)
    body = G.Body(lay, None, 0, (0, 0), stencil=2, fill_diagonals=True, ls_fn=_staircase)
    F = _flags(lay, body)
    for j in range(5):
        for i in range(5):
            f = F[j, i]
            ghost = j < int((i + 1) / 2) * 2
            assert bool(f & G.FILL) == (not (i >= j + 3 or not ghost))


# ---- bilinear interpolation -------------------------------------------------

def _interp_grid(D):
    """Interp01: src on cells (0..3, 0..4, 0..5) over [0,2]x[0,1.5]x[0,0.6],
    1000 everywhere except the corner cells set by the test."""
    dx = [2 / 4, 1.5 / 5, 0.6 / 6][:D]
    src = {}

    def f(i, j, k, n):
        return src.get((i, j, k, n), 1000.0)

    bl = [(1 + 0.5) * dx[0], (2 + 0.5) * dx[1], (3 + 0.5) * dx[2] if D > 2 else 0.0][:D]
    return dx, src, f, bl


def test_bilinear_2d():
    dx, src, f, bl = _interp_grid(2)
    for (i, j), v in {(1, 2): 1, (2, 2): 2, (1, 3): 3, (2, 3): 4}.items():
        src[(i, j, 0, 0)] = float(v)
        src[(i, j, 0, 1)] = -float(v)
    out = {}
    for i in range(5):
        for j in range(5):
            p = [bl[0] + i / 4 * dx[0], bl[1] + j / 4 * dx[1]]
            out[(i, j)] = G.bilinear(p, f, 2, dx, 2, (i, j, 0))
    for i in range(5):
        assert out[(i, 0)][0] == pytest.approx(1 + 0.25 * i, abs=1e-12)
        assert out[(i, 4)][0] == pytest.approx(3 + 0.25 * i, abs=1e-12)
        assert out[(i, 2)][0] == pytest.approx(2 + 0.25 * i, abs=1e-12)
        assert out[(i, 0)][1] == pytest.approx(-(1 + 0.25 * i), abs=1e-12)
        assert out[(i, 4)][1] == pytest.approx(-(3 + 0.25 * i), abs=1e-12)
    for j in range(5):
        assert out[(0, j)][0] == pytest.approx(1 + 0.5 * j, abs=1e-12)
        assert out[(4, j)][0] == pytest.approx(2 + 0.5 * j, abs=1e-12)
        assert out[(2, j)][0] == pytest.approx(1.5 + 0.5 * j, abs=1e-12)
        assert out[(0, j)][1] == pytest.approx(-(1 + 0.5 * j), abs=1e-12)


def test_bilinear_3d():
    dx, src, f, bl = _interp_grid(3)
    vals = {(1, 2, 3): 1, (2, 2, 3): 2, (1, 3, 3): 3, (2, 3, 3): 4, (1, 2, 4): 5, (2, 2, 4): 6, (1, 3, 4): 7, (2, 3, 4): 8}
    for c, v in vals.items():
        src[c + (0,)] = float(v)
    out = {}
    for i in range(5):
        for j in range(5):
            for k in range(5):
                p = [bl[0] + i / 4 * dx[0], bl[1] + j / 4 * dx[1], bl[2] + k / 4 * dx[2]]
                out[(i, j, k)] = G.bilinear(p, f, 3, dx, 1, (i, j, k))[0]
    for i in range(5):
        assert out[(i, 0, 0)] == pytest.approx(1 + 0.25 * i, abs=1e-12)
        assert out[(i, 4, 0)] == pytest.approx(3 + 0.25 * i, abs=1e-12)
        assert out[(i, 0, 4)] == pytest.approx(5 + 0.25 * i, abs=1e-12)
    for k in range(5):
        assert out[(0, 0, k)] == pytest.approx(1 + k, abs=1e-12)
        assert out[(0, 4, k)] == pytest.approx(3 + k, abs=1e-12)
    for j in range(5):
        assert out[(0, j, 2)] == pytest.approx(3 + 0.5 * j, abs=1e-12)


def test_bilinear_c7_reads_component_zero():
    """The last two terms of c7 (Interp_K.H:64-66) come from component 0:
    for component 1 a trilinear field is off by Dx*Dy*Dz*(s010 - s000) of
    component 0."""
    dx = [1.0, 1.0, 1.0]

    def f(i, j, k, n):
        return (1.0 + 2 * i + 3 * j + 5 * k) if n == 0 else (7.0 + i + j + k)

    p = [1.25 + 0.5, 2.5 + 0.5, 3.75 + 0.5]
    v0, v1 = G.bilinear(p, f, 3, dx, 2, (0, 0, 0))
    assert v0 == pytest.approx(1 + 2 * 1.25 + 3 * 2.5 + 5 * 3.75, abs=1e-12)
    exact1 = 7 + 1.25 + 2.5 + 3.75
    quirk = 0.25 * 0.5 * 0.75 * ((f(1, 3, 3, 0) - f(1, 2, 3, 0)) - (f(1, 3, 3, 1) - f(1, 2, 3, 1)))
    assert v1 == pytest.approx(exact1 + quirk, abs=1e-12)


# ---- exact Riemann solver (Toro's tests, intermediate states to 5 d.p.) ----

TORO = [
    # (rhoL, uL, pL, rhoR, uR, pR, p*, u*, rho*L, rho*R, tolerance)
    ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), (0.30313, 0.92745, 0.42632, 0.26557), 1e-5, False),
    ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4), (0.00189, 0.0, 0.02185, 0.02185), 1e-5, False),
    ((1.0, 0.0, 1000.0), (1.0, 0.0, 0.01), (460.894, 19.5975, 0.57506, 5.99924), 1e-5, True),
    ((1.0, 0.0, 0.01), (1.0, 0.0, 100.0), (46.0950, -6.19633, 5.99242, 0.57511), 1e-4, False),
    ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950), (1691.64, 8.68975, 14.2823, 31.0426), 1e-5, True),
]


@pytest.mark.parametrize("case", range(5))
def test_exact_riemann_toro(case):
    L, R, exp, tol, rel = TORO[case]
    PL = [L[0], L[1], 0.0, L[2]]
    PR = [R[0], R[1], 0.0, R[2]]
    p, u, IL, IR, it = G.exact_riemann(PL, PR, 2, 1.4, 1.0)
    assert it < 200
    got = (p, u, IL[0], IR[0])
    for g, e in zip(got, exp):
        bound = abs(e) * tol if rel else tol
        assert abs(g - e) <= max(bound, 1e-12), (case, got, exp)


def test_exact_riemann_scaled_epsilon():
    """Toro test 1 in the low-Mach scaling (UnitDomainTest.H:312-360):
    the same intermediate states in scaled units."""
    rho0, u0, p0 = 0.5, 1.3, 10000.0
    eps = rho0 * u0 * u0 / p0
    PL = [1.0 / rho0, 0.0, 0.0, 1.0 / p0]
    PR = [0.125 / rho0, 0.0, 0.0, 0.1 / p0]
    p, u, IL, IR, it = G.exact_riemann(PL, PR, 2, 1.4, eps)
    assert p == pytest.approx(0.30313 / p0, rel=2e-5)
    assert u == pytest.approx(0.92745 / u0, rel=2e-5)
    assert IL[0] == pytest.approx(0.42632 / rho0, rel=2e-5)
    assert IR[0] == pytest.approx(0.26557 / rho0, rel=2e-5)


# ---- signed distances ------------------------------------------------------

def test_sdf_shapes():
    cyl = G.make_shape(G.CYLINDER, center=(0.5, 0.5, 0.0), axis=(0, 0, 2), radius=0.1)
    assert G.sdf(cyl, 2, 0.5, 0.5, 0) == pytest.approx(0.1)
    assert G.sdf(cyl, 2, 0.8, 0.5, 0) == pytest.approx(-0.2)
    assert G.sdf(cyl, 3, 0.5, 0.7, 9.0) == pytest.approx(-0.1)
    sph = G.make_shape(G.SPHERE, center=(0, 0, 0), radius=1.0, fluid_inside=True)
    assert G.sdf(sph, 3, 2.0, 0, 0) == pytest.approx(1.0)
    pl = G.make_shape(G.PLANE, center=(0.5, 0, 0), axis=(2.0, 0, 0))
    assert G.sdf(pl, 2, 0.25, 0.3, 0) == pytest.approx(0.25)
    u = G.shape_value([G.make_shape(G.SPHERE, (0, 0, 0), radius=1), G.make_shape(G.SPHERE, (3, 0, 0), radius=1)],
                      G.UNION, 2, 1.5, 0, 0)
    assert u == pytest.approx(-0.5)


# ---- the rigid-body fill on the CPU ------------------------------------------

def _cylinder_level(n=24, nbox=2, ngrow=4):
    D = 2
    half = n // nbox
    boxes = [((i * half, 0), ((i + 1) * half - 1, n - 1)) for i in range(nbox)]
    lay = _layout(D, (n, n), boxes=boxes, ngrow=ngrow)
    shape = G.make_shape(G.CYLINDER, center=(0.5, 0.47, 0.0), axis=(0, 0, 1), radius=0.21)
    return lay, shape


def test_rb_fill_fluid_at_rest_is_steady():
    """A uniform gas at rest: every rigid-body condition leaves the
    interface cells at the free state and the body is filled with it."""
    lay, shape = _cylinder_level()
    gamma, eps = 1.4, 1.0
    rho, p = 1.3, 0.7
    glob = np.zeros(lay.domain_shape())
    glob[0] = rho
    glob[3] = p / (gamma - 1)
    for rb in (G.REFLECTIVE, G.NO_SLIP, G.FOEXTRAP):
        buf = lay.alloc()
        lay.scatter(buf, glob)
        lay.fill_boundary(buf)
        body = G.Body(lay, [shape], 0, (0.0, 0.0))
        G.fill_rb(lay, buf, body, rb, gamma, eps)
        out = lay.gather(buf)
        np.testing.assert_allclose(out, glob, rtol=1e-12, atol=1e-14)


def test_rb_fill_reflective_interface_states():
    """Uniform flow past the body: the reflective condition puts the
    interface ghost cells in the intermediate state of the reflected normal
    velocity, so their normal velocity nearly vanishes (all but the small
    intermediate velocity the curvature term of the right pressure makes)
    and their pressure rises where the flow meets the body and falls where
    it leaves it; fluid cells are untouched."""
    lay, shape = _cylinder_level()
    gamma, eps = 1.4, 1.0
    glob = np.zeros(lay.domain_shape())
    glob[0] = 1.0
    glob[1] = 0.3
    glob[3] = 1.0 / (gamma - 1) + 0.5 * 0.3 * 0.3
    buf = lay.alloc()
    lay.scatter(buf, glob)
    lay.fill_boundary(buf)
    body = G.Body(lay, [shape], 0, (0.0, 0.0))
    before = lay.gather(buf)
    G.fill_rb(lay, buf, body, G.REFLECTIVE, gamma, eps)
    out = lay.gather(buf)
    flags = body.field(-1)[0].astype(int)
    nx_, ny_ = body.field(1)[0], body.field(2)[0]
    fluid = (flags & G.GHOST) == 0
    np.testing.assert_array_equal(out[:, 0][:, fluid], before[:, 0][:, fluid])
    iface = ((flags & G.GHOST) != 0) & ((flags & G.INTERFACE) != 0)
    assert iface.sum() > 10
    rho, mx, my, E = (out[c, 0][iface] for c in range(4))
    un = (mx * nx_[iface] + my * ny_[iface]) / rho
    assert np.max(np.abs(un)) < 0.05
    p = (gamma - 1) * (E - 0.5 * (mx * mx + my * my) / rho)
    un_in = 0.3 * nx_[iface]
    big = np.abs(un_in) > 0.15
    assert big.sum() > 4
    assert np.all(np.sign(p[big] - 1.0) == -np.sign(un_in[big]))
    assert np.all(out[0, 0] > 0)


# ---- conditioning of a hierarchy step with a body --------------------------

def _blob_state(D, n, seed):
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    g = np.meshgrid(*([x] * D), indexing="ij")
    shp = (1,) * (3 - D) + (n,) * D
    ph = rng.uniform(0, 2 * np.pi, 3)
    q = np.zeros((D + 2,) + shp)
    q[0] = np.transpose(1 + 0.2 * np.sin(2 * np.pi * g[0] + ph[0]) * np.cos(2 * np.pi * g[-1] + ph[1])).reshape(shp)
    q[D + 1] = np.transpose(1 + 0.1 * np.cos(2 * np.pi * g[-1] + ph[2])).reshape(shp)
    q[1] = 0.3
    return np.array(G.consv_from_primv(list(q), D, 1.4, 1.0))


def _hierarchy_step_with_sphere(limiter_indices, rel_noise):
    from oracle import oracle as O
    from oracle.amr_oracle import OAmr
    D, n = 3, 16
    levels = [O.decompose(D, (0, 0, 0), (n - 1,) * 3, n // 2),
              O.decompose(D, (n // 2,) * 3, (n + n // 2 - 1,) * 3, n // 2)]
    OA = OAmr(D, (0, 0, 0), (n - 1,) * 3, [0.0] * D, [1.0] * D, levels,
              O.Parm(D, limiter=O.VAN_LEER, limiter_indices=limiter_indices), O.MUSCL_HANCOCK, 0.8, ngrow=4)
    OA.set_bodies([G.make_shape(G.SPHERE, (0.5, 0.5, 0.5), radius=0.17)], 0, (0.0,) * D, G.REFLECTIVE, 1.4)
    rng = np.random.default_rng(7)
    for l in range(2):
        u = _blob_state(D, n * 2 ** l, 11)
        if l == 1:
            u = u * (1 + rel_noise * rng.standard_normal(u.shape))
        OA.levels[l].set_dense(u)
    OA.avg_down_all()
    OA.coarse_step()
    return [OA.levels[l].dense() for l in range(2)]


def _max_change(a, b):
    return max(float(np.nanmax(np.abs(x - y))) for x, y in zip(a, b))


def test_oracle_body_limiter_sensitivity():
    """Why the 3D hierarchy-with-body parity case limits every component on
    itself. The reference limits every component on the energy's ratio by
    default, and its ratio has a 0/0 branch (both differences exactly zero:
    phi(1), a full slope; both at the rounding level: an arbitrary ratio).
    Next to the sphere the energy is flat to the last bit while density and
    momentum are not, so a relative change of 1e-15 in the fine level's input
    (the size of the rounding differences between the device's step and the
    restatement's) moves the restatement's own result after one coarse step by
    1e-8 or more; limited component by component the same change stays at
    the rounding level."""
    from oracle import oracle as O
    default = [1 + 3] * O.MAX_NCOMP
    own = list(range(5)) + [4] * (O.MAX_NCOMP - 5)
    base = _hierarchy_step_with_sphere(default, 0.0)
    moved = _hierarchy_step_with_sphere(default, 1e-15)
    assert _max_change(base, moved) > 1e-9
    base = _hierarchy_step_with_sphere(own, 0.0)
    moved = _hierarchy_step_with_sphere(own, 1e-15)
    assert _max_change(base, moved) < 1e-13
