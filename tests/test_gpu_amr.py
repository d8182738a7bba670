"""The AMR coupling on the device against the CPU restatement
(oracle/amr_oracle.py): coarse/fine ghost interpolation with time
interpolation, flux registers, reflux, average_down, tagging, and whole
subcycled hierarchy steps; conservation of the composite totals."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


class _DevArray:
    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 2,
                                         "strides": None}


def read_fab(torch, level, b, fp32=False):
    """The whole fab of box b (valid + ghost cells) as (NC, nz, ny, nx)."""
    a = level.fab(b)
    nx, ny, nz = (a.end[d] - a.begin[d] for d in range(3))
    n = a.nstride * a.ncomp
    t = torch.as_tensor(_DevArray(a.p, n, "<f4" if fp32 else "<f8"), device="cuda")
    flat = t.double().cpu().numpy()
    out = np.empty((a.ncomp, nz, ny, nx))
    for m in range(a.ncomp):
        for k in range(nz):
            for j in range(ny):
                o = m * a.nstride + k * a.kstride + j * a.jstride
                out[m, k, j] = flat[o:o + nx]
    return out, (a.begin[0], a.begin[1], a.begin[2])


def _smooth(D, n, seed=0, blob=2.0):
    from bamrex_b200 import problems
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    g = np.meshgrid(*([x] * D), indexing="ij")
    shp = (1,) * (3 - D) + (n,) * D
    q = np.zeros((D + 2,) + shp)
    ph = rng.uniform(0, 2 * np.pi, 4)
    rho = 1 + 0.3 * np.sin(2 * np.pi * g[0] + ph[0]) * np.cos(2 * np.pi * g[-1] + ph[1])
    r2 = sum((gi - 0.45) ** 2 for gi in g)
    p = 1 + 0.2 * np.cos(2 * np.pi * g[-1] + ph[2]) + blob * (r2 < 0.03)
    q[0] = np.transpose(rho).reshape(shp)
    q[D + 1] = np.transpose(p).reshape(shp)
    for d in range(D):
        q[1 + d] = (0.2 - 0.1 * d) * np.transpose(np.cos(2 * np.pi * g[d] + ph[3])).reshape(shp)
    return problems.consv_from_primv(D, q, 1.4)


def _rel_linf(a, b):
    m = ~np.isnan(b)
    return float(np.max(np.abs(a[m] - b[m])) / max(np.max(np.abs(b[m])), 1e-300))


@pytest.mark.parametrize("D,bc", [(2, 0), (2, 1), (2, 2), (3, 1)])
def test_fill_patch_matches_oracle(torch_cuda, oracle, D, bc):
    """Fine coarse/fine ghosts at the old time, the new time and in between
    are bit-identical to the restatement (time + MC/Barth-Jespersen space
    interpolation, boundary-mapped coarse patches)."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import Coupling
    from oracle.amr_oracle import OCoupling, OLevel
    n = 16 if D == 2 else 8
    hi0 = tuple(n - 1 if d < D else 0 for d in range(3))
    hi1 = tuple(2 * n - 1 if d < D else 0 for d in range(3))
    cboxes = oracle.decompose(D, (0, 0, 0), hi0, 8)
    # two fine boxes touching the low domain faces: periodic images,
    # reflected or extrapolated coarse patch cells, and coarse/fine faces
    fb = [((0, 0, 0), tuple(7 if d < D else 0 for d in range(3))),
          ((8, 0, 0), tuple(15 if d == 0 else (7 if d < D else 0) for d in range(3)))]
    parm = bx.Parm(D, limiter=1)
    s = torch_cuda.cuda.Stream()
    kw = dict(method=bx.MUSCL_HANCOCK, cfl=0.8, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3, stream=s)
    lc = bx.Level(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, cboxes, parm, **kw)
    lf = bx.Level(D, (0, 0, 0), hi1, [0.0] * D, [1.0] * D, fb, parm, **kw)
    C = Coupling(lc, lf, 2)
    oc = OLevel(D, (0, 0, 0), hi0, cboxes, 2, [1.0 / n] * D, (bc,) * 3, (bc,) * 3)
    of = OLevel(D, (0, 0, 0), hi1, fb, 2, [0.5 / n] * D, (bc,) * 3, (bc,) * 3)
    OC = OCoupling(oc, of, 2)
    u_old, u_new, u_f = _smooth(D, n, 1), _smooth(D, n, 2), _smooth(D, 2 * n, 3)
    lc.set_state(u_old)
    oc.set_dense(u_old)
    C.save_coarse_old(0.0, 1.0)
    OC.save_coarse_old(0.0, 1.0)
    lc.set_state(u_new)
    oc.set_dense(u_new)
    lf.set_state(u_f)
    for time in (0.0, 0.375, 1.0):
        C.fill_patch(time)
        lf.sync()
        of.S[:] = np.nan
        of.set_dense(u_f)
        OC.fill_patch(time, [of.S])
        for b in range(len(fb)):
            got, _ = read_fab(torch_cuda, lf, b)
            want = of.fab(b)
            m = ~np.isnan(want)
            assert m.sum() > 0
            np.testing.assert_array_equal(got[m], want[m], err_msg="fine box %d at t=%g" % (b, time))
    C.close()
    lf.close()
    lc.close()


@pytest.mark.parametrize("D,nsteps,reflux", [(2, 3, True), (2, 2, False), (3, 2, True)])
def test_hierarchy_steps_match_oracle(torch_cuda, oracle, D, nsteps, reflux):
    """Whole subcycled coarse steps (fill patch, sweeps with flux-register
    recording, reflux, average_down, dt over levels) against the
    restatement driven on the same grids."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import Amr
    from oracle.amr_oracle import OAmr
    n = 32 if D == 2 else 16
    hi0 = tuple(n - 1 if d < D else 0 for d in range(3))
    bc = 0
    levels = [oracle.decompose(D, (0, 0, 0), hi0, n // 2)]
    lo1, hi1 = n // 2, n + n // 2 - 1  # the middle half, level 1
    levels.append(oracle.decompose(D, tuple(lo1 if d < D else 0 for d in range(3)),
                                   tuple(hi1 if d < D else 0 for d in range(3)), n // 2))
    if D == 2:  # a third level inside the second
        lo2, hi2 = 2 * lo1 + n // 2, 2 * hi1 + 1 - n // 2
        levels.append(oracle.decompose(D, tuple(lo2 if d < D else 0 for d in range(3)),
                                       tuple(hi2 if d < D else 0 for d in range(3)), n // 2))
    parm = bx.Parm(D, limiter=1)
    A = Amr(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, levels[0], parm, cfl=0.8, max_level=len(levels) - 1,
            blocking_factor=8, max_grid_size=64, do_reflux=reflux)
    for l in range(1, len(levels)):
        A.set_level_boxes(l, levels[l])
    OA = OAmr(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, levels, oracle.Parm(D, limiter=1), oracle.MUSCL_HANCOCK, 0.8,
              do_reflux=reflux)
    for l in range(len(levels)):
        u = _smooth(D, n * 2 ** l, 7)
        A.set_state(l, u)
        OA.levels[l].set_dense(u)
    A.avg_down_all()
    OA.avg_down_all()
    for s in range(nsteps):
        # each coarse step from identical inputs: the oracle takes the
        # device state (valid cells) before stepping
        if s:
            for l in range(len(levels)):
                OA.levels[l].set_dense(A.get_state(l))
        dt = A.coarse_step()
        odt = OA.coarse_step()
        assert abs(dt - odt) <= 1e-12 * odt
        for l in range(len(levels)):
            # level l takes 2^l substeps per coarse step; 1e-12 per substep
            e = _rel_linf(A.get_state(l), OA.levels[l].dense())
            assert e <= 1e-12 * 2 ** l, (s, l, e)
    tot, otot = A.conserved_sums(), OA.conserved_sums()
    np.testing.assert_allclose(tot, otot, rtol=1e-12, atol=1e-14 * np.abs(otot).max())
    A.close()


@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 2e-6)])
def test_hierarchy_conserves_periodic(torch_cuda, oracle, precision, tol):
    """Composite totals of a periodic two-level hierarchy stay constant with
    reflux (FP64 to 1e-13, FP32 storage to its rounding)."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import Amr
    D, n = 2, 32
    hi0 = (n - 1, n - 1, 0)
    bc = (bx.BC_PERIODIC,) * 3
    A = Amr(D, (0, 0, 0), hi0, [0.0, 0.0], [1.0, 1.0], oracle.decompose(D, (0, 0, 0), hi0, 16), bx.Parm(D), cfl=0.8,
            bc_lo=bc, bc_hi=bc, max_level=1, blocking_factor=8, max_grid_size=32, precision=precision)
    # fine patches crossing the periodic boundary and in the middle
    A.set_level_boxes(1, [((0, 0, 0), (15, 15, 0)), ((48, 0, 0), (63, 15, 0)), ((24, 24, 0), (39, 39, 0))])
    u = _smooth(D, n, 5)
    A.set_state(0, u)
    A.level(1).set_state(_smooth(D, 2 * n, 6))
    A.avg_down_all()
    s0 = A.conserved_sums()
    for _ in range(4):
        A.coarse_step()
    s1 = A.conserved_sums()
    scale = np.abs(s0).max()
    assert np.all(np.abs(s1 - s0) <= tol * scale), (s1 - s0) / scale
    A.close()


def test_tagging_matches_oracle(torch_cuda, oracle):
    """grad_error on the energy and on the pressure (primitive), and
    state_error on the pressure, are identical to the restatement of
    tagging_K.H (the blast's density is uniform: nothing to tag on rho)."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from oracle.amr_oracle import OLevel, tag_level
    D, n = 3, 24
    hi = (n - 1,) * 3
    boxes = oracle.decompose(D, (0, 0, 0), hi, 12)
    u = problems.blast_3d(n, radius=0.25)
    L = bx.Level(D, (0, 0, 0), hi, [0.0] * 3, [1.0] * 3, boxes, bx.Parm(D))
    L.set_state(u)
    t = L.tag(grad_var=4, grad_threshold=0.1)
    t2 = L.tag(grad_var=0, grad_threshold=0.0, err_var=4, phierr=5.0, err_var_is_primv=True)
    t3 = L.tag(grad_var=4, grad_threshold=0.5, grad_var_is_primv=True)
    t0 = L.tag(grad_var=0, grad_threshold=0.1)
    L.close()
    o = OLevel(D, (0, 0, 0), hi, boxes, 2, [1.0 / n] * 3, (0, 0, 0), (0, 0, 0))
    o.set_dense(u)
    o.lay.fill_boundary(o.S)
    P = oracle.Parm(D)
    np.testing.assert_array_equal(t, tag_level(o, grad_var=4, grad_threshold=0.1))
    np.testing.assert_array_equal(t2, tag_level(o, err_var=4, phierr=5.0, primv=True, parm=P))
    np.testing.assert_array_equal(t3, tag_level(o, grad_var=4, grad_threshold=0.5, primv=True, parm=P))
    assert t0.sum() == 0
    for x in (t, t2, t3):
        assert 0 < x.sum() < x.size


def test_regrid_keeps_fine_data_where_the_coarse_level_moved(torch_cuda, oracle):
    """A regrid that moves level 1 away from part of level 2: the new level
    2 takes the old level-2 values wherever its cells were level-2 cells
    before (AMReX's regrid fills a remade level from its old data first,
    Amr::regrid -> AmrLevel::init(old)), even though the old level 2 is not
    properly nested in the new level 1, and the hierarchy steps on."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import Amr
    D, n = 2, 64
    hi0 = (n - 1, n - 1, 0)
    A = Amr(D, (0, 0, 0), hi0, [0.0] * 3, [1.0] * 3, oracle.decompose(D, (0, 0, 0), hi0, 32), bx.Parm(D),
            max_level=2, blocking_factor=8, max_grid_size=32, n_error_buf=2, phierr=[1.5, 1.5], phierr_var=0)

    def state(lev, c0):
        # a dense square over coarse cells [c0, c0 + 16)^2 at rest, p = 1
        m, s = n * 2 ** lev, 2 ** lev
        u = np.zeros((4, 1, m, m))
        u[0] = 1.0
        u[3] = 2.5
        u[0, 0, c0 * s:(c0 + 16) * s, c0 * s:(c0 + 16) * s] = 2.0
        return u

    try:
        A.init(lambda amr, lev: state(lev, 16))
        assert A.finest_level == 2
        # a fine-scale energy pattern on level 2 that no interpolation from
        # level 1 reproduces
        pat = A.get_state(2)
        j, i = np.indices(pat.shape[2:])
        pat[3, 0] += 0.01 * ((i + 2 * j) % 3)
        A.set_state(2, pat)
        A.set_state(0, state(0, 24))
        A.set_state(1, state(1, 24))
        old1 = A.boxes(1)
        A.regrid(0)
        assert A.finest_level == 2 and A.boxes(1) != old1
        new2 = A.get_state(2)
        kept = ~np.isnan(new2[0]) & ~np.isnan(pat[0])
        assert kept.any() and (~np.isnan(new2[0]) & np.isnan(pat[0])).any()
        np.testing.assert_array_equal(new2[:, kept], pat[:, kept])
        A.coarse_step()
        for lev in range(3):
            s = A.get_state(lev)
            assert np.isfinite(s[:, ~np.isnan(s[0])]).all()
    finally:
        A.close()


def test_blast_regrid_and_step(torch_cuda, oracle):
    """The spherical-blast hierarchy: tag (grad_error >= 0.1 on the
    pressure; the initial density is uniform), build levels 1 and 2 from the
    tags, and step; the boxes satisfy the grid rules and the steps match the
    restatement on the same grids."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.amr import Amr
    from oracle.amr_oracle import OAmr
    D, n = 3, 16
    hi0 = (n - 1,) * 3
    A = Amr(D, (0, 0, 0), hi0, [0.0] * 3, [1.0] * 3, oracle.decompose(D, (0, 0, 0), hi0, 16), bx.Parm(D, limiter=0),
            cfl=0.8, max_level=2, blocking_factor=8, max_grid_size=16, n_error_buf=1, phigrad=[0.1, 0.1],
            phigrad_var=4, phigrad_var_is_primv=True)

    def init(amr, lev):
        m = n * 2 ** lev
        return problems.blast_3d(m, radius=0.25)

    A.init(init)
    assert A.finest_level == 2
    levels = [A.boxes(l) for l in range(3)]
    for l in (1, 2):
        for lo, hi in levels[l]:
            for d in range(3):
                assert lo[d] % 8 == 0 and (hi[d] + 1) % 8 == 0 and hi[d] - lo[d] + 1 <= 16
    OA = OAmr(D, (0, 0, 0), hi0, [0.0] * 3, [1.0] * 3, levels, oracle.Parm(D, limiter=0), oracle.MUSCL_HANCOCK, 0.8)
    for l in range(3):
        OA.levels[l].set_dense(A.get_state(l))
    for s in range(2):
        if s:
            for l in range(3):
                OA.levels[l].set_dense(A.get_state(l))
        A.coarse_step()
        OA.coarse_step()
        for l in range(3):
            assert _rel_linf(A.get_state(l), OA.levels[l].dense()) <= 1e-12 * 2 ** l
    A.close()
