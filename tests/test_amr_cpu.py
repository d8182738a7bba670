"""AMR pieces that run without a GPU: the library's host-side grid
generation (bamrex_cluster_tags) and the CPU restatement of the coupling
(oracle/amr_oracle.py) checked against conservation and consistency
properties."""
import numpy as np
import pytest

from bamrex_b200 import problems


def _blob_tags(D, n, centres, radius):
    x = np.arange(n) + 0.5
    g = np.meshgrid(*([x] * D), indexing="ij")
    t = np.zeros([n] * D, dtype=bool)
    for c in centres:
        t |= sum((gi - ci) ** 2 for gi, ci in zip(g, c)) < radius ** 2
    return t


def _packed(D, t, boxes):
    # packed order: box-major, x fastest; t is indexed [x, y, z]
    out = []
    for lo, hi in boxes:
        sl = tuple(slice(lo[d], hi[d] + 1) for d in range(D))
        out.append(np.transpose(t[sl]).ravel())
    return np.concatenate(out).astype(np.uint8)


@pytest.mark.parametrize("D,n,mgs,bf", [(2, 64, 32, 8), (2, 64, 16, 4), (3, 32, 16, 8)])
def test_cluster_tags_properties(D, n, mgs, bf):
    from bamrex_b200.amr import cluster_tags
    from oracle import oracle as O
    boxes = O.decompose(D, (0, 0, 0), tuple(n - 1 if d < D else 0 for d in range(3)), 16)
    t = _blob_tags(D, n, [(0.3 * n,) * D, (0.7 * n, 0.6 * n, 0.5 * n)[:D]], 0.12 * n)
    nb = 1
    fine = cluster_tags(D, (0, 0, 0), tuple(n - 1 if d < D else 0 for d in range(3)), boxes, _packed(D, t, boxes),
                        ref_ratio=2, blocking_factor=bf, max_grid_size=mgs, n_error_buf=nb, n_proper=1, grid_eff=0.7)
    assert fine
    cover = np.zeros([2 * n] * D, dtype=int)
    for lo, hi in fine:
        for d in range(D):
            assert lo[d] % bf == 0 and (hi[d] + 1) % bf == 0, "blocking factor alignment"
            assert hi[d] - lo[d] + 1 <= mgs, "max_grid_size"
            assert 0 <= lo[d] and hi[d] < 2 * n
        cover[tuple(slice(lo[d], hi[d] + 1) for d in range(D))] += 1
    assert cover.max() == 1, "boxes overlap"
    # every tagged cell (buffered) is refined: level-0 cell c is covered if
    # its fine children are
    tb = t.copy()
    for d in range(D):
        tb = np.maximum.reduce([np.roll(tb, s, axis=d) for s in range(-nb, nb + 1)]) if nb else tb
    child = cover[tuple(slice(0, None, 2) for _ in range(D))] > 0
    assert np.all(child[t]), "a tagged cell is not refined"


def test_cluster_tags_validation():
    from bamrex_b200 import BamrexError
    from bamrex_b200.amr import cluster_tags
    boxes = [((0, 0, 0), (31, 31, 0))]
    tags = np.zeros(32 * 32, dtype=np.uint8)
    with pytest.raises(BamrexError):
        cluster_tags(2, (0, 0, 0), (31, 31, 0), boxes, tags, ref_ratio=2, blocking_factor=6)
    with pytest.raises(BamrexError):
        cluster_tags(2, (0, 0, 0), (31, 31, 0), boxes, tags, ref_ratio=2, blocking_factor=8, max_grid_size=12)
    assert cluster_tags(2, (0, 0, 0), (31, 31, 0), boxes, tags) == []


def _smooth_blob(D, n):
    x = (np.arange(n) + 0.5) / n
    g = np.meshgrid(*([x] * D), indexing="ij")
    shp = (1,) * (3 - D) + (n,) * D
    q = np.zeros((D + 2,) + shp)
    rho = 1 + 0.3 * np.sin(2 * np.pi * g[0])
    r2 = sum((gi - 0.5) ** 2 for gi in g)
    p = 1 + 0.2 * np.cos(2 * np.pi * g[-1]) + 2.0 * (r2 < 0.04)
    q[0] = np.transpose(rho).reshape(shp)
    q[D + 1] = np.transpose(p).reshape(shp)
    for d in range(D):
        q[1 + d] = 0.2 - 0.1 * d
    return problems.consv_from_primv(D, q, 1.4)


@pytest.mark.parametrize("D", [2, 3])
def test_oracle_amr_conserves_with_reflux(oracle, D):
    from oracle.amr_oracle import OAmr
    n = 32 if D == 2 else 16
    q = n // 2
    hi0 = tuple(n - 1 if d < D else 0 for d in range(3))
    fine = [(tuple(q if d < D else 0 for d in range(3)), tuple(3 * q - 1 if d < D else 0 for d in range(3)))]
    bc = (oracle.PERIODIC,) * 3
    u0 = _smooth_blob(D, n)
    drift = {}
    for reflux in (True, False):
        A = OAmr(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, [[((0, 0, 0), hi0)], fine], oracle.Parm(D, limiter=1),
                 oracle.MUSCL_HANCOCK, 0.8, bc_lo=bc, bc_hi=bc, do_reflux=reflux)
        A.levels[0].set_dense(u0)
        A.cpl[1].fill_coarse_patch()
        A.avg_down_all()
        s0 = A.conserved_sums()
        for _ in range(3):
            A.coarse_step()
        drift[reflux] = np.abs(A.conserved_sums() - s0) / np.abs(s0).max()
    assert drift[True].max() <= 1e-13, drift[True]
    assert drift[False].max() > 1e-8, drift[False]


def test_oracle_interp_reproduces_linear_and_averages(oracle):
    from oracle.amr_oracle import _interp, _padded
    D, n, r = 2, 8, 2
    x = np.arange(n)
    Y, X = np.meshgrid(x, x, indexing="ij")
    dense = np.zeros((4, 1, n, n))
    dense[0, 0] = 1.0 + 0.25 * X + 0.125 * Y  # linear: reproduced exactly
    dense[1, 0] = np.where((X + Y) % 3 == 0, 2.0, 1.0)  # rough: bounded, conservative
    dense[2, 0] = 0.5
    dense[3, 0] = 2.0
    P = _padded(dense, D, (0, 0, 0), (0, 0, 0), 2)
    fi = np.arange(2, 2 * n - 2)
    FY, FX = np.meshgrid(fi, fi, indexing="ij")
    w = [FX.ravel(), FY.ravel(), np.zeros(FX.size, dtype=np.int64)]
    v = _interp(P, D, r, 2, w)
    exact = 1.0 + 0.25 * ((w[0] + 0.5) / 2 - 0.5) + 0.125 * ((w[1] + 0.5) / 2 - 0.5)
    np.testing.assert_allclose(v[0], exact, rtol=0, atol=1e-14)
    c = (w[1] // 2, w[0] // 2)
    nb_min = np.minimum.reduce([dense[1, 0][np.clip(c[0] + a, 0, n - 1), np.clip(c[1] + b, 0, n - 1)]
                                for a, b in ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1))])
    nb_max = np.maximum.reduce([dense[1, 0][np.clip(c[0] + a, 0, n - 1), np.clip(c[1] + b, 0, n - 1)]
                                for a, b in ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1))])
    assert np.all(v[1] >= nb_min - 1e-15) and np.all(v[1] <= nb_max + 1e-15)
    # children average to the parent
    m = v[1].reshape(FY.shape)
    avg = 0.25 * (m[0::2, 0::2] + m[1::2, 0::2] + m[0::2, 1::2] + m[1::2, 1::2])
    np.testing.assert_allclose(avg, dense[1, 0][1:n - 1, 1:n - 1], rtol=0, atol=1e-14)


def test_oracle_fine_everywhere_equals_single_fine_level(oracle):
    """A fine level covering the whole domain advances exactly like a single
    level at the fine resolution with the same time steps."""
    from oracle.amr_oracle import OAmr
    D, n = 2, 16
    u0 = _smooth_blob(D, 2 * n)
    A = OAmr(D, (0, 0, 0), (n - 1, n - 1, 0), [0.0, 0.0], [1.0, 1.0],
             [[((0, 0, 0), (n - 1, n - 1, 0))], [((0, 0, 0), (2 * n - 1, 2 * n - 1, 0))]], oracle.Parm(D),
             oracle.MUSCL_HANCOCK, 0.8)
    A.levels[1].set_dense(u0)
    A.avg_down_all()
    dts = []
    for _ in range(2):
        A.coarse_step()
        dts += [A.dt_level[1]] * 2
    lay = oracle.LevelLayout(D, (0, 0, 0), (2 * n - 1, 2 * n - 1, 0), [((0, 0, 0), (2 * n - 1, 2 * n - 1, 0))], 2,
                             [1.0 / (2 * n)] * 2)
    S = lay.alloc()
    lay.scatter(S, u0)
    t = 0.0
    for dt in dts:
        lay.fill_boundary(S)
        S2 = S.copy()
        lay.advance_explicit(S, S2, t, dt, oracle.MUSCL_HANCOCK, oracle.Parm(D))
        t += dt
    np.testing.assert_array_equal(A.levels[1].dense(), lay.gather(S))


def _random_level_boxes(rng, D, n, align):
    cuts = []
    for d in range(3):
        if d < D:
            c = [0]
            while c[-1] < n:
                c.append(min(n, c[-1] + align * int(rng.integers(1, 5))))
            cuts.append(list(zip(c[:-1], [x - 1 for x in c[1:]])))
        else:
            cuts.append([(0, 0)])
    keep = rng.uniform(0.4, 1.0)
    boxes = [((x0, y0, z0), (x1, y1, z1)) for (z0, z1) in cuts[2] for (y0, y1) in cuts[1] for (x0, x1) in cuts[0]
             if rng.random() < keep]
    return boxes or [((0, 0, 0), (cuts[0][0][1], cuts[1][0][1], cuts[2][0][1]))]


@pytest.mark.parametrize("seed", range(6))
def test_cluster_tags_matches_dense_restatement(seed):
    """The library's grid generation works box by box in blocked space; the
    oracle buffers, erodes and blocks cell masks over the whole domain.  The
    box lists agree exactly over ragged, partly covered levels, periodic and
    non-periodic sides, both refinement ratios and several buffers."""
    from bamrex_b200.amr import cluster_tags
    from oracle import amr_oracle as AO
    rng = np.random.default_rng(1000 + seed)
    for _ in range(12):
        D = int(rng.integers(1, 4))
        ratio = int(rng.choice([2, 4]))
        bf = 2 * ratio * int(rng.integers(1, 3))
        c = bf // ratio
        n = c * int(rng.integers(2, {1: 40, 2: 14, 3: 7}[D]))
        boxes = _random_level_boxes(rng, D, n, int(rng.choice([1, 2, c])))
        t = rng.random([n] * D) < rng.choice([0.002, 0.02, 0.2])
        per = tuple(int(rng.random() < 0.4) if d < D else 0 for d in range(3))
        kw = dict(ref_ratio=ratio, blocking_factor=bf, max_grid_size=bf * int(rng.integers(1, 5)),
                  n_error_buf=int(rng.integers(0, 4)), n_proper=int(rng.integers(0, 3)),
                  grid_eff=float(rng.choice([0.5, 0.7, 0.9])), periodic=per)
        hi = tuple(n - 1 if d < D else 0 for d in range(3))
        tags = _packed(D, t, boxes)
        got = cluster_tags(D, (0, 0, 0), hi, boxes, tags, **kw)
        want = AO.cluster_tags_dense(D, (0, 0, 0), hi, boxes, tags, **kw)
        assert got == want, (D, n, kw)


def test_cluster_tags_threaded_matches_dense_restatement():
    """A level large enough (256^3 cells, 64^3 blocked cells) that the tag
    scan, the allowed-cell test and the clipping run on several host threads
    still gives exactly the restatement's boxes: sparse random tags and a
    tagged spherical shell, periodic and non-periodic sides."""
    from bamrex_b200.amr import cluster_tags
    from oracle import amr_oracle as AO
    rng = np.random.default_rng(4242)
    n = 256
    hi = (n - 1,) * 3
    z, y, x = np.meshgrid(*([np.arange(n) + 0.5] * 3), indexing="ij")
    shell = np.abs(np.sqrt((x - 128) ** 2 + (y - 120) ** 2 + (z - 136) ** 2) - 70) < 2
    for per in ((0, 0, 0), (1, 0, 1)):
        boxes = _random_level_boxes(rng, 3, n, 4)
        t = shell | (rng.random([n] * 3) < 0.0005)
        kw = dict(ref_ratio=2, blocking_factor=8, max_grid_size=32, n_error_buf=2, n_proper=1, grid_eff=0.7,
                  periodic=per)
        tags = _packed(3, t, boxes)
        got = cluster_tags(3, (0, 0, 0), hi, boxes, tags, **kw)
        want = AO.cluster_tags_dense(3, (0, 0, 0), hi, boxes, tags, **kw)
        assert len(got) > 100 and got == want


def test_tag_extra_restatement_small_cases():
    """box_error, interface_error and ghost_error of the restatement on
    hand-checked cells: the box tags the cells whose centres it contains,
    |level set| <= lstol and interface flags tag, solid cells away from the
    interface are cleared even where another criterion tagged them."""
    import numpy as np
    from oracle.amr_oracle import tag_level_extra
    D = 2
    boxes = [((0, 0, 0), (3, 1, 0)), ((0, 2, 0), (3, 3, 0))]
    dx = [0.25, 0.25, 1.0]
    tags = np.zeros(16, dtype=np.uint8)
    tags[0] = 1  # (0, 0) from another criterion
    out = tag_level_extra(tags, boxes, (0, 0, 0), D, dx, (0.0, 0.0, 0.0), box=((0.3, 0.3), (0.6, 0.9)))
    # centres 0.375, 0.625 in x (0.625 > 0.6: out), 0.375 ... 0.875 in y
    want = np.zeros((4, 4), dtype=np.uint8)
    want[1:4, 1] = 1
    got = np.zeros((4, 4), dtype=np.uint8)
    got[0:2] = out[:8].reshape(2, 4)
    got[2:4] = out[8:].reshape(2, 4)
    want[0, 0] = 1
    np.testing.assert_array_equal(got, want)
    ls = np.full((1, 4, 4), 1.0)
    ls[0, 3, 3] = 0.01
    flags = np.zeros((1, 4, 4), dtype=np.int64)
    flags[0, 0, 0] = 1          # solid, not at the interface: cleared
    flags[0, 0, 1] = 1 | 2      # solid at the interface: tagged
    flags[0, 2, 0] = 2          # fluid at the interface: tagged
    out = tag_level_extra(tags, boxes, (0, 0, 0), D, dx, (0.0, 0.0, 0.0), ls=ls, flags=flags, lstol=0.05)
    got = np.zeros((4, 4), dtype=np.uint8)
    got[0:2] = out[:8].reshape(2, 4)
    got[2:4] = out[8:].reshape(2, 4)
    want = np.zeros((4, 4), dtype=np.uint8)
    want[0, 1] = want[2, 0] = want[3, 3] = 1
    np.testing.assert_array_equal(got, want)
    # without lstol only ghost_error applies
    out = tag_level_extra(np.ones(16, dtype=np.uint8), boxes, (0, 0, 0), D, dx, (0.0, 0.0, 0.0), ls=ls, flags=flags)
    assert out[0] == 0 and out[1] == 1 and out.sum() == 15
