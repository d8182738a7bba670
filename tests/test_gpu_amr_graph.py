"""Coarse steps replayed as CUDA graphs (bamrex_amr_set_graph): the time
steps computed on the device and the whole subcycled recursion captured once
per state of the levels' buffers give the host-driven coarse step's result
bit for bit: every level's state, every coarse dt and the time, over
several steps, with regrids between them, FP32 storage, a rigid body on
every level and a stop time that clamps the last step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _smooth(D, n, seed, blob=2.0):
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


def _nested(D, n):
    from bamrex_b200.level import decompose
    hi0 = tuple(n - 1 if d < D else 0 for d in range(3))
    levels = [decompose(D, (0, 0, 0), hi0, n // 2)]
    lo1, hi1 = n // 2, n + n // 2 - 1
    levels.append(decompose(D, tuple(lo1 if d < D else 0 for d in range(3)),
                            tuple(hi1 if d < D else 0 for d in range(3)), n // 2))
    if D == 2:
        lo2, hi2 = 2 * lo1 + n // 2, 2 * hi1 + 1 - n // 2
        levels.append(decompose(D, tuple(lo2 if d < D else 0 for d in range(3)),
                                tuple(hi2 if d < D else 0 for d in range(3)), n // 2))
    return hi0, levels


def _pair(D, n, graph, precision=0, body=False):
    import bamrex_b200 as bx
    from bamrex_b200.amr import Amr
    hi0, levels = _nested(D, n)
    A = Amr(D, (0, 0, 0), hi0, [0.0] * D, [1.0] * D, levels[0], bx.Parm(D, limiter=1), cfl=0.8,
            max_level=len(levels) - 1, blocking_factor=8, max_grid_size=64, precision=precision,
            ngrow=4 if body else 2)
    A.set_graph(graph)
    for l in range(1, len(levels)):
        A.set_level_boxes(l, levels[l])
    if body:
        A.set_body(dict(kind=bx.SDF_CYLINDER, center=(0.5, 0.5, 0.0), axis=(0, 0, 1), radius=0.1))
    for l in range(len(levels)):
        A.set_state(l, _smooth(D, n * 2 ** l, 11))
    A.avg_down_all()
    return A


def _same(A, B, what):
    assert A.time == B.time, what
    for l in range(A.finest_level + 1):
        a, b = A.get_state(l), B.get_state(l)
        np.testing.assert_array_equal(a, b, err_msg="%s, level %d" % (what, l))


@pytest.mark.parametrize("D,precision,body", [(2, 0, False), (2, 1, False), (3, 0, False), (2, 0, True)])
def test_graph_coarse_steps_equal_host_steps(torch_cuda, D, precision, body):
    n = 32 if D == 2 else 16
    A = _pair(D, n, False, precision, body)
    B = _pair(D, n, True, precision, body)
    steps = 6
    for s in range(steps):
        da, db = A.coarse_step(), B.coarse_step()
        assert da == db, (s, da, db)
        assert A.dt_level() == B.dt_level()
        _same(A, B, "coarse step %d" % s)
    caps, reps, kern = B.graph_stats()
    # the first step after the levels were set takes the host path
    assert reps == steps - 1 and 1 <= caps <= 2 and kern > 0, (caps, reps, kern)
    assert A.graph_stats()[1] == 0
    tot_a, tot_b = A.conserved_sums(), B.conserved_sums()
    np.testing.assert_array_equal(tot_a, tot_b)
    A.close()
    B.close()


def test_graph_steps_to_stop_time(torch_cuda):
    """The last step is clamped to the stop time on the device as the host
    clamps it."""
    A = _pair(2, 32, False)
    B = _pair(2, 32, True)
    for _ in range(2):
        A.coarse_step()
        B.coarse_step()
    stop = A.time + 1.5 * A.dt_level()[0]
    dts = []
    for s in range(2):
        da, db = A.coarse_step(stop), B.coarse_step(stop)
        assert da == db, (s, da, db)
        dts.append(da)
        _same(A, B, "step %d to the stop time" % s)
    assert dts[1] < 0.9 * dts[0]  # the clamped step
    assert abs(A.time - stop) <= 1e-15 * stop
    A.close()
    B.close()


def test_graph_steps_with_regrids(torch_cuda):
    """A 3D blast hierarchy that regrids every 4 coarse steps: host steps at
    the regrids and the first step after, graph replays between them."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.amr import Amr

    def make(graph):
        n = 16
        A = Amr(3, (0, 0, 0), (n - 1,) * 3, [0.0] * 3, [1.0] * 3, [((0, 0, 0), (n - 1,) * 3)],
                bx.Parm(3, limiter=0), cfl=0.8, max_level=2, blocking_factor=8, max_grid_size=16, n_error_buf=1,
                phigrad=[0.1, 0.1], phigrad_var=4, phigrad_var_is_primv=True, regrid_int=4)
        A.set_graph(graph)
        A.init(lambda amr, lev: problems.blast_3d(n * 2 ** lev, radius=0.25))
        return A

    A, B = make(False), make(True)
    assert A.finest_level == 2
    for s in range(10):
        da, db = A.coarse_step(), B.coarse_step()
        assert da == db, (s, da, db)
        assert [A.boxes(l) for l in range(A.finest_level + 1)] == [B.boxes(l) for l in range(B.finest_level + 1)]
        _same(A, B, "coarse step %d" % s)
    assert B.graph_stats()[1] >= 4
    A.close()
    B.close()
