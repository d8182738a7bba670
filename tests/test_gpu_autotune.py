"""The sweep work decomposition is free to change: every segment shape the
autotuner may pick gives the same state bit for bit, and the tuner returns
one of its candidates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_segments_do_not_change_results(oracle, tmp_path, monkeypatch):
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.autotune import S_CANDIDATES, X_CANDIDATES, tune_segments
    n = 256
    hi = (n - 1, n - 1, 0)
    boxes = oracle.decompose(2, (0, 0, 0), hi, 128)
    u0 = problems.quadrant_2d(n)
    parm = bx.Parm(2, limiter=bx.MINBEE)
    ref = None
    for xs, ss in ((0, 0), (32, 16), (64, 24), (256, 48), (128, 256)):
        lev = bx.Level(2, (0, 0, 0), hi, [0, 0], [1, 1], boxes, parm, cfl=0.8, x_segment=xs, s_segment=ss)
        lev.set_state(u0)
        lev.run(3, use_graph=False)
        out = lev.get_state()
        lev.close()
        if ref is None:
            ref = out
        else:
            np.testing.assert_array_equal(out, ref)
    monkeypatch.setenv("BAMREX_TUNE_CACHE", str(tmp_path))
    x, s, table = tune_segments(2, (0, 0, 0), hi, [0, 0], [1, 1], boxes, parm, u0, steps=2)
    assert x in (0,) + X_CANDIDATES and s in (0,) + S_CANDIDATES
    assert "auto" in table
    x2, s2, _ = tune_segments(2, (0, 0, 0), hi, [0, 0], [1, 1], boxes, parm, u0, steps=2)
    assert (x2, s2) == (x, s)  # from the cache


def test_kernel_tuner_picks_measured_kinds(oracle, tmp_path, monkeypatch):
    """tune_sweeps times every kernel kind per direction and then segment
    lengths; its choice builds a level whose steps match the oracle, and the
    second call comes from the cache."""
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.autotune import tune_sweeps
    monkeypatch.setenv("BAMREX_TUNE_CACHE", str(tmp_path))
    D, n = 3, 48
    hi = (n - 1,) * 3
    boxes = oracle.decompose(D, (0, 0, 0), hi, 24)
    u0 = problems.blast_3d(n, radius=0.25)
    parm = bx.Parm(D, limiter=bx.MINBEE)
    r = tune_sweeps(D, (0, 0, 0), hi, [0.0] * 3, [1.0] * 3, boxes, parm, u0, steps=2)
    assert {"auto", "tma", "wave", "march"} <= set(r["table"])
    assert all(k in (bx.STAGING_REGISTERS, bx.STAGING_TMA, bx.STAGING_WAVE) for k in r["staging_dir"][:D])
    lev = bx.Level(D, (0, 0, 0), hi, [0.0] * 3, [1.0] * 3, boxes, parm, cfl=0.8, staging_dir=r["staging_dir"],
                   x_mode=r["x_mode"], x_segment=r["x_segment"], s_segment=r["s_segment"])
    assert [lev.staging(d) for d in range(D)] == list(r["staging_dir"][:D])
    lay = oracle.LevelLayout(D, (0, 0, 0), hi, boxes, 2, [1.0 / n] * D)
    S1, S2 = lay.alloc(), lay.alloc()
    lay.scatter(S1, u0)
    lay.fill_boundary(S1)
    dt = lay.est_time_step(S1, 1.4, 1.0, 0.8)
    S2[:] = S1
    lay.advance_explicit(S1, S2, 0.0, dt, oracle.MUSCL_HANCOCK, oracle.Parm(D, limiter=oracle.MINBEE))
    lev.set_state(u0)
    lev.advance(0.0, dt)
    got, ref = lev.get_state(), lay.gather(S1)
    lev.close()
    for c in range(D + 2):
        assert np.max(np.abs(got[c] - ref[c])) <= 1e-12 * np.max(np.abs(ref[c]))
    assert tune_sweeps(D, (0, 0, 0), hi, [0.0] * 3, [1.0] * 3, boxes, parm, u0, steps=2) == r
