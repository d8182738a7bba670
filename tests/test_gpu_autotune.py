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
