"""Checkpoint and restart of a device hierarchy (amr.checkPoint() /
AmrLevelAdv::checkPoint / restart, Source/main.cpp:96-99,
Source/AmrLevelAdv.cpp:95-113): a run restarted from a checkpoint continues
the uninterrupted run bit for bit, across regrids, directly and through the
inputs-file runner (amr.check_int / amr.restart)."""
import numpy as np
import pytest

from test_gpu_inputs import INPUTS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _states(amr):
    return [(amr.boxes(lev), amr.get_state(lev)) for lev in range(amr.finest_level + 1)]


def _assert_same(a, b):
    assert len(a) == len(b)
    for (ba, sa), (bb, sb) in zip(a, b):
        assert ba == bb
        np.testing.assert_array_equal(sa, sb)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32_storage"])
def test_restart_continues_bit_for_bit(torch_cuda, tmp_path, precision):
    from bamrex_b200 import inputs as I
    from bamrex_b200.checkpoint import read_checkpoint, write_checkpoint
    pp = I.ParmParse.from_text(INPUTS)
    s = I.read_settings(pp, 2)
    s.max_level = 2
    s.phigrad = [0.1, 0.1]
    amr = I.make_amr(s, I.INITIAL_DATA["QuadrantProblem"](pp, s), precision=precision)
    for _ in range(3):  # the regrid of step 2 has happened
        amr.coarse_step(s.stop_time)
    path = str(tmp_path / "chk00003")
    write_checkpoint(path, amr)
    ck = read_checkpoint(path)
    assert ck["coarse_steps"] == amr.coarse_steps == 3 and ck["time"] == amr.time
    for _ in range(4):  # regrids at steps 4 and 6
        amr.coarse_step(s.stop_time)
    ref, t_ref = _states(amr), amr.time
    assert amr.finest_level == 2
    amr.close()

    s.restart = path
    amr2 = I.restart_amr(s, precision=precision)
    assert amr2.coarse_steps == 3 and amr2.time == ck["time"]
    for _ in range(4):
        amr2.coarse_step(s.stop_time)
    assert amr2.time == t_ref
    _assert_same(_states(amr2), ref)
    amr2.close()


def test_inputs_run_restarts_from_its_checkpoint(torch_cuda, tmp_path):
    """max_step 4 with amr.check_int 2 writes chk00002 and chk00004; a run
    restarted from chk00002 writes the same final plotfile and checkpoint."""
    from bamrex_b200 import inputs as I
    from bamrex_b200 import plotfile as P
    from bamrex_b200.checkpoint import read_checkpoint
    f = tmp_path / "inputs"
    f.write_text(INPUTS)
    a = str(tmp_path / "a")
    I.main(["--problem", "QuadrantProblem", "--dim", "2", str(f), "amr.plot_file=%s/plt" % a, "amr.check_int=2",
            "amr.check_file=%s/chk" % a])
    names = sorted(p.name for p in (tmp_path / "a").iterdir())
    assert names == ["chk00002", "chk00004", "plt00000", "plt00002", "plt00004"]
    b = str(tmp_path / "b")
    I.main(["--problem", "QuadrantProblem", "--dim", "2", str(f), "amr.plot_file=%s/plt" % b, "amr.check_int=2",
            "amr.check_file=%s/chk" % b, "amr.restart=%s/chk00002" % a])
    # the restarted run continues at step 2: no initial plotfile
    assert sorted(p.name for p in (tmp_path / "b").iterdir()) == ["chk00004", "plt00004"]
    pa, pb = P.read_plotfile(a + "/plt00004"), P.read_plotfile(b + "/plt00004")
    assert pa["time"] == pb["time"]
    for (_, _, ba, fa), (_, _, bb, fb) in zip(pa["levels"], pb["levels"]):
        assert ba == bb
        for x, y in zip(fa, fb):
            np.testing.assert_array_equal(x, y)
    ca, cb = read_checkpoint(a + "/chk00004"), read_checkpoint(b + "/chk00004")
    assert ca["dt_level"] == cb["dt_level"] and ca["coarse_steps"] == cb["coarse_steps"] == 4
