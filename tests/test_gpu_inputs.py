"""The reference's run from an inputs file (python -m bamrex_b200.inputs)
on the device: its plotfiles hold exactly the state of the same hierarchy
stepped through bamrex_b200.amr.Amr directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

INPUTS = """
max_step  = 4
stop_time = 0.3
prob.adiabatic = 1.4
geometry.is_periodic = 0 0
geometry.prob_lo = 0 0
geometry.prob_hi = 1 1
amr.n_cell = 64 64
adv.cfl = 0.8
adv.num_method = muscl_hancock
limiting.limiter = minbee
amr.max_level = 1
amr.ref_ratio = 2
amr.regrid_int = 2
amr.blocking_factor = 8
amr.max_grid_size = 32
amr.plot_int = 2
tagging.max_phigrad_lev = 1
tagging.phigrad = 0.1
init.density_TR = 1.5
init.velocity_x_TR = 0
init.velocity_y_TR = 0
init.pressure_TR = 1.5
init.density_TL = 0.5323
init.velocity_x_TL = 1.206
init.velocity_y_TL = 0
init.pressure_TL = 0.3
init.density_BL = 0.138
init.velocity_x_BL = 1.206
init.velocity_y_BL = 1.206
init.pressure_BL = 0.029
init.density_BR = 0.5323
init.velocity_x_BR = 0
init.velocity_y_BR = 1.206
init.pressure_BR = 0.3
"""


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def test_inputs_run_matches_direct_hierarchy(torch_cuda, tmp_path):
    from bamrex_b200 import inputs as I
    from bamrex_b200 import plotfile as P
    f = tmp_path / "inputs"
    f.write_text(INPUTS)
    prefix = str(tmp_path / "out" / "plt")
    I.main(["--problem", "QuadrantProblem", "--dim", "2", str(f), "amr.plot_file=" + prefix])
    names = sorted(p.name for p in (tmp_path / "out").iterdir())
    assert names == ["plt00000", "plt00002", "plt00004"]

    pp = I.ParmParse.from_text(INPUTS)
    s = I.read_settings(pp, 2)
    amr = I.make_amr(s, I.INITIAL_DATA["QuadrantProblem"](pp, s))
    for _ in range(4):
        amr.coarse_step(s.stop_time)
    got = P.read_plotfile(prefix + "00004")
    assert got["time"] == amr.time and got["varnames"] == ["density", "mom_x", "mom_y", "energy"]
    assert len(got["levels"]) == amr.finest_level + 1 == 2
    for lev, (_, _, boxes, fabs) in enumerate(got["levels"]):
        assert boxes == amr.boxes(lev)
        glob = amr.get_state(lev)
        dlo, _ = amr.domain(lev)
        for (lo, hi), fab in zip(boxes, fabs):
            sl = tuple(slice(lo[d] - dlo[d], hi[d] - dlo[d] + 1) if d < 2 else slice(0, 1) for d in (2, 1, 0))
            np.testing.assert_array_equal(fab, glob[(slice(None),) + sl])
    amr.close()
