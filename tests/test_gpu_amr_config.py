"""The 3D spherical-blast hierarchy as the bench builds it (3 levels, ratio
2, blocking factor 8, boxes cut to a max_grid_size drawn per box from
{16, 32, 48, 64}, grad_error on rho >= 0.1, subcycling), one coarse step
from identical inputs against the restatement (oracle/amr_oracle.py) on the
same grids: every level within 1e-12 * 2^level relative L-infinity (level l
takes 2^l substeps) and the composite totals within 1e-12.

The base is 128^3 (the restatement's fill-patch and register arithmetic run
in numpy, about half a minute per coarse step at this size); the device code
path is the one of the 256^3 configuration."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel_linf(a, b):
    m = ~np.isnan(b)
    return float(np.max(np.abs(a[m] - b[m])) / max(np.max(np.abs(b[m])), 1e-300))


def test_blast_hierarchy_coarse_step_matches_oracle(oracle):
    import torch
    assert torch.cuda.is_available()
    from bamrex_b200.amr import blast_hierarchy
    from oracle.amr_oracle import OAmr
    n0 = 128
    hi = (n0 - 1,) * 3
    A, _ = blast_hierarchy(n0)
    levels = [A.boxes(lev) for lev in range(A.finest_level + 1)]
    assert len(levels) == 3 and all(len(b) > 0 for b in levels)
    kinds = [[A.level(lev).staging(d) for d in range(3)] for lev in range(3)]
    OA = OAmr(3, (0, 0, 0), hi, [0.0] * 3, [1.0] * 3, levels, oracle.Parm(3, limiter=oracle.MINBEE),
              oracle.MUSCL_HANCOCK, 0.8)
    for lev in range(3):
        OA.levels[lev].set_dense(A.get_state(lev))
    dt = A.coarse_step()
    odt = OA.coarse_step()
    assert abs(dt - odt) <= 1e-12 * odt
    for lev in range(3):
        e = _rel_linf(A.get_state(lev), OA.levels[lev].dense())
        print("level %d: %d boxes, kernels %s, rel L-inf %.2e" % (lev, len(levels[lev]), kinds[lev], e))
        assert e <= 1e-12 * 2 ** lev, (lev, e)
    tot, otot = A.conserved_sums(), OA.conserved_sums()
    np.testing.assert_allclose(tot, otot, rtol=1e-12, atol=1e-14 * np.abs(otot).max())
    A.close()
