"""Device memory of destroyed levels: a freed level arena of 64 MiB or more
is kept whole and handed to the next level that fits it, and
bamrex_release_memory gives every kept page back to the driver.  Levels made
on kept, pooled or fresh memory step alike."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_levels_on_kept_and_released_memory_step_alike():
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200._abi import lib
    n = 2048  # two FP64 state buffers of ~135 MB each: a kept-size arena
    hi = (n - 1, n - 1, 0)
    u0 = problems.quadrant_2d(n)
    outs = []
    for k in range(4):
        if k == 3:
            assert lib().bamrex_release_memory() == 0
        lev = bx.Level(2, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], [((0, 0, 0), hi)], bx.Parm(2, limiter=0), cfl=0.8)
        lev.set_state(u0)
        lev.run(2)
        outs.append(lev.get_state())
        if k == 1:
            # a second level alive beside a kept block takes pool memory
            other = bx.Level(2, (0, 0, 0), hi, [0.0, 0.0], [1.0, 1.0], [((0, 0, 0), hi)], bx.Parm(2, limiter=0),
                             cfl=0.8)
            other.set_state(u0)
            other.run(2)
            outs.append(other.get_state())
            other.close()
        lev.close()
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
