"""bamrex_conserved_sums_noalloc (static device scratch, no allocation)
against the level's own conserved sums, called through the C ABI.  Kept in
a file collected last so it also runs after every other test in the same
process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(level, stream=None, edit=None):
    from bamrex_b200._abi import Array4, Box, lib
    nb = len(level.boxes)
    boxes = (Box * nb)(*[Box.make(lo, hi) for lo, hi in level.boxes])
    fabs = (Array4 * nb)(*[level.fab(b) for b in range(nb)])
    if edit:
        edit(fabs)
    dx = (ctypes.c_double * 3)(*(list(level.dx) + [1.0] * (3 - len(level.dx))))
    out = (ctypes.c_double * level.NC)()
    rc = lib().bamrex_conserved_sums_noalloc(level.D, boxes, fabs, nb, dx, out, stream)
    return rc, np.array(list(out))


# 1D, 2D and 3D; boxes of 16 cells (one thread per cell) and of 64 (several
# cells per thread in the strided accumulation); the default stream and the
# level's own stream
@pytest.mark.parametrize("D,n,mgs,own_stream", [(1, 4096, 64, False), (2, 256, 16, False), (2, 256, 64, True),
                                                (3, 48, 16, False), (3, 64, 64, True)])
def test_noalloc_sums_equal_level_sums(oracle, D, n, mgs, own_stream):
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
    lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D))
    lev.set_state(problems.random_states(D, tuple(reversed([n if d < D else 1 for d in range(3)])), seed=11))
    stream = lev.stream_handle() if own_stream else None
    a1 = lev.conserved_sums()
    rc1, b1 = _noalloc(lev, stream)
    a2 = lev.conserved_sums()
    rc2, b2 = _noalloc(lev, stream)
    assert rc1 == 0 and rc2 == 0
    np.testing.assert_array_equal(b1, a1)
    np.testing.assert_array_equal(b2, a2)
    np.testing.assert_array_equal(a1, a2)
    # a step changes the state: both paths follow it
    lev.advance(0.0, 1e-4)
    lev.sync()
    np.testing.assert_array_equal(_noalloc(lev, stream)[1], lev.conserved_sums())
    lev.close()


def test_noalloc_rejects_bad_fabs(oracle):
    """A fab that does not cover its box, or has too few components, is
    refused on the host before anything is launched."""
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200._abi import ERR_ARG, lib
    D, n = 2, 64
    hi = (n - 1, n - 1, 0)
    lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, oracle.decompose(D, (0, 0, 0), hi, 32), bx.Parm(D))
    lev.set_state(problems.random_states(D, (1, n, n), seed=3))

    def short(f):
        f[1].end[0] = f[1].begin[0] + 4

    def few(f):
        f[2].ncomp = D + 1

    rc, _ = _noalloc(lev, edit=short)
    assert rc == ERR_ARG and b"does not cover" in lib().bamrex_last_error()
    rc, _ = _noalloc(lev, edit=few)
    assert rc == ERR_ARG and b"too few components" in lib().bamrex_last_error()
    # the scratch is untouched by the refused calls: a good call still agrees
    rc, got = _noalloc(lev)
    assert rc == 0
    np.testing.assert_array_equal(got, lev.conserved_sums())
    lev.close()


def test_noalloc_rejects_too_many_boxes():
    from bamrex_b200._abi import ERR_ARG, Array4, Box, lib
    n = 4097
    boxes = (Box * n)(*[Box.make((i, 0, 0), (i, 0, 0)) for i in range(n)])
    fabs = (Array4 * n)()
    dx = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    out = (ctypes.c_double * 3)()
    rc = lib().bamrex_conserved_sums_noalloc(1, boxes, fabs, n, dx, out, None)
    assert rc == ERR_ARG
    assert b"4096" in lib().bamrex_last_error()
