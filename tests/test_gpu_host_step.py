"""bamrex_level_step_host: one step of a host-resident state, streamed in
slabs (uploads, sweeps, downloads overlapped), equals copy_in + advance +
est_time_step + copy_out bit for bit; levels it cannot stream take the
plain sequence and give the same result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _level(D, n, mgs, bc, method=0, precision=0, x_mode=0, staging=0):
    import bamrex_b200 as bx
    from bamrex_b200.level import decompose
    hi = tuple(x - 1 for x in n)
    boxes = decompose(D, (0,) * D, hi, mgs)
    return bx.Level(D, (0,) * D, hi, [0.0] * D, [1.0] * D, boxes, bx.Parm(D), method=method, cfl=0.8,
                    bc_lo=(bc,) * D, bc_hi=(bc,) * D, precision=precision, x_mode=x_mode, staging=staging)


def _state(D, n, seed):
    from bamrex_b200 import problems
    if D == 2 and n[0] == n[1]:
        return problems.quadrant_2d(n[0])
    return problems.random_states(D, tuple(n[d] if d < D else 1 for d in (2, 1, 0)), seed=seed)


CASES = [
    # D, n, max_grid_size, bc, method, precision, x_mode, slabs
    (2, (96, 96), 96, 0, 0, 0, 0, 4),
    (2, (96, 96), 96, 0, 0, 0, 0, 7),
    (2, (130, 70), 130, 2, 0, 0, 2, 5),
    (2, (96, 96), 96, 0, 1, 0, 0, 3),
    (2, (96, 96), 96, 0, 0, 1, 0, 6),
    (3, (24, 20, 28), 28, 0, 0, 0, 0, 5),
    (3, (24, 20, 28), 28, 2, 0, 1, 0, 4),
    # not streamable: several boxes; periodic in the last direction
    (2, (64, 64), 32, 0, 0, 0, 0, 4),
    (2, (64, 64), 64, 1, 0, 0, 0, 4),
]


# the slabs swept by every kernel kind (registers, TMA march, wavefront): a
# slab takes the whole box's tensor maps and lane-group shape
STAGED = [(2, (96, 96), 96, 0, 0, 0, 0, 4, k) for k in (1, 2, 3)] + \
    [(3, (24, 20, 28), 28, 0, 0, 0, 0, 5, k) for k in (1, 2, 3)] + [(3, (24, 20, 28), 28, 2, 0, 1, 0, 4, 3)]


@pytest.mark.parametrize("case", CASES + STAGED, ids=[str(c) for c in CASES + STAGED])
def test_step_host_equals_plain_step(torch_cuda, case):
    torch = torch_cuda
    D, n, mgs, bc, method, prec, xm, slabs = case[:8]
    st = case[8] if len(case) > 8 else 0
    u0 = _state(D, n, seed=3)
    ref_lev = _level(D, n, mgs, bc, method, prec, xm, st)
    ref_lev.set_state(u0)
    dt = ref_lev.estTimeStep()
    ref_lev.advance(0.0, dt)
    ref = ref_lev.get_state()
    ref_next = ref_lev.estTimeStep()
    ref_lev.close()

    lev = _level(D, n, mgs, bc, method, prec, xm, st)
    packed = lev.packing.pack(u0)
    h = torch.tensor(packed).pin_memory()
    out = torch.empty_like(h).pin_memory()
    for k in range(2):  # twice: the second reuses the streams and events
        nxt = lev.step_host_ptr(h.data_ptr(), out.data_ptr(), dt, slabs)
        got = lev.packing.unpack(out.numpy())
        np.testing.assert_array_equal(got, ref)
        assert nxt == ref_next
    # in place (the same host buffer in and out)
    lev.step_host_ptr(h.data_ptr(), h.data_ptr(), dt, slabs)
    np.testing.assert_array_equal(lev.packing.unpack(h.numpy()), ref)
    # the device state is the step's result
    np.testing.assert_array_equal(lev.get_state(), ref)
    lev.close()


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[4], CASES[5], CASES[7]], ids=lambda c: str(c))
def test_run_host_equals_device_run(torch_cuda, case):
    """bamrex_level_run_host (host round trip every step, copies of
    consecutive steps overlapped, dt on the device) equals the
    device-stepped run of the same steps bit for bit, time included."""
    torch = torch_cuda
    D, n, mgs, bc, method, prec, xm, slabs = case
    u0 = _state(D, n, seed=5)
    ref_lev = _level(D, n, mgs, bc, method, prec, xm)
    ref_lev.set_state(u0)
    t_ref, steps = ref_lev.run(4, use_graph=False)
    assert steps == 4
    ref = ref_lev.get_state()
    ref_next = ref_lev.estTimeStep()
    ref_lev.close()

    lev = _level(D, n, mgs, bc, method, prec, xm)
    lev.set_state(u0)
    dt0 = lev.estTimeStep()
    h = torch.tensor(lev.packing.pack(u0)).pin_memory()
    t, nxt = lev.run_host_ptr(h.data_ptr(), 4, dt0, 0.0, slabs)
    np.testing.assert_array_equal(lev.packing.unpack(h.numpy()), ref)
    assert t == t_ref
    assert nxt == ref_next
    lev.close()
