"""The device side of the multi-rank level on one GPU: two Levels hold the
two halves of the boxes (as two ranks would), their halo buffers are packed
and unpacked by the library and handed across in this process (no
collective), and after the split steps the union equals one Level over all
boxes bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("D,n,mgs,bc", [(2, 128, 32, 0), (2, 96, 32, 1), (3, 32, 16, 2)])
def test_two_levels_with_device_halos_equal_one(oracle, D, n, mgs, bc):
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.distributed import DeviceEngine, HaloPlan, partition
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
    owners = partition(boxes, 2)
    u0 = problems.random_states(D, tuple(reversed([n if d < D else 1 for d in range(3)])), seed=8) if D == 2 \
        else problems.blast_3d(n, radius=0.3)
    kw = dict(cfl=0.8, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
    parm = bx.Parm(D, limiter=bx.VAN_LEER)
    ranks = []
    for r in range(2):
        mine = [boxes[b] for b in range(len(boxes)) if owners[b] == r]
        lev = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, mine, parm, **kw)
        full = np.zeros_like(u0)
        lev.set_state(u0)
        eng = DeviceEngine(lev)
        plan = HaloPlan(D, (0, 0, 0), hi, boxes, owners, 2, (bc,) * 3, (bc,) * 3, r)
        bufs = []
        for d in range(D):
            send, recv = plan.dirs[d]
            eng.set_halo(d, send, recv)
            bufs.append((eng.buffer(send["cells"]), eng.buffer(recv["cells"])))
        ranks.append((lev, eng, plan, bufs))
        del full
    ref = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, parm, **kw)
    ref.set_state(u0)
    NC = D + 2
    for step in range(3):
        ws = max(e.wave_speed() for _, e, _, _ in ranks)
        dt = 0.8 * min(1.0 / n / ws for _ in range(D))
        for d in range(D):
            for lev, e, plan, bufs in ranks:
                e.pack(d, bufs[d][0])
            for r, (lev, e, plan, bufs) in enumerate(ranks):
                peer = ranks[1 - r]
                recv = plan.dirs[d][1]
                psend = peer[2].dirs[d][0]
                # the receiving level's stream waits for the sender's pack
                e.stream.wait_stream(peer[1].stream)
                with e.stream_context():
                    for p, start, cnt in recv["peers"]:
                        ps = [q for q in psend["peers"] if q[0] == r][0]
                        bufs[d][1][start * NC:(start + cnt) * NC] = peer[3][d][0][ps[1] * NC:(ps[1] + cnt) * NC]
            for r, (lev, e, plan, bufs) in enumerate(ranks):
                # a rank packs its next buffer only after the peer copied this one
                e.stream.wait_stream(ranks[1 - r][1].stream)
            for lev, e, plan, bufs in ranks:
                e.unpack(d, bufs[d][1])
                e.fill_dir(d)
                e.sweep_dir(d, dt, d == D - 1)
        ref.advance(0.0, dt)
    torch.cuda.synchronize()
    got = np.full_like(u0, np.nan)
    for lev, e, plan, bufs in ranks:
        part = np.full_like(u0, np.nan)
        packed = np.empty(lev.packing.size)
        lev.copy_out_ptr(packed.ctypes.data)
        lev.sync()
        lev.packing.unpack(packed, part)
        m = ~np.isnan(part)
        got[m] = part[m]
    want = ref.get_state()
    assert not np.isnan(got).any()
    np.testing.assert_array_equal(got, want)
    for lev, *_ in ranks:
        lev.close()
    ref.close()


@pytest.mark.parametrize("D,n,mgs,stop", [(2, 128, 32, -1.0), (3, 32, 16, -1.0), (2, 128, 64, 0.01)])
def test_device_dt_split_run_equals_level_run(oracle, D, n, mgs, stop):
    """The split step with dt on the device (bamrex_level_dist_*: the wave
    speed copied to a buffer, dt computed from it on the level's stream, the
    sweeps reading it) equals the level's own device-stepped run bit for
    bit, time and step count included, also when the stop time ends it."""
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.distributed import DeviceEngine, DistLevel
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
    u0 = problems.quadrant_2d(n) if D == 2 else problems.blast_3d(n, radius=0.3)
    parm = bx.Parm(D, limiter=bx.MINBEE)
    a = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, parm, cfl=0.8)
    b = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, parm, cfl=0.8)
    try:
        a.set_state(u0)
        b.set_state(u0)
        dl = DistLevel(DeviceEngine(a), D, (0, 0, 0), hi, boxes, [0] * len(boxes), 2, (0, 0, 0), (0, 0, 0),
                       [1.0 / n] * D, 0.8, 0, 1, None)
        t_a, _, steps_a = dl.run_device(7, 0.0, stop)
        t_b, steps_b = b.run(7, stop_time=stop, use_graph=False)
        assert steps_a == steps_b and t_a == t_b
        if stop > 0:
            assert steps_a < 7 and t_a == stop
        np.testing.assert_array_equal(a.get_state(), b.get_state())
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("D,n,mgs,staging", [(2, 128, 32, 0), (2, 128, 32, 2), (2, 128, 32, 3), (3, 32, 16, 3)])
def test_split_sweep_parts_equal_level_run(oracle, D, n, mgs, staging):
    """The overlapped schedule's sweeps on one GPU: each direction swept in
    two launches over complementary box sets (bamrex_level_set_sweep_split /
    sweep_dir_device_part; every other box in part 1) with the register,
    TMA-march and wavefront kernels equals the level's own device-stepped
    run bit for bit."""
    import torch
    assert torch.cuda.is_available()
    import bamrex_b200 as bx
    from bamrex_b200 import problems
    from bamrex_b200.distributed import DeviceEngine
    hi = tuple(n - 1 if d < D else 0 for d in range(3))
    boxes = oracle.decompose(D, (0, 0, 0), hi, mgs)
    u0 = problems.quadrant_2d(n) if D == 2 else problems.blast_3d(n, radius=0.3)
    parm = bx.Parm(D, limiter=bx.MINBEE)
    a = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, parm, cfl=0.8, staging=staging)
    b = bx.Level(D, (0, 0, 0), hi, [0.0] * D, [1.0] * D, boxes, parm, cfl=0.8, staging=staging)
    try:
        a.set_state(u0)
        b.set_state(u0)
        e = DeviceEngine(a)
        for d in range(D):
            e.set_split(d, list(range(d % 2, len(boxes), 2)))
        ws = e.ws_buffer()
        e.begin(0.0, -1.0)
        e.wave_speed_into(ws)
        e.device_dt(ws, True)
        for _ in range(5):
            for d in range(D):
                e.fill_dir_device(d)
                e.sweep_dir_device_part(d, d == D - 1, 0)
                e.sweep_dir_device_part(d, d == D - 1, 1)
            e.wave_speed_into(ws)
            e.device_dt(ws, False)
        t_a, _, steps_a = e.end()
        t_b, steps_b = b.run(5, use_graph=False)
        assert steps_a == steps_b == 5 and t_a == t_b
        np.testing.assert_array_equal(a.get_state(), b.get_state())
    finally:
        a.close()
        b.close()
