"""The multi-rank level on CPU: two gloo ranks, each owning part of the
boxes, step with halo exchange between sweeps and a max-reduced time step;
the gathered result equals the single-process run bit for bit.  The compute
engine is the CPU oracle; the host logic (partition, halo plan, exchange,
dt) is the one the device path uses."""
import os
import socket

import numpy as np
import pytest


class OracleEngine:
    """CPU engine for DistLevel over the oracle's per-box layout."""

    def __init__(self, lay, parm, method, dx=None, cfl=0.8):
        import torch
        self.torch, self.device = torch, "cpu"
        self.lay, self.parm, self.method = lay, parm, method
        self.NC = lay.NC
        self.S = [lay.alloc(), lay.alloc()]
        self.cur = 0
        self.halo = {}
        self.dx, self.cfl = dx, cfl

    def set_halo(self, d, send, recv):
        self.halo[d] = (send, recv)

    def stream_context(self):
        import contextlib
        return contextlib.nullcontext()

    def buffer(self, cells):
        return self.torch.zeros(max(1, cells * self.NC), dtype=self.torch.float64)

    def _region(self, lb, lo, hi):
        bg = self.lay.begins[lb]
        f = self.lay.fab(self.S[self.cur], lb)
        return f, (slice(None), slice(lo[2] - bg[2], hi[2] - bg[2] + 1), slice(lo[1] - bg[1], hi[1] - bg[1] + 1),
                   slice(lo[0] - bg[0], hi[0] - bg[0] + 1))

    def pack(self, d, buf):
        b = buf.numpy()
        for (lb, lo, hi, off) in self.halo[d][0]["regions"]:
            f, sl = self._region(lb, lo, hi)
            v = f[sl].reshape(self.NC, -1)
            b[off * self.NC: off * self.NC + v.size] = v.ravel()

    def unpack(self, d, buf):
        b = buf.numpy()
        for (lb, lo, hi, off) in self.halo[d][1]["regions"]:
            f, sl = self._region(lb, lo, hi)
            shape = f[sl].shape
            f[sl] = b[off * self.NC: off * self.NC + int(np.prod(shape))].reshape(shape)

    def fill_dir(self, d):
        self.lay.fill_boundary(self.S[self.cur])

    def sweep_dir(self, d, dt, reduce_ws):
        self.lay.sweep_dir(self.S[self.cur], self.S[self.cur ^ 1], d, dt, self.method, self.parm)
        self.cur ^= 1

    def wave_speed(self):
        return self.lay.max_wave_speed(self.S[self.cur], self.parm.adiabatic, self.parm.epsilon)

    # the device-dt protocol (bamrex_level_dist_*), mirrored on the host:
    # step scalars, the dt kernel's arithmetic, sweeps skipped once done
    def ws_buffer(self):
        return self.torch.zeros(1, dtype=self.torch.float64)

    def begin(self, time, stop_time):
        self.time, self.stop, self.dt, self.steps, self.done = time, stop_time, 0.0, 0, False
        self.start = self.cur

    def wave_speed_into(self, ws):
        ws[0] = self.wave_speed()

    def device_dt(self, ws, first):
        if self.done:
            return
        if not first:
            self.time = self.time + self.dt
            self.steps += 1
        ms = float(ws[0])
        dt_est = 1.0e20
        for d in range(len(self.dx)):
            dt_est = min(dt_est, self.dx[d] / ms)
        dt_est *= self.cfl
        dt0 = dt_est
        if self.stop >= 0.0:
            eps = 0.001 * dt0
            if self.time + dt0 > self.stop - eps:
                dt0 = self.stop - self.time
            if not self.time < self.stop:
                self.done = True
        self.dt = dt0

    def fill_dir_device(self, d):
        if not self.done:
            self.fill_dir(d)

    def sweep_dir_device(self, d, reduce_ws):
        if self.done:
            self.cur ^= 1
            return
        self.sweep_dir(d, self.dt, reduce_ws)

    # the split sweep: part 0 (boxes without remote ghost cells in d) runs
    # before the received halo is unpacked, part 1 after; each part takes
    # its boxes' cells from a full sweep of the input as it is at that time
    def set_split(self, d, edge):
        if not hasattr(self, "edge"):
            self.edge = {}
        self.edge[d] = set(edge)

    def sweep_dir_device_part(self, d, reduce_ws, part):
        if not self.done:
            tmp = self.lay.alloc()
            self.lay.sweep_dir(self.S[self.cur], tmp, d, self.dt, self.method, self.parm)
            out = self.S[self.cur ^ 1]
            for lb, (lo, hi) in enumerate(self.lay.boxes):
                if (lb in self.edge[d]) != (part == 1):
                    continue
                bg = self.lay.begins[lb]
                sl = (slice(None), slice(lo[2] - bg[2], hi[2] - bg[2] + 1), slice(lo[1] - bg[1], hi[1] - bg[1] + 1),
                      slice(lo[0] - bg[0], hi[0] - bg[0] + 1))
                self.lay.fab(out, lb)[sl] = self.lay.fab(tmp, lb)[sl]
        if part == 1:
            self.cur ^= 1

    def end(self):
        if self.done:
            self.cur = self.start ^ ((self.steps * len(self.dx)) & 1)
        return self.time, self.dt, self.steps


def _case(name):
    from bamrex_b200 import problems
    if name == "quadrant2d":
        n = 64
        return 2, n, 16, problems.quadrant_2d(n), (0, 0, 0), 0
    if name == "periodic2d":
        n = 48
        return 2, n, 16, problems.random_states(2, (1, n, n), seed=4), (1, 1, 1), 1
    n = 16
    return 3, n, 8, problems.blast_3d(n, radius=0.3), (2, 2, 2), 1


def _worker(rank, world, port, name, nsteps, out, device_dt=False, stop_time=-1.0, overlap=False):
    import torch.distributed as dist
    from bamrex_b200.distributed import DistLevel, partition
    from oracle import oracle as O
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        D, n, mgs, u0, bc, lim = _case(name)
        hi = tuple(n - 1 if d < D else 0 for d in range(3))
        boxes = O.decompose(D, (0, 0, 0), hi, mgs)
        owners = partition(boxes, world)
        local = [b for b in range(len(boxes)) if owners[b] == rank]
        dx = [1.0 / n] * D
        lay = O.LevelLayout(D, (0, 0, 0), hi, [boxes[b] for b in local], 2, dx, bc_lo=bc, bc_hi=bc)
        eng = OracleEngine(lay, O.Parm(D, limiter=lim), O.MUSCL_HANCOCK, dx, 0.8)
        lay.scatter(eng.S[0], u0)
        if not overlap:
            # the engine's split sweep stays unused: the plain schedule
            del OracleEngine.set_split
        dl = DistLevel(eng, D, (0, 0, 0), hi, boxes, owners, 2, bc, bc, dx, 0.8, rank, world, dist, overlap=overlap)
        assert dl.overlap == overlap
        if device_dt:
            t_end, _, taken = dl.run_device(nsteps, 0.0, stop_time)
            dts = (t_end, taken)
        else:
            dts = dl.run(nsteps)
        glob = lay.gather(eng.S[eng.cur])
        # rank 0 collects every rank's boxes and compares with one process
        parts = [None] * world
        dist.all_gather_object(parts, (glob, dts))
        if rank == 0:
            full = np.full_like(parts[0][0], np.nan)
            for g, _ in parts:
                m = ~np.isnan(g)
                full[m] = g[m]
            ref_lay = O.LevelLayout(D, (0, 0, 0), hi, boxes, 2, dx, bc_lo=bc, bc_hi=bc)
            if device_dt:
                ref, t, rdts = O.run_level(ref_lay, u0, O.Parm(D, limiter=lim), O.MUSCL_HANCOCK, 0.8, nsteps=nsteps,
                                           stop_time=stop_time if stop_time >= 0 else None)
                same_dt = float(dts == (t, len(rdts)))
            else:
                ref, t, rdts = O.run_level(ref_lay, u0, O.Parm(D, limiter=lim), O.MUSCL_HANCOCK, 0.8, nsteps=nsteps)
                same_dt = float(rdts == dts)
            np.save(out, np.array([float(np.array_equal(full, ref)), same_dt, float(np.sum(owners)),
                                   float(np.abs(full - ref).max())]))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("name", ["quadrant2d", "periodic2d", "blast3d"])
def test_two_ranks_equal_one(tmp_path, name):
    import torch.multiprocessing as mp
    out = str(tmp_path / "r.npy")
    mp.spawn(_worker, args=(2, _free_port(), name, 4, out), nprocs=2, join=True)
    same, same_dt, owned, diff = np.load(out)
    assert owned > 0, "both ranks own boxes"
    assert same_dt == 1.0
    assert same == 1.0, diff


@pytest.mark.parametrize("name,stop_time", [("quadrant2d", -1.0), ("periodic2d", -1.0), ("blast3d", -1.0),
                                            ("quadrant2d", 0.015)])
def test_two_ranks_device_dt_equal_one(tmp_path, name, stop_time):
    """The run with dt kept on the device (the wave speed all-reduced in a
    buffer, dt computed from it where the sweeps read it; no host wait
    inside the run): same state, time and step count as one process, also
    when the stop time ends the run early."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "r.npy")
    mp.spawn(_worker, args=(2, _free_port(), name, 6, out, True, stop_time), nprocs=2, join=True)
    same, same_dt, owned, diff = np.load(out)
    assert owned > 0, "both ranks own boxes"
    assert same_dt == 1.0
    assert same == 1.0, diff


def test_partition_and_plan_symmetry():
    """Every region a rank receives from a peer is one the peer sends, in the
    same order and size."""
    from bamrex_b200.distributed import HaloPlan, partition
    from oracle import oracle as O
    D, n = 2, 64
    boxes = O.decompose(D, (0, 0, 0), (n - 1, n - 1, 0), 16)
    for world in (2, 3, 4):
        owners = partition(boxes, world)
        assert sorted(set(owners)) == list(range(world))
        plans = [HaloPlan(D, (0, 0, 0), (n - 1, n - 1, 0), boxes, owners, 2, (1, 1, 1), (1, 1, 1), r)
                 for r in range(world)]
        for d in range(D):
            for r in range(world):
                send = plans[r].dirs[d][0]
                for peer, start, cnt in send["peers"]:
                    recv = plans[peer].dirs[d][1]
                    match = [p for p in recv["peers"] if p[0] == r]
                    assert match and match[0][2] == cnt


@pytest.mark.parametrize("name,stop_time", [("quadrant2d", -1.0), ("periodic2d", -1.0), ("blast3d", -1.0),
                                            ("quadrant2d", 0.015)])
def test_two_ranks_overlapped_equal_one(tmp_path, name, stop_time):
    """The overlapped schedule (each direction: pack and post the halo,
    fill and sweep the boxes without remote ghost cells while it is in
    flight, then unpack and sweep the rest): the same state, time and step
    count as one process, bit for bit."""
    import torch.multiprocessing as mp
    out = str(tmp_path / "r.npy")
    mp.spawn(_worker, args=(2, _free_port(), name, 6, out, True, stop_time, True), nprocs=2, join=True)
    same, same_dt, owned, diff = np.load(out)
    assert owned > 0, "both ranks own boxes"
    assert same_dt == 1.0
    assert same == 1.0, diff
