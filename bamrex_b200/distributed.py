"""A level over several processes, one GPU per rank: box partition, halo
exchange plan, and the split step with the ghost slabs of other ranks'
boxes exchanged between sweeps (the FillBoundary of fill_consv_boundary
after every sweep, Source/AmrLevelAdv_advance.cpp:356) and the time step
from the max wave speed over all ranks (the ParReduce of max_wave_speed,
Source/System/Euler/Euler.cpp:46-74, computeNewDt, Source/AmrLevelAdv.cpp:
537-619).

The host logic here is independent of the compute engine: ``DeviceEngine``
drives a device ``Level`` over NCCL; tests drive the same logic with a CPU
engine over gloo.
"""
from __future__ import annotations

import numpy as np

from . import _abi


# ------------------------------------------------------------------ partition
def _morton(x, y, z):
    code = 0
    for bit in range(21):
        code |= ((x >> bit) & 1) << (3 * bit) | ((y >> bit) & 1) << (3 * bit + 1) | ((z >> bit) & 1) << (3 * bit + 2)
    return code


def partition(boxes, nranks):
    """Owner rank of every box: boxes in Morton order of their lower corner,
    cut into nranks contiguous runs of about equal cell counts (the idea of
    AMReX's space-filling-curve DistributionMapping)."""
    if not boxes:
        return []
    unit = min(max(1, min(hi[d] - lo[d] + 1 for d in range(3))) for lo, hi in boxes)
    order = sorted(range(len(boxes)), key=lambda b: _morton(*[(boxes[b][0][d] // unit) & 0x1FFFFF for d in range(3)]))
    cells = [int(np.prod([hi[d] - lo[d] + 1 for d in range(3)])) for lo, hi in boxes]
    total = sum(cells)
    owners = [0] * len(boxes)
    acc = 0
    for b in order:
        owners[b] = min(nranks - 1, acc * nranks // total) if total else 0
        acc += cells[b]
    return owners


# ------------------------------------------------------------------ halo plan
def _intersect(a_lo, a_hi, b_lo, b_hi):
    lo = [max(a_lo[d], b_lo[d]) for d in range(3)]
    hi = [min(a_hi[d], b_hi[d]) for d in range(3)]
    return (lo, hi) if all(lo[d] <= hi[d] for d in range(3)) else None


def halo_ops(D, dom_lo, dom_hi, boxes, ngrow, bc_lo, bc_hi, d):
    """Every ghost region of direction d whose source is another box, for
    all boxes, in a canonical order: (dst box, side, src box, dst lo, dst hi,
    shift).  Physical (non-periodic) boundaries are not listed: each box
    fills those from its own cells."""
    ops = []
    g = ngrow
    dlo, dhi = dom_lo[d], dom_hi[d]
    length = dhi - dlo + 1
    for b, (lo, hi) in enumerate(boxes):
        if lo[d] != dlo and lo[d] < dlo + g:
            raise ValueError("box %d starts within the ghost width of a domain face" % b)
        if hi[d] != dhi and hi[d] > dhi - g:
            raise ValueError("box %d ends within the ghost width of a domain face" % b)
        for side in (0, 1):
            slo, shi = list(lo), list(hi)
            if side == 0:
                slo[d], shi[d] = lo[d] - g, lo[d] - 1
            else:
                slo[d], shi[d] = hi[d] + 1, hi[d] + g
            parts = []
            ilo, ihi = list(slo), list(shi)
            ilo[d], ihi[d] = max(slo[d], dlo), min(shi[d], dhi)
            if ilo[d] <= ihi[d]:
                parts.append((ilo, ihi, 0))
            bc = bc_lo[d] if side == 0 else bc_hi[d]
            if bc == _abi.BC_PERIODIC:
                olo, ohi = list(slo), list(shi)
                if side == 0:
                    ohi[d] = min(shi[d], dlo - 1)
                else:
                    olo[d] = max(slo[d], dhi + 1)
                if olo[d] <= ohi[d]:
                    parts.append((olo, ohi, length if side == 0 else -length))
            for plo, phi, sh in parts:
                qlo, qhi = list(plo), list(phi)
                qlo[d] += sh
                qhi[d] += sh
                for s, (blo, bhi) in enumerate(boxes):
                    if s == b and sh == 0:
                        continue
                    x = _intersect(qlo, qhi, blo, bhi)
                    if x is None:
                        continue
                    xlo, xhi = x
                    dst_lo, dst_hi = list(xlo), list(xhi)
                    dst_lo[d] -= sh
                    dst_hi[d] -= sh
                    ops.append((b, side, s, tuple(dst_lo), tuple(dst_hi), sh))
    return ops


class HaloPlan:
    """Per direction: this rank's send and receive regions, grouped by peer
    rank (ascending), each group in the canonical order of halo_ops, so the
    two sides of every pair agree on the buffer layout."""

    def __init__(self, D, dom_lo, dom_hi, boxes, owners, ngrow, bc_lo, bc_hi, rank):
        self.rank = rank
        self.local = [b for b in range(len(boxes)) if owners[b] == rank]
        self.local_index = {b: i for i, b in enumerate(self.local)}
        self.dirs = []
        for d in range(D):
            ops = halo_ops(D, dom_lo, dom_hi, boxes, ngrow, bc_lo, bc_hi, d)
            send, recv = {}, {}
            for (b, side, s, dlo, dhi, sh) in ops:
                if owners[b] == owners[s]:
                    continue  # a local copy: the level's own ghost fill
                if owners[s] == rank:
                    slo, shi = list(dlo), list(dhi)
                    slo[d] += sh
                    shi[d] += sh
                    send.setdefault(owners[b], []).append((self.local_index[s], tuple(slo), tuple(shi)))
                if owners[b] == rank:
                    recv.setdefault(owners[s], []).append((self.local_index[b], dlo, dhi))
            self.dirs.append((self._layout(send), self._layout(recv)))

    @staticmethod
    def _layout(groups):
        regions, peers, off = [], [], 0
        for peer in sorted(groups):
            start = off
            for (lb, lo, hi) in groups[peer]:
                n = int(np.prod([hi[q] - lo[q] + 1 for q in range(3)]))
                regions.append((lb, lo, hi, off))
                off += n
            peers.append((peer, start, off - start))
        return dict(regions=regions, peers=peers, cells=off)


# ------------------------------------------------------------------ engines
class DeviceEngine:
    """The device Level of this rank's boxes; buffers are CUDA tensors."""

    def __init__(self, level):
        import torch
        self.torch = torch
        self.device = "cuda"
        self.level = level
        self.NC = level.NC
        # the level's stream, so buffer traffic and NCCL order with its kernels
        self.stream = torch.cuda.ExternalStream(level.stream_handle())

    def stream_context(self):
        return self.torch.cuda.stream(self.stream)

    def set_halo(self, d, send, recv):
        from ._abi import Region, check, lib

        def regions(lst):
            arr = (Region * max(1, len(lst)))()
            for i, (lb, lo, hi, off) in enumerate(lst):
                arr[i].box = lb
                for q in range(3):
                    arr[i].lo[q] = lo[q]
                    arr[i].hi[q] = hi[q]
                arr[i].offset = off
            return arr

        sr, rr = regions(send["regions"]), regions(recv["regions"])
        check(lib().bamrex_level_set_halo(self.level._h, d, sr, len(send["regions"]), rr, len(recv["regions"])),
              self.level._h)

    def buffer(self, cells):
        with self.stream_context():
            return self.torch.zeros(max(1, cells * self.NC), dtype=self.torch.float64, device="cuda")

    def pack(self, d, buf):
        import ctypes
        from ._abi import check, lib
        check(lib().bamrex_level_halo_pack(self.level._h, d, ctypes.c_void_p(buf.data_ptr())), self.level._h)

    def unpack(self, d, buf):
        import ctypes
        from ._abi import check, lib
        check(lib().bamrex_level_halo_unpack(self.level._h, d, ctypes.c_void_p(buf.data_ptr())), self.level._h)

    def fill_dir(self, d):
        from ._abi import check, lib
        check(lib().bamrex_level_fill_dir(self.level._h, d), self.level._h)

    def sweep_dir(self, d, dt, reduce_ws):
        from ._abi import check, lib
        check(lib().bamrex_level_sweep_dir(self.level._h, d, dt, 1 if reduce_ws else 0), self.level._h)

    def wave_speed(self):
        import ctypes
        from ._abi import check, lib
        out = ctypes.c_double()
        check(lib().bamrex_level_wave_speed(self.level._h, ctypes.byref(out)), self.level._h)
        return out.value

    # the step with dt on the device (bamrex_level_dist_*): nothing here waits
    def ws_buffer(self):
        with self.stream_context():
            return self.torch.zeros(1, dtype=self.torch.float64, device="cuda")

    def begin(self, time, stop_time):
        from ._abi import check, lib
        check(lib().bamrex_level_dist_begin(self.level._h, float(time), float(stop_time)), self.level._h)

    def wave_speed_into(self, ws):
        import ctypes
        from ._abi import check, lib
        check(lib().bamrex_level_wave_speed_async(self.level._h, ctypes.c_void_p(ws.data_ptr())), self.level._h)

    def device_dt(self, ws, first):
        import ctypes
        from ._abi import check, lib
        check(lib().bamrex_level_dist_dt(self.level._h, ctypes.c_void_p(ws.data_ptr()), 1 if first else 0),
              self.level._h)

    def fill_dir_device(self, d):
        from ._abi import check, lib
        check(lib().bamrex_level_fill_dir_device(self.level._h, d), self.level._h)

    def sweep_dir_device(self, d, reduce_ws):
        from ._abi import check, lib
        check(lib().bamrex_level_sweep_dir_device(self.level._h, d, 1 if reduce_ws else 0), self.level._h)

    def set_split(self, d, edge_boxes):
        """Direction d's sweep in two parts: part 1 the local boxes listed
        (their ghost cells come from other ranks), part 0 the others."""
        import ctypes
        from ._abi import check, lib
        arr = (ctypes.c_int * max(1, len(edge_boxes)))(*edge_boxes)
        check(lib().bamrex_level_set_sweep_split(self.level._h, d, arr, len(edge_boxes)), self.level._h)

    def sweep_dir_device_part(self, d, reduce_ws, part):
        from ._abi import check, lib
        check(lib().bamrex_level_sweep_dir_device_part(self.level._h, d, 1 if reduce_ws else 0, part), self.level._h)

    def end(self):
        """(time, next dt, steps taken); waits for the level's stream."""
        import ctypes
        from ._abi import check, lib
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        check(lib().bamrex_level_dist_end(self.level._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(n)),
              self.level._h)
        return t.value, dt.value, n.value


class DistLevel:
    """The split step of one level whose boxes are spread over the ranks of
    a torch.distributed process group."""

    def __init__(self, engine, D, dom_lo, dom_hi, boxes, owners, ngrow, bc_lo, bc_hi, dx, cfl, rank, world, dist,
                 overlap=True):
        self.e, self.D, self.dx, self.cfl = engine, D, list(dx), cfl
        self.rank, self.world, self.dist = rank, world, dist
        self.plan = HaloPlan(D, dom_lo, dom_hi, boxes, owners, ngrow, bc_lo, bc_hi, rank)
        self.bufs = []
        for d in range(D):
            send, recv = self.plan.dirs[d]
            engine.set_halo(d, send, recv)
            self.bufs.append((engine.buffer(send["cells"]), engine.buffer(recv["cells"])))
        # interior sweeps while halos travel: per direction the local boxes
        # that receive ghost cells from other ranks are swept after the
        # exchange, every other box while it is in flight
        self.overlap = bool(overlap) and world > 1 and hasattr(engine, "set_split")
        if self.overlap:
            for d in range(D):
                edge = sorted({lb for (lb, _lo, _hi, _off) in self.plan.dirs[d][1]["regions"]})
                engine.set_split(d, edge)

    def exchange_start(self, d):
        """Pack direction d's halo and post its sends and receives (every
        rank posts the same pairs in the same order); returns the requests."""
        send, recv = self.plan.dirs[d]
        sbuf, rbuf = self.bufs[d]
        self.e.pack(d, sbuf)
        NC = self.e.NC
        # one batch (an NCCL group): separate sends and receives of a pair of
        # ranks, each posting its receive first, could wait on each other in
        # the pair's stream
        ops = [self.dist.P2POp(self.dist.irecv, rbuf[start * NC:(start + n) * NC], peer)
               for peer, start, n in recv["peers"]]
        ops += [self.dist.P2POp(self.dist.isend, sbuf[start * NC:(start + n) * NC], peer)
                for peer, start, n in send["peers"]]
        if not ops:
            return []
        with self.e.stream_context():
            return self.dist.batch_isend_irecv(ops)

    def exchange_finish(self, d, reqs):
        """Wait for direction d's requests (with NCCL: the level's stream
        waits, the host does not) and unpack the received ghost cells."""
        with self.e.stream_context():
            for r in reqs:
                r.wait()
        self.e.unpack(d, self.bufs[d][1])

    def exchange(self, d):
        self.exchange_finish(d, self.exchange_start(d))

    def global_wave_speed(self):
        ws = self.e.wave_speed()
        if self.world > 1:
            with self.e.stream_context():
                t = self.e.torch.tensor([ws], dtype=self.e.torch.float64, device=self.e.device)
                self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
                ws = float(t.item())
        return ws

    def est_time_step(self):
        """cfl * min_d dx_d / max wave speed over all ranks
        (AmrLevelAdv::estTimeStep, Source/AmrLevelAdv.cpp:395-477)."""
        ws = self.global_wave_speed()
        dt = 1.0e20
        for d in range(self.D):
            dt = min(dt, self.dx[d] / ws)
        return dt * self.cfl

    def advance(self, dt):
        for d in range(self.D):
            if self.world > 1:
                self.exchange(d)
            self.e.fill_dir(d)
            self.e.sweep_dir(d, dt, d == self.D - 1)

    def run(self, nsteps):
        """nsteps steps with dt computed on the host each step (two waits a
        step); returns the dts."""
        dts = []
        for _ in range(nsteps):
            dt = self.est_time_step()
            self.advance(dt)
            dts.append(dt)
        return dts

    def _global_max_into(self, ws):
        self.e.wave_speed_into(ws)
        if self.dist is not None:
            with self.e.stream_context():
                self.dist.all_reduce(ws, op=self.dist.ReduceOp.MAX)

    def run_device(self, nsteps, time=0.0, stop_time=-1.0):
        """nsteps steps with dt kept on the device: this rank's max wave speed
        is all-reduced in a device buffer and the next dt computed from it on
        the level's stream, so the host enqueues the whole run without
        waiting (computeNewDt across ranks, Source/AmrLevelAdv.cpp:487-619).
        Returns (time, next dt, steps taken)."""
        if not hasattr(self, "_ws"):
            self._ws = self.e.ws_buffer()
        ws = self._ws
        self.e.begin(time, stop_time)
        try:
            self._global_max_into(ws)
            self.e.device_dt(ws, True)
            for _ in range(nsteps):
                for d in range(self.D):
                    last = d == self.D - 1
                    if self.overlap:
                        # the interior boxes sweep while the halo is in flight
                        reqs = self.exchange_start(d)
                        self.e.fill_dir_device(d)
                        self.e.sweep_dir_device_part(d, last, 0)
                        self.exchange_finish(d, reqs)
                        self.e.sweep_dir_device_part(d, last, 1)
                        continue
                    if self.world > 1:
                        self.exchange(d)
                    self.e.fill_dir_device(d)
                    self.e.sweep_dir_device(d, last)
                self._global_max_into(ws)
                self.e.device_dt(ws, False)
        except BaseException:
            try:
                self.e.end()
            except Exception:
                pass
            raise
        return self.e.end()
