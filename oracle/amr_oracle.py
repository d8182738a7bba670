"""TEST INFRASTRUCTURE ONLY -- CPU restatement of the AMR glue.

Checks the device coarse/fine coupling (libbamrex_cuda.so, amr.cu /
amr_kernels.cu) operation by operation: fine ghost interpolation with time
interpolation, flux registers (CrseInit / FineAdd), reflux, average_down,
errorEst tagging, and the subcycled hierarchy step (timeStep recursion with
computeInitialDt / computeNewDt and post_timestep, Source/AmrLevelAdv.cpp:
487-652; flux scaling and register calls, Source/AmrLevelAdv_advance.cpp:
192-254).  The AMReX arithmetic behind those call sites is not part of the
reference, so parity with AMReX itself is unpinned; this restates the
methods the device code documents (time interpolation as
alpha*old + beta*new; monotonized-central slopes with a Barth-Jespersen
scale; mean of the r^D children; reflux by -/+ register / volume), in the
same order of floating-point operations.  Level sweeps use the C oracle
(bamrex_oracle.c).  Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def _cell_slices(lay, b, lo, hi):
    """Slices of fab b for the cell range [lo, hi] (inclusive, 3D)."""
    bg = lay.begins[b]
    return (slice(None), slice(lo[2] - bg[2], hi[2] - bg[2] + 1), slice(lo[1] - bg[1], hi[1] - bg[1] + 1),
            slice(lo[0] - bg[0], hi[0] - bg[0] + 1))


class OLevel:
    """One level: an oracle LevelLayout and its current state buffer."""

    def __init__(self, D, dom_lo, dom_hi, boxes, ngrow, dx, bc_lo, bc_hi):
        self.D, self.NC, self.ngrow = D, D + 2, ngrow
        self.dom_lo = tuple(dom_lo) + (0,) * (3 - len(dom_lo))
        self.dom_hi = tuple(dom_hi) + (0,) * (3 - len(dom_hi))
        self.boxes = [(tuple(lo) + (0,) * (3 - len(lo)), tuple(hi) + (0,) * (3 - len(hi))) for lo, hi in boxes]
        self.dx = list(dx)
        self.bc_lo, self.bc_hi = tuple(bc_lo), tuple(bc_hi)
        self.lay = O.LevelLayout(D, self.dom_lo, self.dom_hi, self.boxes, ngrow, dx, self.bc_lo, self.bc_hi)
        self.S = self.lay.alloc()
        n = [self.dom_hi[d] - self.dom_lo[d] + 1 for d in range(3)]
        self.owner = -np.ones((n[2], n[1], n[0]), dtype=np.int64)
        for b, (lo, hi) in enumerate(self.boxes):
            self.owner[lo[2] - self.dom_lo[2]:hi[2] - self.dom_lo[2] + 1, lo[1] - self.dom_lo[1]:hi[1] - self.dom_lo[1] + 1,
                       lo[0] - self.dom_lo[0]:hi[0] - self.dom_lo[0] + 1] = b

    def set_dense(self, glob):
        self.lay.scatter(self.S, glob)

    def dense(self, buf=None):
        return self.lay.gather(self.S if buf is None else buf)

    def fab(self, b, buf=None):
        return self.lay.fab(self.S if buf is None else buf, b)

    def vol(self):
        v = 1.0
        for d in range(self.D):
            v *= self.dx[d]
        return v


def _padded(dense, D, bc_lo, bc_hi, pad):
    """The dense coarse array padded by `pad` cells in each active direction,
    pad cells mapped into the domain by the boundary rules (periodic, mirror
    with the normal momentum negated, or extrapolation)."""
    NC = dense.shape[0]
    n = [dense.shape[3], dense.shape[2], dense.shape[1]]
    idx, neg = [], []
    for d in range(3):
        if d >= D:
            idx.append(np.arange(n[d]))
            neg.append(np.zeros(n[d], dtype=bool))
            continue
        x = np.arange(-pad, n[d] + pad)
        m = x.copy()
        ng = np.zeros(len(x), dtype=bool)
        for side, sel in ((0, x < 0), (1, x >= n[d])):
            bc = bc_lo[d] if side == 0 else bc_hi[d]
            if bc == O.PERIODIC:
                m[sel] = x[sel] % n[d]
            elif bc == O.REFLECTIVE:
                m[sel] = (-1 - x[sel]) if side == 0 else (2 * n[d] - 1 - x[sel])
                ng[sel] = True
            else:
                m[sel] = 0 if side == 0 else n[d] - 1
        idx.append(m)
        neg.append(ng)
    P = dense[:, idx[2][:, None, None], idx[1][None, :, None], idx[0][None, None, :]].copy()
    for d in range(D):
        sl = [slice(None)] * 3
        shape = [1, 1, 1]
        shape[2 - d] = len(neg[d])
        flip = neg[d].reshape(shape)
        comp = P[1 + d]
        P[1 + d] = np.where(flip, -comp, comp)
    return P


def _interp(P, D, r, pad, w):
    """Fine values at wrapped fine cells w (3 x N int arrays, coarse-domain
    relative) from the padded coarse array P; returns (NC, N)."""
    c = [w[d] // r if d < D else w[d] for d in range(3)]
    xi = [((2 * (w[d] - c[d] * r) + 1 - r) / (2.0 * r)) if d < D else np.zeros(w[d].shape) for d in range(3)]
    pc = [c[d] + pad if d < D else c[d] for d in range(3)]
    xmax = (r - 1) / (2.0 * r)
    NC = P.shape[0]
    out = np.empty((NC, len(w[0])))

    def at(m, off):
        q = [pc[d] + off[d] for d in range(3)]
        return P[m, q[2], q[1], q[0]]

    with np.errstate(divide="ignore", invalid="ignore"):
        for m in range(NC):
            uc = at(m, (0, 0, 0))
            umin, umax = uc.copy(), uc.copy()
            ext = np.zeros_like(uc)
            slopes = []
            for d in range(D):
                e = [0, 0, 0]
                e[d] = -1
                ul = at(m, e)
                e[d] = 1
                ur = at(m, e)
                dc = 0.5 * (ur - ul)
                dl = 2.0 * (uc - ul)
                dr = 2.0 * (ur - uc)
                sl = np.where(dl * dr > 0.0, np.copysign(np.minimum(np.abs(dc), np.minimum(np.abs(dl), np.abs(dr))), dc),
                              0.0)
                slopes.append(sl)
                umin = np.minimum(umin, np.minimum(ul, ur))
                umax = np.maximum(umax, np.maximum(ul, ur))
                ext = ext + np.abs(sl) * xmax
            alpha = np.ones_like(uc)
            pos = ext > 0.0
            alpha = np.where(pos, np.minimum(alpha, (umax - uc) / ext), alpha)
            alpha = np.where(pos, np.minimum(alpha, (uc - umin) / ext), alpha)
            s = np.zeros_like(uc)
            for d in range(D):
                s = s + slopes[d] * xi[d]
            out[m] = uc + alpha * s
    return out


class OCoupling:
    """Coarse/fine coupling of two oracle levels."""

    def __init__(self, crse: OLevel, fine: OLevel, r):
        self.c, self.f, self.r = crse, fine, r
        self.D, self.NC = crse.D, crse.NC
        self.old = None
        self.t_old = self.t_new = 0.0
        self._build_register()

    # -- coarse data at a time
    def _coarse_dense(self, time):
        new = self.c.dense()
        if self.old is None:
            return new
        span = self.t_new - self.t_old
        teps = 1e-3 * span
        if abs(time - self.t_old) < teps:
            return self.old
        if abs(time - self.t_new) < teps:
            return new
        a_old = (self.t_new - time) / span
        a_new = (time - self.t_old) / span
        return a_old * self.old + a_new * new

    def save_coarse_old(self, t_old, t_new):
        self.old = self.c.dense()
        self.t_old, self.t_new = t_old, t_new

    def _fill_cells(self, b, cells_unwrapped, shift, P, pad, bufs):
        """Interpolate fine cells (3 x N, unwrapped) of box b into bufs."""
        f, r, D = self.f, self.r, self.D
        w = [cells_unwrapped[d] + shift[d] - (self.c.dom_lo[d] * r if d < D else 0) for d in range(3)]
        vals = _interp(P, D, r, pad, w)
        for buf in bufs:
            fab = f.lay.fab(buf, b)
            bg = f.lay.begins[b]
            ii = cells_unwrapped[0] - bg[0]
            jj = cells_unwrapped[1] - bg[1]
            kk = cells_unwrapped[2] - bg[2]
            for m in range(self.NC):
                fab[m, kk, jj, ii] = vals[m]

    def fill_patch(self, time, bufs):
        """Coarse/fine ghost cells of every fine box (face slabs of depth
        ngrow, inside the domain or its periodic image, not covered by fine
        boxes) into each buffer of bufs."""
        f, D, r = self.f, self.D, self.r
        pad = 2
        P = _padded(self._coarse_dense(time), D, self.c.bc_lo, self.c.bc_hi, pad)
        g = f.ngrow
        for b, (lo, hi) in enumerate(f.boxes):
            for d in range(D):
                dlo, dhi = f.dom_lo[d], f.dom_hi[d]
                n = dhi - dlo + 1
                for side in (0, 1):
                    rng = [np.arange(lo[q], hi[q] + 1) for q in range(3)]
                    rng[d] = np.arange(lo[d] - g, lo[d]) if side == 0 else np.arange(hi[d] + 1, hi[d] + g + 1)
                    Z, Y, X = np.meshgrid(rng[2], rng[1], rng[0], indexing="ij")
                    cells = [X.ravel(), Y.ravel(), Z.ravel()]
                    pos = cells[d]
                    inside = (pos >= dlo) & (pos <= dhi)
                    periodic = (f.bc_lo[d] if side == 0 else f.bc_hi[d]) == O.PERIODIC
                    shift = np.zeros(len(pos), dtype=np.int64)
                    if periodic:
                        shift = np.where(inside, 0, n if side == 0 else -n)
                        keep = np.ones(len(pos), dtype=bool)
                    else:
                        keep = inside
                    wrapped = [cells[q] + (shift if q == d else 0) for q in range(3)]
                    own = np.full(len(pos), -1, dtype=np.int64)
                    own[keep] = f.owner[wrapped[2][keep] - f.dom_lo[2], wrapped[1][keep] - f.dom_lo[1],
                                        wrapped[0][keep] - f.dom_lo[0]]
                    keep = keep & (own < 0)
                    if not keep.any():
                        continue
                    sel = [cells[q][keep] for q in range(3)]
                    sh = [np.zeros(keep.sum(), dtype=np.int64) for _ in range(3)]
                    sh[d] = shift[keep]
                    self._fill_cells(b, sel, sh, P, pad, bufs)

    def fill_coarse_patch(self):
        f, D = self.f, self.D
        pad = 2
        P = _padded(self.c.dense(), D, self.c.bc_lo, self.c.bc_hi, pad)
        for b, (lo, hi) in enumerate(f.boxes):
            rng = [np.arange(lo[q], hi[q] + 1) for q in range(3)]
            Z, Y, X = np.meshgrid(rng[2], rng[1], rng[0], indexing="ij")
            cells = [X.ravel(), Y.ravel(), Z.ravel()]
            self._fill_cells(b, cells, [np.zeros(len(cells[0]), dtype=np.int64)] * 3, P, pad, [f.S])

    # -- flux registers
    def _build_register(self):
        f, c, r, D = self.f, self.c, self.r, self.D
        self.slots = []
        for d in range(D):
            slots = []
            n = f.dom_hi[d] - f.dom_lo[d] + 1
            for b, (lo, hi) in enumerate(f.boxes):
                for side in (0, 1):
                    pos = lo[d] - 1 if side == 0 else hi[d] + 1
                    shift = 0
                    if pos < f.dom_lo[d] or pos > f.dom_hi[d]:
                        if (f.bc_lo[d] if side == 0 else f.bc_hi[d]) != O.PERIODIC:
                            continue
                        shift = n if side == 0 else -n
                    fface = lo[d] if side == 0 else hi[d] + 1
                    rng = [np.arange(lo[q], hi[q] + 1) if q < D else np.zeros(1, dtype=np.int64) for q in range(3)]
                    rng[d] = np.array([pos + shift])
                    seen = set()
                    for kf in rng[2]:
                        for jf in rng[1]:
                            for i_f in rng[0]:
                                w = (int(i_f), int(jf), int(kf))
                                if f.owner[w[2] - f.dom_lo[2], w[1] - f.dom_lo[1], w[0] - f.dom_lo[0]] >= 0:
                                    continue
                                B = tuple(w[q] // r if q < D else w[q] for q in range(3))
                                if B in seen:
                                    continue
                                seen.add(B)
                                cb = int(c.owner[B[2] - c.dom_lo[2], B[1] - c.dom_lo[1], B[0] - c.dom_lo[0]])
                                assert cb >= 0, "not properly nested"
                                cface = list(B)
                                cface[d] = B[d] + (1 if side == 0 else 0)
                                ffaces = []
                                tz = r if (D > 2 and d != 2) else 1
                                ty = r if (D > 1 and d != 1) else 1
                                tx = r if d != 0 else 1
                                for a2 in range(tz):
                                    for a1 in range(ty):
                                        for a0 in range(tx):
                                            fi = fface if d == 0 else B[0] * r + a0
                                            fj = fface if d == 1 else (B[1] * r + a1 if D > 1 else 0)
                                            fk = fface if d == 2 else (B[2] * r + a2 if D > 2 else 0)
                                            ffaces.append((fi, fj, fk))
                                slots.append(dict(B=B, cb=cb, cface=tuple(cface), b=b, ffaces=ffaces,
                                                  sign=-1 if side == 0 else 1))
            # the device orders slots by fine box, side, piece, then coarse
            # cell z-y-x; the values do not depend on the order
            self.slots.append(slots)
        self.reg = [np.zeros((self.NC, len(s))) for s in self.slots]

    def crse_init(self, fluxes, dt):
        c, D = self.c, self.D
        for d in range(D):
            s = dt
            for e in range(D):
                if e != d:
                    s *= c.dx[e]
            for q, sl in enumerate(self.slots[d]):
                cb = sl["cb"]
                lo = c.boxes[cb][0]
                i, j, k = sl["cface"]
                F = fluxes[d][cb][:, k - lo[2], j - lo[1], i - lo[0]]
                self.reg[d][:, q] = -(F * s)

    def fine_add(self, fluxes, dt):
        f, D = self.f, self.D
        for d in range(D):
            s = dt
            for e in range(D):
                if e != d:
                    s *= f.dx[e]
            for q, sl in enumerate(self.slots[d]):
                lo = f.boxes[sl["b"]][0]
                acc = self.reg[d][:, q].copy()
                for (i, j, k) in sl["ffaces"]:
                    acc = acc + fluxes[d][sl["b"]][:, k - lo[2], j - lo[1], i - lo[0]] * s
                self.reg[d][:, q] = acc

    def reflux(self):
        c = self.c
        vol = c.vol()
        for d in range(self.D):
            for q, sl in enumerate(self.slots[d]):
                i, j, k = sl["B"]
                fab = c.fab(sl["cb"])
                bg = c.lay.begins[sl["cb"]]
                fab[:, k - bg[2], j - bg[1], i - bg[0]] = fab[:, k - bg[2], j - bg[1], i - bg[0]] + \
                    (float(sl["sign"]) * self.reg[d][:, q]) / vol

    def avg_down(self):
        c, f, r, D = self.c, self.f, self.r, self.D
        rz = r if D > 2 else 1
        ry = r if D > 1 else 1
        w = 1.0 / (r * ry * rz)
        fd = f.dense()
        for cb, (clo, chi) in enumerate(c.boxes):
            for b, (lo, hi) in enumerate(f.boxes):
                flo = [lo[q] // r if q < D else lo[q] for q in range(3)]
                fhi = [hi[q] // r if q < D else hi[q] for q in range(3)]
                xlo = [max(clo[q], flo[q]) for q in range(3)]
                xhi = [min(chi[q], fhi[q]) for q in range(3)]
                if any(xlo[q] > xhi[q] for q in range(3)):
                    continue
                s = 0.0
                for kk in range(rz):
                    for jj in range(ry):
                        for ii in range(r):
                            zs = slice(xlo[2] * (r if D > 2 else 1) + kk - f.dom_lo[2],
                                       (xhi[2] + 1) * (r if D > 2 else 1) - f.dom_lo[2], rz)
                            ys = slice(xlo[1] * (r if D > 1 else 1) + jj - f.dom_lo[1],
                                       (xhi[1] + 1) * (r if D > 1 else 1) - f.dom_lo[1], ry)
                            xs = slice(xlo[0] * r + ii - f.dom_lo[0], (xhi[0] + 1) * r - f.dom_lo[0], r)
                            s = s + fd[:, zs, ys, xs]
                c.fab(cb)[_cell_slices(c.lay, cb, xlo, xhi)] = s * w


def tag_level(lev: OLevel, grad_var=0, grad_threshold=0.0, err_var=None, phierr=0.0, primv=False, parm=None):
    """errorEst tags of the valid cells in packed (box-major, x-fastest)
    order; ghost cells of lev.S must be filled (fill_boundary + fill_patch)."""
    D = lev.D
    out = []
    for b, (lo, hi) in enumerate(lev.boxes):
        fab = lev.fab(b)
        bg = lev.lay.begins[b]

        def val(var, off):
            sl = [slice(None)]
            for q in (2, 1, 0):
                a = lo[q] - bg[q] + off[q]
                sl.append(slice(a, a + hi[q] - lo[q] + 1))
            U = fab[tuple(sl)]
            if not primv:
                return U[var]
            rho = U[0]
            inv = 1.0 / rho
            q = [rho] + [U[1 + d] * inv for d in range(D)]
            usq = q[1] * q[1]
            for d in range(1, D):
                usq = usq + q[1 + d] * q[1 + d]
            p = (parm.adiabatic - 1) * (U[1 + D] - (0.5 * parm.epsilon) * U[0] * usq)
            return (q + [p])[var]

        t = np.zeros((hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1), dtype=np.uint8)
        if err_var is not None:
            t |= (val(err_var, (0, 0, 0)) >= phierr).astype(np.uint8)
        if grad_threshold > 0:
            v = val(grad_var, (0, 0, 0))
            g = np.zeros_like(v)
            for d in range(D):
                e = [0, 0, 0]
                e[d] = -1
                a = np.abs(val(grad_var, e) - v)
                e[d] = 1
                a = np.maximum(a, np.abs(v - val(grad_var, e)))
                g = np.maximum(g, a) if d else a
            t |= (g >= grad_threshold * np.maximum(np.abs(v), 1e-14)).astype(np.uint8)
        out.append(t.ravel())
    return np.concatenate(out)


def tag_level_extra(tags, boxes, dom_lo, D, dx, prob_lo, box=None, ls=None, flags=None, lstol=None):
    """The criteria errorEst applies after grad_error / state_error
    (Source/AmrLevelAdv.cpp:780-830), on packed tags: box_error
    (Source/Src_K/tagging_K.H:87-103: the cell centre (i + 1/2) dx + prob_lo
    inside box = (lo, hi) in every direction), interface_error
    (tagging_K.H:62-72, with lstol: at the interface or |level set| <=
    lstol) and ghost_error (tagging_K.H:74-84: a ghost cell not at the
    interface is cleared; whenever there is a body, flags given).  ls and
    flags are global (nz, ny, nx) arrays of the valid cells (level set,
    GFM flags: 1 ghost, 2 interface)."""
    out = np.array(tags, dtype=np.uint8).copy()
    o = 0
    for lo, hi in boxes:
        shp = (hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1)
        m = shp[0] * shp[1] * shp[2]
        t = out[o:o + m].reshape(shp)
        if box is not None:
            inside = np.ones(shp, dtype=bool)
            for d in range(D):
                p = (np.arange(lo[d], hi[d] + 1) + 0.5) * dx[d] + prob_lo[d]
                ok = (box[0][d] <= p) & (p <= box[1][d])
                inside &= ok.reshape([-1 if q == 2 - d else 1 for q in range(3)])
            t[inside] = 1
        if flags is not None:
            sl = tuple(slice(lo[q] - dom_lo[q], hi[q] - dom_lo[q] + 1) for q in (2, 1, 0))
            F = flags[sl].astype(np.int64)
            if lstol is not None:
                t[((F & 2) != 0) | (np.abs(ls[sl]) <= lstol)] = 1
            t[((F & 1) != 0) & ((F & 2) == 0)] = 0
        o += m
    return out


class OAmr:
    """The subcycled hierarchy on oracle levels with fixed grids."""

    def __init__(self, D, dom_lo, dom_hi, prob_lo, prob_hi, level_boxes, parm, method, cfl, ratio=2, ngrow=2,
                 bc_lo=(0, 0, 0), bc_hi=(0, 0, 0), do_reflux=True):
        self.D, self.r, self.parm, self.method, self.cfl = D, ratio, parm, method, cfl
        self.do_reflux = do_reflux
        self.levels, self.cpl = [], [None]
        for l, boxes in enumerate(level_boxes):
            f = ratio ** l
            lo = [dom_lo[d] * f if d < D else 0 for d in range(3)]
            hi = [(dom_hi[d] + 1) * f - 1 if d < D else 0 for d in range(3)]
            dx = [(prob_hi[d] - prob_lo[d]) / (hi[d] - lo[d] + 1) for d in range(D)]
            self.levels.append(OLevel(D, lo, hi, boxes, ngrow, dx, bc_lo, bc_hi))
            if l > 0:
                self.cpl.append(OCoupling(self.levels[l - 1], self.levels[l], ratio))
        self.dt_level = [0.0] * len(self.levels)
        self.steps = 0
        self.time = 0.0
        self.bodies = None

    def set_bodies(self, shapes, combine, prob_lo, rb_bc, adiabatic, epsilon=1.0, stencil=2, fill_diagonals=False):
        """A static rigid body on every level (its level set at the level's
        resolution, as every AmrLevelAdv level builds in initData); each
        level's advance then runs FillRBGhostCells after its coarse/fine
        ghost fill (Source/AmrLevelAdv_advance.cpp:108-116)."""
        from oracle import gfm_oracle as G
        self.bodies = [G.Body(L.lay, shapes, combine, prob_lo, stencil=stencil, fill_diagonals=fill_diagonals)
                       for L in self.levels]
        self.body_args = (rb_bc, adiabatic, epsilon)

    def avg_down_all(self):
        for l in range(len(self.levels) - 1, 0, -1):
            self.cpl[l].avg_down()

    def compute_dt(self, stop_time):
        nl = len(self.levels)
        dt_min = []
        for L in self.levels:
            L.lay.fill_boundary(L.S)
            dt_min.append(L.lay.est_time_step(L.S, self.parm.adiabatic, self.parm.epsilon, self.cfl))
        dt0 = 1.0e100
        nf = 1
        for l in range(nl):
            if l > 0:
                nf *= self.r
            dt0 = min(dt0, nf * dt_min[l])
        eps = 0.001 * dt0
        if stop_time >= 0.0 and (self.time + dt0) > (stop_time - eps):
            dt0 = stop_time - self.time
        nf = 1
        for l in range(nl):
            if l > 0:
                nf *= self.r
            self.dt_level[l] = dt0 / nf

    def _advance(self, l, time, dt):
        L = self.levels[l]
        L.lay.fill_boundary(L.S)
        if l > 0:
            self.cpl[l].fill_patch(time, [L.S])
        if self.bodies is not None:
            from oracle import gfm_oracle as G
            G.fill_rb(L.lay, L.S, self.bodies[l], *self.body_args)
        S2 = L.S.copy()
        fl = L.lay.advance_explicit_fluxes(L.S, S2, time, dt, self.method, self.parm)
        if l + 1 < len(self.levels):
            self.cpl[l + 1].crse_init(fl, dt)
        if l > 0:
            self.cpl[l].fine_add(fl, dt)

    def time_step(self, l, time):
        dt = self.dt_level[l]
        finest = len(self.levels) - 1
        if l < finest:
            self.cpl[l + 1].save_coarse_old(time, time + dt)
        self._advance(l, time, dt)
        if l < finest:
            dtf = self.dt_level[l + 1]
            for i in range(self.r):
                self.time_step(l + 1, time + i * dtf)
            if self.do_reflux:
                self.cpl[l + 1].reflux()
            self.cpl[l + 1].avg_down()

    def coarse_step(self, stop_time=-1.0):
        self.compute_dt(stop_time)
        self.time_step(0, self.time)
        self.time += self.dt_level[0]
        self.steps += 1
        return self.dt_level[0]

    def conserved_sums(self):
        NC = self.D + 2
        tot = np.zeros(NC)
        for l, L in enumerate(self.levels):
            d = L.dense()
            v = L.vol()
            cov = np.zeros(d.shape[1:], dtype=bool)
            if l + 1 < len(self.levels):
                F = self.levels[l + 1]
                for lo, hi in F.boxes:
                    sl = tuple(slice(lo[q] // self.r - L.dom_lo[q], hi[q] // self.r - L.dom_lo[q] + 1)
                               if q < self.D else slice(None) for q in (2, 1, 0))
                    cov[sl] = True
            m = ~np.isnan(d[0]) & ~cov
            tot += np.array([d[n][m].sum() for n in range(NC)]) * v
        return tot


# ----------------------------------------------------------------------
# grid generation (bamrex_cluster_tags), dense restatement
# ----------------------------------------------------------------------

def _shift_mask(m, d, s, periodic, outside):
    """out[x] = m[x + s] along axis d (wrapped, or `outside` past the ends)."""
    n = m.shape[d]
    if periodic:
        return np.roll(m, -s, axis=d)
    out = np.full_like(m, outside)
    if abs(s) < n:
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        src[d] = slice(s, n) if s >= 0 else slice(0, n + s)
        dst[d] = slice(0, n - s) if s >= 0 else slice(-s, n)
        out[tuple(dst)] = m[tuple(src)]
    return out


def _sweep(m, d, rad, periodic, use_and, outside):
    if rad <= 0:
        return m
    acc = None
    for s in range(-rad, rad + 1):
        sh = _shift_mask(m, d, s, periodic, outside)
        acc = sh if acc is None else ((acc & sh) if use_and else (acc | sh))
    return acc


def _cluster(btag, D, eff, lo, hi, depth, out):
    sub = btag[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1]
    if not sub.any():
        return
    idx = np.nonzero(sub)
    base = list(lo)
    lo = [base[d] + int(idx[d].min()) for d in range(3)]
    hi = [base[d] + int(idx[d].max()) for d in range(3)]
    sub = btag[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1]
    vol = sub.size
    nt = int(sub.sum())
    all_unit = all(hi[d] == lo[d] for d in range(D))
    if nt >= eff * vol or all_unit or depth > 64:
        out.append((tuple(lo), tuple(hi)))
        return
    sig = [sub.sum(axis=tuple(a for a in range(3) if a != d)).astype(np.int64) for d in range(D)]
    best_d, best_cut = -1, 0
    best_score = -1
    for d in range(D):
        n = len(sig[d])
        for x in range(1, n - 1):
            if sig[d][x] == 0:
                score = n * 4 - abs(2 * x - n)
                if score > best_score:
                    best_score, best_d, best_cut = score, d, x
    if best_d < 0:
        best_jump = 0
        for d in range(D):
            n = len(sig[d])
            if n < 4:
                continue
            lap = np.zeros(n, dtype=np.int64)
            lap[1:n - 1] = sig[d][:n - 2] - 2 * sig[d][1:n - 1] + sig[d][2:]
            for x in range(1, n - 2):
                if (lap[x] > 0 and lap[x + 1] < 0) or (lap[x] < 0 and lap[x + 1] > 0):
                    jump = abs(int(lap[x]) - int(lap[x + 1]))
                    if jump > best_jump:
                        best_jump, best_d, best_cut = jump, d, x + 1
    if best_d < 0:
        ln = 0
        for d in range(D):
            if hi[d] - lo[d] + 1 > ln:
                ln, best_d = hi[d] - lo[d] + 1, d
        best_cut = ln // 2
    ahi = list(hi)
    ahi[best_d] = lo[best_d] + best_cut - 1
    clo = list(lo)
    clo[best_d] = lo[best_d] + best_cut
    _cluster(btag, D, eff, lo, ahi, depth + 1, out)
    _cluster(btag, D, eff, clo, hi, depth + 1, out)


def _clip(allowed, D, lo, hi, out):
    sub = allowed[lo[0]:hi[0] + 1, lo[1]:hi[1] + 1, lo[2]:hi[2] + 1]
    nin = int(sub.sum())
    if nin == 0:
        return
    if nin == sub.size:
        out.append((tuple(lo), tuple(hi)))
        return
    best_d, ln = 0, 0
    for d in range(D):
        if hi[d] - lo[d] + 1 > ln:
            ln, best_d = hi[d] - lo[d] + 1, d
    ahi = list(hi)
    ahi[best_d] = lo[best_d] + ln // 2 - 1
    clo = list(lo)
    clo[best_d] = lo[best_d] + ln // 2
    _clip(allowed, D, lo, ahi, out)
    _clip(allowed, D, clo, hi, out)


def _chop(lo, hi, D, mgs, out):
    for d in range(D):
        ln = hi[d] - lo[d] + 1
        if ln > mgs:
            pieces = (ln + mgs - 1) // mgs
            base, extra = ln // pieces, ln % pieces
            a = lo[d]
            for p in range(pieces):
                qlo, qhi = list(lo), list(hi)
                qlo[d] = a
                qhi[d] = a + base + (1 if p < extra else 0) - 1
                a = qhi[d] + 1
                _chop(qlo, qhi, D, mgs, out)
            return
    out.append((tuple(lo), tuple(hi)))


def cluster_tags_dense(D, dom_lo, dom_hi, boxes, tags_packed, ref_ratio=2, blocking_factor=8, max_grid_size=32,
                       n_error_buf=2, n_proper=1, grid_eff=0.7, periodic=(0, 0, 0)):
    """Level l+1 boxes from level-l tags, on cell masks over the whole
    domain: buffer the tags by n_error_buf (per direction), erode the box
    coverage by n_proper (cells across a non-periodic side count as covered,
    periodic sides wrap), drop buffered tags outside the eroded coverage,
    block by blocking_factor / ref_ratio (tagged if any footprint cell is,
    allowed if every one is), cluster the blocked tags by signatures (a zero
    of the signature nearest the middle, else the strongest inflection,
    else halve the longest side) until a box is grid_eff full, split the
    clusters into allowed pieces, chop at max_grid_size, order by
    (z, y, x) of the lower corner and refine."""
    dl = [dom_lo[d] if d < D else 0 for d in range(3)]
    n = [dom_hi[d] - dom_lo[d] + 1 if d < D else 1 for d in range(3)]
    c = blocking_factor // ref_ratio
    cc = [c if d < D else 1 for d in range(3)]
    nt = [n[d] // cc[d] for d in range(3)]
    tag = np.zeros(n, dtype=bool)
    cov = np.zeros(n, dtype=bool)
    off = 0
    for lo, hi in boxes:
        lo = tuple(lo) + (0,) * (3 - len(lo))
        hi = tuple(hi) + (0,) * (3 - len(hi))
        ext = [hi[d] - lo[d] + 1 for d in range(3)]
        vol = ext[0] * ext[1] * ext[2]
        blk = np.asarray(tags_packed[off:off + vol]).reshape(ext[2], ext[1], ext[0]).transpose(2, 1, 0) != 0
        off += vol
        sl = tuple(slice(lo[d] - dl[d], hi[d] - dl[d] + 1) for d in range(3))
        cov[sl] = True
        tag[sl] = blk
    for d in range(D):
        tag = _sweep(tag, d, n_error_buf, bool(periodic[d]), False, False)
    allowed = cov
    for d in range(D):
        allowed = _sweep(allowed, d, n_proper, bool(periodic[d]), True, True)
    tag = tag & allowed
    btag = tag.reshape(nt[0], cc[0], nt[1], cc[1], nt[2], cc[2]).any(axis=(1, 3, 5))
    ball = allowed.reshape(nt[0], cc[0], nt[1], cc[1], nt[2], cc[2]).all(axis=(1, 3, 5))
    btag = btag & ball
    clusters = []
    _cluster(btag, D, grid_eff, [0, 0, 0], [nt[0] - 1, nt[1] - 1, nt[2] - 1], 0, clusters)
    clipped = []
    for lo, hi in clusters:
        _clip(ball, D, list(lo), list(hi), clipped)
    mgs_t = max_grid_size // blocking_factor
    chopped = []
    for lo, hi in clipped:
        _chop(list(lo), list(hi), D, mgs_t, chopped)
    chopped.sort(key=lambda b: (b[0][2], b[0][1], b[0][0]))
    out = []
    for lo, hi in chopped:
        flo = tuple((lo[d] * c + dl[d]) * ref_ratio if d < D else 0 for d in range(3))
        fhi = tuple(((hi[d] + 1) * c + dl[d]) * ref_ratio - 1 if d < D else 0 for d in range(3))
        out.append((flo, fhi))
    return out
