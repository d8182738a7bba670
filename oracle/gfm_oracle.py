"""CPU restatement of BAMReX's ghost-fluid rigid body (test infrastructure:
the checker of the GPU path in tests/, never part of the product).

Follows, in operation order:
  signed distances   Source/Geometry/PlaneSDF.H:30-41, SphereSDF.H:28-37,
                     CylinderSDF.H:36-50, UnionSDF.H:24-33, IntersectionSDF.H:24-39
  level set          fill_from_IF, Source/AmrLevelAdv_LSinit.cpp:13-35
  normals            fill_ls_normals, Source/Geometry/Normals.cpp:12-54
  flags              build_gfm_flags, Source/GFM/GFMFlag.cpp:6-83
  interpolation      bilinear_interp, Source/GFM/Interp_K.H:17-75
  exact Riemann      EulerExactRiemannSolver, Source/System/Euler/RiemannSolver.H:112-275,
                     Euler.H:139-165, 248-333; newton_raphson, RootFinding.H:27-40
  interface fill     fill_ghost_rb, Source/GFM/RigidBody.cpp:24-170
  extrapolation      extrapolate_from_boundary, Source/GFM/Extrapolate.cc:9-37,
                     Extrapolate.H:47-117; fast_sweep, Source/GFM/FastSweep.H:17-214

One deliberate difference: the reference writes each interface ghost cell
in place while its loop runs, so a later cell whose interpolation stencil
reaches an earlier one reads the new value (and under OpenMP tiling the
outcome depends on the thread schedule).  Here every interface cell reads
the state from before the fill.  With an exact distance function the 2D
stencil of a cell reflected 1.5 dx into the fluid lies in the fluid, so the
two agree there.

Pinned to the reference's own tests: the flag patterns of
Tests/GFMFlag01.cpp and Tests/GFMFlag02.cpp, the interpolated values of
Tests/Interp01.cpp, and the intermediate states of Toro's five Riemann
problems (Tests/ExactRiemann01.cpp with Tests/UnitDomainTest.H:99-310); see
tests/test_gfm_cpu.py.
"""
from __future__ import annotations

import math

import numpy as np

PLANE, SPHERE, CYLINDER = 0, 1, 2
UNION, INTERSECTION = 0, 1
REFLECTIVE, NO_SLIP, FOEXTRAP = 0, 1, 2
GHOST, INTERFACE, FILL = 1, 2, 4
PERIODIC = 1


# ---- signed distances (> 0 in the body) -----------------------------------

def make_shape(kind, center=(0.0, 0.0, 0.0), axis=(0.0, 0.0, 1.0), radius=0.0, fluid_inside=False):
    """Constructor arithmetic of the SDF classes (axis / normal normalised
    for planes and cylinders)."""
    c = [float(center[q]) if q < len(center) else 0.0 for q in range(3)]
    a = [float(axis[q]) if q < len(axis) else 0.0 for q in range(3)]
    if kind in (PLANE, CYLINDER):
        mag = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
        a = [a[0] / mag, a[1] / mag, a[2] / mag]
    return {"kind": kind, "c": c, "a": a, "r": float(radius), "sign": 1 if fluid_inside else -1}


def sdf(s, D, x, y, z):
    p = [x, y if D > 1 else 0.0, z if D > 2 else 0.0]
    rx, ry, rz = p[0] - s["c"][0], p[1] - s["c"][1], p[2] - s["c"][2]
    a = s["a"]
    if s["kind"] == PLANE:
        return -1 * (rx * a[0] + ry * a[1] + rz * a[2])
    if s["kind"] == SPHERE:
        t = rx * rx
        if D > 1:
            t = t + ry * ry
        if D > 2:
            t = t + rz * rz
        return (math.sqrt(t) - s["r"]) * s["sign"]
    dot = rx * a[0] + ry * a[1] + rz * a[2]
    tx, ty, tz = rx - dot * a[0], ry - dot * a[1], rz - dot * a[2]
    return (math.sqrt(tx * tx + ty * ty + tz * tz) - s["r"]) * s["sign"]


def shape_value(shapes, combine, D, x, y, z):
    f1 = sdf(shapes[0], D, x, y, z)
    if len(shapes) == 1:
        return f1
    f2 = sdf(shapes[1], D, x, y, z)
    if combine == UNION:
        outside = min(max(f1, f2), 0.0)
        inside = math.sqrt(max(f1, 0.0) * max(f1, 0.0) + max(f2, 0.0) * max(f2, 0.0))
        return inside + outside
    inside = max(min(f1, f2), 0.0)
    outside = -math.sqrt(min(f1, 0.0) * min(f1, 0.0) + min(f2, 0.0) * min(f2, 0.0))
    return inside + outside


# ---- level set, normals, flags on the fabs of an oracle LevelLayout --------

class Body:
    """Level set (D+1 components on every fab cell) and flags (valid cells)
    of one level; fabs indexed like LevelLayout.fab: [comp, k, j, i]."""

    def __init__(self, layout, shapes, combine, prob_lo, stencil=2, fill_diagonals=False, ls_fn=None):
        """ls_fn(i, j, k): a level set given per cell instead of shapes (the
        reference's flag tests set the MultiFab directly)."""
        self.lay = layout
        D = layout.D
        self.D = D
        dx = layout.dx
        plo = [float(prob_lo[q]) if q < len(prob_lo) else 0.0 for q in range(3)]
        self.ls, self.flags = [], []
        for b in range(len(layout.boxes)):
            nc, nz, ny, nx = layout.shapes[b]
            bg = layout.begins[b]
            L = np.zeros((D + 1, nz, ny, nx))
            for kk in range(nz):
                for jj in range(ny):
                    for ii in range(nx):
                        i, j, k = bg[0] + ii, bg[1] + jj, bg[2] + kk
                        if ls_fn is not None:
                            L[0, kk, jj, ii] = ls_fn(i, j, k)
                        else:
                            L[0, kk, jj, ii] = shape_value(shapes, combine, D, (i + 0.5) * dx[0] + plo[0],
                                                           (j + 0.5) * dx[1] + plo[1], (k + 0.5) * dx[2] + plo[2])
            # normals on the fab shrunk by one
            sh = [1 if d < D else 0 for d in range(3)]
            for kk in range(sh[2], nz - sh[2]):
                for jj in range(sh[1], ny - sh[1]):
                    for ii in range(sh[0], nx - sh[0]):
                        nv = [0.0, 0.0, 0.0]
                        for d in range(D):
                            o = [0, 0, 0]
                            o[d] = 1
                            lp = L[0, kk + o[2], jj + o[1], ii + o[0]]
                            lm = L[0, kk - o[2], jj - o[1], ii - o[0]]
                            l0 = L[0, kk, jj, ii]
                            nv[d] = ((lp - l0) if abs(lp) < abs(lm) else (l0 - lm)) / dx[d]
                            L[1 + d, kk, jj, ii] = nv[d]
                        m2 = nv[0] * nv[0]
                        for d in range(1, D):
                            m2 = m2 + nv[d] * nv[d]
                        mag = math.sqrt(m2)
                        if mag != 0:
                            for d in range(D):
                                L[1 + d, kk, jj, ii] = nv[d] / -mag
            self.ls.append(L)
            # flags of the valid cells (stored on the whole fab, 0 in ghosts)
            F = np.zeros((nz, ny, nx), dtype=np.int64)
            lo, hi = layout.boxes[b]
            for k in range(lo[2], hi[2] + 1):
                for j in range(lo[1], hi[1] + 1):
                    for i in range(lo[0], hi[0] + 1):
                        ii, jj, kk = i - bg[0], j - bg[1], k - bg[2]
                        F[kk, jj, ii] = self._flag(L[0], ii, jj, kk, stencil, fill_diagonals)
            self.flags.append(F)

    def _flag(self, ls, i, j, k, stencil, diag):
        D = self.D
        l0 = ls[k, j, i]

        def at(di, dj, dk):
            return ls[k + dk, j + dj, i + di]

        flag = 0
        if l0 >= 0:
            flag |= GHOST
        iface = False
        for d in range(D):
            o = [0, 0, 0]
            o[d] = 1
            iface = iface or (l0 * at(*o) <= 0) or (l0 * at(-o[0], -o[1], -o[2]) <= 0)
        if iface:
            flag |= INTERFACE
        if l0 >= 0:
            close = False
            if not diag:
                for s in range(-stencil, stencil + 1):
                    for d in range(D):
                        o = [0, 0, 0]
                        o[d] = s
                        close = close or (l0 * at(*o) <= 0)
            else:
                for ii in range(-stencil, stencil + 1):
                    jr = stencil - abs(ii) if D >= 2 else 0
                    for jj in range(-jr, jr + 1):
                        kr = jr - abs(jj) if D == 3 else 0
                        for kk in range(-kr, kr + 1):
                            close = close or (l0 * at(ii, jj, kk) <= 0)
            if close:
                flag |= FILL
        return flag

    def field(self, which):
        """Level set / normal component / flags of the valid cells as a
        global (nz, ny, nx) array."""
        lay = self.lay
        n = [lay.dom_hi[d] - lay.dom_lo[d] + 1 for d in range(3)]
        out = np.full((n[2], n[1], n[0]), np.nan)
        for b, (lo, hi) in enumerate(lay.boxes):
            bg = lay.begins[b]
            src = self.flags[b] if which < 0 else self.ls[b][which]
            out[lo[2] - lay.dom_lo[2]:hi[2] - lay.dom_lo[2] + 1, lo[1] - lay.dom_lo[1]:hi[1] - lay.dom_lo[1] + 1,
                lo[0] - lay.dom_lo[0]:hi[0] - lay.dom_lo[0] + 1] = \
                src[lo[2] - bg[2]:hi[2] - bg[2] + 1, lo[1] - bg[1]:hi[1] - bg[1] + 1, lo[0] - bg[0]:hi[0] - bg[0] + 1]
        return out


# ---- bilinear interpolation (origin at index 0, Interp_K.H) ---------------

def bilinear(p, src, D, dx, ncomp, cell):
    """src(i, j, k, n) -> value; p the point measured from index 0.  Returns
    the ncomp interpolated values (c7 of Interp_K.H:64-66 takes its last two
    terms from component 0)."""
    ijk = [p[d] / dx[d] - 0.5 for d in range(D)] + [0.0] * (3 - D)
    i0 = [int(ijk[d]) if d < D else cell[d] for d in range(3)]
    i1 = [int(math.ceil(ijk[d])) if d < D else cell[d] for d in range(3)]
    Dx = [ijk[d] - i0[d] if d < D else 0.0 for d in range(3)]
    out = []
    for n in range(ncomp):
        s000 = src(i0[0], i0[1], i0[2], n)
        s100 = src(i1[0], i0[1], i0[2], n)
        s010 = src(i0[0], i1[1], i0[2], n)
        s110 = src(i1[0], i1[1], i0[2], n)
        s001 = src(i0[0], i0[1], i1[2], n)
        s101 = src(i1[0], i0[1], i1[2], n)
        s011 = src(i0[0], i1[1], i1[2], n)
        s111 = src(i1[0], i1[1], i1[2], n)
        c0 = s000
        c1 = s100 - s000
        c2 = s010 - s000
        c3 = s001 - s000
        c4 = s110 - s010 - s100 + s000
        c5 = s011 - s001 - s010 + s000
        c6 = s101 - s001 - s100 + s000
        c7 = s111 - s011 - s101 - s110 + s100 + s001 + src(i0[0], i1[1], i0[2], 0) - src(i0[0], i0[1], i0[2], 0)
        out.append(c0 + c1 * Dx[0] + c2 * Dx[1] + c3 * Dx[2] + c4 * Dx[0] * Dx[1] + c5 * Dx[1] * Dx[2]
                   + c6 * Dx[2] * Dx[0] + c7 * Dx[0] * Dx[1] * Dx[2])
    return out


# ---- exact Riemann solver (interface at x = 0, direction 0) -----------------

def sound_speed(q, gamma, eps):
    return math.sqrt(gamma * q[-1] / (q[0] * eps))


def _one_side(p, q, gamma):
    pK = q[-1]
    if p > pK:
        A = 2 / ((gamma + 1) * q[0])
        B = ((gamma - 1) / (gamma + 1)) * pK
        return (p - pK) * math.sqrt(A / (p + B))
    cK = sound_speed(q, gamma, 1)
    return 2 * cK / (gamma - 1) * (math.pow(p / pK, (gamma - 1) / (2 * gamma)) - 1)


def _one_side_deriv(p, q, gamma):
    pK = q[-1]
    if p > pK:
        A = 2 / ((gamma + 1) * q[0])
        B = ((gamma - 1) / (gamma + 1)) * pK
        return math.sqrt(A / (p + B)) * (1 - (p - pK) / (2 * (B + p)))
    cK = sound_speed(q, gamma, 1)
    return math.pow(p / pK, -(gamma + 1) / (2 * gamma)) / (q[0] * cK)


def consv_from_primv(q, D, gamma, eps):
    U = [q[0]] + [q[0] * q[1 + d] for d in range(D)]
    vie = q[1 + D] / (gamma - 1)
    usq = q[1] * q[1]
    for d in range(1, D):
        usq = usq + q[1 + d] * q[1 + d]
    return U + [vie + 0.5 * eps * q[0] * usq]


def exact_riemann(L, R, D, gamma, eps, max_iter=200):
    """p*, u*, primitive left / right intermediate states, iterations."""
    cL, cR = sound_speed(L, gamma, 1), sound_speed(R, gamma, 1)
    p = 0.5 * (L[-1] + R[-1]) - 0.125 * math.sqrt(eps) * (R[1] - L[1]) * (L[0] + R[0]) * (cL + cR)
    p = max(1e-6, p)
    it = 0
    while True:
        it += 1
        prev = p
        f = _one_side(prev, L, gamma) + _one_side(prev, R, gamma) + math.sqrt(eps) * (R[1] - L[1])
        fd = _one_side_deriv(prev, L, gamma) + _one_side_deriv(prev, R, gamma)
        p = prev - f / fd
        if not (abs(p - prev) >= 1e-8 * abs(prev)) or it >= max_iter:
            break
    u = 0.5 * (L[1] + R[1]) + 0.5 * (_one_side(p, R, gamma) - _one_side(p, L, gamma)) / math.sqrt(eps)
    IL, IR = list(L), list(R)
    IL[1] = IR[1] = u
    IL[-1] = IR[-1] = p
    for I, K in ((IL, L), (IR, R)):
        pK = K[-1]
        if p > pK:
            pr, ar = p / pK, (gamma - 1) / (gamma + 1)
            I[0] = K[0] * (pr + ar) / (ar * pr + 1)
        else:
            I[0] = K[0] * math.pow(p / pK, 1 / gamma)
    return p, u, IL, IR, it


# ---- the rigid-body ghost fill of a level ---------------------------------

def _fill_boundary_inner(lay, buf):
    """FillBoundary: ghost cells whose image (periodic shifts only) is a
    valid cell of some box."""
    D, NC = lay.D, lay.NC
    n = [lay.dom_hi[d] - lay.dom_lo[d] + 1 for d in range(3)]
    own = -np.ones((n[2], n[1], n[0]), dtype=np.int64)
    for b, (lo, hi) in enumerate(lay.boxes):
        own[lo[2] - lay.dom_lo[2]:hi[2] - lay.dom_lo[2] + 1, lo[1] - lay.dom_lo[1]:hi[1] - lay.dom_lo[1] + 1,
            lo[0] - lay.dom_lo[0]:hi[0] - lay.dom_lo[0] + 1] = b
    fabs = [lay.fab(buf, b) for b in range(len(lay.boxes))]
    for b, (lo, hi) in enumerate(lay.boxes):
        f = fabs[b]
        bg = lay.begins[b]
        _, nz, ny, nx = lay.shapes[b]
        for kk in range(nz):
            for jj in range(ny):
                for ii in range(nx):
                    c = [bg[0] + ii, bg[1] + jj, bg[2] + kk]
                    if all(lo[d] <= c[d] <= hi[d] for d in range(3)):
                        continue
                    m = list(c)
                    ok = True
                    for d in range(D):
                        dl, dh = lay.dom_lo[d], lay.dom_hi[d]
                        if m[d] < dl or m[d] > dh:
                            bc = lay.bc_lo[d] if m[d] < dl else lay.bc_hi[d]
                            if bc != PERIODIC:
                                ok = False
                                break
                            m[d] = dl + ((m[d] - dl) % (dh - dl + 1))
                    if not ok:
                        continue
                    s = own[m[2] - lay.dom_lo[2], m[1] - lay.dom_lo[1], m[0] - lay.dom_lo[0]]
                    if s < 0:
                        continue
                    sb = lay.begins[s]
                    f[:, kk, jj, ii] = fabs[s][:, m[2] - sb[2], m[1] - sb[1], m[0] - sb[0]]


def _sweep_orders(D):
    """(s_i, s_j, s_k) of fast_sweep's loops in their order (FastSweep.H)."""
    if D == 1:
        return [(1, 1, 1), (-1, 1, 1)]
    if D == 2:
        return [(1, 1, 1), (-1, 1, 1), (-1, -1, 1), (1, -1, 1)]
    return [(1, 1, 1), (1, 1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1), (1, -1, 1), (1, -1, -1)]


def _extrapolate_box(lay, f, L, F, b):
    """extrapolate_from_boundary on one box: two fast sweeps, in place."""
    D, NC = lay.D, lay.NC
    lo, hi = lay.boxes[b]
    bg = lay.begins[b]
    dx = lay.dx
    for _ in range(2):
        for s in _sweep_orders(D):
            ks = range(lo[2], hi[2] + 1) if s[2] > 0 else range(hi[2], lo[2] - 1, -1)
            js = range(lo[1], hi[1] + 1) if s[1] > 0 else range(hi[1], lo[1] - 1, -1)
            is_ = range(lo[0], hi[0] + 1) if s[0] > 0 else range(hi[0], lo[0] - 1, -1)
            for k in ks:
                for j in js:
                    for i in is_:
                        ii, jj, kk = i - bg[0], j - bg[1], k - bg[2]
                        flag = F[kk, jj, ii]
                        if (flag & INTERFACE) or not (flag & GHOST):
                            continue
                        sflip = -1 if L[0, kk, jj, ii] >= 0 else 1
                        w, nb = [], []
                        for d in range(D):
                            nd = L[1 + d, kk, jj, ii] / dx[d] * sflip
                            o = [0, 0, 0]
                            o[d] = 1 if nd < 0 else -1
                            w.append(abs(nd))
                            nb.append((kk + o[2], jj + o[1], ii + o[0]))
                        den = w[0]
                        for d in range(1, D):
                            den = den + w[d]
                        for m in range(NC):
                            num = 0.0 + w[0] * f[m][nb[0]]
                            for d in range(1, D):
                                num = num + w[d] * f[m][nb[d]]
                            # the reference divides in long double
                            f[m, kk, jj, ii] = float(np.longdouble(num) / np.longdouble(den))


def fill_rb(lay, buf, body, rb_bc, gamma, eps):
    """FillRBGhostCells + fill_consv_boundary on a level state `buf` whose
    ghost cells are filled (FillPatch).  Returns the number of interface
    cells whose exact Riemann solve reached the iteration cap."""
    D, NC = lay.D, lay.NC
    dx = lay.dx
    unconverged = 0
    pending = []
    for b, (lo, hi) in enumerate(lay.boxes):
        f = lay.fab(buf, b)
        L, F = body.ls[b], body.flags[b]
        bg = lay.begins[b]

        def src(i, j, k, n, f=f, bg=bg):
            idx = (k - bg[2], j - bg[1], i - bg[0])
            if any(q < 0 or q >= s for q, s in zip(idx, f.shape[1:])):
                raise IndexError("interpolation stencil outside the fab: more ghost cells needed")
            return float(f[n, idx[0], idx[1], idx[2]])

        for k in range(lo[2], hi[2] + 1):
            for j in range(lo[1], hi[1] + 1):
                for i in range(lo[0], hi[0] + 1):
                    ii, jj, kk = i - bg[0], j - bg[1], k - bg[2]
                    flag = F[kk, jj, ii]
                    if not ((flag & INTERFACE) and (flag & GHOST)):
                        continue
                    idx = (i, j, k)
                    nrm = [float(L[1 + d, kk, jj, ii]) for d in range(D)]
                    reach = float(L[0, kk, jj, ii]) + 1.5 * dx[0]
                    xr = [(idx[d] + 0.5) * dx[d] + reach * nrm[d] for d in range(D)]
                    U = bilinear(xr, src, D, dx, NC, idx)
                    if rb_bc != FOEXTRAP:
                        q = [U[0]] + [U[1 + d] / U[0] for d in range(D)]
                        usq = q[1] * q[1]
                        for d in range(1, D):
                            usq = usq + q[1 + d] * q[1 + d]
                        q.append((gamma - 1) * (U[1 + D] - 0.5 * eps * U[0] * usq))
                        if rb_bc == NO_SLIP:
                            for d in range(D):
                                q[1 + d] *= -1
                            U = consv_from_primv(q, D, gamma, eps)
                        else:
                            un = q[1] * nrm[0]
                            for d in range(1, D):
                                un = un + q[1 + d] * nrm[d]
                            ut = [q[1 + d] - un * nrm[d] for d in range(D)]
                            o = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
                            curv = -(0.5 * (1.0 / dx[0]) * (L[1, kk, jj, ii + 1] - L[1, kk, jj, ii - 1]))
                            for d in range(1, D):
                                a = L[1 + d, kk + o[d][2], jj + o[d][1], ii + o[d][0]]
                                z = L[1 + d, kk - o[d][2], jj - o[d][1], ii - o[d][0]]
                                curv = curv - (0.5 * (1.0 / dx[d]) * (a - z))
                            ut2 = ut[0] * ut[0]
                            for d in range(1, D):
                                ut2 = ut2 + ut[d] * ut[d]
                            utl = math.sqrt(ut2)
                            mid = [utl, 0.0][:D - 1]
                            PL = [q[0], -un] + mid + [q[1 + D]]
                            pR = max(q[1 + D] - q[0] * ut2 * curv * 2 * 1.5 * dx[0], 1e-14)
                            PR = [q[0], un] + mid + [pR]
                            p, u, IL, IR, it = exact_riemann(PL, PR, D, gamma, eps)
                            if it >= 200:
                                unconverged += 1
                            I = consv_from_primv(IL, D, gamma, eps)
                            U = [I[0]] + [-I[1] * nrm[d] + ut[d] * I[0] for d in range(D)] + [I[1 + D]]
                    pending.append((b, kk, jj, ii, U))
    for b, kk, jj, ii, U in pending:
        lay.fab(buf, b)[:, kk, jj, ii] = U
    _fill_boundary_inner(lay, buf)
    for _ in range(D + 1):
        for b in range(len(lay.boxes)):
            _extrapolate_box(lay, lay.fab(buf, b), body.ls[b], body.flags[b], b)
        _fill_boundary_inner(lay, buf)
    lay.fill_boundary(buf)
    return unconverged
