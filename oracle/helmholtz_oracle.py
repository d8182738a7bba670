"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the pressure Helmholtz
operator, its smoother, the multigrid V-cycle and the BiCGStab solve.

Follows, in operation order:
  * mlalapgrad_adotx (Source/LinearSolver/MLALapGrad_2D_K.H:9-33,
    MLALapGrad_3D_K.H:9-38);
  * alapgrad_gsrb (MLALapGrad_2D_K.H:180-230: Gauss-Seidel; MLALapGrad_3D_K.H:
    258-324: over-relaxed with omega = 1.15), with a domain face handled as
    the boundary value cf * x(cell) (cf = +1 Neumann, -1 Dirichlet) whose
    part the smoother moves to the left-hand side (the cf / delta terms);
  * averageDownCoeffs (MLALaplacianGrad.H:950-986) for the coarse operators;
  * the pointwise residual of the reference's own solver test
    (Tests/MLABecLapGrad01.cpp:153-204) and its unit-domain coefficients
    (:70-128), for the known-answer checks.
The MLMG cycle of AMReX is not part of the reference: the V-cycle and
BiCGStab here restate the method the device code documents, and solves are
compared by their residual, not bit for bit.  Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

PERIODIC, NEUMANN, DIRICHLET = 0, 1, 2


def _axis(d):
    return 2 - d  # arrays are (nz, ny, nx)


def _neighbours(x, d, bc_lo, bc_hi):
    """(x at cell - e_d, cf_lo, x at cell + e_d, cf_hi) with boundary values."""
    ax = _axis(d)
    xm = np.roll(x, 1, axis=ax)
    xp = np.roll(x, -1, axis=ax)
    cfm = np.zeros(x.shape)
    cfp = np.zeros(x.shape)
    sl0 = [slice(None)] * 3
    sl0[ax] = 0
    sl1 = [slice(None)] * 3
    sl1[ax] = -1
    sl0, sl1 = tuple(sl0), tuple(sl1)
    if bc_lo[d] != PERIODIC:
        f = 1.0 if bc_lo[d] == NEUMANN else -1.0
        cfm[sl0] = f
        xm[sl0] = f * x[sl0]
    if bc_hi[d] != PERIODIC:
        f = 1.0 if bc_hi[d] == NEUMANN else -1.0
        cfp[sl1] = f
        xp[sl1] = f * x[sl1]
    return xm, cfm, xp, cfp


def _face_lo_hi(b, d):
    ax = _axis(d)
    n = b.shape[ax] - 1
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[ax] = slice(0, n)
    hi[ax] = slice(1, n + 1)
    return b[tuple(lo)], b[tuple(hi)]


class Op:
    def __init__(self, D, n, dx, bc_lo, bc_hi, ascal=1.0, bscal=1.0, cscal=0.0, a=None, b=None, c=None):
        self.D = D
        self.n = tuple(n) + (1,) * (3 - len(n))
        self.shape = (self.n[2], self.n[1], self.n[0])
        self.dx = list(dx) + [1.0] * (3 - len(dx))
        self.bc_lo, self.bc_hi = tuple(bc_lo) + (0,) * 3, tuple(bc_hi) + (0,) * 3
        self.ascal, self.bscal, self.cscal = ascal, bscal, cscal
        self.a = np.ones(self.shape) if a is None else a
        self.b = b if b is not None else [np.ones(self.face_shape(d)) for d in range(D)]
        self.c = c  # list of D cell arrays or None

    def face_shape(self, d):
        s = list(self.shape)
        s[_axis(d)] += 1
        return tuple(s)

    def apply(self, x):
        dxinv = [1.0 / self.dx[d] for d in range(3)]
        v = self.ascal * self.a * x
        nb = [_neighbours(x, d, self.bc_lo, self.bc_hi) for d in range(self.D)]
        for d in range(self.D):
            dh = self.bscal * dxinv[d] * dxinv[d]
            bl, bh = _face_lo_hi(self.b[d], d)
            xm, _, xp, _ = nb[d]
            v = v - dh * (bh * (xp - x) - bl * (x - xm))
        if self.c is not None:
            for d in range(self.D):
                xm, _, xp, _ = nb[d]
                chd = self.cscal * self.c[d] * 0.5 * dxinv[d]
                v = v + chd * (xp - xm)
        return v

    def gsrb(self, phi, rhs, color):
        D = self.D
        phi = phi.copy()
        Z, Y, X = np.meshgrid(*[np.arange(s) for s in self.shape], indexing="ij")
        mask = ((X + Y + Z + color) % 2) == 0
        dh = [self.bscal / (self.dx[d] * self.dx[d]) for d in range(3)]
        cdh = [self.cscal / (2 * self.dx[d]) for d in range(3)]
        cc = [self.c[d] if self.c is not None else np.zeros(self.shape) for d in range(D)]
        nb = [_neighbours(phi, d, self.bc_lo, self.bc_hi) for d in range(D)]
        bl = [_face_lo_hi(self.b[d], d)[0] for d in range(D)]
        bh = [_face_lo_hi(self.b[d], d)[1] for d in range(D)]
        gamma = self.ascal * self.a
        for d in range(D):
            gamma = gamma + dh[d] * (bl[d] + bh[d])
        delta = dh[0] * (bl[0] * nb[0][1] + bh[0] * nb[0][3])
        for d in range(1, D):
            delta = delta + dh[d] * (bl[d] * nb[d][1] + bh[d] * nb[d][3])
        for d in range(D):
            delta = delta + cdh[d] * cc[d] * (nb[d][1] - nb[d][3])
        rho = dh[0] * (bl[0] * nb[0][0] + bh[0] * nb[0][2])
        for d in range(1, D):
            rho = rho + dh[d] * (bl[d] * nb[d][0] + bh[d] * nb[d][2])
        for d in range(D):
            rho = rho - cdh[d] * cc[d] * (nb[d][2] - nb[d][0])
        if D == 3:
            omega = 1.15
            g_m_d = gamma - delta
            res = rhs - (gamma * phi - rho)
            new = phi + omega / g_m_d * res
        else:
            new = (rhs + rho - phi * delta) / (gamma - delta)
        phi[mask] = new[mask]
        return phi

    def coarsen(self):
        D = self.D
        w = 0.5 ** D

        def avg_cells(f):
            out = 0.0
            for kk in range(2 if D > 2 else 1):
                for jj in range(2 if D > 1 else 1):
                    for ii in range(2):
                        out = out + f[kk::2 if D > 2 else 1, jj::2 if D > 1 else 1, ii::2]
            return out * w

        nc = [self.n[q] // 2 if q < D else self.n[q] for q in range(3)]
        a = avg_cells(self.a)
        c = [avg_cells(cd) for cd in self.c] if self.c is not None else None
        b = []
        wf = 0.5 ** (D - 1)
        for d in range(D):
            fb = self.b[d]
            s = 0.0
            others = [q for q in range(D) if q != d]
            for t2 in range(2 if len(others) > 1 else 1):
                for t1 in range(2 if len(others) > 0 else 1):
                    sl = [slice(None)] * 3
                    sl[_axis(d)] = slice(0, None, 2)
                    if len(others) > 0:
                        sl[_axis(others[0])] = slice(t1, None, 2)
                    if len(others) > 1:
                        sl[_axis(others[1])] = slice(t2, None, 2)
                    s = s + fb[tuple(sl)]
            b.append(s * wf)
        dxc = [self.dx[q] * 2 if q < D else self.dx[q] for q in range(3)]
        return Op(D, nc, dxc, self.bc_lo, self.bc_hi, self.ascal, self.bscal, self.cscal, a, b, c)


def hierarchy(op, max_levels=0):
    ops = [op]
    while True:
        o = ops[-1]
        if max_levels and len(ops) >= max_levels:
            break
        if not all(o.n[q] % 2 == 0 and o.n[q] >= 4 for q in range(o.D)):
            break
        ops.append(o.coarsen())
    return ops


def vcycle(ops, r, nu1=2, nu2=2, bottom=16, l=0):
    o = ops[l]
    phi = np.zeros(o.shape)
    if l == len(ops) - 1:
        for _ in range(bottom):
            phi = o.gsrb(phi, r, 0)
            phi = o.gsrb(phi, r, 1)
        return phi
    for _ in range(nu1):
        phi = o.gsrb(phi, r, 0)
        phi = o.gsrb(phi, r, 1)
    res = r - o.apply(phi)
    D = o.D
    rc = 0.0
    for kk in range(2 if D > 2 else 1):
        for jj in range(2 if D > 1 else 1):
            for ii in range(2):
                rc = rc + res[kk::2 if D > 2 else 1, jj::2 if D > 1 else 1, ii::2]
    rc = rc * (0.5 ** D)
    ec = vcycle(ops, rc, nu1, nu2, bottom, l + 1)
    e = ec
    for q in range(D):
        e = np.repeat(e, 2, axis=_axis(q))
    phi = phi + e
    for _ in range(nu2):
        phi = o.gsrb(phi, r, 0)
        phi = o.gsrb(phi, r, 1)
    return phi


def bicgstab(ops, b, x0=None, tol_rel=1e-12, max_iter=200, **kw):
    A = ops[0]
    x = np.zeros(A.shape) if x0 is None else x0.copy()
    r = b - A.apply(x)
    rh = r.copy()
    rho = alpha = omega = 1.0
    p = np.zeros(A.shape)
    v = np.zeros(A.shape)
    bn = np.sqrt((b * b).sum())
    it = 0
    while np.sqrt((r * r).sum()) > tol_rel * bn and it < max_iter:
        rho_old = rho
        rho = (rh * r).sum()
        beta = (rho / rho_old) * (alpha / omega)
        p = r + beta * (p - omega * v)
        ph = vcycle(ops, p, **kw)
        v = A.apply(ph)
        alpha = rho / (rh * v).sum()
        s = r - alpha * v
        sh = vcycle(ops, s, **kw)
        t = A.apply(sh)
        omega = (t * s).sum() / (t * t).sum()
        x = x + alpha * ph + omega * sh
        r = s - omega * t
        it += 1
    return x, it, np.sqrt((r * r).sum()) / bn


# ---------------------------------------------------------------- the
# reference's unit-domain solver test (Tests/MLABecLapGrad01.cpp)
def unit_domain_problem(D, ncell=8):
    """Coefficients and source of MLABecLapGradTest::setup on [0,1]^D with
    ncell cells per side: alpha, gamma (c), beta on faces from the cell
    field beta_cc on the grown box, source; Neumann boundaries."""
    dx = 1.0 / ncell
    c = (np.arange(-1, ncell + 1) + 0.5) * dx  # grown by one
    g = np.meshgrid(*([c] * D), indexing="ij")  # g[0] = x ...

    def sinpi(v):
        return np.sin(np.pi * v)

    def cospi(v):
        return np.cos(np.pi * v)

    x = g[0]
    y = g[1] if D > 1 else None
    z = g[2] if D > 2 else None
    alpha = sinpi(2 * x) ** 2
    src = sinpi(2 * x) ** 3
    gam0 = cospi(x) ** 4
    beta_cc = sinpi(2 * x) + 2
    if D > 1:
        alpha = alpha * cospi(4 * y) ** 2
        src = src * cospi(4 * y)
        gam0 = gam0 * cospi(2 * y) ** 2
        gam1 = cospi(3 * x) ** 2 * sinpi(2 * y) ** 4
        beta_cc = beta_cc + 0.5 * cospi(4 * y)
    if D > 2:
        alpha = alpha * sinpi(6 * z) ** 2
        src = src * cospi(2 * z) ** 2
        gam0 = gam0 * cospi(3 * z) ** 2
        gam1 = gam1 * cospi(z) ** 4
        gam2 = (sinpi(3 * x) + 1) ** 2 * cospi(3 * y) ** 2 * sinpi(2 * z) ** 4
        beta_cc = beta_cc + cospi(z) ** 2
    src = src + 0.2

    def inner(f):
        return np.transpose(f[tuple(slice(1, -1) for _ in range(D))]).reshape(
            (1,) * (3 - D) + (ncell,) * D)

    gam = [inner(gam0)] + ([inner(gam1)] if D > 1 else []) + ([inner(gam2)] if D > 2 else [])
    bcc = np.transpose(beta_cc)  # (z, y, x) with the ghost layer
    bcc = bcc.reshape((1,) * (3 - D) + bcc.shape)
    faces = []
    for d in range(D):
        ax = _axis(d)
        lo = [slice(1, -1)] * 3
        hi = [slice(1, -1)] * 3
        for q in range(3 - D):
            lo[q] = slice(None)
            hi[q] = slice(None)
        lo[ax] = slice(0, ncell + 1)
        hi[ax] = slice(1, ncell + 2)
        faces.append(0.5 * (bcc[tuple(lo)] + bcc[tuple(hi)]))
    return inner(alpha), faces, gam, inner(src), dx


def reference_residual(a, b, c, alpha, faces, gam, rhs, soln, dx, D):
    """The test's residual (Tests/MLABecLapGrad01.cpp:153-204) on the
    interior cells (the solution grown by nothing: interior only)."""
    inner = tuple(slice(None) if q < 3 - D else slice(1, -1) for q in range(3))
    s = soln
    ddx = 1 / (dx * dx)
    idx = 1 / dx
    aterm = a * alpha * s
    bsum = 0.0
    csum = 0.0
    for d in range(D):
        ax = _axis(d)
        bl, bh = _face_lo_hi(faces[d], d)
        sp = np.roll(s, -1, axis=ax)
        sm = np.roll(s, 1, axis=ax)
        bsum = bsum + ddx * (bh * (sp - s) - bl * (s - sm))
        csum = csum + idx * gam[d] * (sp - sm)
    bterm = -b * bsum
    cterm = 0.5 * c * csum
    return (aterm + bterm + cterm - rhs)[inner]
