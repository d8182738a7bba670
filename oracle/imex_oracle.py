"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the IMEX step.

advance_imex_rk (Source/IMEX/IMEX_RK.cpp:23-86, 196-235) with the tableaux of
Source/IMEX/ButcherTableau.cpp:5-98 (stage states by the two-output
conservative_update, Source/Fluxes/Update.H:216-300; later stages start from
compute_pressure, Source/IMEX/IMEX_O1.cpp:292-378) and, per stage, the
linearised pressure equation of compute_flux_imex_o1:
  * explicit advection: advance_rusanov_adv and advance_MUSCL_rusanov_adv
    with its local half step (Source/IMEX/IMEX_Fluxes.cpp:11-323), adv_flux
    and kinetic_energy (Source/IMEX_K/euler_K.H), minmod (Limiters.H:76-81);
  * compute_enthalpy, compute_ke, compute_velocity, pressure_source_vector
    (Source/IMEX/IMEX_O1.cpp:178-290, 420-453);
  * the pressure operator of setup_pressure_op (IMEX_O1.cpp:570-614: A = 1,
    B = dt^2, C = -eps dt / 2 for the split kinetic energy, a = eps / (gamma
    - 1), b = average_cellcenter_to_face of the enthalpy, c = u^n) solved
    with oracle.helmholtz_oracle;
  * update_momentum_flux, update_energy_flux (IMEX_O1.cpp:480-556) and the
    conservative update (Source/Fluxes/Update.H:99-130 multiplication form).
Ghost cells: periodic images, first-order extrapolation (transmissive) or
even reflection with the normal momentum negated (reflective), filled one
direction after the other (x, y, z) over the ghosts already filled, the
pressure likewise without the sign change (bamrexBCData::fill_consv_boundary
and fill_pressure_boundary, Source/BoundaryConditions/BCs.cpp:215-442).
Every array operation is one IEEE operation in the reference's order, so
with the pressure given the step reproduces the device bit for bit; the
pressure solve itself is compared through its residual.  Only tests/ import
this module.
"""
from __future__ import annotations

import numpy as np

from . import helmholtz_oracle as HO

TRANSMISSIVE, PERIODIC, REFLECTIVE = 0, 1, 2
RUSANOV, MUSCL_RUSANOV = 0, 1
REUSE_PRESSURE, CONSERVATIVE, CONSERVATIVE_EX = 0, 1, 2
KE_CONSERVATIVE, KE_EX, KE_SPLIT = 0, 1, 2


def _ax(d):
    return 3 - d  # padded state arrays are (comp, z, y, x); scalars use _sax


def _sax(d):
    return 2 - d


def fill(u, D, G, bc_lo, bc_hi, vector=True):
    """Pad the valid array u ((NC, nz, ny, nx) if vector else (nz, ny, nx))
    by G ghost cells in each of the first D directions."""
    out = u
    for d in range(D):
        ax = _ax(d) if vector else _sax(d)
        for side, bc in ((0, bc_lo[d]), (1, bc_hi[d])):
            pad = [(0, 0)] * out.ndim
            pad[ax] = (G, 0) if side == 0 else (0, G)
            mode = {PERIODIC: "wrap", TRANSMISSIVE: "edge", REFLECTIVE: "symmetric"}[bc]
            if bc == PERIODIC and side == 1:
                continue  # both sides at once below
            if bc == PERIODIC:
                pad[ax] = (G, G)
            new = np.pad(out, pad, mode=mode)
            if bc == REFLECTIVE and vector:
                sl = [slice(None)] * new.ndim
                sl[0] = 1 + d
                sl[ax] = slice(0, G) if side == 0 else slice(new.shape[ax] - G, None)
                new[tuple(sl)] = -new[tuple(sl)]
            out = new
    return out


class Grid:
    """Index helper for arrays padded by G in the first D directions."""

    def __init__(self, D, n, G):
        self.D, self.G = D, G
        self.n = list(n) + [1] * (3 - len(n))

    def sl(self, lo, hi, comp=None):
        """Slices (z, y, x) for the cell range [lo, hi) given in valid
        coordinates (lo may be negative, hi may exceed n)."""
        s = []
        for d in (2, 1, 0):
            g = self.G if d < self.D else 0
            s.append(slice(lo[d] + g, hi[d] + g))
        return tuple(s) if comp is None else (comp,) + tuple(s)


def _rng(D, n, grow):
    lo = [(-grow if d < D else 0) for d in range(3)]
    hi = [(n[d] + grow if d < D else 1) for d in range(3)]
    return lo, hi


def _shift(lo, hi, d, s):
    lo = list(lo)
    hi = list(hi)
    lo[d] += s
    hi[d] += s
    return lo, hi


def kinetic_energy(U, D, eps):
    m2 = U[1] * U[1]
    for d in range(1, D):
        m2 = m2 + U[1 + d] * U[1 + d]
    return eps * m2 / (2 * U[0])


def adv_flux(U, D, d, eps):
    """adv_flux<d> of every cell of U (NC, ...)."""
    ud = U[1 + d] / U[0]
    F = np.empty_like(U)
    F[0] = U[1 + d]
    for n in range(1, D + 1):
        F[n] = U[n] * ud
    F[1 + D] = ud * kinetic_energy(U, D, eps)
    return F


def minmod(a, b):
    return np.where((a > 0) & (b > 0), np.fmin(a, b), np.where((a < 0) & (b < 0), np.fmax(a, b), 0.0))


def explicit_update(Upad, G, D, n, dx, dt, eps, method, local_time_step=True, Upad_update=None):
    """State advanced by the advection fluxes of Upad on the valid box grown
    by one (Uex, padded by 1; the update applies to Upad_update, default
    Upad) and the advection fluxes on the faces of that box (list over d of
    arrays (NC, ...) with one more face along d)."""
    grid = Grid(D, n, G)
    lo1, hi1 = _rng(D, n, 1)
    NC = D + 2
    faces = []
    if method == RUSANOV:
        # physical fluxes on the box grown by 2, Rusanov fluxes on faces
        for d in range(D):
            flo, fhi = list(lo1), list(hi1)
            fhi[d] += 1  # faces lo1[d] .. hi1[d]
            R = Upad[(slice(None),) + grid.sl(flo, fhi)]
            Lo, Lh = _shift(flo, fhi, d, -1)
            L = Upad[(slice(None),) + grid.sl(Lo, Lh)]
            FR, FL = adv_flux(R, D, d, eps), adv_flux(L, D, d, eps)
            umax = np.maximum(np.fabs(R[1 + d] / R[0]), np.fabs(L[1 + d] / L[0]))
            faces.append(0.5 * ((FR + FL) - umax * (R - L)))
    else:
        # reconstruction on the box grown by 2
        lo2, hi2 = _rng(D, n, 2)
        C = Upad[(slice(None),) + grid.sl(lo2, hi2)]
        SL, SR = [], []
        hdtdx = [0.5 * (dt / dx[d]) for d in range(D)]
        for d in range(D):
            a, b = _shift(lo2, hi2, d, -1)
            Um = Upad[(slice(None),) + grid.sl(a, b)]
            a, b = _shift(lo2, hi2, d, 1)
            Up = Upad[(slice(None),) + grid.sl(a, b)]
            hdelta = 0.5 * minmod(C - Um, Up - C)
            sl_, sr_ = C - hdelta, C + hdelta
            if local_time_step:
                FLd, FRd = adv_flux(sl_, D, d, eps), adv_flux(sr_, D, d, eps)
                upd = hdtdx[d] * (FRd - FLd)
                sl_, sr_ = sl_ - upd, sr_ - upd
            SL.append(sl_)
            SR.append(sr_)
        g2 = Grid(D, n, 2)
        for d in range(D):
            flo, fhi = list(lo1), list(hi1)
            fhi[d] += 1
            L_i = SL[d][(slice(None),) + g2.sl(flo, fhi)]          # left state of cell i
            a, b = _shift(flo, fhi, d, -1)
            R_im = SR[d][(slice(None),) + g2.sl(a, b)]              # right state of cell i-1
            FL, FR = adv_flux(L_i, D, d, eps), adv_flux(R_im, D, d, eps)
            umax = np.maximum(np.fabs(L_i[1 + d] / L_i[0]), np.fabs(R_im[1 + d] / R_im[0]))
            faces.append(0.5 * ((FL + FR) - umax * (L_i - R_im)))
    # update on the grown box
    U1 = (Upad if Upad_update is None else Upad_update)[(slice(None),) + grid.sl(lo1, hi1)]
    acc = None
    for d in range(D):
        F = faces[d]
        n_f = F.shape[_ax(d)]
        s_hi = [slice(None)] * 4
        s_lo = [slice(None)] * 4
        s_hi[_ax(d)] = slice(1, n_f)
        s_lo[_ax(d)] = slice(0, n_f - 1)
        term = (dt / dx[d]) * (F[tuple(s_hi)] - F[tuple(s_lo)])
        acc = term if acc is None else acc + term
    Uex = U1 - acc
    return Uex, faces


def stage_flux(Uimp, Uexp, p, D, dx, dt, parm_gamma, eps, bc_lo, bc_hi, method=RUSANOV,
               enthalpy_method=REUSE_PRESSURE, ke_method=KE_EX, local_time_step=True, p_new=None, tol_rel=1e-14,
               max_iter=400):
    """compute_flux_imex_o1 (Source/IMEX/IMEX_O1.cpp:19-176): fluxes of one
    implicit stage of size dt from the explicit-stage state Uexp (advection
    fluxes, enthalpy, kinetic energy, velocity) applied to Uimp.  U*: valid
    states (NC, nz, ny, nx); p: valid pressure (nz, ny, nx).  p_new: use
    this pressure instead of solving (to compare the steps around the solve
    bit for bit).  Returns a dict of the solved pressure, the fluxes on the
    valid faces and the intermediate fields."""
    NC = D + 2
    U = Uexp
    n = [U.shape[3], U.shape[2], U.shape[1]]
    G = 3 if method == MUSCL_RUSANOV else 2
    adia = parm_gamma
    Upad = fill(U, D, G, bc_lo, bc_hi)
    Upad_imp = fill(Uimp, D, G, bc_lo, bc_hi)
    grid = Grid(D, n, G)
    lo0, hi0 = _rng(D, n, 0)
    lo1, hi1 = _rng(D, n, 1)
    Uex, afaces = explicit_update(Upad, G, D, n, dx, dt, eps, method, local_time_step, Upad_imp)  # padded by 1
    g1 = Grid(D, n, 1)
    U_in1 = Upad[(slice(None),) + grid.sl(lo1, hi1)]
    ppad = fill(p, D, 1, bc_lo, bc_hi, vector=False)
    # enthalpy on the grown box (compute_enthalpy)
    if enthalpy_method == REUSE_PRESSURE:
        enth = ppad * adia / ((adia - 1) * Uex[0])
        p0 = p
    else:
        src = U_in1 if enthalpy_method == CONSERVATIVE else Uex
        enth = adia * (src[1 + D] - kinetic_energy(src, D, eps)) / Uex[0]
        pfull = (adia - 1) * (Uex[1 + D] - kinetic_energy(Uex, D, eps))
        p0 = pfull[g1.sl(lo0, hi0)]
    # kinetic energy and velocity on the valid box
    Uv = U
    Uexv = Uex[(slice(None),) + g1.sl(lo0, hi0)]
    if ke_method == KE_CONSERVATIVE:
        ke = kinetic_energy(Uv, D, eps)
    elif ke_method == KE_EX:
        ke = kinetic_energy(Uexv, D, eps)
    else:
        dot = Uv[1] * Uexv[1]
        for d in range(1, D):
            dot = dot + Uv[1 + d] * Uexv[1 + d]
        ke = 0.5 * eps * dot / Uv[0]
    vel = [Uv[1 + d] / Uv[0] for d in range(D)]
    # pressure_source_vector
    hdtdx = [0.5 * dt * (1.0 / dx[d]) for d in range(D)]
    acc = None
    for d in range(D):
        a, b = _shift(lo0, hi0, d, 1)
        ep = enth[g1.sl(a, b)] * Uex[(1 + d,) + g1.sl(a, b)]
        a, b = _shift(lo0, hi0, d, -1)
        em = enth[g1.sl(a, b)] * Uex[(1 + d,) + g1.sl(a, b)]
        term = hdtdx[d] * (ep - em)
        acc = term if acc is None else acc + term
    rhs = eps * (Uexv[1 + D] - ke - acc)
    # pressure operator
    bfaces = []
    for d in range(D):
        flo, fhi = list(lo0), list(hi0)
        fhi[d] += 1
        a, b = _shift(flo, fhi, d, -1)
        bfaces.append(0.5 * (enth[g1.sl(a, b)] + enth[g1.sl(flo, fhi)]))
    linbc = lambda b: HO.PERIODIC if b == PERIODIC else HO.NEUMANN
    split = ke_method == KE_SPLIT
    op = HO.Op(D, n[:D], list(dx), [linbc(b) for b in bc_lo[:D]], [linbc(b) for b in bc_hi[:D]], ascal=1.0,
               bscal=dt * dt, cscal=(-0.5 * eps * dt) if split else 0.0,
               a=np.full(rhs.shape, eps / (adia - 1)), b=bfaces, c=vel if split else None)
    if p_new is None:
        ops = HO.hierarchy(op)
        p_new, iters, rel = HO.bicgstab(ops, rhs, x0=p0, tol_rel=tol_rel, max_iter=max_iter)
    pn = fill(p_new, D, 1, bc_lo, bc_hi, vector=False)
    # fluxes on the valid faces
    heps = 0.5 / eps
    hdtdxe = [hdtdx[d] / eps for d in range(D)]
    fluxes = []
    for d in range(D):
        F = afaces[d]
        sl = [slice(None)] * 4
        for e in range(D):
            if e != d:
                sl[_ax(e)] = slice(1, F.shape[_ax(e)] - 1)  # the grown box's faces -> valid faces
        sl[_ax(d)] = slice(1, F.shape[_ax(d)] - 1)
        F = F[tuple(sl)].copy()
        flo, fhi = list(lo0), list(hi0)
        fhi[d] += 1
        a, b = _shift(flo, fhi, d, -1)
        pi, pm = pn[g1.sl(flo, fhi)], pn[g1.sl(a, b)]
        hi_, hm = enth[g1.sl(flo, fhi)], enth[g1.sl(a, b)]
        mi, mm = Uex[(1 + d,) + g1.sl(flo, fhi)], Uex[(1 + d,) + g1.sl(a, b)]
        F[1 + d] = F[1 + d] + heps * (pi + pm)
        F[1 + D] = F[1 + D] + (0.5 * (hi_ * mi + hm * mm) - hdtdxe[d] * ((hi_ + hm) * (pi - pm)))
        fluxes.append(F)
    return {"p": p_new, "fluxes": fluxes, "Uex": Uex, "enth": enth, "ke": ke, "rhs": rhs, "op": op,
            "bfaces": bfaces}


def _fdiff(F, d):
    nf = F.shape[_ax(d)]
    s_hi = [slice(None)] * 4
    s_lo = [slice(None)] * 4
    s_hi[_ax(d)] = slice(1, nf)
    s_lo[_ax(d)] = slice(0, nf - 1)
    return F[tuple(s_hi)] - F[tuple(s_lo)]


def conservative_update(U, fluxes, D, dx, dt):
    """Update.H:99-130: out = in - dt idx_x dFx - dt idx_y dFy [- ...]."""
    out = U.copy()
    for d in range(D):
        out = out - (dt * (1.0 / dx[d])) * _fdiff(fluxes[d], d)
    return out


def imex_step(U, p, D, dx, dt, parm_gamma, eps, bc_lo, bc_hi, method=RUSANOV, enthalpy_method=REUSE_PRESSURE,
              ke_method=KE_EX, p_new=None, tol_rel=1e-14, max_iter=400):
    """One SP111 step: stage_flux with Uimp = Uexp = U and dt, then the
    conservative update.  Returns stage_flux's dict plus the new state "U"."""
    r = stage_flux(U, U, p, D, dx, dt, parm_gamma, eps, bc_lo, bc_hi, method, enthalpy_method, ke_method, True,
                   p_new, tol_rel, max_iter)
    r["U"] = conservative_update(U, r["fluxes"], D, dx, dt)
    return r


# IMEXButcherTableau (Source/IMEX/ButcherTableau.cpp:5-98): A_imp, A_exp, b
def tableau(name):
    if name == "SP111":
        return [[1.0]], [[0.0]], [1.0]
    if name == "SSP222":
        a = 1 - 1 / np.sqrt(2)
        return [[a, 0.0], [1 - 2 * a, a]], [[0.0, 0.0], [1.0, 0.0]], [0.5, 0.5]
    if name == "SASSP322":
        return ([[0.5, 0, 0], [-0.5, 0.5, 0], [0, 0.5, 0.5]], [[0, 0, 0], [0, 0, 0], [0, 1, 0]], [0, 0.5, 0.5])
    if name == "SASSP332":
        return ([[0.25, 0, 0], [0, 0.25, 0], [1 / 3, 1 / 3, 1 / 3]], [[0, 0, 0], [0.5, 0, 0], [0.5, 0.5, 0]],
                [1 / 3, 1 / 3, 1 / 3])
    if name == "SSP433":
        al, be, et = 0.24169426078821, 0.06042356519705, 0.12915286960590
        return ([[al, 0, 0, 0], [-al, al, 0, 0], [0, 1 - al, al, 0], [be, et, 0.5 - be - et - al, al]],
                [[0, 0, 0, 0], [0, 0, 0, 0], [0, 1, 0, 0], [0, 0.25, 0.25, 0]], [0, 1 / 6, 1 / 6, 2 / 3])
    raise ValueError(name)


def stage_states(U, F, dts_imp, dts_exp, D, dx):
    """conservative_update with two outputs (Update.H:216-300): each
    output = in - sum over the earlier stages of (dt_i idx_x dFx + dt_i
    idx_y dFy [+ ...])."""
    outs = []
    for dts in (dts_imp, dts_exp):
        out = U.copy()
        for i, Fi in enumerate(F):
            acc = None
            for d in range(D):
                t = (dts[i] * (1.0 / dx[d])) * _fdiff(Fi[d], d)
                acc = t if acc is None else acc + t
            out = out - acc
        outs.append(out)
    return outs


def stage_pressure(Unew, Uold, D, dx, adt, adia, eps, bc_lo, bc_hi, method, ke_method):
    """compute_pressure (IMEX_O1.cpp:292-378) for the linearised scheme on
    the valid cells."""
    if ke_method == KE_SPLIT:
        dot = Uold[1] * Unew[1]
        for d in range(1, D):
            dot = dot + Uold[1 + d] * Unew[1 + d]
        return (adia - 1) * (Unew[1 + D] - 0.5 * eps * dot / Uold[0])
    if ke_method == KE_EX:
        n = [Unew.shape[3], Unew.shape[2], Unew.shape[1]]
        G = 3 if method == MUSCL_RUSANOV else 2
        Op = fill(Uold, D, G, bc_lo, bc_hi)
        ex, _ = explicit_update(Op, G, D, n, dx, adt, eps, method, local_time_step=False)
        ex = ex[(slice(None),) + Grid(D, n, 1).sl(*_rng(D, n, 0))]
        m2 = ex[1] * ex[1]
        for d in range(1, D):
            m2 = m2 + ex[1 + d] * ex[1 + d]
        return (adia - 1) * (Unew[1 + D] - 0.5 * eps * m2 / Unew[0])
    return pressure_of(Unew, D, adia, eps)


def imex_rk_step(U, p, D, dx, dt, parm_gamma, eps, bc_lo, bc_hi, method=RUSANOV, enthalpy_method=REUSE_PRESSURE,
                 ke_method=KE_EX, name="SP111", p_stages=None, tol_rel=1e-14, max_iter=400):
    """advance_imex_rk (Source/IMEX/IMEX_RK.cpp:23-86) with the named
    tableau: per stage the two stage states, the stage pressure (stages after
    the first), the stage fluxes; then the b-weighted flux sum (sum_fluxes)
    and the conservative update.  p_stages: the pressure of each stage's
    solve to use instead of solving."""
    Ai, Ae, b = tableau(name)
    s = len(b)
    F, stages = [], []
    Uexp_prev = None
    for st in range(s):
        dti = [Ai[st][i] * dt for i in range(s)]
        dte = [Ae[st][i] * dt for i in range(s)]
        Uimp, Uexp = stage_states(U, F, dti, dte, D, dx)
        adt = Ai[st][st] * dt
        if st > 0:
            p = stage_pressure(Uexp, Uexp_prev, D, dx, adt, parm_gamma, eps, bc_lo, bc_hi, method, ke_method)
        r = stage_flux(Uimp, Uexp, p, D, dx, adt, parm_gamma, eps, bc_lo, bc_hi, method, enthalpy_method, ke_method,
                       name == "SP111", None if p_stages is None else p_stages[st], tol_rel, max_iter)
        r["Uimp"], r["Uexp"], r["p_in"] = Uimp, Uexp, p
        stages.append(r)
        p = r["p"]
        F.append(r["fluxes"])
        Uexp_prev = Uexp
    fsum = []
    for d in range(D):
        acc = F[0][d] * b[0]
        for i in range(1, s):
            acc = acc + F[i][d] * b[i]
        fsum.append(acc)
    return {"U": conservative_update(U, fsum, D, dx, dt), "p": p, "fluxes": fsum, "stages": stages}


def pressure_of(U, D, adia, eps):
    """(gamma - 1)(E - eps |m|^2 / (2 rho)) (euler_K.H pressure)."""
    return (adia - 1) * (U[1 + D] - kinetic_energy(U, D, eps))


def advective_time_step(U, D, dx, cfl):
    """cfl / max (|m_x| / dx + |m_y| / dy [+ |m_z| / dz]) / rho
    (max_dx_scaled_speed, Source/System/Euler/Euler.cpp:107-129)."""
    s = np.fabs(U[1]) / dx[0]
    for d in range(1, D):
        s = s + np.fabs(U[1 + d]) / dx[d]
    return (1.0 / np.max(s / U[0])) * cfl
