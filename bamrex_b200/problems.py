"""Seeded initial data for the explicit-path workloads.

Each generator returns the conserved state as a float64 array of shape
(NC, nz, ny, nx), with cell centres x = prob_lo + (i + 0.5) dx as in the
reference's problem setups.
"""
from __future__ import annotations

import numpy as np

DEFAULT_SEED = 20261203


def consv_from_primv(D, q, adiabatic, epsilon=1.0):
    """Vectorised consv_from_primv (Source/System/Euler/Euler.H:138-165).
    q: (NC, ...) primitive array (rho, u.., p)."""
    u = np.empty_like(q)
    u[0] = q[0]
    for d in range(D):
        u[1 + d] = q[0] * q[1 + d]
    u_sq = q[1] * q[1]
    for d in range(1, D):
        u_sq = u_sq + q[1 + d] * q[1 + d]
    u[1 + D] = q[1 + D] / (adiabatic - 1) + 0.5 * epsilon * q[0] * u_sq
    return u


def sod_1d(n=400, adiabatic=1.4):
    """1D Sod shock tube on [0,1]: (rho,u,p) = (1,0,1) for x < 0.5, else
    (0.125,0,0.1) (cell-centre test as Exec/RiemannProblem/Prob.cpp:104-109)."""
    x = (np.arange(n) + 0.5) / n
    q = np.zeros((3, 1, 1, n))
    left = x < 0.5
    q[0, 0, 0] = np.where(left, 1.0, 0.125)
    q[2, 0, 0] = np.where(left, 1.0, 0.1)
    return consv_from_primv(1, q, adiabatic)


def quadrant_2d(n=4096, seed=DEFAULT_SEED, adiabatic=1.4, ny=None):
    """2D four-quadrant Riemann problem on [0,1]^2.  Quadrant states from
    numpy.random.default_rng(seed), drawn in the order TR, TL, BL, BR, each
    (rho ~ U[0.1,1.5], u ~ U[-1,1], v ~ U[-1,1], p ~ U[0.03,1.5]); quadrant
    rule as Exec/QuadrantProblem/Prob.cpp:85-94; then rho *= 1 + 1e-3 N(0,1)
    per cell from the same stream."""
    ny = n if ny is None else ny
    rng = np.random.default_rng(seed)
    states = {}
    for name in ("TR", "TL", "BL", "BR"):
        rho = rng.uniform(0.1, 1.5)
        u = rng.uniform(-1.0, 1.0)
        v = rng.uniform(-1.0, 1.0)
        p = rng.uniform(0.03, 1.5)
        states[name] = (rho, u, v, p)
    x = (np.arange(n) + 0.5) / n
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    q = np.empty((4, 1, ny, n))
    sel = {
        "TR": (X > 0.5) & (Y > 0.5),
        "TL": (X < 0.5) & (Y > 0.5),
        "BL": (X < 0.5) & (Y < 0.5),
    }
    sel["BR"] = ~(sel["TR"] | sel["TL"] | sel["BL"])
    for name, m in sel.items():
        for c in range(4):
            q[c, 0][m] = states[name][c]
    q[0, 0] *= 1.0 + 1e-3 * rng.standard_normal((ny, n))
    return consv_from_primv(2, q, adiabatic)


def blast_3d(n=256, adiabatic=1.4, radius=0.2, centre=(0.5, 0.5, 0.5)):
    """3D spherical blast on [0,1]^3: rho = 1, u = 0, p = 10 for r < radius
    around the centre, else 0.1 (radial rule as
    Exec/CylindricalExplosion/Prob.cpp:79-91, centre moved)."""
    c = (np.arange(n) + 0.5) / n
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    r2 = (X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2
    q = np.zeros((5, n, n, n))
    q[0] = 1.0
    q[4] = np.where(r2 < radius * radius, 10.0, 0.1)
    return consv_from_primv(3, q, adiabatic)


def isentropic_vortex(D, n, prob_lo, prob_hi, centre, strength=5.0, scale=1.0, rho_bg=1.0, vel_bg=(0.0, 0.0, 0.0),
                      p_bg=1.0, adiabatic=1.4, epsilon=1.0):
    """The isentropic vortex of Exec/IsentropicVortex/Prob.cpp:87-123 at
    time 0 on the cell centres of an n-cell box over [prob_lo, prob_hi]
    (2D or 3D, the vortex uniform along z): with r^2 = |x - centre|^2 /
    scale^2, dT = -(gamma-1) lambda^2 / (8 gamma pi^2) exp(1 - r^2),
    rho = rho_bg + (1 + dT)^(1/(gamma-1)) - 1, p = p_bg + (1 + dT)^(gamma/
    (gamma-1)) - 1, (u, v) = vel_bg + lambda / (2 pi) exp((1 - r^2)/2) (-y,
    x) / scale.  scale = 1 is the reference's unit-core vortex."""
    nx, ny = n[0], n[1]
    nz = n[2] if D > 2 else 1
    dx = [(prob_hi[d] - prob_lo[d]) / n[d] for d in range(D)]
    x = (prob_lo[0] + (np.arange(nx) + 0.5) * dx[0] - centre[0]) / scale
    y = (prob_lo[1] + (np.arange(ny) + 0.5) * dx[1] - centre[1]) / scale
    X, Y = np.meshgrid(x, y)
    r_sq = X * X + Y * Y
    lam = strength
    dT = -(adiabatic - 1) * lam * lam / (8 * adiabatic * np.pi * np.pi) * np.exp(1 - r_sq)
    vel_mult = lam / (2 * np.pi) * np.exp((1 - r_sq) * 0.5)
    q = np.zeros((D + 2, nz, ny, nx))
    q[0] = rho_bg + (1 + dT) ** (1 / (adiabatic - 1)) - 1
    q[1] = vel_bg[0] - vel_mult * Y
    q[2] = vel_bg[1] + vel_mult * X
    if D > 2:
        q[3] = vel_bg[2]
    q[1 + D] = p_bg + (1 + dT) ** (adiabatic / (adiabatic - 1)) - 1
    return consv_from_primv(D, q, adiabatic, epsilon)


def random_states(D, shape, seed=DEFAULT_SEED, adiabatic=1.4):
    """Random cells as Profiling/explicit_scaling.cpp:220-260: rho, p in
    [1,2], velocities in [-1,1] (our own seeded stream)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    q = np.empty((D + 2, nz, ny, nx))
    q[0] = rng.uniform(1.0, 2.0, (nz, ny, nx))
    for d in range(D):
        q[1 + d] = rng.uniform(-1.0, 1.0, (nz, ny, nx))
    q[1 + D] = rng.uniform(1.0, 2.0, (nz, ny, nx))
    return consv_from_primv(D, q, adiabatic)


def gaussian_random_field(shape, corr_cells, seed, rng=None):
    """Unit-variance periodic Gaussian random field on a grid of `shape`
    (nz, ny, nx): white noise filtered in Fourier space by a Gaussian of
    correlation length corr_cells cells."""
    rng = np.random.default_rng(seed) if rng is None else rng
    w = rng.standard_normal(shape)
    k = np.meshgrid(*[np.fft.fftfreq(n) for n in shape], indexing="ij")
    k2 = sum(ki ** 2 for ki in k)
    filt = np.exp(-0.5 * (2 * np.pi * corr_cells) ** 2 * k2)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    return (g - g.mean()) / g.std()


def low_mach_pressure_problem(n=2048, seed=DEFAULT_SEED, log_sigma=1.0, corr_cells=32, mach=0.01, adiabatic=1.4,
                              cfl=0.8):
    """The 2D IMEX pressure solve workload: density a lognormal field
    (log-sigma 1.0, correlation length 32 cells), beta = 1/rho on cells,
    the Helmholtz scalars of setup_pressure_op (Source/IMEX/IMEX_O1.cpp:
    592-596): A = 1, a = epsilon / (gamma - 1) with epsilon = Mach^2, B = dt^2
    with dt from the flow CFL at speed `mach`, and a seeded smooth right-hand
    side.  Returns dict(rho, beta_cc, a, B, rhs, dx) with (1, n, n) arrays."""
    rng = np.random.default_rng(seed)
    g = gaussian_random_field((n, n), corr_cells, seed, rng)
    rho = np.exp(log_sigma * g)
    eps = mach * mach
    dx = 1.0 / n
    dt = cfl * dx / mach
    rhs = gaussian_random_field((n, n), 2 * corr_cells, seed + 1, rng)
    return dict(rho=rho[None], beta_cc=(1.0 / rho)[None], a=eps / (adiabatic - 1), B=dt * dt, rhs=rhs[None], dx=dx)


def low_mach_state(n=2048, seed=DEFAULT_SEED, log_sigma=1.0, corr_cells=32, amplitude=0.01, adiabatic=1.4,
                   epsilon=1.0):
    """The 2D low-Mach IMEX state: density lognormal (log-sigma 1.0,
    correlation length 32 cells), velocity the curl of a seeded stream
    function (a Gaussian random field, central differences on the periodic
    grid) scaled to peak speed `amplitude`, pressure 1/gamma, so the sound
    speed is O(1) and the Mach number about `amplitude`.  Returns
    (U (4, 1, n, n), p (1, n, n))."""
    rng = np.random.default_rng(seed)
    rho = np.exp(log_sigma * gaussian_random_field((n, n), corr_cells, seed, rng))
    psi = gaussian_random_field((n, n), corr_cells, seed + 2, rng)
    u = 0.5 * (np.roll(psi, -1, axis=0) - np.roll(psi, 1, axis=0))   # d psi / dy (rows are y)
    v = -0.5 * (np.roll(psi, -1, axis=1) - np.roll(psi, 1, axis=1))  # -d psi / dx
    scale = amplitude / np.max(np.sqrt(u * u + v * v))
    u, v = u * scale, v * scale
    p = np.full((n, n), 1.0 / adiabatic)
    U = np.empty((4, 1, n, n))
    U[0, 0] = rho
    U[1, 0] = rho * u
    U[2, 0] = rho * v
    U[3, 0] = p / (adiabatic - 1) + 0.5 * epsilon * rho * (u * u + v * v)
    return U, p[None]
