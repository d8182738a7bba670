"""Seeded initial data of the workloads (bamrex_b200/problems.py)."""
import math

import numpy as np

from bamrex_b200 import problems


def test_isentropic_vortex_matches_the_reference_formula():
    """Exec/IsentropicVortex/Prob.cpp:87-123 at time 0: background state far
    away, the temperature dip and the swirl at the core, counter-clockwise
    rotation, uniform along z."""
    g, lam, scale = 1.4, 5.0, 0.1
    n = (40, 40, 4)
    U = problems.isentropic_vortex(3, n, [0.0, 0.0, 0.0], [1.0, 1.0, 0.1], centre=(0.5, 0.5), strength=lam,
                                   scale=scale, vel_bg=(0.2, 0.0, 0.0), adiabatic=g)
    rho = U[0]
    u, v = U[1] / rho, U[2] / rho
    p = (g - 1) * (U[4] - 0.5 * rho * (u * u + v * v + (U[3] / rho) ** 2))
    # a far corner cell is the background state to ~exp(-half the domain^2 / scale^2)
    assert abs(rho[0, 0, 0] - 1.0) < 1e-10 and abs(u[0, 0, 0] - 0.2) < 1e-9 and abs(p[0, 0, 0] - 1.0) < 1e-9
    # the cell nearest the centre against the formula
    x = ((19 + 0.5) / 40 - 0.5) / scale
    r2 = 2 * x * x
    dT = -(g - 1) * lam * lam / (8 * g * math.pi ** 2) * math.exp(1 - r2)
    assert abs(rho[0, 19, 19] - ((1 + dT) ** (1 / (g - 1)))) < 1e-12
    assert abs(p[0, 19, 19] - ((1 + dT) ** (g / (g - 1)))) < 1e-12
    # counter-clockwise: v > 0 right of the centre, u < background above it
    assert v[0, 20, 25] > 0 and u[0, 25, 20] < 0.2
    np.testing.assert_array_equal(U[:, 0], U[:, 3])
