"""The Helmholtz restatement (oracle/helmholtz_oracle.py) against the
reference's own solver test (Tests/MLABecLapGrad01.cpp: unit domain, 8 cells
per side, Neumann boundaries, (A, B, C) = (1, 2, 0) and (1, 2, -4), interior
residual <= 1e-12 ||rhs||_2), and properties of the operator and cycle."""
import numpy as np
import pytest


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("abc", [(1, 2, 0), (1, 2, -4)])
def test_oracle_solves_reference_unit_domain(D, abc):
    from oracle import helmholtz_oracle as H
    a, b, c = abc
    alpha, faces, gam, src, dx = H.unit_domain_problem(D, 8)
    op = H.Op(D, (8,) * D, [dx] * D, (H.NEUMANN,) * 3, (H.NEUMANN,) * 3, a, b, c, alpha, faces, gam if c else None)
    x, it, rr = H.bicgstab(H.hierarchy(op), src, tol_rel=1e-12)
    res = H.reference_residual(a, b, c, alpha, faces, gam, src, x, dx, D)
    assert np.abs(res).max() <= 1e-12 * np.sqrt((src * src).sum())
    assert it <= 20


def test_operator_symmetric_without_c():
    from oracle import helmholtz_oracle as H
    rng = np.random.default_rng(1)
    n = 16
    faces = [rng.uniform(0.5, 2.0, (1, n, n + 1)), rng.uniform(0.5, 2.0, (1, n + 1, n))]
    faces[0][:, :, n] = faces[0][:, :, 0]  # one face across the periodic boundary
    faces[1][:, n, :] = faces[1][:, 0, :]
    for bc in (H.PERIODIC, H.NEUMANN, H.DIRICHLET):
        op = H.Op(2, (n, n), [1.0 / n] * 2, (bc,) * 3, (bc,) * 3, 0.3, 1e-3, 0.0, rng.uniform(1, 2, (1, n, n)), faces)
        x, y = rng.standard_normal((1, n, n)), rng.standard_normal((1, n, n))
        assert abs((op.apply(x) * y).sum() - (x * op.apply(y)).sum()) <= 1e-12 * np.abs(op.apply(x)).sum()


def test_vcycle_contracts_on_low_mach_problem():
    from bamrex_b200 import problems
    from oracle import helmholtz_oracle as H
    p = problems.low_mach_pressure_problem(n=64, corr_cells=4)
    op = H.Op(2, (64, 64), [p["dx"]] * 2, (0, 0, 0), (0, 0, 0), 1.0, p["B"], 0.0, np.full((1, 64, 64), p["a"]), None)
    bcc = p["beta_cc"]
    op.b = [0.5 * (np.roll(bcc, 1, axis=2 - d) + bcc) for d in range(2)]
    op.b = [np.concatenate([b, b[:, :, :1]], axis=2) if d == 0 else np.concatenate([b, b[:, :1, :]], axis=1)
            for d, b in enumerate(op.b)]
    ops = H.hierarchy(op)
    x, it, rr = H.bicgstab(ops, p["rhs"], tol_rel=1e-8)
    assert rr <= 1e-8 and it <= 30
