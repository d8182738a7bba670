"""CPU-side checks of the product library: it loads, it exports every symbol
include/bamrex_cuda.h declares, and its host-only logic (Parm defaults,
status strings, argument validation, packing) behaves like the reference.
No device computation runs here."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"BAMREX_API\s+[\w\s\*]*?\b(bamrex_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import bamrex_b200
    L = bamrex_b200.lib()
    decl = _declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
    # and the Python binding declares a signature for each of them
    from bamrex_b200._abi import SIGNATURES
    assert sorted(SIGNATURES) == decl


def test_abi_version_and_status_strings():
    import bamrex_b200
    L = bamrex_b200.lib()
    assert L.bamrex_abi_version() == 4
    assert L.bamrex_status_string(0) == b"ok"
    assert b"argument" in L.bamrex_status_string(1)


def test_region_timers_record_host_phases():
    """The region timers (the BL_PROFILE / TinyProfiler counterpart) time
    host-side phases; grid generation is host code, so it runs here."""
    import bamrex_b200 as bx
    from bamrex_b200.amr import cluster_tags
    prev = bx.profile_enable(True)
    try:
        bx.profile_reset()
        assert bx.profile_report() == []
        tags = np.zeros((32, 32), dtype=np.int8)
        tags[10:14, 12:20] = 1
        for _ in range(2):
            cluster_tags(2, (0, 0, 0), (31, 31, 0), [((0, 0, 0), (31, 31, 0))], tags, ref_ratio=2,
                         blocking_factor=8, max_grid_size=32)
        rows = {r[0]: r for r in bx.profile_report()}
        assert rows["bamrex_cluster_tags"][1] == 2
        for phase in ("cluster_tags:mark", "cluster_tags:cluster", "cluster_tags:clip_chop"):
            assert rows[phase][1] == 2 and rows[phase][2] >= 0
        assert rows["bamrex_cluster_tags"][2] >= rows["cluster_tags:cluster"][2]
        bx.profile_enable(False)
        bx.profile_reset()
        cluster_tags(2, (0, 0, 0), (31, 31, 0), [((0, 0, 0), (31, 31, 0))], tags)
        assert bx.profile_report() == []
    finally:
        bx.profile_enable(prev)
        bx.profile_reset()


@pytest.mark.parametrize("D", [1, 2, 3])
def test_parm_defaults_match_fluidsystem(D):
    """FluidSystem::set_parm_defaults + init_parm (FluidSystem.cpp:52-101)."""
    from bamrex_b200._abi import CParm, lib
    p = CParm()
    assert lib().bamrex_parm_set_defaults(ctypes.byref(p), D) == 0
    assert p.adiabatic == -1 and p.epsilon == 1 and p.Re == 1 and p.eos_mu == 28.96
    assert p.limiter == 1  # van_leer
    assert list(p.limiter_indices) == [1 + D] * 8  # UInd::E
    assert not any(p.limit_on_primv)
    p.adiabatic = 1.4
    assert lib().bamrex_parm_init(ctypes.byref(p)) == 0
    g = 1.4
    exp = [g, g + 1, g - 1, 1 / (g + 1), 1 / (g - 1), (g + 1) / (2 * g), (g - 1) / (2 * g), g / (g + 1), g / (g - 1)]
    assert list(p.adia) == exp
    assert p.R_spec == 8.3145 / (28.96 * 1e-3)
    assert p.need_primitive_for_limiting == 0
    p.limit_on_primv[0] = 1
    lib().bamrex_parm_init(ctypes.byref(p))
    assert p.need_primitive_for_limiting == 1


def test_argument_validation_without_device():
    """Bad arguments are rejected on the host with BAMREX_ERR_ARG before any
    device work (null pointers, bad dimension/direction, unsupported method)."""
    from bamrex_b200._abi import Array4, Box, CParm, lib
    L = lib()
    p = CParm()
    L.bamrex_parm_set_defaults(ctypes.byref(p), 2)
    p.adiabatic = 1.4
    b = Box.make((0, 0, 0), (7, 7, 0))
    dx = (ctypes.c_double * 3)(0.1, 0.1, 1.0)
    a = Array4()
    assert L.bamrex_compute_flux(0, 0, 2, 0.0, ctypes.byref(b), a, a, dx, 0.01, ctypes.byref(p), None) == 1
    assert L.bamrex_compute_flux(0, 2, 2, 0.0, ctypes.byref(b), a, a, dx, 0.01, ctypes.byref(p), None) == 1
    assert L.bamrex_compute_flux(2, 0, 2, 0.0, ctypes.byref(b), a, a, dx, 0.01, ctypes.byref(p), None) == 1
    assert L.bamrex_sweep_box(3, 0, 2, ctypes.byref(b), a, a, a, dx, 0.01, ctypes.byref(p), None) == 1
    assert L.bamrex_level_create(None, None, None) == 1
    assert L.bamrex_last_error()


def test_packing_roundtrip():
    from bamrex_b200 import Packing, decompose
    D = 3
    boxes = decompose(D, (0, 0, 0), (9, 6, 4), 4)
    pk = Packing(D, (0, 0, 0), boxes)
    g = np.random.default_rng(0).standard_normal((5, 5, 7, 10))
    packed = pk.pack(g)
    assert packed.size == g.size
    np.testing.assert_array_equal(pk.unpack(packed), g)


def test_problem_generators_are_seeded_and_physical():
    from bamrex_b200 import problems
    a = problems.quadrant_2d(64, seed=3)
    b = problems.quadrant_2d(64, seed=3)
    np.testing.assert_array_equal(a, b)
    assert a.shape == (4, 1, 64, 64)
    rho, E = a[0], a[3]
    assert (rho > 0).all()
    p = 0.4 * (E - 0.5 * (a[1] ** 2 + a[2] ** 2) / rho)
    assert (p > 0).all()
    s = problems.sod_1d(400)
    assert s.shape == (3, 1, 1, 400) and s[0, 0, 0, 0] == 1.0 and s[0, 0, 0, -1] == 0.125
