"""The C++ host surface (include/bamrex/level.hpp) compiles with a plain C++
compiler against the C ABI, and (on a GPU) reproduces the oracle's Sod run."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "sod_level.cpp")


def _build(tmp_path):
    import bamrex_b200
    bamrex_b200.lib()
    exe = str(tmp_path / "sod_level")
    libdir = os.path.join(ROOT, "bamrex_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    os.path.join(libdir, "libbamrex_cuda.so"), "-Wl,-rpath," + libdir], check=True)
    return exe


def test_cpp_host_compiles(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_cpp_host_sod_matches_oracle(tmp_path, oracle):
    exe = _build(tmp_path)
    out = str(tmp_path / "sod.txt")
    subprocess.run([exe, out], check=True)
    vals = open(out).read().split()
    steps, t = int(vals[0]), float(vals[1])
    u = np.array([float(v) for v in vals[2:]]).reshape(3, 1, 1, 400)
    from bamrex_b200 import problems
    lay = oracle.LevelLayout(1, (0, 0, 0), (399, 0, 0), [((0, 0, 0), (399, 0, 0))], 2, [1.0 / 400])
    ref, t_ref, dts = oracle.run_level(lay, problems.sod_1d(400), oracle.Parm(1), oracle.MUSCL_HANCOCK, 0.9,
                                       stop_time=0.2)
    assert steps == len(dts) and abs(t - t_ref) <= 1e-14
    err = max(np.max(np.abs(u[c] - ref[c])) / np.max(np.abs(ref[c])) for c in range(3))
    assert err <= 1e-10
