"""Generate tests/golden/reference_known_answers.json from the BAMReX test
sources (read as text; nothing of the reference is compiled or run).

Sources parsed:
  Tests/hllc_test.H     Toro et al. (2020) left/right states and expected
                        wave-speed estimates for the Toro (1994) estimator
  Tests/HLLC01.cpp      the tolerances each fixture is checked with
  Tests/BoxTest.H       primitive/conserved state pairs (gamma=1.6, eps=0.5)
  Tests/Euler01.cpp     tolerances and expected max wave speed
  Tests/Limiters01.cpp  minmod known answers

Usage: python tests/golden/make_golden.py --ref /path/to/BAMReX
       (or BAMREX_REFERENCE=/path/to/BAMReX python tests/golden/make_golden.py)
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))


def _class_body(src: str, name: str) -> str:
    m = re.search(r"class\s+%s\s*:\s*public\s+\w+\s*\{" % re.escape(name), src)
    if not m:
        raise ValueError(name)
    i, depth = m.end(), 1
    while depth:
        depth += {"{": 1, "}": -1}.get(src[i], 0)
        i += 1
    return src[m.end():i - 1]


def _real(body: str, var: str) -> float:
    m = re.search(r"Real\s+%s\s*=\s*([-+0-9.eE]+)\s*;" % re.escape(var), body)
    if not m:
        raise ValueError(var)
    return float(m.group(1))


def toro_fixtures(ref: str):
    src = open(os.path.join(ref, "Tests", "hllc_test.H")).read()
    tests = open(os.path.join(ref, "Tests", "HLLC01.cpp")).read()
    out = []
    for name in ["Toro2020Test1", "Toro2020Test2", "Toro2020Test4", "Toro2020Test5", "Toro2020Test7",
                 "Toro2020Test5Scaled"]:
        body = _class_body(src, name)
        f = {k: _real(body, k) for k in ["density_L", "u_L", "p_L", "density_R", "u_R", "p_R",
                                          "exp_To_S_L", "exp_To_S_R", "adiabatic"]}
        # expected S* from the fixture's own formula (hllc_test.H, exp_To_S_interm)
        sL, sR = f["exp_To_S_L"], f["exp_To_S_R"]
        f["exp_To_S_interm"] = ((f["p_R"] - f["p_L"] + f["density_L"] * f["u_L"] * (sL - f["u_L"])
                                 - f["density_R"] * f["u_R"] * (sR - f["u_R"]))
                                / (f["density_L"] * (sL - f["u_L"]) - f["density_R"] * (sR - f["u_R"])))
        scaled = name.endswith("Scaled")
        if scaled:
            rho0, u0, p0 = _real(body, "density_0"), _real(body, "u_0"), _real(body, "p_0")
            f["epsilon"] = rho0 * u0 * u0 / p0
            f["primv_L"] = [f["density_L"] / rho0, f["u_L"] / u0, f["p_L"] / p0]
            f["primv_R"] = [f["density_R"] / rho0, f["u_R"] / u0, f["p_R"] / p0]
            f["speed_scale"] = 1.0 / u0
        else:
            f["epsilon"] = 1.0
            f["primv_L"] = [f["density_L"], f["u_L"], f["p_L"]]
            f["primv_R"] = [f["density_R"], f["u_R"], f["p_R"]]
            f["speed_scale"] = 1.0
        # tolerances of the WaveSpeedEstToro1994 test for this fixture
        m = re.search(r"TEST_F\(%s,\s*WaveSpeedEstToro1994\)\s*\{(.*?)\n\}" % name, tests, re.S)
        tol = re.findall(r"EXPECT_NEAR\(\s*(S_L|S_R|S_interm)\s*,[^,]+,\s*([0-9.eE+-]+)", m.group(1))
        f["tol"] = {k: float(v) for k, v in tol}
        f["name"] = name
        out.append(f)
    return out


def _gpu_array(body: str, name: str, dim: int):
    m = re.search(r"#if AMREX_SPACEDIM == 3(.*?)#elif AMREX_SPACEDIM == 2(.*?)#elif AMREX_SPACEDIM == 1(.*?)#endif",
                  body, re.S)
    block = {3: m.group(1), 2: m.group(2), 1: m.group(3)}[dim]
    mm = re.search(r"%s\s*\{([^}]*)\}" % re.escape(name), block)
    return [float(x) for x in mm.group(1).replace("\n", " ").split(",")]


def box_fixtures(ref: str):
    src = open(os.path.join(ref, "Tests", "BoxTest.H")).read()
    adia = float(re.search(r"const amrex::Real adia\s*=\s*([0-9.]+)", src).group(1))
    eps = float(re.search(r"const amrex::Real eps\s*=\s*([0-9.]+)", src).group(1))
    out = {"adiabatic": adia, "epsilon": eps, "tol": 1e-12, "dims": {}}
    for D in (1, 2, 3):
        out["dims"][str(D)] = {k: _gpu_array(src, k, D) for k in ["primv_L", "primv_R", "consv_L", "consv_R"]}
    # Euler01.cpp:44-66 expected max wave speed (2D and 3D): |v| + c with eps
    e01 = open(os.path.join(ref, "Tests", "Euler01.cpp")).read()
    m3 = re.search(r"#if AMREX_SPACEDIM == 3\s*//.*?const Real expected = (.*?);", e01, re.S)
    m2 = re.search(r"#elif AMREX_SPACEDIM == 2\s*//.*?const Real expected = (.*?);", e01, re.S)

    def ev(expr):
        return eval(expr.replace("sqrt", "math.sqrt"), {"math": math})

    out["max_wave_speed"] = {"3": ev(m3.group(1)), "2": ev(m2.group(1)), "rtol": 1e-12}
    # BoxTest::setup(true): 4^D domain, cells with all indices < 2 hold consv_L, others consv_R
    out["layout"] = {"ncell": 4, "split": 2}
    return out


def minmod_cases(ref: str):
    src = open(os.path.join(ref, "Tests", "Limiters01.cpp")).read()
    return [[float(a), float(b), float(c)]
            for a, b, c in re.findall(r"EXPECT_EQ\(minmod\(([-0-9.]+),\s*([-0-9.]+)\),\s*([-0-9.]+)\)", src)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BAMREX_REFERENCE"),
                    help="the BAMReX source tree (default: $BAMREX_REFERENCE)")
    ap.add_argument("--out", default=os.path.join(HERE, "reference_known_answers.json"))
    a = ap.parse_args()
    if not a.ref:
        ap.error("give the BAMReX source tree with --ref or $BAMREX_REFERENCE")
    data = {
        "source": "BAMReX Tests/{hllc_test.H,HLLC01.cpp,BoxTest.H,Euler01.cpp,Limiters01.cpp}",
        "toro_wave_speeds": toro_fixtures(a.ref),
        "box_test": box_fixtures(a.ref),
        "minmod": minmod_cases(a.ref),
    }
    with open(a.out, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
