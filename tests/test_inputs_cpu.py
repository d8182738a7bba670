"""Inputs files in the reference's format (bamrex_b200/inputs.py) and
plotfiles (bamrex_b200/plotfile.py), on the host.

The settings cases follow the reference's readers: main
(Source/main.cpp:23-50), AmrLevelAdv::read_params
(Source/AmrLevelAdv.cpp:836-916), FluidSystem::ReadParameters
(Source/System/FluidSystem.cpp:10-71, FluidSystem.H:91-137),
bamrexBCData::build (Source/BoundaryConditions/BCs.cpp:28-83, 215-221),
get_tagging_params (Source/Tagging_params.cpp:24-70) and SDF::make_sdf
(Source/Geometry/MakeSDF.cpp:20-140). The main loop is driven through a
stand-in hierarchy whose coarse step advances time by a fixed dt, clamped
to the stop time, as Amr::coarseTimeStep clamps it."""
import os

import numpy as np
import pytest

from bamrex_b200 import _abi
from bamrex_b200 import inputs as I
from bamrex_b200 import plotfile as P

QUADRANT_2D = """
# four-quadrant Riemann problem
max_step  = 1000
stop_time = 0.25

prob.adiabatic = 1.4
prob.epsilon   = 0.5

geometry.is_periodic = 0 0 0
geometry.coord_sys   = 0        # Cartesian
geometry.prob_lo     = 0.0 0.0 0.0
geometry.prob_hi     = 2.0 1.0 1.0
amr.n_cell           = 256 128 128

adv.cfl        = 0.8
adv.num_method = muscl_hancock
limiting.limiter = minbee
limiting.density = "density"
limiting.mom     = u_x u_y
limiting.energy  = p

bc.x = transmissive reflective
bc.y = reflective transmissive

amr.max_level       = 2
amr.ref_ratio       = 2 2 2 2
amr.regrid_int      = 2
amr.blocking_factor = 8
amr.max_grid_size   = 64
amr.plot_int        = 10
amr.plot_file       = out/plt

tagging.max_phierr_lev = 2
tagging.phierr         = 1.01 1.1 1.5
"""


def _pp(text=QUADRANT_2D, overrides=()):
    return I.ParmParse.from_text(text, overrides)


# ---- the file format -------------------------------------------------------

def test_parse_comments_quotes_last_definition():
    pp = _pp("a = 1 2  # two\nb = \"x y\"\n# c = 3\na = 7\nflag = true\n")
    assert pp.queryarr("a", int) == [7]
    assert pp.get("b") == "x y"
    assert not pp.contains("c")
    assert pp.get("flag", bool) is True
    assert pp.query("missing", int, 5) == 5
    with pytest.raises(I.InputsError, match="not found"):
        pp.get("missing")
    with pytest.raises(I.InputsError, match="cannot read"):
        pp.get("b", float)


def test_parse_prefix_file_include_and_command_line(tmp_path):
    (tmp_path / "base").write_text("adv.cfl = 0.5\nadv.num_method = hllc\n")
    (tmp_path / "inputs").write_text("FILE = base\nadv.cfl = 0.7\n")
    pp = I.ParmParse.from_file(str(tmp_path / "inputs"), ["adv.num_method=slic", "amr.n_cell=8", "16"])
    adv = pp.sub("adv")
    assert adv.get("cfl", float) == 0.7
    assert adv.get("num_method") == "slic"
    assert pp.sub("amr").getarr("n_cell", int) == [8, 16]
    assert pp.sub("adv").names() == ["cfl", "num_method"]


@pytest.mark.parametrize("bad", ["just words here", "= 3"])
def test_parse_rejects_malformed_lines(bad):
    with pytest.raises(I.InputsError):
        _pp(bad)


# ---- settings ------------------------------------------------------------

def test_quadrant_settings():
    s = I.read_settings(_pp(), 2)
    assert (s.max_step, s.stop_time, s.strt_time) == (1000, 0.25, 0.0)
    assert s.plot_at == [0.25]
    assert s.n_cell == (256, 128) and s.dom_hi == (255, 127)
    assert s.prob_lo == (0.0, 0.0) and s.prob_hi == (2.0, 1.0)
    assert s.cfl == 0.8 and s.method == _abi.MUSCL_HANCOCK and s.do_reflux
    p = s.parm
    assert (p.adiabatic, p.epsilon, p.limiter) == (1.4, 0.5, _abi.MINBEE)
    # density on density, momenta on the velocities, energy on the pressure
    assert p.limiter_indices[:4] == [0, 1, 2, 3]
    assert p.limit_on_primv[:4] == [False, True, True, True]
    assert (s.bc_lo, s.bc_hi) == ((_abi.BC_TRANSMISSIVE, _abi.BC_REFLECTIVE), (_abi.BC_REFLECTIVE, _abi.BC_TRANSMISSIVE))
    assert (s.max_level, s.ref_ratio, s.regrid_int, s.blocking_factor, s.max_grid_size) == (2, 2, 2, 8, 64)
    assert s.phierr == [1.01, 1.1] and s.phierr_var == 0 and not s.phierr_var_is_primv
    assert s.phigrad == []
    assert s.plot_int == 10 and s.plot_file == "out/plt"
    assert s.body is None


def test_defaults_of_the_reference():
    s = I.read_settings(_pp(QUADRANT_2D.replace("limiting.", "#limiting.").replace("prob.epsilon", "#")), 2)
    p = s.parm
    assert p.limiter == _abi.VAN_LEER and p.epsilon == 1.0
    assert p.limiter_indices == [3] * 8 and p.limit_on_primv == [False] * 8  # every component on UInd::E
    s3 = I.read_settings(_pp(QUADRANT_2D.replace("bc.", "#bc.")), 3)
    assert s3.bc_lo == (_abi.BC_TRANSMISSIVE,) * 3 and s3.n_cell == (256, 128, 128)
    assert s3.parm.limiter_indices[:5] == [0, 1, 2, 4, 4]  # mom_z keeps UInd::E


def test_variable_names():
    assert I.variable_index(3, "energy") == (4, False)
    assert I.variable_index(3, "p") == (4, True)
    assert I.variable_index(2, "u_z") == (3, True)  # QInd::W is 3 whatever the dimension
    assert I.variable_index(2, "T") == (4, True)
    with pytest.raises(I.InputsError, match="Invalid variable name"):
        I.variable_index(2, "pressure")


def test_periodic_geometry_overrides_faces():
    s = I.read_settings(_pp(QUADRANT_2D.replace("is_periodic = 0 0 0", "is_periodic = 1 0 0")), 2)
    assert s.bc_lo[0] == s.bc_hi[0] == _abi.BC_PERIODIC
    txt = QUADRANT_2D.replace("bc.x = transmissive reflective", "bc.x = periodic periodic")
    with pytest.raises(I.InputsError, match="is_periodic"):
        I.read_settings(_pp(txt), 2)


@pytest.mark.parametrize("text, exc, match", [
    ("bc.x = transmissive wall\n", I.InputsError, "Invalid BC type"),
    ("bc.x = gresho transmissive\n", NotImplementedError, "bc.x = gresho"),
    ("bc.rb = slip\n", I.InputsError, "Invalid rigid body BC"),
    ("adv.num_method = upwind\n", I.InputsError, "Invalid numerical method"),
    ("adv.num_method = imex\n", NotImplementedError, "imex"),
    ("adv.visc_method = op_split_explicit\n", NotImplementedError, "visc"),
    ("limiting.limiter = minmod\n", I.InputsError, "limiting.limiter"),
    ("limiting.energy = pressure\n", I.InputsError, "Invalid variable name"),
    ("geometry.coord_sys = 1\n", I.InputsError, "coord_sys = 0"),
    ("strt_time = -1\n", I.InputsError, "non-negative strt_time"),
    ("tagging.max_box_lev = 1\ntagging.box_x = 0.1 0.2\n", I.InputsError, "box_y"),
    ("amr.ref_ratio = 4 4\n", NotImplementedError, "ratio 2"),
    ("amr.ref_ratio = 2 4\n", NotImplementedError, "one ratio"),
    ("ls.geom_type = box\n", NotImplementedError, "geom_type = box"),
    ("ls.geom_type = teapot\n", I.InputsError, "Invalid geometry"),
])
def test_refusals(text, exc, match):
    with pytest.raises(exc, match=match):
        I.read_settings(_pp(QUADRANT_2D + text), 2)


@pytest.mark.parametrize("drop, match", [
    ("adv.num_method", "adv.num_method not found"),
    ("prob.adiabatic", "prob.adiabatic not found"),
    ("amr.n_cell", "amr.n_cell not found"),
])
def test_required_settings(drop, match):
    with pytest.raises(I.InputsError, match=match):
        I.read_settings(_pp(QUADRANT_2D.replace(drop, "#" + drop)), 2)


def test_time_limits():
    no_limits = QUADRANT_2D.replace("max_step", "#").replace("stop_time", "#")
    with pytest.raises(I.InputsError, match="neither max_step nor stop_time"):
        I.read_settings(_pp(no_limits), 2)
    # read_params reads stop_time with get() even when max_step is set
    with pytest.raises(I.InputsError, match="stop_time not found"):
        I.read_settings(_pp(QUADRANT_2D.replace("stop_time", "#")), 2)
    s = I.read_settings(_pp(QUADRANT_2D + "amr.plot_at = 0.2 0.1\n"), 2)
    assert s.plot_at == [0.1, 0.2, 0.25]


def test_rigid_bodies():
    cyl = ("ls.geom_type = cylinder\nls.cylinder_radius = 0.1\nls.cylinder_center = 0.5 0.5 0\n"
           "ls.cylinder_axis = 0 0 1\nls.cylinder_has_fluid_inside = false\nbc.rb = no_slip\n")
    s = I.read_settings(_pp(QUADRANT_2D + cyl), 2)
    (sh,) = s.body["shapes"]
    assert sh == dict(kind=_abi.SDF_CYLINDER, radius=0.1, center=(0.5, 0.5, 0.0), axis=(0.0, 0.0, 1.0),
                      fluid_inside=False)
    assert s.body["rb_bc"] == _abi.RB_NO_SLIP and s.rb_bc == _abi.RB_NO_SLIP
    two = ("ls.geom_type = two_spheres\n" + "".join(
        "ls.sphere%d_center = %g 0.5 0.5\nls.sphere%d_radius = 0.3\nls.sphere%d_has_fluid_inside = 0\n" % (k, c, k, k)
        for k, c in ((1, 0.4), (2, 0.6))))
    s = I.read_settings(_pp(QUADRANT_2D + two), 3)
    assert s.body["combine"] == _abi.SDF_INTERSECTION and len(s.body["shapes"]) == 2
    assert s.body["shapes"][1]["center"] == (0.6, 0.5, 0.5) and s.rb_bc == _abi.RB_REFLECTIVE
    plane = "ls.geom_type = plane\nls.plane_point = 0.5 0 0\nls.plane_normal = 1 1 0\n"
    s = I.read_settings(_pp(QUADRANT_2D + plane), 2)
    assert s.body["shapes"][0]["kind"] == _abi.SDF_PLANE and s.body["shapes"][0]["axis"] == (1.0, 1.0, 0.0)
    assert I.read_settings(_pp(QUADRANT_2D + "ls.geom_type = all_regular\n"), 2).body is None
    with pytest.raises(I.InputsError, match="sphere_radius not found"):
        I.read_settings(_pp(QUADRANT_2D + "ls.geom_type = sphere\nls.sphere_center = 0 0 0\n"), 2)


def test_amr_arguments():
    s = I.read_settings(_pp(), 2)
    kw = I.amr_kwargs(s)
    boxes = kw["boxes"]
    cells = sum((hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) for lo, hi in boxes)
    assert cells == 256 * 128 and max(hi[0] - lo[0] + 1 for lo, hi in boxes) == 64
    assert kw["ngrow"] == 2 and kw["regrid_int"] == 2 and kw["max_level"] == 2
    assert kw["phierr"] == [1.01, 1.1] and kw["bc_lo"] == s.bc_lo
    single = I.read_settings(_pp(QUADRANT_2D.replace("amr.max_level       = 2", "amr.max_level = 0")), 2)
    assert I.amr_kwargs(single)["regrid_int"] == 0
    body = I.read_settings(_pp(QUADRANT_2D + "ls.geom_type = sphere\nls.sphere_center = 1 0.5 0\n"
                               "ls.sphere_radius = 0.1\nls.sphere_has_fluid_inside = 0\n"), 2)
    assert I.amr_kwargs(body)["ngrow"] == 4
    # interface and box tagging (Tagging_params.cpp:66-84): lstol padded with
    # zeros to max_int_lev, the refine box from box_x / box_y
    tagged = I.read_settings(_pp(QUADRANT_2D + "tagging.max_int_lev = 3\ntagging.lstol = 0.1 0.05\n"
                                 "tagging.max_box_lev = 1\ntagging.box_x = 0.1 0.4\ntagging.box_y = 0.2 0.3\n"), 2)
    kw = I.amr_kwargs(tagged)
    assert kw["max_int_lev"] == 3 and kw["lstol"] == [0.1, 0.05, 0.0]
    assert kw["max_box_lev"] == 1 and kw["refine_box"] == ([0.1, 0.2], [0.4, 0.3])
    plain = I.amr_kwargs(s)
    assert plain["max_int_lev"] == -1 and plain["max_box_lev"] == -1 and plain["refine_box"] is None


# ---- the main loop ---------------------------------------------------------

class _StandInAmr:
    def __init__(self, dt, time=0.0, coarse_steps=0):
        self.dt, self.time, self.calls = dt, time, []
        self.coarse_steps = coarse_steps

    def coarse_step(self, stop_time=-1.0):
        dt = self.dt
        if stop_time >= 0 and self.time + dt > stop_time:
            dt = stop_time - self.time
        self.calls.append(stop_time)
        self.time += dt
        self.coarse_steps += 1
        return dt


def _loop(text, dt, start_step=0, start_time=None):
    s = I.read_settings(_pp(text), 2)
    amr = _StandInAmr(dt, s.strt_time if start_time is None else start_time, start_step)
    plots, checks = [], []
    t, n = I.run(amr, s, on_plot=lambda a, k, tt: plots.append(k), on_check=lambda a, k, tt: checks.append(k))
    return s, amr, t, n, plots, checks


def test_main_loop_stop_time_and_plot_times():
    txt = QUADRANT_2D.replace("amr.plot_int        = 10", "amr.plot_int = 4") + "amr.check_int = 5\namr.plot_at = 0.1\n"
    s, amr, t, n, plots, checks = _loop(txt, 0.03)
    # 0.03 x 3, clamp to 0.1, then 0.03 x 5, clamp to 0.25
    assert n == 9 and abs(t - 0.25) < 1e-15
    assert amr.calls == [0.1] * 4 + [0.25] * 5
    assert plots == [0, 4, 8, 9]  # at the start, every 4 steps, at the end
    assert checks == [5, 9]


def test_main_loop_plot_at_adds_a_plotfile():
    txt = QUADRANT_2D.replace("amr.plot_int        = 10", "amr.plot_int = -1") + "amr.plot_at = 0.1\n"
    s, amr, t, n, plots, checks = _loop(txt, 0.03)
    assert plots == [4, 9]  # the plot_at time, then the end
    assert checks == [9]


def test_main_loop_max_step():
    txt = QUADRANT_2D.replace("max_step  = 1000", "max_step = 3").replace("amr.plot_int        = 10",
                                                                       "amr.plot_files_output = 0")
    s, amr, t, n, plots, checks = _loop(txt, 0.01)
    assert n == 3 and abs(t - 0.03) < 1e-15 and plots == [] and checks == [3]


# ---- plotfiles -------------------------------------------------------------

def _levels(D, rng):
    def fabs(boxes):
        return [rng.standard_normal((D + 2,) + tuple(hi[d] - lo[d] + 1 if d < D else 1 for d in (2, 1, 0)))
                for lo, hi in boxes]
    pad = (0,) * (3 - D)
    b0 = [((0,) * D + pad, (7,) + (15,) * (D - 1) + pad), ((8,) + (0,) * (D - 1) + pad, (15,) * D + pad)]
    b1 = [((8,) * D + pad, (15,) * D + pad), ((16,) + (8,) * (D - 1) + pad, (23,) + (15,) * (D - 1) + pad)]
    return [((0, 0, 0), (15,) * D + pad, b0, fabs(b0)), ((0, 0, 0), (31,) * D + pad, b1, fabs(b1))]


@pytest.mark.parametrize("D", [2, 3])
def test_plotfile_round_trip(tmp_path, D):
    rng = np.random.default_rng(5)
    levels = _levels(D, rng)
    names = ["density"] + ["mom_" + "xyz"[d] for d in range(D)] + ["energy"]
    path = str(tmp_path / "plt00010")
    P.write_plotfile(path, D, 0.125, [0.0] * D, [2.0] + [1.0] * (D - 1), levels, names, 2, [10, 20])
    got = P.read_plotfile(path)
    assert got["varnames"] == names and got["spacedim"] == D and got["time"] == 0.125
    assert got["level_steps"] == [10, 20] and got["ref_ratio"] == 2
    assert got["prob_hi"] == [2.0] + [1.0] * (D - 1)
    for (dlo, dhi, boxes, fabs), (glo, ghi, gboxes, gfabs) in zip(levels, got["levels"]):
        assert (tuple(glo), tuple(ghi)) == (dlo, dhi)
        assert gboxes == boxes
        for a, b in zip(fabs, gfabs):
            np.testing.assert_array_equal(a, b)
    hdr = open(os.path.join(path, "Header")).read().split("\n")
    assert hdr[0] == "HyperCLaw-V1.1" and hdr[1] == str(D + 2) and hdr[2:D + 4] == names
    assert hdr[D + 4] == str(D) and hdr[D + 6] == "1"  # dimension, finest level
    cell_h = open(os.path.join(path, "Level_1", "Cell_H")).read().split("\n")
    assert cell_h[:5] == ["1", "0", str(D + 2), "0", "(2 0"]
    assert cell_h[5:9] == [P._box_str(D, *b) for b in levels[1][2]] + [")", "2"]
    assert cell_h[9] == "FabOnDisk: Cell_D_00000 0" and cell_h[10].startswith("FabOnDisk: Cell_D_00000 ")
    assert cell_h[12] == "2,%d" % (D + 2)
    mins = [float(x) for x in cell_h[13].rstrip(",").split(",")]
    assert mins == [float(v) for v in levels[1][3][0].reshape(D + 2, -1).min(axis=1)]


def test_plotfile_rejects_mismatched_fab(tmp_path):
    levels = _levels(2, np.random.default_rng(1))
    dlo, dhi, boxes, fabs = levels[0]
    fabs = [fabs[0][:, :, :3]] + fabs[1:]
    with pytest.raises(ValueError, match="expected"):
        P.write_plotfile(str(tmp_path / "p"), 2, 0.0, [0, 0], [1, 1], [(dlo, dhi, boxes, fabs)],
                         ["density", "mom_x", "mom_y", "energy"])


# ---- initial data read from the inputs -------------------------------------

QUADRANT_STATES = "".join(
    "init.density_%s = %g\ninit.velocity_x_%s = %g\ninit.velocity_y_%s = %g\ninit.pressure_%s = %g\n"
    % (q, r, q, u, q, v, q, p) for q, r, u, v, p in (("TR", 0.5313, 0, 0, 0.4), ("TL", 1, 0.7276, 0, 1),
                                                     ("BL", 0.8, 0, 0, 1), ("BR", 1, 0, 0.7276, 1)))


class _Centres:
    def __init__(self, D, n):
        self.D, self.n = D, n

    def cell_centres(self, lev):
        x = (np.arange(self.n) + 0.5) / self.n
        return [x, x if self.D > 1 else np.zeros(1), x if self.D > 2 else np.zeros(1)]


@pytest.mark.parametrize("D", [2, 3])
def test_quadrant_initial_data(D):
    from bamrex_b200.problems import consv_from_primv
    pp = _pp(QUADRANT_2D + QUADRANT_STATES)
    s = I.read_settings(pp, D)
    u = I.INITIAL_DATA["QuadrantProblem"](pp, s)(_Centres(D, 8), 0)
    assert u.shape == (D + 2,) + ((8,) if D == 3 else (1,)) + (8, 8)
    for (j, i), prim in (((7, 7), (0.5313, 0, 0, 0.4)), ((7, 0), (1, 0.7276, 0, 1)), ((0, 0), (0.8, 0, 0, 1)),
                         ((0, 7), (1, 0, 0.7276, 1))):
        q = np.array(list(prim[:3]) + [0.0] * (D - 2) + [prim[3]]).reshape(D + 2, 1)
        np.testing.assert_array_equal(u[:, 0, j, i], consv_from_primv(D, q, 1.4, 0.5)[:, 0])
    with pytest.raises(I.InputsError, match="init.pressure_BR not found"):
        I.INITIAL_DATA["QuadrantProblem"](_pp(QUADRANT_2D + QUADRANT_STATES.replace("init.pressure_BR", "#")), s)


def test_plotfile_names():
    assert I.plotfile_name("out/plt", 10) == "out/plt00010"
    assert I.plotfile_name("chk", 123456) == "chk123456"


class _Level:
    """Cell centres and domain of one level over [lo, hi]^D with n cells."""

    def __init__(self, D, n, lo=0.0, hi=1.0):
        self.D, self.n, self.lo, self.hi = D, n, lo, hi

    def cell_centres(self, lev):
        x = self.lo + (np.arange(self.n) + 0.5) * (self.hi - self.lo) / self.n
        return [x if d < self.D else np.zeros(1) for d in range(3)]

    def domain(self, lev):
        return (0, 0, 0), tuple(self.n - 1 if d < self.D else 0 for d in range(3))


def _prim(D, rho, vel, p):
    from bamrex_b200.problems import consv_from_primv
    q = np.array([rho] + list(vel) + [p], dtype=np.float64).reshape(D + 2, 1)
    return consv_from_primv(D, q, 1.4, 0.5)[:, 0]


RIEMANN = ("init.density_L = 1\ninit.velocity_L = 0.75\ninit.pressure_L = 1\n"
           "init.density_R = 0.125\ninit.velocity_R = 0\ninit.pressure_R = 0.1\n")


@pytest.mark.parametrize("D", [1, 2, 3])
def test_riemann_initial_data(D):
    pp = _pp(QUADRANT_2D + RIEMANN)
    s = I.read_settings(pp, D)
    u = I.INITIAL_DATA["RiemannProblem"](pp, s)(_Level(D, 8), 0)
    vel_l = [0.75] + [0.0] * (D - 1) if D == 1 else [0.0, 0.75] + [0.0] * (D - 2)
    left, right = _prim(D, 1, vel_l, 1), _prim(D, 0.125, [0.0] * D, 0.1)
    if D == 1:  # split at the middle of [0, 2] in x
        np.testing.assert_array_equal(u[:, 0, 0, 7], left)
    else:       # split at y = 0.5
        np.testing.assert_array_equal(u[:, 0, 3, 7], left)
        np.testing.assert_array_equal(u[:, 0, 4, 0], right)


def test_explosion_initial_data():
    text = QUADRANT_2D + ("init.density_in = 1\ninit.pressure_in = 10\ninit.density_out = 0.125\n"
                          "init.pressure_out = 0.1\ninit.radius = 0.4\n")
    pp = _pp(text)
    s = I.read_settings(pp, 3)
    u = I.INITIAL_DATA["CylindricalExplosion"](pp, s)(_Level(3, 10, 0.0, 2.0), 0)
    inside, outside = _prim(3, 1, [0, 0, 0], 10), _prim(3, 0.125, [0, 0, 0], 0.1)
    np.testing.assert_array_equal(u[:, 5, 5, 5], inside)   # centre (1.1, 1.1, 1.1): r = 0.17
    np.testing.assert_array_equal(u[:, 0, 5, 5], outside)  # z far from 1
    pp = _pp(text + "init.force_cylindrical = true\n")
    u = I.INITIAL_DATA["CylindricalExplosion"](pp, s)(_Level(3, 10, 0.0, 2.0), 0)
    np.testing.assert_array_equal(u[:, 0, 5, 5], inside)   # a cylinder along z
    pp = _pp(text + "init.setup_as_rp = 1\n")
    with pytest.raises(I.InputsError, match="sym.rot_axis not found"):
        I.INITIAL_DATA["CylindricalExplosion"](pp, I.read_settings(pp, 2))
    pp = _pp(text + "init.setup_as_rp = 1\nsym.rot_axis = 1\n")
    u = I.INITIAL_DATA["CylindricalExplosion"](pp, I.read_settings(pp, 2))(_Level(2, 10), 0)
    np.testing.assert_array_equal(u[:, 0, 1, 9], _prim(2, 1, [0, 0], 10))  # r = y = 0.15
    np.testing.assert_array_equal(u[:, 0, 4, 0], _prim(2, 0.125, [0, 0], 0.1))  # r = y = 0.45
    with pytest.raises(I.InputsError, match="init.radius not found"):
        I.INITIAL_DATA["CylindricalExplosion"](_pp(text.replace("init.radius", "#")), s)


def test_vortex_initial_data():
    from bamrex_b200.problems import isentropic_vortex
    text = QUADRANT_2D + ("init.lambda = 5\ninit.density_bg = 1\ninit.u_bg = 0.1\ninit.v_bg = 0.2\n"
                          "init.w_bg = 0\ninit.pressure_bg = 1\ninit.x_c = 1\ninit.y_c = 0.5\n")
    pp = _pp(text)
    s = I.read_settings(pp, 2)
    u = I.INITIAL_DATA["IsentropicVortex"](pp, s)(_Level(2, 16), 0)
    ref = isentropic_vortex(2, [16, 16, 1], [0.0, 0.0], [2.0, 1.0], (1.0, 0.5), strength=5.0, vel_bg=(0.1, 0.2, 0.0),
                            adiabatic=1.4, epsilon=0.5)
    np.testing.assert_array_equal(u, ref)


# ---- arithmetic values (ParmParse evaluates them against other entries) ------

def test_expressions():
    pp = _pp("D = 0.01\nM = 2\nadia = 1.4\np_amb = 1\nrho_amb = 1\n"
             "t_0 = (D*6/(M*sqrt(adia*p_amb/rho_amb)))\nstop_time = t_0+0.0015\n"
             "amr.plot_at = t_0 t_0+0.0002\namr.n_cell = 2*4 2^3\nhalf = 3/2\n"
             "init.r = 0.25\ninit.area = pi*r^2\nr = 7\nloop_a = loop_b\nloop_b = \"loop_a + 1\"\n")
    t0 = 0.01 * 6 / (2 * (1.4 ** 0.5))
    assert pp.get("t_0", float) == pytest.approx(t0, rel=1e-15)
    assert pp.get("stop_time", float) == pytest.approx(t0 + 0.0015, rel=1e-15)
    assert pp.sub("amr").getarr("plot_at", float) == pytest.approx([t0, t0 + 0.0002], rel=1e-15)
    assert pp.sub("amr").getarr("n_cell", int) == [8, 8]
    assert pp.sub("init").get("area", float) == pytest.approx(3.141592653589793 / 16)  # init.r before r
    with pytest.raises(I.InputsError, match="cannot read"):
        pp.get("half", int)
    with pytest.raises(I.InputsError, match="refers to itself"):
        pp.get("loop_a", float)
    with pytest.raises(I.InputsError, match="single value"):  # unquoted spaces make three values
        _pp("a = b\nb = 1 + 2\n").get("a", float)
    with pytest.raises(I.InputsError, match="unknown name"):
        _pp("x = y + 1\n").get("x", float)
    with pytest.raises(I.InputsError, match="cannot read"):
        _pp("x = __import__('os')\n").get("x", float)
    # evaluated in double as ParmParse does: a tower of powers overflows at
    # once instead of growing an unbounded integer
    with pytest.raises(I.InputsError, match="cannot read"):
        _pp("x = 9^9^9\n").get("x", float)
    with pytest.raises(I.InputsError, match="cannot read"):
        _pp("n = 10^400\n").get("n", int)
    assert _pp("n = 2^10\n").get("n", int) == 1024


def test_missing_include_is_an_inputs_error(tmp_path):
    (tmp_path / "inputs").write_text("FILE = not_there\n")
    with pytest.raises(I.InputsError, match="FILE = not_there: no such file"):
        I.ParmParse.from_file(str(tmp_path / "inputs"))


def test_main_loop_after_a_restart():
    """A hierarchy restarted at coarse step 4 keeps counting: max_step counts
    the steps before the restart, no initial plotfile, the next plot and
    checkpoint on the original cadence."""
    text = QUADRANT_2D.replace("amr.plot_int        = 10", "amr.plot_int = 4") + \
        "max_step = 10\nstop_time = 100\namr.check_int = 3\n"
    s, amr, t, n, plots, checks = _loop(text, 0.1, start_step=4, start_time=0.4)
    assert n == 10 and len(amr.calls) == 6
    assert plots == [8, 10] and checks == [6, 9, 10]
    assert s.restart == ""
    assert I.read_settings(_pp(QUADRANT_2D + "amr.restart = chk00010\n"), 2).restart == "chk00010"
