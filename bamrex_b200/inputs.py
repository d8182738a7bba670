"""Run settings from an inputs file in the reference's format, and the
reference's main loop over a device hierarchy.

The reference reads every setting through AMReX ParmParse: `max_step`,
`strt_time`, `stop_time` and `amr.plot_at` in main (Source/main.cpp:23-50);
`adv.*` in AmrLevelAdv::read_params (Source/AmrLevelAdv.cpp:836-916);
`prob.*` and `limiting.*` in FluidSystem::ReadParameters
(Source/System/FluidSystem.cpp:10-50, defaults 52-71, variable names
Source/System/FluidSystem.H:91-137); `bc.*` in bamrexBCData::build
(Source/BoundaryConditions/BCs.cpp:28-83, periodic geometry overriding the
face types at 215-221, names BCTypes.H:10-67); `tagging.*` in
get_tagging_params (Source/Tagging_params.cpp:24-70); `ls.*` in SDF::make_sdf
(Source/Geometry/MakeSDF.cpp:20-140); `geometry.*` and `amr.*` are AMReX's
own Geometry and Amr settings. `read_settings` maps them onto this
package's Parm, Amr and rigid-body descriptors with the same names,
defaults and refusals; settings of parts this package does not build
(viscosity, tracers, rigid bodies other than planes, spheres and cylinders,
interface tagging) raise NotImplementedError naming the setting.

The file format is ParmParse's: `name = value value ...` up to the end of
the line, `#` starts a comment, a double-quoted value is one token, a
number may be an arithmetic expression over other entries (`t_0 = D*6/M`,
`stop_time = t_0+0.0015`; + - * / ^, sqrt, exp, log, sin, cos, ..., pi),
`FILE = path` reads another inputs file in place (a relative path from
the working directory, as AMReX opens it, else from the including file's
directory), and when a name is
defined more than once the last definition is the one read. Command-line
`name=value` arguments after the file are read as later definitions.
"""
from __future__ import annotations

import ast
import math
import operator
import os
import shlex
from dataclasses import dataclass, field

from . import _abi
from .level import Parm


class InputsError(ValueError):
    """A setting is missing or malformed (where the reference aborts)."""


# ----------------------------------------------------------------------
# ParmParse-format table
# ----------------------------------------------------------------------

def _tokens(line: str):
    lex = shlex.shlex(line, posix=True)
    lex.whitespace_split = True
    lex.commenters = "#"
    lex.quotes = '"'
    lex.escape = ""
    try:
        return list(lex)
    except ValueError as e:
        raise InputsError("cannot split %r: %s" % (line.strip(), e)) from None


_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
           ast.Pow: operator.pow, ast.Mod: operator.mod}
_UNOPS = {ast.UAdd: operator.pos, ast.USub: operator.neg}
_FUNCS = {"sqrt": math.sqrt, "exp": math.exp, "log": math.log, "log10": math.log10, "sin": math.sin,
          "cos": math.cos, "tan": math.tan, "asin": math.asin, "acos": math.acos, "atan": math.atan,
          "atan2": math.atan2, "sinh": math.sinh, "cosh": math.cosh, "tanh": math.tanh, "abs": abs,
          "fabs": abs, "floor": math.floor, "ceil": math.ceil, "pow": math.pow, "min": min, "max": max}
_CONSTS = {"pi": math.pi}


def _eval_expr(text: str, symbol):
    """Value of an arithmetic expression (+ - * / ^ **, parentheses, the
    functions of _FUNCS, pi) whose names are looked up by symbol(name),
    evaluated in double precision."""
    try:
        tree = ast.parse(text.replace("^", "**"), mode="eval")
    except SyntaxError:
        raise ValueError(text) from None

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)) \
                and not isinstance(node.value, bool):
            # in double, as ParmParse evaluates: 9^9^9 overflows instead of
            # building an unbounded integer
            return float(node.value)
        if isinstance(node, ast.BinOp) and type(node.op) in _BINOPS:
            return _BINOPS[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp) and type(node.op) in _UNOPS:
            return _UNOPS[type(node.op)](ev(node.operand))
        if isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in _FUNCS \
                and not node.keywords:
            return _FUNCS[node.func.id](*[ev(a) for a in node.args])
        if isinstance(node, ast.Name):
            return _CONSTS[node.id] if node.id in _CONSTS else symbol(node.id)
        if isinstance(node, ast.Attribute):
            parts = []
            while isinstance(node, ast.Attribute):
                parts.append(node.attr)
                node = node.value
            if isinstance(node, ast.Name):
                return symbol(".".join([node.id] + parts[::-1]))
        raise ValueError(text)
    return ev(tree)


def parse_text(text: str, base_dir: str = ".", table=None, _depth=0):
    """Definitions of an inputs text as [(name, [values...])] in file order."""
    if _depth > 16:
        raise InputsError("FILE includes nested more than 16 deep")
    table = [] if table is None else table
    for lineno, raw in enumerate(text.splitlines(), 1):
        toks = _tokens(raw.replace("=", " = ", 1) if "=" in raw else raw)
        if not toks:
            continue
        if len(toks) < 2 or toks[1] != "=":
            raise InputsError("line %d: expected 'name = value ...': %r" % (lineno, raw.strip()))
        name, values = toks[0], toks[2:]
        if name == "FILE":
            if len(values) != 1:
                raise InputsError("line %d: FILE takes one path" % lineno)
            path = values[0]
            if not os.path.isabs(path) and not os.path.exists(path):
                path = os.path.join(base_dir, path)
            if not os.path.exists(path):
                raise InputsError("line %d: FILE = %s: no such file (from the working directory or %s)"
                                  % (lineno, values[0], base_dir))
            with open(path) as f:
                parse_text(f.read(), os.path.dirname(path), table, _depth + 1)
            continue
        table.append((name, values))
    return table


def parse_args(args, table=None):
    """Command-line definitions after the inputs file: `name=value ...`
    (the values of one name run up to the next `name=`)."""
    table = [] if table is None else table
    i = 0
    args = list(args)
    while i < len(args):
        a = args[i]
        if "=" not in a:
            raise InputsError("command-line setting without '=': %r" % a)
        name, first = a.split("=", 1)
        if not name:
            raise InputsError("command-line setting without a name: %r" % a)
        values = [first] if first else []
        i += 1
        while i < len(args) and "=" not in args[i]:
            values.append(args[i])
            i += 1
        table.append((name, values))
    return table


class ParmParse:
    """Typed reads of a definition table under a prefix (`adv`, `amr`, ...),
    as amrex::ParmParse(prefix)."""

    def __init__(self, table, prefix: str = ""):
        self._table = table
        self.prefix = prefix

    @classmethod
    def from_file(cls, path: str, overrides=()):
        with open(path) as f:
            table = parse_text(f.read(), os.path.dirname(os.path.abspath(path)))
        parse_args(overrides, table)
        return cls(table)

    @classmethod
    def from_text(cls, text: str, overrides=()):
        table = parse_text(text)
        parse_args(overrides, table)
        return cls(table)

    def sub(self, prefix: str) -> "ParmParse":
        return ParmParse(self._table, prefix)

    def _full(self, name):
        return "%s.%s" % (self.prefix, name) if self.prefix else name

    def _last(self, name):
        full = self._full(name)
        for n, v in reversed(self._table):
            if n == full:
                return v
        return None

    def contains(self, name) -> bool:
        return self._last(name) is not None

    def names(self):
        p = self.prefix + "." if self.prefix else ""
        return sorted({n[len(p):] for n, _ in self._table if n.startswith(p)})

    def _symbol(self, name, seen):
        """A number-valued entry named in an expression: under this prefix
        first, then as written."""
        for full in ((self._full(name), name) if self.prefix else (name,)):
            if full in seen:
                raise InputsError("%s refers to itself" % full)
            for n, v in reversed(self._table):
                if n == full:
                    if len(v) != 1:
                        raise InputsError("%s: an expression needs a single value" % full)
                    return self._convert(full, v[0], float, seen | {full})
        raise InputsError("unknown name %r in an expression" % name)

    def _convert(self, full, tok, typ, seen=frozenset()):
        try:
            if typ is bool:
                t = tok.lower()
                if t in ("true", "t", "1"):
                    return True
                if t in ("false", "f", "0"):
                    return False
                raise ValueError(tok)
            if typ in (int, float):
                try:
                    return typ(tok)
                except ValueError:
                    v = _eval_expr(tok, lambda name: self._symbol(name, seen | {full}))
                    if typ is int:
                        if float(v) != int(v):
                            raise ValueError(tok)
                        return int(v)
                    return float(v)
            return str(tok)
        except InputsError:
            raise
        except (ValueError, ZeroDivisionError, OverflowError, TypeError):
            raise InputsError("%s: cannot read %r as %s" % (full, tok, typ.__name__)) from None

    def query(self, name, typ=str, default=None):
        v = self._last(name)
        if v is None:
            return default
        if not v:
            raise InputsError("%s: no value" % self._full(name))
        return self._convert(self._full(name), v[0], typ)

    def get(self, name, typ=str):
        v = self.query(name, typ)
        if v is None:
            raise InputsError("ParmParse::get(): %s not found in the inputs" % self._full(name))
        return v

    def queryarr(self, name, typ=str, default=None, n=None):
        v = self._last(name)
        if v is None:
            return default
        if n is not None and len(v) < n:
            raise InputsError("%s: %d values, %d needed" % (self._full(name), len(v), n))
        vals = [self._convert(self._full(name), t, typ) for t in v]
        return vals[:n] if n is not None else vals

    def getarr(self, name, typ=str, n=None):
        v = self.queryarr(name, typ, n=n)
        if v is None:
            raise InputsError("ParmParse::getarr(): %s not found in the inputs" % self._full(name))
        return v


# ----------------------------------------------------------------------
# name tables of the reference
# ----------------------------------------------------------------------

METHODS = {"muscl_hancock": _abi.MUSCL_HANCOCK, "hllc": _abi.HLLC, "imex": _abi.IMEX, "rcm": _abi.RCM,
           "slic": _abi.SLIC, "force": _abi.FORCE, "lax_friedrichs": _abi.LAX_FRIEDRICHS}
EXPLICIT_METHODS = (_abi.MUSCL_HANCOCK, _abi.HLLC, _abi.SLIC, _abi.FORCE, _abi.LAX_FRIEDRICHS)
BC_NAMES = ("transmissive", "reflective", "periodic", "gresho", "pressure_outlet", "coaxial_jet", "supersonic_jet")
RB_NAMES = {"reflective": _abi.RB_REFLECTIVE, "no_slip": _abi.RB_NO_SLIP}
NOT_BUILT_GEOMETRY = ("box", "cone", "equilateral_wedge", "guitton_nozzle", "polygon_union")


def variable_index(D: int, name: str):
    """(index, is_primitive) of a variable name (FluidSystem::VariableIndex /
    VariableIsPrimitive). The primitive indices are the reference's QInd
    constants, so in 2D `u_z` names slot 3, the pressure, as there."""
    cons = {"density": 0, "mom_x": 1, "mom_y": 2, "mom_z": 3, "energy": 1 + D}
    prim = {"u_x": 1, "u_y": 2, "u_z": 3, "p": 1 + D, "T": 2 + D, "eta": 3 + D, "zeta": 4 + D, "kappa": 5 + D}
    if name in cons:
        return cons[name], False
    if name in prim:
        return prim[name], True
    raise InputsError("Invalid variable name " + name)


# ----------------------------------------------------------------------
# settings
# ----------------------------------------------------------------------

@dataclass
class Settings:
    """Everything a run of the reference reads, in this package's terms."""
    spacedim: int
    # main (Source/main.cpp:23-50)
    max_step: int = -1
    strt_time: float = 0.0
    stop_time: float = -1.0
    plot_at: list = field(default_factory=list)
    # geometry.* (AMReX Geometry)
    n_cell: tuple = ()
    prob_lo: tuple = ()
    prob_hi: tuple = ()
    is_periodic: tuple = ()
    # adv.* (AmrLevelAdv::read_params)
    cfl: float = 0.9
    method: int = _abi.MUSCL_HANCOCK
    method_name: str = "muscl_hancock"
    do_reflux: bool = True
    verbose: int = 0
    # prob.* and limiting.* (FluidSystem::ReadParameters)
    parm: Parm = None
    # bc.* (bamrexBCData::build)
    bc_lo: tuple = ()
    bc_hi: tuple = ()
    rb_bc: int = _abi.RB_REFLECTIVE
    # amr.* (AMReX Amr)
    max_level: int = 0
    ref_ratio: int = 2
    regrid_int: int = 1
    blocking_factor: int = 8
    max_grid_size: int = 32
    n_error_buf: int = 1
    grid_eff: float = 0.7
    n_proper: int = 1
    plot_int: int = -1
    plot_per: float = -1.0
    plot_file: str = "plt"
    plot_files_output: bool = True
    check_int: int = -1
    check_file: str = "chk"
    checkpoint_files_output: bool = True
    restart: str = ""
    # tagging.* (get_tagging_params)
    phierr: list = field(default_factory=list)
    phierr_var: int = 0
    phierr_var_is_primv: bool = False
    phigrad: list = field(default_factory=list)
    phigrad_var: int = 0
    phigrad_var_is_primv: bool = False
    max_int_lev: int = -1
    lstol: list = field(default_factory=list)
    max_box_lev: int = -1
    refine_box: tuple | None = None
    # ls.* (SDF::make_sdf): shapes for bamrex_b200.level.body_desc, or None
    body: dict | None = None

    @property
    def dom_lo(self):
        return (0,) * self.spacedim

    @property
    def dom_hi(self):
        return tuple(n - 1 for n in self.n_cell)


def _shape_flag(ls, name):
    return ls.get(name, bool)


def read_body(D: int, ls: ParmParse, rb_bc: int):
    """ls.* -> {'shapes': [...], 'combine': ..., 'rb_bc': ...} or None
    (SDF::make_sdf, Source/Geometry/MakeSDF.cpp:20-140)."""
    geom_type = ls.query("geom_type", str, "")
    if geom_type in ("", "all_regular"):
        return None
    if geom_type == "sphere":
        shapes = [dict(kind=_abi.SDF_SPHERE, center=tuple(ls.getarr("sphere_center", float, n=D)),
                       radius=ls.get("sphere_radius", float),
                       fluid_inside=_shape_flag(ls, "sphere_has_fluid_inside"))]
        combine = _abi.SDF_UNION
    elif geom_type == "two_spheres":
        shapes = [dict(kind=_abi.SDF_SPHERE, center=tuple(ls.getarr("sphere%d_center" % k, float, n=D)),
                       radius=ls.get("sphere%d_radius" % k, float),
                       fluid_inside=_shape_flag(ls, "sphere%d_has_fluid_inside" % k)) for k in (1, 2)]
        combine = _abi.SDF_INTERSECTION
    elif geom_type == "cylinder":
        shapes = [dict(kind=_abi.SDF_CYLINDER, radius=ls.get("cylinder_radius", float),
                       center=tuple(ls.getarr("cylinder_center", float, n=3)),
                       axis=tuple(ls.getarr("cylinder_axis", float, n=3)),
                       fluid_inside=_shape_flag(ls, "cylinder_has_fluid_inside"))]
        combine = _abi.SDF_UNION
    elif geom_type == "plane":
        shapes = [dict(kind=_abi.SDF_PLANE, center=tuple(ls.getarr("plane_point", float, n=3)),
                       axis=tuple(ls.getarr("plane_normal", float, n=3)))]
        combine = _abi.SDF_UNION
    elif geom_type in NOT_BUILT_GEOMETRY:
        raise NotImplementedError("ls.geom_type = %s: only plane, sphere, two_spheres and cylinder bodies are "
                                  "built" % geom_type)
    else:
        raise InputsError("Invalid geometry type " + geom_type)
    return {"shapes": shapes, "combine": combine, "rb_bc": rb_bc}


def read_settings(pp: ParmParse, spacedim: int) -> Settings:
    """Settings of a run with `spacedim` dimensions (the reference fixes it
    at compile time) from an inputs table."""
    D = spacedim
    if D not in (1, 2, 3):
        raise InputsError("spacedim must be 1, 2 or 3")
    s = Settings(spacedim=D)

    # main
    s.max_step = pp.query("max_step", int, -1)
    s.strt_time = pp.query("strt_time", float, 0.0)
    s.stop_time = pp.query("stop_time", float, -1.0)
    if s.strt_time < 0.0:
        raise InputsError("MUST SPECIFY a non-negative strt_time")
    if s.max_step < 0 and s.stop_time < 0.0:
        raise InputsError("Exiting because neither max_step nor stop_time is non-negative.")
    amr = pp.sub("amr")
    s.plot_at = sorted(amr.queryarr("plot_at", float, []) + [s.stop_time])

    # geometry
    geo = pp.sub("geometry")
    if geo.query("coord_sys", int, 0) != 0:
        raise InputsError("Please set geom.coord_sys = 0")
    s.n_cell = tuple(amr.getarr("n_cell", int, n=D))
    if any(n < 1 for n in s.n_cell):
        raise InputsError("amr.n_cell must be positive")
    s.prob_lo = tuple(geo.getarr("prob_lo", float, n=D))
    s.prob_hi = tuple(geo.getarr("prob_hi", float, n=D))
    s.is_periodic = tuple(bool(v) for v in geo.queryarr("is_periodic", int, [0] * D, n=D))

    # adv
    adv = pp.sub("adv")
    s.verbose = adv.query("v", int, 0)
    s.cfl = adv.query("cfl", float, 0.9)
    s.do_reflux = adv.query("do_reflux", bool, True)
    s.method_name = adv.get("num_method", str)
    if s.method_name not in METHODS:
        raise InputsError("Invalid numerical method \"%s\". Valid options are muscl_hancock, hllc, and imex"
                          % s.method_name)
    s.method = METHODS[s.method_name]
    if s.method not in EXPLICIT_METHODS:
        raise NotImplementedError("adv.num_method = %s: AMR hierarchies here step the explicit methods "
                                  "(muscl_hancock, hllc, slic, force, lax_friedrichs); the IMEX step is "
                                  "bamrex_b200.imex.Imex on a single level" % s.method_name)
    if adv.query("visc_method", str, ""):
        raise NotImplementedError("adv.visc_method: viscous terms are not built")
    if adv.query("do_tracers", int, 0):
        raise NotImplementedError("adv.do_tracers: tracer particles are not built")
    pp.get("stop_time", float)  # read_params requires it even with max_step set
    prob = pp.sub("prob")
    if prob.query("system", str, "fluid") != "fluid":
        raise NotImplementedError("prob.system: only the fluid (Euler) system is built")

    # prob / limiting
    adiabatic = prob.get("adiabatic", float)
    epsilon = prob.query("epsilon", float, 1.0)
    lim = pp.sub("limiting")
    limiter_name = lim.query("limiter", str, "van_leer")
    if limiter_name not in _abi.LIMITERS:
        raise InputsError("limiting.limiter: %r is not one of minbee, van_leer, van_albada, superbee"
                          % limiter_name)
    idx = [1 + D] * _abi.MAX_NCOMP
    prim = [False] * _abi.MAX_NCOMP
    density = lim.query("density", str, "")
    energy = lim.query("energy", str, "")
    mom = lim.queryarr("mom", str, [])
    if density:
        idx[0], prim[0] = variable_index(D, density)
    if energy:
        idx[1 + D], prim[1 + D] = variable_index(D, energy)
    for d in range(D):
        if d < len(mom) and mom[d]:
            idx[1 + d], prim[1 + d] = variable_index(D, mom[d])
    s.parm = Parm(D, adiabatic=adiabatic, epsilon=epsilon, limiter=_abi.LIMITERS[limiter_name],
                  limiter_indices=idx, limit_on_primv=prim)

    # bc
    bc = pp.sub("bc")
    lo, hi = [], []
    for d, axis in zip(range(D), "xyz"):
        pair = bc.getarr(axis, str, n=2) if bc.contains(axis) else ["transmissive", "transmissive"]
        for name in pair:
            if name not in BC_NAMES:
                raise InputsError("Invalid BC type specified")
            if name not in _abi.BCS:
                raise NotImplementedError("bc.%s = %s: only transmissive, reflective and periodic faces are built"
                                          % (axis, name))
        a, b = _abi.BCS[pair[0]], _abi.BCS[pair[1]]
        if s.is_periodic[d]:
            a = b = _abi.BC_PERIODIC
        elif _abi.BC_PERIODIC in (a, b):
            raise InputsError("bc.%s = periodic needs geometry.is_periodic set in that direction" % axis)
        lo.append(a)
        hi.append(b)
    s.bc_lo, s.bc_hi = tuple(lo), tuple(hi)
    rb = bc.query("rb", str, "reflective")
    if rb not in RB_NAMES:
        raise InputsError("Invalid rigid body BC type specified")
    s.rb_bc = RB_NAMES[rb]

    # amr
    s.max_level = amr.query("max_level", int, 0)
    ratios = amr.queryarr("ref_ratio", int, [2])
    used = ratios[:max(s.max_level, 1)]
    if any(r != used[0] for r in used):
        raise NotImplementedError("amr.ref_ratio: one ratio for every level pair")
    s.ref_ratio = used[0]
    if s.max_level > 0 and s.ref_ratio != 2:
        raise NotImplementedError("amr.ref_ratio = %d: the coarse/fine glue is built for ratio 2" % s.ref_ratio)
    s.regrid_int = amr.queryarr("regrid_int", int, [1])[0]
    s.blocking_factor = amr.queryarr("blocking_factor", int, [8])[0]
    s.max_grid_size = amr.queryarr("max_grid_size", int, [32 if D == 3 else 128])[0]
    s.n_error_buf = amr.queryarr("n_error_buf", int, [1])[0]
    s.grid_eff = amr.query("grid_eff", float, 0.7)
    s.n_proper = amr.query("n_proper", int, 1)
    s.plot_int = amr.query("plot_int", int, -1)
    s.plot_per = amr.query("plot_per", float, -1.0)
    s.plot_file = amr.query("plot_file", str, "plt")
    s.plot_files_output = amr.query("plot_files_output", bool, True)
    s.check_int = amr.query("check_int", int, -1)
    s.check_file = amr.query("check_file", str, "chk")
    s.checkpoint_files_output = amr.query("checkpoint_files_output", bool, True)
    # amr.restart names a checkpoint of this library (bamrex_b200.checkpoint);
    # AMReX's own checkpoint files are not read
    s.restart = amr.query("restart", str, "")

    # tagging
    tg = pp.sub("tagging")
    # interface tagging: |level set| <= lstol[lev] or an interface cell
    # (Tagging_params.cpp:66-71; lstol sized max_int_lev, zeros where the
    # inputs give fewer values)
    s.max_int_lev = tg.query("max_int_lev", int, -1)
    if s.max_int_lev > 0:
        vals = tg.queryarr("lstol", float, []) or []
        s.lstol = (list(vals) + [0.0] * s.max_int_lev)[:s.max_int_lev]
    # box tagging: the box_x / box_y / box_z intervals (Tagging_params.cpp:72-84)
    s.max_box_lev = tg.query("max_box_lev", int, -1)
    if s.max_box_lev != -1:
        lo, hi = [], []
        for nm in ("box_x", "box_y", "box_z")[:D]:
            v = tg.getarr(nm, float, n=2)
            lo.append(v[0])
            hi.append(v[1])
        s.refine_box = (lo, hi)
    for kind in ("phierr", "phigrad"):
        max_lev = tg.query("max_%s_lev" % kind, int, -1)
        if max_lev == -1:
            continue
        vals = tg.queryarr(kind, float, [1.0e20] * max_lev)
        var = tg.query("%s_var" % kind, str, "")
        vi, vp = variable_index(D, var) if var else (0, False)
        setattr(s, kind, vals[:max_lev])
        setattr(s, kind + "_var", vi)
        setattr(s, kind + "_var_is_primv", vp)

    # rigid bodies
    s.body = read_body(D, pp.sub("ls"), s.rb_bc)
    return s


# ----------------------------------------------------------------------
# the hierarchy and the main loop
# ----------------------------------------------------------------------

def amr_kwargs(s: Settings, ngrow: int | None = None, precision=_abi.FP64):
    """Keyword arguments of bamrex_b200.amr.Amr for these settings (base
    grids: the domain chopped at amr.max_grid_size)."""
    from .level import decompose
    pad = (0,) * (3 - s.spacedim)
    boxes = decompose(s.spacedim, s.dom_lo + pad, s.dom_hi + pad, s.max_grid_size)
    if ngrow is None:
        ngrow = 4 if s.body is not None else 2
    return dict(spacedim=s.spacedim, dom_lo=s.dom_lo, dom_hi=s.dom_hi, prob_lo=list(s.prob_lo),
                prob_hi=list(s.prob_hi), boxes=boxes, parm=s.parm, method=s.method, cfl=s.cfl, ngrow=ngrow,
                bc_lo=s.bc_lo, bc_hi=s.bc_hi, precision=precision, max_level=s.max_level, ref_ratio=s.ref_ratio,
                blocking_factor=s.blocking_factor, max_grid_size=s.max_grid_size, n_error_buf=s.n_error_buf,
                n_proper=s.n_proper, grid_eff=s.grid_eff, regrid_int=s.regrid_int if s.max_level > 0 else 0,
                do_reflux=s.do_reflux, phigrad=s.phigrad, phigrad_var=s.phigrad_var,
                phigrad_var_is_primv=s.phigrad_var_is_primv, phierr=s.phierr, phierr_var=s.phierr_var,
                phierr_var_is_primv=s.phierr_var_is_primv, max_int_lev=s.max_int_lev, lstol=s.lstol,
                max_box_lev=s.max_box_lev, refine_box=s.refine_box)


def make_amr(s: Settings, initial_data=None, ngrow: int | None = None, precision=_abi.FP64, base_boxes=None):
    """The device hierarchy of these settings with its rigid body; with
    `initial_data(amr, lev) -> (NC, nz, ny, nx) array` the initial
    hierarchy is built as Amr::init does (level 0, then tag, new level,
    initial data, up to amr.max_level).  base_boxes replaces the base
    level's grids (a restart takes the checkpoint's)."""
    from .amr import Amr
    kw = amr_kwargs(s, ngrow, precision)
    if base_boxes is not None:
        kw["boxes"] = base_boxes
    a = Amr(**kw)
    if s.body is not None:
        b = s.body
        a.set_body(b["shapes"], combine=b["combine"], rb_bc=b["rb_bc"])
    if initial_data is not None:
        a.init(initial_data, s.strt_time)
    a.time = s.strt_time
    return a


def plot_due(s: Settings, step: int, time: float, dt: float) -> bool:
    """AMReX Amr's plot trigger after a coarse step: every amr.plot_int coarse
    steps, or when the step crossed a multiple of amr.plot_per."""
    if not s.plot_files_output:
        return False
    if s.plot_int > 0 and step % s.plot_int == 0:
        return True
    if s.plot_per > 0 and dt > 0:
        return math.floor((time + 1e-12 * dt) / s.plot_per) > math.floor((time - dt + 1e-12 * dt) / s.plot_per)
    return False


def restart_amr(s: Settings, ngrow: int | None = None, precision=_abi.FP64):
    """The hierarchy of these settings continuing the checkpoint amr.restart
    (AmrLevelAdv::restart, Source/AmrLevelAdv.cpp:95-104): the checkpoint's
    grids, state, time and stepping, these settings otherwise."""
    from .checkpoint import restart_amr as _restart
    return _restart(s.restart, lambda boxes: make_amr(s, None, ngrow, precision, base_boxes=boxes))


def run(amr, s: Settings, on_plot=None, on_check=None):
    """The reference's main loop (Source/main.cpp:68-107) on a hierarchy
    made by make_amr: coarse steps clamped to the next of amr.plot_at and
    stop_time, until max_step steps or stop_time. `on_plot(amr, step,
    time)` is called where AMReX writes a plotfile (at the start when
    amr.plot_int or amr.plot_per is set, after plot_int steps, on crossing
    a multiple of plot_per, at each plot_at time, and at the end) and
    `on_check(amr, step, time)` where it writes a checkpoint (after
    check_int steps and at the end). A restarted hierarchy keeps counting
    coarse steps from its checkpoint (max_step counts them all) and writes
    no initial plotfile. Returns (time, coarse steps)."""
    steps = amr.coarse_steps
    restarted = steps > 0
    last_plot = last_check = steps if restarted else -1
    if on_plot is not None and s.plot_files_output and (s.plot_int > 0 or s.plot_per > 0) and not restarted:
        on_plot(amr, steps, amr.time)
        last_plot = steps
    i_plot = 0
    next_stop = s.plot_at[i_plot]
    while (steps < s.max_step or s.max_step < 0) and (amr.time < s.stop_time or s.stop_time < 0.0):
        dt = amr.coarse_step(next_stop)
        steps += 1
        if on_plot is not None and plot_due(s, steps, amr.time, dt):
            on_plot(amr, steps, amr.time)
            last_plot = steps
        if on_check is not None and s.checkpoint_files_output and s.check_int > 0 and steps % s.check_int == 0:
            on_check(amr, steps, amr.time)
            last_check = steps
        if amr.time >= next_stop * (1 - 1e-12):
            i_plot += 1
            if i_plot >= len(s.plot_at):
                continue
            next_stop = s.plot_at[i_plot]
            if on_plot is not None and s.plot_files_output and last_plot < steps:
                on_plot(amr, steps, amr.time)
                last_plot = steps
    if on_check is not None and s.checkpoint_files_output and last_check < steps:
        on_check(amr, steps, amr.time)
    if on_plot is not None and s.plot_files_output and last_plot < steps:
        on_plot(amr, steps, amr.time)
    return amr.time, steps


# ----------------------------------------------------------------------
# initial data read from the inputs
# ----------------------------------------------------------------------

def quadrant_initial_data(pp: ParmParse, s: Settings):
    """initdata of the reference's four-quadrant problem
    (Exec/QuadrantProblem/Prob.cpp:19-95): the primitive states
    init.{density,velocity_x,velocity_y,pressure}_{TR,TL,BL,BR} placed by
    the quadrant of the cell centre about (0.5, 0.5) (a centre on x = 0.5
    or y = 0.5 falls to BR, as there); zero z velocity. Returns
    fn(amr, lev) -> (NC, nz, ny, nx) conserved state of level lev."""
    import numpy as np
    from .problems import consv_from_primv
    D = s.spacedim
    if D < 2:
        raise InputsError("the quadrant problem needs two or three dimensions")
    init = pp.sub("init")
    states = {}
    for q in ("TR", "TL", "BL", "BR"):
        prim = [init.get("density_" + q, float), init.get("velocity_x_" + q, float),
                init.get("velocity_y_" + q, float)] + [0.0] * (D - 2) + [init.get("pressure_" + q, float)]
        states[q] = consv_from_primv(D, np.array(prim, dtype=np.float64).reshape(D + 2, 1),
                                     s.parm.adiabatic, s.parm.epsilon)[:, 0]

    def fn(amr, lev):
        x, y, z = amr.cell_centres(lev)
        X = np.broadcast_to(x[None, None, :], (len(z), len(y), len(x)))
        Y = np.broadcast_to(y[None, :, None], X.shape)
        out = np.empty((D + 2,) + X.shape)
        tr, tl, bl = (X > 0.5) & (Y > 0.5), (X < 0.5) & (Y > 0.5), (X < 0.5) & (Y < 0.5)
        br = ~(tr | tl | bl)
        for mask, q in ((tr, "TR"), (tl, "TL"), (bl, "BL"), (br, "BR")):
            for n in range(D + 2):
                out[n][mask] = states[q][n]
        return out
    return fn


def _two_states(s, prim_a, prim_b):
    import numpy as np
    from .problems import consv_from_primv
    D = s.spacedim
    out = []
    for prim in (prim_a, prim_b):
        q = np.array(prim, dtype=np.float64).reshape(D + 2, 1)
        out.append(consv_from_primv(D, q, s.parm.adiabatic, s.parm.epsilon)[:, 0])
    return out


def _fill(D, mask, inside, outside):
    import numpy as np
    out = np.empty((D + 2,) + mask.shape)
    for n in range(D + 2):
        out[n] = np.where(mask, inside[n], outside[n])
    return out


def _mesh(amr, lev):
    import numpy as np
    x, y, z = amr.cell_centres(lev)
    shape = (len(z), len(y), len(x))
    return (np.broadcast_to(x[None, None, :], shape), np.broadcast_to(y[None, :, None], shape),
            np.broadcast_to(z[:, None, None], shape))


def riemann_initial_data(pp: ParmParse, s: Settings):
    """initdata_euler of the reference's Riemann problem
    (Exec/RiemannProblem/Prob.cpp:33-118): init.{density,velocity,
    pressure}_{L,R}; in 1D the left state where x < (prob_lo + prob_hi)/2
    with the velocity along x, in 2D and 3D the left state where y < 0.5 (a
    fixed 0.5, as there) with the velocity along y. The exact-solution file
    the reference also writes is not written."""
    D = s.spacedim
    init = pp.sub("init")
    vals = {k: init.get(k, float) for k in ("density_L", "velocity_L", "pressure_L", "density_R", "velocity_R",
                                            "pressure_R")}
    vel = lambda v: [v] + [0.0] * (D - 1) if D == 1 else [0.0, v] + [0.0] * (D - 2)
    left, right = _two_states(s, [vals["density_L"]] + vel(vals["velocity_L"]) + [vals["pressure_L"]],
                              [vals["density_R"]] + vel(vals["velocity_R"]) + [vals["pressure_R"]])

    def fn(amr, lev):
        X, Y, _ = _mesh(amr, lev)
        mask = X < (s.prob_lo[0] + s.prob_hi[0]) * 0.5 if D == 1 else Y < 0.5
        return _fill(D, mask, left, right)
    return fn


def explosion_initial_data(pp: ParmParse, s: Settings):
    """initdata of the reference's cylindrical explosion
    (Exec/CylindricalExplosion/Prob.cpp:20-92): init.{density,pressure}_in
    at rest where r < init.radius, init.{density,pressure}_out elsewhere,
    r the distance from (1, 1, 1) (1D: r = x; 2D with init.setup_as_rp: x
    or y by sym.rot_axis; 3D with init.force_cylindrical: the distance from
    the line x = y = 1). init.radius has no default there (an unset value
    is read uninitialised); here it is required."""
    import numpy as np
    D = s.spacedim
    init = pp.sub("init")
    d_in, p_in = init.get("density_in", float), init.get("pressure_in", float)
    d_out, p_out = init.get("density_out", float), init.get("pressure_out", float)
    radius = init.get("radius", float)
    as_rp = init.query("setup_as_rp", bool, False)
    cylindrical = init.query("force_cylindrical", bool, False)
    rot_axis = pp.sub("sym").get("rot_axis", int) if as_rp else 0
    inside, outside = _two_states(s, [d_in] + [0.0] * D + [p_in], [d_out] + [0.0] * D + [p_out])

    def fn(amr, lev):
        X, Y, Z = _mesh(amr, lev)
        if D == 1:
            r = X
        elif D == 2:
            r = (X if rot_axis == 0 else Y) if as_rp else np.sqrt((X - 1) * (X - 1) + (Y - 1) * (Y - 1))
        elif cylindrical:
            r = np.sqrt((X - 1) * (X - 1) + (Y - 1) * (Y - 1))
        else:
            r = np.sqrt((X - 1) * (X - 1) + (Y - 1) * (Y - 1) + (Z - 1) * (Z - 1))
        return _fill(D, r < radius, inside, outside)
    return fn


def vortex_initial_data(pp: ParmParse, s: Settings):
    """initdata of the reference's isentropic vortex
    (Exec/IsentropicVortex/Prob.cpp:25-123 at time 0): init.lambda,
    init.{density,u,v,w,pressure}_bg, centre (init.x_c, init.y_c). The
    exact-solution file the reference also writes is not written."""
    from .problems import isentropic_vortex
    D = s.spacedim
    if D < 2:
        raise InputsError("the isentropic vortex needs two or three dimensions")
    init = pp.sub("init")
    lam = init.get("lambda", float)
    rho, p = init.get("density_bg", float), init.get("pressure_bg", float)
    vel = (init.get("u_bg", float), init.get("v_bg", float), init.get("w_bg", float))
    centre = (init.get("x_c", float), init.get("y_c", float))

    def fn(amr, lev):
        lo, hi = amr.domain(lev)
        n = [hi[d] - lo[d] + 1 for d in range(3)]
        return isentropic_vortex(D, n, list(s.prob_lo), list(s.prob_hi), centre, strength=lam, rho_bg=rho,
                                 vel_bg=vel, p_bg=p, adiabatic=s.parm.adiabatic, epsilon=s.parm.epsilon)
    return fn


INITIAL_DATA = {"QuadrantProblem": quadrant_initial_data, "RiemannProblem": riemann_initial_data,
                "CylindricalExplosion": explosion_initial_data, "IsentropicVortex": vortex_initial_data}


def plotfile_name(prefix: str, step: int) -> str:
    """AMReX's plotfile and checkpoint naming: the prefix and the coarse
    step in at least five digits."""
    return "%s%05d" % (prefix, step)


def main(argv=None):
    """python -m bamrex_b200.inputs --problem QuadrantProblem --dim 2 INPUTS
    [name=value ...]: the reference's executable for that problem on the
    device, with its plotfiles."""
    import argparse
    from .plotfile import write_amr_plotfile
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--problem", required=True, choices=sorted(INITIAL_DATA))
    ap.add_argument("--dim", type=int, required=True, choices=(1, 2, 3))
    ap.add_argument("--fp32-storage", action="store_true")
    ap.add_argument("inputs")
    ap.add_argument("overrides", nargs="*")
    a = ap.parse_args(argv)
    pp = ParmParse.from_file(a.inputs, a.overrides)
    s = read_settings(pp, a.dim)
    fn = INITIAL_DATA[a.problem](pp, s)
    prec = _abi.FP32_STORAGE if a.fp32_storage else _abi.FP64
    if s.restart:
        amr = restart_amr(s, precision=prec)
        print("restarted from %s at t = %.10g, coarse step %d" % (s.restart, amr.time, amr.coarse_steps))
    else:
        amr = make_amr(s, fn, precision=prec)

    def plot(amr_, step, time):
        path = plotfile_name(s.plot_file, step)
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        write_amr_plotfile(path, amr_, step)
        print("wrote %s at t = %.6g" % (path, time))

    def check(amr_, step, time):
        from .checkpoint import write_checkpoint
        path = plotfile_name(s.check_file, step)
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        write_checkpoint(path, amr_)
        print("wrote %s at t = %.6g" % (path, time))

    t, n = run(amr, s, on_plot=plot, on_check=check)
    print("%d coarse steps, t = %.10g" % (n, t))
    amr.close()


if __name__ == "__main__":
    main()
